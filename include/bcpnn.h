/*
 * bcpnn.h -- C ABI of the B200 BCPNN simulation core (libgsbn_b200.so).
 *
 * This is the layer under the drop-in procedures ProcUpdLazy, ProcExchangeSpike
 * and ProcSpkRec of the C++ engine.  It replaces, for one network held on one
 * GPU, what gsbn does per tick through Pop/Proj objects, SyncVector mirrors and
 * per-object CUDA streams (src/gsbn/procedures/ProcUpdLazy.cpp,
 * ProcUpdLazy/Pop.cpp, ProcUpdLazy/Proj.cpp).  Conventions:
 *
 *   - plain C types, caller-owned host buffers, library-owned device buffers;
 *   - every call returns an int status (BCPNN_OK == 0); no exception crosses
 *     the boundary; bcpnn_last_error() gives the message of the last failure;
 *   - one CUDA stream per network handle; a handle is not thread-safe;
 *   - the simulation state keeps the names and the row-major layouts of gsbn's
 *     Database vectors (dsup_<pop>, pij_<proj>, ... ; row = dest_hcu*C + slot,
 *     cell = row*M + mcu) at the read/write boundary, whatever the device
 *     layout is.
 *
 * Numerics: plain FP32 with the same expression trees as gsbn's CPU path;
 * exp/log and the random streams follow include/bcpnn_numerics.h, so a CPU
 * replay with the same definitions is bit-identical.
 */
#ifndef BCPNN_H
#define BCPNN_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define BCPNN_OK 0
#define BCPNN_ERR_INVALID (-1)   /* bad argument (null pointer, size, index) */
#define BCPNN_ERR_CUDA (-2)      /* a CUDA runtime call failed               */
#define BCPNN_ERR_NOT_FOUND (-3) /* unknown state vector name                */
#define BCPNN_ERR_SIZE (-4)      /* buffer size does not match the vector    */
#define BCPNN_ERR_STATE (-5)     /* call not valid in the current state      */
#define BCPNN_ERR_DEVICE (-6)    /* a kernel reported an error word          */

/* element types reported by bcpnn_state_info */
#define BCPNN_F32 0
#define BCPNN_I32 1
#define BCPNN_I8 2

typedef struct bcpnn_net bcpnn_net;

/* One population: gsbn PopParam (src/gsbn/proto/gsbn.proto:38-59) fields used
   by ProcUpdLazy/Pop.cpp:17-40. */
typedef struct bcpnn_pop_desc {
  int32_t hcu_num;
  int32_t mcu_num;   /* 1 .. 512 */
  float taum;
  float wtagain;
  float maxfq;
  float igain;
  float wgain;
  float lgbias;
  float snoise;
  float taua;        /* ProcUpdMulti only: adaptation time constant (gsbn.proto:52, default 0.05) */
  float adgain;      /* ProcUpdMulti only: adaptation gain (gsbn.proto:51, default 1)           */
} bcpnn_pop_desc;

/* One projection: gsbn ProjParam (gsbn.proto:61-74) fields used by
   ProcUpdLazy/Proj.cpp:16-52. */
typedef struct bcpnn_proj_desc {
  int32_t src_pop;
  int32_t dest_pop;
  float tauzi;
  float tauzj;
  float taue;
  float taup;
  float maxfq;
  float bgain;
  float wgain;
  float tauepsc;   /* <= 0 means "not set": tauepsc defaults to tauzi       */
  float slot_num;  /* float in the schema; dim_conn = min(Hs*Ms, (int)slot) */
} bcpnn_proj_desc;

typedef struct bcpnn_net_desc {
  int32_t n_pops;
  const bcpnn_pop_desc* pops;
  int32_t n_projs;
  const bcpnn_proj_desc* projs;
  float dt;                  /* GenParam.dt                                   */
  uint32_t seed;             /* Philox key word 0 (ProcUpdLazy argi "seed")   */
  float poisson_noise_hz;    /* ProcUpdLazy argf "poisson-noise-hz" (0: off)  */
  int32_t exchange_spikes;   /* 1: ProcExchangeSpike runs every tick          */
  int32_t device;            /* CUDA device ordinal                           */
  int32_t max_ticks_per_run; /* capacity of the per-run spike log             */
  int32_t tick_threads;      /* CTA size of the tick kernel: 512 (0 = default)
                                or 256 (two CTAs per SM, HCUs of <= 256 MCUs) */
  int32_t fp64_tables;       /* 0: gsbn's closed-form trace decay in float (bit
                                parity with the reference CPU path); 1: per
                                elapsed-tick propagators expm(d A) built in FP64
                                on the GPU and rounded once to float -- robust
                                when time constants nearly coincide, not
                                bit-identical to the reference */
  int32_t update_variant;    /* 0: ProcUpdLazy; 1: ProcUpdMulti (row-only updates
                                that replay a ring of postsynaptic spikes,
                                adaptation in the population; per-tick launches) */
  int32_t spike_buffer_size; /* ProcUpdMulti argi "spike buffer size" (1 .. 1024;
                                0 means 1) */
} bcpnn_net_desc;

/* Build a network on the device with gsbn's initial values.  Limits: at most
   4096 populations, 4096 projections, 8 projections into one population, 512
   MCUs per HCU, and one HCU's resident state must fit in shared memory.
   Replaces ProcUpdLazy::init_new (ProcUpdLazy.cpp:8-46), Pop::init_new
   (ProcUpdLazy/Pop.cpp:8-65) and Proj::init_new (ProcUpdLazy/Proj.cpp:6-107). */
int bcpnn_net_create(const bcpnn_net_desc* desc, bcpnn_net** out);

/* Release every device buffer and the stream of the network. */
int bcpnn_net_destroy(bcpnn_net* net);

/* Connection table of one projection: ii (source MCU or -1) and di (delay in
   ticks, 1..31) for all dest_hcu*C slots.  Replaces ProcInitConn::add_row
   (ProcInitConn.cpp:92-103) writing ii_<proj>/di_<proj>. */
int bcpnn_set_conn(bcpnn_net* net, int32_t proj, const int32_t* ii, const int32_t* di, size_t n_slots);

/* Stimulus for the following ticks: lginp for every MCU of the network (row
   lginp-idx of .lginp) and wmask for every HCU (row wmask-idx of .wmask), as
   ProcExtGen publishes them (ProcExtGen.cpp:126-144) and Pop::update_sup_cpu
   reads them (ProcUpdLazy/Pop.cpp:327-332). */
int bcpnn_set_stimulus(bcpnn_net* net, const float* lginp, size_t n_mcu, const float* wmask_row, size_t n_hcu);

/* Device-resident stimulus tables, uploaded once: n_lginp_rows rows of
   total-MCU lginp values and n_wmask_rows rows of total-HCU wmask values, the
   device copy of what ProcExtGen keeps in .lginp/.wmask (ProcExtGen.cpp:57-103).
   bcpnn_use_stimulus selects the rows used by the following runs without any
   host->device copy; bcpnn_set_stimulus switches back to host-set values. */
int bcpnn_upload_stimuli(bcpnn_net* net, int32_t n_lginp_rows, const float* lginp_rows, int32_t n_wmask_rows,
                         const float* wmask_rows);
int bcpnn_use_stimulus(bcpnn_net* net, int32_t lginp_row, int32_t wmask_row);

/* The same from ProcExtGen's pattern-index rows (.lgidx, one MCU index per
   HCU; any other value means no input to that HCU): the library computes
   lginp = log(1+eps) on the indexed MCU and log(0+eps) elsewhere
   (ProcExtGen.cpp:130-144) with its own float log, on the device.  Both
   rows are copied on the network's stream: a page-locked row is read when
   the stream reaches the copy, so keep it unchanged until the next
   bcpnn_sync; a pageable row is staged before the call returns. */
int bcpnn_set_stimulus_idx(bcpnn_net* net, const int32_t* lgidx_row, size_t n_hcu, float eps, const float* wmask_row,
                           size_t n_wmask);
int bcpnn_upload_stimuli_idx(bcpnn_net* net, int32_t n_lgidx_rows, const int32_t* lgidx_rows, float eps,
                             int32_t n_wmask_rows, const float* wmask_rows);

/* bcpnn_upload_stimuli_idx queued on the network's stream without a wait,
   for a caller that uploads a run schedule's tables once per pass (as
   ProcExtGen reads its stimulus file once, ProcExtGen.cpp:57-103, and picks
   rows per segment): the pattern-index and mask rows are copied from the
   caller's buffers (page-locked: read when the stream reaches the copies, so
   keep them unchanged until the next bcpnn_sync) and the lginp rows computed
   on the device.  The device tables grow, with a wait and a device
   allocation, only when a call has more rows than every earlier one; then
   bcpnn_use_stimulus selects rows.  At most 65535 pattern-index rows. */
int bcpnn_upload_stimuli_idx_async(bcpnn_net* net, int32_t n_lgidx_rows, const int32_t* lgidx_rows, float eps,
                                   int32_t n_wmask_rows, const float* wmask_rows);

/* External spike replay of one population (ProcUpdLazy args "external spike",
   ProcUpdLazy/Pop.cpp:67-110 and fill_spike :389-409): n entries, entry k
   overrides the spikes of tick ticks[k] with idx[offsets[k] .. offsets[k+1]);
   offsets holds n + 1 non-negative, non-decreasing values.  Ticks outside
   [0, 2^24) are ignored (no run reaches them).  Once set, every tick is
   overridden (ticks not listed give no spikes); a later call replaces the
   table. */
int bcpnn_set_ext_spikes(bcpnn_net* net, int32_t pop, int32_t n, const int32_t* ticks, const int32_t* offsets,
                         const int32_t* idx);

/* Structural-plasticity pruning of projection `proj`, on the device:
   every connected slot row whose row tick ti is below threshold_t, or none of
   whose weights reaches wp or wn (w >= wp or w <= wn), is disconnected
   (ii = -1, di = 0, ti = 0, pi = 0, ei = 0, and pij, eij, zj2 of its cells set
   to 0).  removed_src (cap >= H*C entries) receives the source MCUs of the
   removed rows in row order, *n_removed their number.  Replaces
   ProcStructuralPlasticity's Prj::prune / remove_conn
   (ProcStructuralPlasticity/Prj.cpp:69-92, 130-165).  Synchronises. */
int bcpnn_prune(bcpnn_net* net, int32_t proj, int32_t threshold_t, float wp, float wn, int32_t* removed_src,
                size_t cap, int32_t* n_removed);

/* Key of population `pop`'s random streams: Philox key (seed, key_pop*16 +
   stream) instead of (desc->seed, pop*16 + stream).  Lets a population of a
   batch (many independent networks built as one multi-population network)
   draw exactly the numbers it would draw as population key_pop of a network
   of its own with that seed.  No counterpart in the reference (its RNG is
   unseeded, src/gsbn/Random.cpp:5-13). */
int bcpnn_set_pop_rng(bcpnn_net* net, int32_t pop, uint32_t seed, uint32_t key_pop);

/* Advance n_ticks ticks with simstep first_simstep, first_simstep+1, ... .
   prn is the plasticity of every tick of the run; old_prn is the value of
   GlobalVar "old-prn" at the first tick (an all-cells catch-up runs first when
   it differs from prn).  Asynchronous on the network's stream.  Replaces
   ProcUpdLazy::update_gpu (ProcUpdLazy.cpp:128-180) called once per tick,
   plus the ProcExchangeSpike copy (ProcExchangeSpike.cpp:94-139) when
   desc->exchange_spikes is set. */
int bcpnn_run(bcpnn_net* net, int32_t first_simstep, int32_t n_ticks, float prn, float old_prn);

/* Restore gsbn's initial values in every state vector (Pop.cpp:59-65,
   Proj.cpp:88-105) and restart the tick count; connectivity, stimulus and
   replay tables are kept.  Asynchronous, on the device. */
int bcpnn_reset(bcpnn_net* net);

/* The cudaStream_t (as void*) the network's work is queued on, for callers
   that time or order their own work against it. */
int bcpnn_get_stream(const bcpnn_net* net, void** stream);

/* Wait for all work queued on the network's stream. */
int bcpnn_sync(bcpnn_net* net);

/* Number of 32-bit words of one tick of population `pop` in the spike log. */
int bcpnn_spike_log_words(const bcpnn_net* net, int32_t pop, int32_t* words);

/* Copy the spike log of the last run for population `pop`: n_ticks rows of
   bcpnn_spike_log_words() words; bit (i & 31) of word (i >> 5) is MCU i of the
   population (index h*M + m, as ProcSpkRec writes it, ProcSpkRec/Pop.cpp:30-52).
   Synchronises the stream. */
int bcpnn_get_spike_log(bcpnn_net* net, int32_t pop, uint32_t* out, size_t n_words);

/* The same copy queued without waiting for it: the host can queue the next
   segment's stimulus and run behind it, and the device runs the segments
   back to back.  The log is copied on the network's stream into one of two
   device staging buffers and from there to `out` on a second stream of the
   network, so the next run does not wait for the host copy.  `out` must stay
   valid, and is only complete, after the next bcpnn_sync (which waits for
   both streams and reports a device error of the runs); with page-locked
   `out` the copy is asynchronous, with pageable memory the driver may
   complete it before returning.  A later bcpnn_run does not disturb a queued
   copy (stream order). */
int bcpnn_get_spike_log_async(bcpnn_net* net, int32_t pop, uint32_t* out, size_t n_words);

/* ProcCheck's recall counters on the device (ProcCheck/Pop.cpp:36-44
   update_counter, :46-60 check_result), so a recall segment's evaluation
   needs no spike log on the host.  bcpnn_check_count adds, for every MCU of
   population `pop`, its spikes in ticks k0 .. k1-1 of the last run (0-based
   within the run) to the population's counters (zero at creation).
   bcpnn_check_result_async queues, per HCU, the MCU with the most counted
   spikes (the first on ties, -1 when none spiked) and that count into
   idx/cnt (n_hcu = the population's HCUs) and clears the counters; like the
   asynchronous spike log (and on the same second stream), idx/cnt are
   complete after the next bcpnn_sync.
   The caller walks ProcCheck's tick cursor (which ticks count, when a
   segment is evaluated) and compares idx/cnt with the expected pattern. */
int bcpnn_check_count(bcpnn_net* net, int32_t pop, int32_t k0, int32_t k1);
int bcpnn_check_result_async(bcpnn_net* net, int32_t pop, int32_t* idx, int32_t* cnt, size_t n_hcu);

/* Per tick of the last run, one byte per projection: bit 0 set if row 9 was in
   .ssi_<proj>, bit 1 if MCU 9 was in .ssj_<proj> (the debug flags ProcSpkRec
   writes to ssi_pop_/ssj_pop_<proj>.csv, ProcSpkRec/Prj.cpp:95-138).  out has
   n_ticks * n_projs bytes, tick-major. */
int bcpnn_get_ss_flags(bcpnn_net* net, uint8_t* out, size_t n_bytes);

/* Size and element type of a named state vector (gsbn Database names, e.g.
   "pij_0", "dsup_1", "spike_0", ".counter_0"). */
int bcpnn_state_info(const bcpnn_net* net, const char* name, int32_t* type, size_t* count);

/* Copy a named state vector to / from host memory in gsbn's layout.  Replaces
   Database::sync_vector_* + SyncVector::cpu_data/mutable_cpu_data
   (include/gsbn/Database.hpp, src/gsbn/SyncVector.cu:277-322).
   Synchronises the stream. */
int bcpnn_read_state(bcpnn_net* net, const char* name, void* host, size_t bytes);
int bcpnn_write_state(bcpnn_net* net, const char* name, const void* host, size_t bytes);

/* The same read as bcpnn_read_state, for callers that cannot allocate device
   memory: an embedding whose device memory is entirely pre-reserved by its
   own pool or budget (a cudaMalloc there fails or breaks the embedder's
   accounting), or a simulation loop that must not stall on cudaMalloc/
   cudaFree, which can synchronise the whole device.  bcpnn_read_state may
   cudaMalloc a staging buffer the first time it gathers a cell field
   (pij/eij/zi2/zj2 are interleaved on the device); this entry point gathers
   into a fixed 4 MiB array compiled into the library instead, which every GPU
   that loads the library keeps until the process exits, and allocates
   nothing.  Limits: a cell field read this way has at most 1048576 elements
   (larger ones return BCPNN_ERR_SIZE); .siq_<proj> is not offered.  The first
   call on a device looks up the array's device address and keeps it (make
   that first call before any stream capture; the kept address assumes the
   device is not reset with cudaDeviceReset while the library is loaded).
   All calls on a device share the array: calls that overlap on the GPU (from
   several threads or handles at once) race, so serialise them; each call
   synchronises its network's stream before it returns.  No counterpart in
   the reference, which reads state through SyncVector host mirrors. */
int bcpnn_read_state_noalloc(bcpnn_net* net, const char* name, void* host, size_t bytes);

/* Cumulative cell updates since creation: out[0] row cells, out[1] column
   cells (active post MCUs x dim_conn, as gsbn's column loop counts them),
   out[2] all-cells catch-up cells.  Synchronises the stream. */
int bcpnn_counters(bcpnn_net* net, uint64_t out[3]);

/* Number of kernels this library launched for the network since creation. */
int bcpnn_kernel_launches(const bcpnn_net* net, uint64_t* out);

/* Failure-detection self-test (no counterpart in the reference, whose
   errors all abort): runs the bounded grid-barrier wait of the persistent tick
   kernel on an arrival count that never completes.  Every wait gives up after
   limit_ns (1e5 .. 2e9 ns) and sets the barrier bit of the network's error
   word; the call then returns BCPNN_ERR_DEVICE with the timeout in
   bcpnn_last_error, and the network stays usable.  Nothing traps or spins
   without bound. */
int bcpnn_selftest_barrier_timeout(bcpnn_net* net, int64_t limit_ns);

/* Numerics self-test (no counterpart in the reference): the decay closed
   forms divide by a multiplication with a correctly rounded double
   reciprocal, RN_float(a * RN_double(1/b)), and fall back to a warp-uniform
   exact division (zero and infinite operands by their exact results, a
   double-precision quotient rounded once for subnormal or extreme operands)
   where the quotient is subnormal.  This runs n_pairs float pairs drawn from
   `seed` (with biased draws of zero, infinite, subnormal, extreme-exponent
   and near-midpoint quotients) through both forms and `/` on the network's
   device and reports how many pairs were compared (NaN operands skipped) and
   how many quotients of either form differed from `/` in any bit (NaN
   results compare equal). */
int bcpnn_selftest_division(bcpnn_net* net, uint64_t n_pairs, uint64_t seed, uint64_t* tested, uint64_t* mismatches);

/* Phase probe of the tick kernel (no counterpart in the reference): in a
   library built with -DBCPNN_PHASE_PROBE, copies per CTA (up to max_ctas) the
   32 counters of kernel phases -- SM clock cycles summed over ticks; slots
   0-9 group A (barrier wait, support, softmax, spikes, j-traces, column wait,
   rows, end of rows, join wait, staging), 16-29 group B (barrier wait, join
   wait, staging, column units of the grid, delay queue, spike wait, unit
   publication), slot 31 the tick count; slots 14 and 15 count the closed-form
   decays done by the exact fallback and by the reciprocal form -- sets
   *n_ctas and, if reset, zeroes them.  The default build returns
   BCPNN_ERR_STATE. */
int bcpnn_phase_probe(bcpnn_net* net, uint64_t* out, int32_t max_ctas, int32_t* n_ctas, int32_t reset);

/* Message of the last failing call on this handle ("" if none). */
const char* bcpnn_last_error(const bcpnn_net* net);

/* Static description of a status code. */
const char* bcpnn_status_string(int status);

#ifdef __cplusplus
}
#endif

#endif /* BCPNN_H */
