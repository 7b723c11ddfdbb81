/*
 * bcpnn_batch.h -- C ABI of the batch engine: many independent networks of
 * uneven size advanced together on one GPU by one persistent kernel per run.
 *
 * A member is a whole gsbn network of one population (H HCUs x M MCUs) with
 * one recurrent projection (src_pop = dest_pop = 0), its own connectivity,
 * stimulus tables and Philox seed: exactly what ProcUpdLazy (Pop.cpp,
 * Proj.cpp) computes for that network alone, tick by tick, bit for bit.
 * Members share the schedule: every run advances all of them over the same
 * ticks with the same prn, each reading its own stimulus rows.
 *
 * No counterpart in the reference: gsbn runs one network per process.  The
 * entry points mirror the single-network ones of bcpnn.h:
 *   bcpnn_batch_create            bcpnn_net_create, once per member
 *   bcpnn_batch_set_conn          bcpnn_set_conn (ProcInitConn add_row)
 *   bcpnn_batch_upload_stimuli_idx bcpnn_upload_stimuli_idx (ProcExtGen tables)
 *   bcpnn_batch_use_stimulus      bcpnn_use_stimulus (ProcExtGen's lgidx-row /
 *                                 wmask-idx, one row index for all members)
 *   bcpnn_batch_run               bcpnn_run (n calls of ProcUpdLazy::update +
 *                                 ProcExchangeSpike, every member)
 *   bcpnn_batch_read_state        bcpnn_read_state (gsbn names and layouts)
 *   bcpnn_batch_get_spike_log     bcpnn_get_spike_log
 *
 * Execution: a cooperative launch of as many CTAs as fit on the GPU at once.
 * Per tick, phase A gives every (member, HCU) item to one warp (items are
 * assigned to warps by a longest-processing-time schedule over estimated
 * costs): population update, j-traces and the HCU's active rows with the
 * ordered epsc sum; then a grid barrier; phase B spreads over all warps the
 * column updates of the tick's spikes, in units of 64 slots, and their
 * fan-out into the delay queue; then a grid barrier.  The delay queue is
 * event driven: a spike sets one bit per fan-out slot in the destination
 * HCU's arrival ring at the tick the row becomes active, instead of every
 * slot's shift register being stepped every tick; bcpnn_batch_read_state
 * rebuilds gsbn's qi/.siq from the ring.
 *
 * Errors: int status codes of bcpnn.h (BCPNN_OK, BCPNN_ERR_*), message in
 * bcpnn_batch_last_error.  Not thread-safe per handle.
 */
#ifndef BCPNN_BATCH_H
#define BCPNN_BATCH_H

#include <stddef.h>
#include <stdint.h>

#include "bcpnn.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct bcpnn_batch bcpnn_batch;

typedef struct bcpnn_batch_member {
  bcpnn_pop_desc pop;    /* hcu_num, mcu_num (1 .. 64), taum, ... as for one network */
  bcpnn_proj_desc proj;  /* src_pop = dest_pop = 0; slot_num gives C = min(H*M, slot_num) */
  uint32_t seed;         /* Philox key (seed, population 0): the member's stream as a network of its own */
} bcpnn_batch_member;

typedef struct bcpnn_batch_desc {
  int32_t n_members;
  const bcpnn_batch_member* members;
  float dt;
  float poisson_noise_hz;   /* project-defined input noise, as bcpnn_net_desc */
  int32_t device;
  int32_t max_ticks_per_run;
  int32_t threads;          /* CTA size of the batch kernel: 256, 384 or 512 (0: 512) */
  int32_t lpt_weights[3];   /* item cost model of the warp schedule: cost = w0 + w1*M + w2*C/32
                               ({0,0,0}: the default 64, 4, 1) */
} bcpnn_batch_desc;

int bcpnn_batch_create(const bcpnn_batch_desc* desc, bcpnn_batch** out);
int bcpnn_batch_destroy(bcpnn_batch* b);

/* connectivity of one member: H*C source MCU indices (-1: empty slot) and
   delays (1 .. 31), as bcpnn_set_conn */
int bcpnn_batch_set_conn(bcpnn_batch* b, int32_t member, const int32_t* ii, const int32_t* di, size_t n);

/* stimulus tables of one member (rows of H pattern indices, rows of H mask
   values), as bcpnn_upload_stimuli_idx; lginp = log(1+eps) on the indexed
   MCU, log(eps) elsewhere (ProcExtGen.cpp:130-144) */
int bcpnn_batch_upload_stimuli_idx(bcpnn_batch* b, int32_t member, int32_t n_lgidx_rows, const int32_t* lgidx_rows,
                                   float eps, int32_t n_wmask_rows, const float* wmask_rows);

/* the stimulus rows the next runs use, the same row index for every member */
int bcpnn_batch_use_stimulus(bcpnn_batch* b, int32_t lgidx_row, int32_t wmask_row);

/* n_ticks ticks of every member from first_simstep, prn as bcpnn_run (the
   all-cells catch-up at a change of prn included) */
int bcpnn_batch_run(bcpnn_batch* b, int32_t first_simstep, int32_t n_ticks, float prn, float old_prn);

/* every member back to gsbn's initial state (connectivity, stimulus kept) */
int bcpnn_batch_reset(bcpnn_batch* b);
int bcpnn_batch_sync(bcpnn_batch* b);
int bcpnn_batch_get_stream(const bcpnn_batch* b, void** stream);

/* a member's state vector in gsbn's name and layout (names of bcpnn_read_state
   with index 0: "pij_0", "qi_0", "dsup_0", ...) */
int bcpnn_batch_state_info(bcpnn_batch* b, int32_t member, const char* name, int32_t* type, size_t* count);
int bcpnn_batch_read_state(bcpnn_batch* b, int32_t member, const char* name, void* host, size_t bytes);

/* a member's spike log of the last run: n_ticks rows of ceil(H*M/32) words */
int bcpnn_batch_get_spike_log(bcpnn_batch* b, int32_t member, uint32_t* out, size_t n_words);

/* cumulative cell updates of all members: row cells, column cells, all-cells */
int bcpnn_batch_counters(bcpnn_batch* b, uint64_t out[3]);
int bcpnn_batch_kernel_launches(const bcpnn_batch* b, uint64_t* out);

/* The schedule tuner: times candidate launch shapes -- CTA size 256, 384 or
   512 and item cost models of the warp schedule -- on probe_ticks training ticks
   followed by probe_ticks recall ticks (the catch-up at the switch included),
   from the current state, restoring nothing (call it on a fresh or reset
   batch; reset afterwards).  The fastest becomes the batch's shape;
   out[0..3] = threads, cost weights w0, w1, w2; *us_per_tick its time. */
int bcpnn_batch_tune(bcpnn_batch* b, int32_t probe_ticks, int32_t lgidx_train, int32_t wmask_train,
                     int32_t lgidx_recall, int32_t wmask_recall, int32_t out[4], float* us_per_tick);

const char* bcpnn_batch_last_error(const bcpnn_batch* b);

/* Phase probe of the batch kernel, as bcpnn_phase_probe: in a library built
   with -DBCPNN_PHASE_PROBE, per CTA 32 counters -- [0] phase A SM cycles
   summed over warps and ticks, [1] the slowest warp's phase A summed over
   ticks, [2], [3] the same for phase B, [4], [5] the waits of the two grid
   barriers, [6] ticks, [7] units, [8] items; the default build returns
   BCPNN_ERR_STATE. */
int bcpnn_batch_phase_probe(bcpnn_batch* b, uint64_t* out, int32_t max_ctas, int32_t* n_ctas, int32_t reset);

#ifdef __cplusplus
}
#endif

#endif /* BCPNN_BATCH_H */
