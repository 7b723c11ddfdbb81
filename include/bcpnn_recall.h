/* Replicate recall engine: the recall phase (prn = 0) of one trained
 * population with a full recurrent projection, run for R independent noise
 * replicates at once, with the synaptic support as a BF16 tensor-core
 * contraction.  No counterpart in the reference (gsbn runs one network per
 * process); it reproduces what gsbn's ProcUpdLazy does in recall for each
 * replicate, under these conditions:
 *
 *   - prn = 0: the plasticity rate kp is 0, so w_ij and b_j stay as the
 *     prn-change catch-up left them (Proj.cpp:289 recomputes w_ij once at the
 *     switch; the row and j-trace updates only rewrite them when kp != 0,
 *     Proj.cpp:352-356, 445-451).  The traces P/E/Z keep moving in gsbn but
 *     never reach the spikes again, so the engine does not carry them.
 *   - one projection, source = destination population, every destination HCU
 *     holds one slot per source MCU (C = H*M) and every delay is 1 tick: the
 *     rows active at tick t are the MCUs that spiked at t-3 (the exchange
 *     after the tick, then the queue bit set at t-2 and read out at t-1,
 *     ProcExchangeSpike.cpp:94-139, Proj.cpp:621-664).
 *
 * Per tick t and replicate r the engine computes (same order as gsbn):
 *   population update with epsc(t-1): sup, dsup, softmax/WTA with the
 *   population-MCU-0 max seed (Pop.cpp:229-323), Philox spikes with seed
 *   seed_base + r, Poisson input noise;
 *   epsc(t) = epsc(t-1) * (1 - kepsc) + S(t-3) . W  (Proj.cpp:310-363 decay,
 *   :445-451 ordered sum over active rows), where S is the 0/1 spike matrix
 *   [R x N] (exact in BF16) and W [N x N] holds w_ij rounded once to BF16; the
 *   products accumulate in FP32 in tensor memory.
 *
 * Limits: N = H*M a multiple of 256, M dividing 256 (HCUs never straddle a
 * 256-column tile), R a multiple of 128, one population.  sm_100a only.
 * desc.contraction selects an FP32 form of the contraction (W kept in FP32,
 * SIMT multiply-adds) with everything else unchanged.
 */
#ifndef BCPNN_RECALL_H
#define BCPNN_RECALL_H

#include <stddef.h>
#include <stdint.h>

#include "bcpnn.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct bcpnn_recall bcpnn_recall;

typedef struct bcpnn_recall_desc {
  int32_t hcu_num, mcu_num;  /* H, M */
  int32_t replicates;        /* R */
  bcpnn_pop_desc pop;        /* taum, wtagain, maxfq, igain, wgain, lgbias, snoise */
  float dt;
  float kepsc;               /* epsc decay rate of the projection (dt/tauepsc, else dt/tauzi) */
  uint32_t seed_base;        /* replicate r uses Philox key seed_base + r */
  float poisson_noise_hz;
  int32_t device;
  int32_t contraction;       /* BCPNN_RECALL_BF16 (0) or BCPNN_RECALL_FP32 (1) */
} bcpnn_recall_desc;

/* The form of the support contraction S(t-3) . W:
   BCPNN_RECALL_BF16  W rounded once to BF16, tcgen05 tensor-core MMA with
                      FP32 accumulation in tensor memory;
   BCPNN_RECALL_FP32  W kept in FP32, FP32 fused multiply-adds on the SIMT
                      pipes (the same engine at full precision, for measuring
                      the BF16 form against).
   Both accumulate in FP32 in an order of their own, not gsbn's row order, and
   share the population kernel and the epsc epilogue. */
enum { BCPNN_RECALL_BF16 = 0, BCPNN_RECALL_FP32 = 1 };

int bcpnn_recall_create(const bcpnn_recall_desc* d, bcpnn_recall** out);
int bcpnn_recall_destroy(bcpnn_recall* r);

/* Trained state, shared by every replicate: W[i*N + j] = w_ij from source MCU
   i to destination MCU j (float; rounded to BF16 here in the BF16 form), bj[N], and the
   population state at the end of tick first-1: epsc[N], dsup[N], the spikes
   of ticks first-3, first-2 and first-1 (int8 [N] each; in a gsbn network
   these are .siq, bit 0 of qi and si of the slots, by source MCU). */
int bcpnn_recall_load(bcpnn_recall* r, const float* w, const float* bj, const float* epsc, const float* dsup,
                      const int8_t* spikes_tm3, const int8_t* spikes_tm2, const int8_t* spikes_tm1);

/* Per-replicate stimulus: lgidx[R*H] (MCU index per HCU, anything else = no
   input; lginp = log(1+eps) / log(0+eps) as ProcExtGen computes it) and
   wmask[R*H]. */
int bcpnn_recall_set_cues(bcpnn_recall* r, const int32_t* lgidx, float eps, const float* wmask);

/* Ticks first .. first+n-1.  Spikes of ticks count_first .. count_last are
   added to the per-replicate MCU counters (ProcCheck's counting window).
   Asynchronous on the engine's stream. */
int bcpnn_recall_run(bcpnn_recall* r, int32_t first, int32_t n_ticks, int32_t count_first, int32_t count_last);

/* Zero the counters. */
int bcpnn_recall_clear_counts(bcpnn_recall* r);

/* Rows row0 .. row0+n_rows-1 (replicates) of a per-replicate array, after
   the last tick run: "dsup" and "epsc" (float [N] per row), "spike" (int8
   [N], the last tick), "counts" (uint8 [N]).  Synchronises. */
int bcpnn_recall_read(bcpnn_recall* r, const char* name, int32_t row0, int32_t n_rows, void* host, size_t bytes);

/* Overwrite rows of "dsup", "epsc" (float) or of the spike history
   "spike_tm3" / "spike_tm2" / "spike_tm1" (int8, relative to the next tick to
   run). */
int bcpnn_recall_write(bcpnn_recall* r, const char* name, int32_t row0, int32_t n_rows, const void* host,
                       size_t bytes);

int bcpnn_recall_get_stream(const bcpnn_recall* r, void** stream);

/* In-place timing of the contraction kernel: with timing on, bcpnn_recall_run
   records a CUDA event pair around every contraction launch on the engine's
   stream -- each launch timed where it runs, beside the population update of
   the same tick -- and adds the elapsed times up when the run synchronises.
   bcpnn_recall_timing(r, on) switches it and clears the sums;
   bcpnn_recall_contraction_time reads the summed milliseconds and launches. */
int bcpnn_recall_timing(bcpnn_recall* r, int32_t on);
int bcpnn_recall_contraction_time(const bcpnn_recall* r, double* total_ms, uint64_t* n_launches);
int bcpnn_recall_launches(const bcpnn_recall* r, uint64_t* out);
const char* bcpnn_recall_last_error(const bcpnn_recall* r);

#ifdef __cplusplus
}
#endif

#endif
