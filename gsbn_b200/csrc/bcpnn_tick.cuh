/*
 * bcpnn_tick.cuh -- the tick of the plain FP32 path: one CTA per (population,
 * destination HCU), all state that only this HCU uses kept in shared memory
 * for the whole launch.
 *
 * What one tick of gsbn does for destination HCU h (ProcUpdLazy.cpp:88-124):
 *   population update      Pop.cpp:229-323   support, softmax/WTA, spikes
 *   external spike replay  Pop.cpp:389-409
 *   per incoming projection:
 *     j-traces and bias    Proj.cpp:310-363
 *     active rows          Proj.cpp:365-479, 667-720 (ordered epsc sum)
 *     active columns       Proj.cpp:481-536, 722-760
 *     delay queue          Proj.cpp:621-630, 645-664 (next tick's rows)
 * reads, from other HCUs, only (a) the previous tick's presynaptic spikes and
 * (b) the population's MCU-0 support terms, which seed every HCU's softmax
 * maximum (Pop.cpp:270).  So the per-MCU traces, the delay queue and the
 * active-row list of h live in shared memory; only spikes, the MCU-0 seed
 * values, cells, row traces and logs go through global memory per tick, and
 * everything is written back to the gsbn-layout arrays at the end of the
 * launch.
 *
 * Launch forms (same code):
 *   - persistent: one cooperative launch per run, a bounded grid barrier
 *     between ticks (tick t+1 reads what other CTAs published in tick t);
 *   - one launch per tick when the grid cannot be co-resident.
 * The next tick's first row chunk (its traces, cells and decay-table entries)
 * is staged into shared memory before the barrier, so its loads overlap the
 * wait.
 */

#include "bcpnn_device.cuh"

/* This header is compiled once per CTA size: the includer defines
   BCPNN_TICK_THREADS (512 or 256) and BCPNN_TICK_NS, the namespace the
   variant lives in.  512 threads suit large HCUs (one CTA per SM); 256
   threads let two CTAs share an SM, for batches of small HCUs. */
#ifndef BCPNN_TICK_THREADS
#define BCPNN_TICK_THREADS 512
#define BCPNN_TICK_NS t512
#endif

namespace bcpnn {
namespace BCPNN_TICK_NS {

constexpr int kBlock = BCPNN_TICK_THREADS;
constexpr int kWarps = kBlock / 32;
constexpr int kRowChunkCells = kBlock; /* row cells staged per chunk (one per thread) */
constexpr int kMinBlocks = kBlock <= 256 ? 2 : 1;

/* The CTA is split in two warp groups that run concurrently inside a tick:
   group A (warps 0-7): support, softmax, spikes, j-traces, active rows;
   group B (warps 8-15): delay queue (next tick's rows), then, once A has
   published the spike list, the column updates.  A column cell whose row is
   also active this tick must see the row update first: B leaves those cells,
   and all threads do them after the groups join. */
constexpr int kGroup = kBlock / 2;
constexpr int kGroupWarps = kGroup / 32;
constexpr int kBarA = 1, kBarB = 2, kBarSpikes = 3, kBarRows = 4;
constexpr int kDQ = 4; /* delay-queue chunks of kGroup slots compacted together */

__device__ __forceinline__ void group_sync(int id) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(kGroup) : "memory");
}

/* phase probe (BCPNN_PHASE_PROBE): the recording thread adds the cycles since
   its previous mark to slot `slot` of its CTA's row of g_phase_probe, slot
   0-15 for group A's thread and 16 + slot for group B's */
#ifdef BCPNN_PHASE_PROBE
#define PROBE_DECL long long probe_t = clock64(); const bool probe_on = (threadIdx.x % kGroup) == 0
#define PROBE(slot)                                                                 \
  do {                                                                              \
    if (probe_on) {                                                                 \
      const long long t_ = clock64();                                               \
      g_probe_smem[(threadIdx.x < kGroup ? 0 : 16) + (slot)] += (unsigned long long)(t_ - probe_t); \
      probe_t = t_;                                                                 \
    }                                                                               \
  } while (0)
#define PROBE_TICK()                                                                \
  do {                                                                              \
    if (threadIdx.x == 0) g_probe_smem[kProbeTicks] += 1;                           \
  } while (0)
#define PROBE_BEGIN()                                                               \
  do {                                                                              \
    if (threadIdx.x < kProbeSlots) g_probe_smem[threadIdx.x] = 0;                   \
    __syncthreads();                                                                \
  } while (0)
#define PROBE_FLUSH()                                                               \
  do {                                                                              \
    __syncthreads();                                                                \
    if (threadIdx.x < kProbeSlots && blockIdx.x < kProbeCtas)                       \
      atomicAdd(&g_phase_probe[blockIdx.x * kProbeSlots + threadIdx.x], g_probe_smem[threadIdx.x]); \
  } while (0)
#else
#define PROBE_DECL do {} while (0)
#define PROBE(slot) do {} while (0)
#define PROBE_TICK() do {} while (0)
#define PROBE_BEGIN() do {} while (0)
#define PROBE_FLUSH() do {} while (0)
#endif

/* ordered compaction within a warp group (see block_prefix) */
__device__ __forceinline__ int group_prefix(bool flag, int gtid, int bar_id, int* s_warp, int* s_total, int* total) {
  int lane = gtid & 31, warp = gtid >> 5;
  unsigned m = __ballot_sync(0xffffffffu, flag);
  int before = __popc(m & ((1u << lane) - 1u));
  if (lane == 0) s_warp[warp] = __popc(m);
  group_sync(bar_id);
  if (warp == 0) {
    int c = lane < kGroupWarps ? s_warp[lane] : 0;
    int incl = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane < kGroupWarps) s_warp[lane] = incl - c;
    if (lane == 31) *s_total = incl;
  }
  group_sync(bar_id);
  int base = s_warp[warp];
  *total = *s_total;
  __syncwarp();
  return base + before;
}

__device__ __forceinline__ float group_max(float v, int gtid, int bar_id, float* s_red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    float w = __shfl_xor_sync(0xffffffffu, v, o);
    v = (w > v) ? w : v;
  }
  int lane = gtid & 31, warp = gtid >> 5;
  if (lane == 0) s_red[warp] = v;
  group_sync(bar_id);
  float r = s_red[lane % kGroupWarps];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    float w = __shfl_xor_sync(0xffffffffu, r, o);
    r = (w > r) ? w : r;
  }
  return r;
}

/* shared-memory layout of a CTA, in 32-bit words from the dynamic base;
   float4 arrays first (16-byte alignment) */
struct TickLayout {
  int stg_rtr, stg_rA, stg_rB;   /* [rows] float4: row traces (pi,ei,zi), table parts 2,3   */
  int stg_cv, stg_cA, stg_cB;    /* [kRowChunkCells] float4: cell, table parts 0,1          */
  int stg_rR, stg_cR;            /* [rows] / [kRowChunkCells] 2 x double2: divisor reciprocals */
  int stg_row, stg_ti;           /* [rows] int                                             */
  int stg_tv, stg_wv;            /* [kRowChunkCells] int / float                           */
  int w_dsup, w_act, w_spkl, w_pi, w_w, w_lg;
  int w_spkp;                    /* [2][M] int: spike lists by tick parity (deferred columns) */
  int w_spk, w_skip;             /* bytes                                                  */
  int st_dsup, st_act, st_cnt;
  int st_q[kMaxIn];              /* per incoming projection (QView) */
  int total;
};

/* words of one projection's resident block: pj ej zj epsc bj [M]; ii di qi
   [C]; list [2][C]; bits [2][ceil(C/32)]; nlist [2] */
__host__ __device__ inline int qblock_words(int M, int C) { return 5 * M + 5 * C + 2 * ((C + 31) / 32) + 2; }

__host__ __device__ inline int row_chunk_rows(int M) {
  int r = kRowChunkCells / M;
  if (r < 1) r = 1;
  return r;
}

__host__ __device__ inline void tick_layout(int M, int n_in, const int* C, TickLayout& L) {
  const int rows = (row_chunk_rows(M) + 3) & ~3; /* rows of one chunk, padded to 16 bytes */
  int o = 0;
  L.stg_rtr = o; o += 4 * rows;
  L.stg_rA = o; o += 4 * rows;
  L.stg_rB = o; o += 4 * rows;
  L.stg_cv = o; o += 4 * kRowChunkCells;
  L.stg_cA = o; o += 4 * kRowChunkCells;
  L.stg_cB = o; o += 4 * kRowChunkCells;
  L.stg_rR = o; o += 8 * rows;
  L.stg_cR = o; o += 8 * kRowChunkCells;
  L.stg_row = o; o += rows;
  L.stg_ti = o; o += rows;
  L.stg_tv = o; o += kRowChunkCells;
  L.stg_wv = o; o += kRowChunkCells;
  L.w_dsup = o; o += M;
  L.w_lg = o; o += M;
  L.w_act = o; o += M;
  L.w_spkl = o; o += M;
  L.w_pi = o; o += rows;
  L.w_w = o; o += kRowChunkCells;
  L.w_spkp = o; o += 2 * M;
  L.w_spk = o; o += (M + 3) / 4;
  L.w_skip = o; o += (kRowChunkCells + 3) / 4;
  L.st_dsup = o; o += M;
  L.st_act = o; o += M;
  L.st_cnt = o; o += M;
  for (int q = 0; q < kMaxIn; ++q) {
    L.st_q[q] = o;
    if (q < n_in) o += qblock_words(M, C[q]);
  }
  L.total = o;
}

/* views of projection q's resident block; list/bits/nlist by tick parity */
struct QView {
  float *pj, *ej, *zj, *epsc, *bj;
  int *ii, *di, *qi;
  int* list;      /* [2][C] */
  uint32_t* bits; /* [2][W] */
  int* nlist;     /* [2] */
  int W;
};

__device__ __forceinline__ QView qview(float* sm, const TickLayout& L, int q, int M, int C) {
  QView v;
  float* b = sm + L.st_q[q];
  v.pj = b;
  v.ej = b + M;
  v.zj = b + 2 * M;
  v.epsc = b + 3 * M;
  v.bj = b + 4 * M;
  int* ib = (int*)(b + 5 * M);
  v.ii = ib;
  v.di = ib + C;
  v.qi = ib + 2 * C;
  v.list = ib + 3 * C;
  v.W = (C + 31) / 32;
  v.bits = (uint32_t*)(ib + 5 * C);
  v.nlist = ib + 5 * C + 2 * v.W;
  return v;
}

/* Stage rows [base, base+nr) of `list` of projection J for a tick at
   `simstep`: row traces, cells of the chunk, and the decay-table entries for
   their elapsed ticks.  Threads gtid, gtid+gsize, ... of a group of gsize. */
__device__ __forceinline__ void stage_rows(const ProjDev& J, const int* list, int base, int nr, int M, int simstep,
                                           const float4* tab, const double2* rtab, int tlen, float* sm,
                                           const TickLayout& L, int gtid, int gsize) {
  float4* rtr = (float4*)(sm + L.stg_rtr);
  float4* rA = (float4*)(sm + L.stg_rA);
  float4* rB = (float4*)(sm + L.stg_rB);
  float4* cv = (float4*)(sm + L.stg_cv);
  float4* cA = (float4*)(sm + L.stg_cA);
  float4* cB = (float4*)(sm + L.stg_cB);
  double2* rR = (double2*)(sm + L.stg_rR);
  double2* cR = (double2*)(sm + L.stg_cR);
  int* srow = (int*)(sm + L.stg_row);
  int* sti = (int*)(sm + L.stg_ti);
  int* stv = (int*)(sm + L.stg_tv);
  float* swv = sm + L.stg_wv;
  for (int t = gtid; t < nr; t += gsize) {
    int r = list[base + t];
    int ti = J.ti[r];
    float pi = J.pi[r], ei = J.ei[r], zi = J.zi[r];
    int pdt = simstep - ti;
    float4 A = make_float4(0, 0, 0, 0), B = A;
    double2 R0 = make_double2(0, 0), R1 = R0;
    if (pdt > 0 && pdt < tlen) {
      A = tab[(size_t)pdt * 4 + 2];
      B = tab[(size_t)pdt * 4 + 3];
      R0 = rtab[(size_t)pdt * 4 + 2];
      R1 = rtab[(size_t)pdt * 4 + 3];
    }
    srow[t] = r;
    sti[t] = ti;
    rtr[t] = make_float4(pi, ei, zi, 0.0f);
    rA[t] = A;
    rB[t] = B;
    rR[2 * t] = R0;
    rR[2 * t + 1] = R1;
  }
  for (int c = gtid; c < nr * M; c += gsize) {
    int rr = c / M;
    int j = c - rr * M;
    size_t index = (size_t)list[base + rr] * M + j;
    int tv = __ldcg(J.tij + index); /* cells and tij: other CTAs write them (deferred columns) */
    float4 c4 = __ldcg(J.cell + index);
    float wv = J.wij[index];
    int pdt = simstep - tv;
    float4 A = make_float4(0, 0, 0, 0), B = A;
    double2 R0 = make_double2(0, 0), R1 = R0;
    if (pdt > 0 && pdt < tlen) {
      A = tab[(size_t)pdt * 4 + 0];
      B = tab[(size_t)pdt * 4 + 1];
      R0 = rtab[(size_t)pdt * 4 + 0];
      R1 = rtab[(size_t)pdt * 4 + 1];
    }
    stv[c] = tv;
    cv[c] = c4;
    swv[c] = wv;
    cA[c] = A;
    cB[c] = B;
    cR[2 * c] = R0;
    cR[2 * c + 1] = R1;
  }
}

__device__ __forceinline__ bool tid_is_zero() { return threadIdx.x == 0; }

__device__ __forceinline__ unsigned long long globaltimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void atomic_add_release(unsigned int* p, unsigned int v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ unsigned int load_acquire(const unsigned int* p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

/* Grid-wide barrier of a cooperative launch: arrival counter `bar` (zero at
   launch) must reach `target`.  The wait is bounded: after kBarrierNs, or as
   soon as another CTA has set an error word, it gives up, sets kErrBarrier
   and returns false, and every CTA leaves its tick loop. */
constexpr unsigned long long kBarrierNs = 2000000000ull;

__device__ __forceinline__ bool grid_sync(unsigned int* bar, unsigned int target, int* err, int* s_ok,
                                          unsigned long long limit_ns = kBarrierNs) {
  __syncthreads();
  if (threadIdx.x == 0) {
    atomic_add_release(bar, 1u);
    unsigned long long t0 = globaltimer_ns();
    int ok = 1;
    while (load_acquire(bar) < target) {
      if (*(volatile int*)err) {
        ok = 0;
        break;
      }
      if (globaltimer_ns() - t0 > limit_ns) {
        atomicOr(err, kErrBarrier);
        ok = 0;
        break;
      }
      __nanosleep(20);
    }
    *s_ok = ok;
  }
  __syncthreads();
  return *s_ok != 0;
}

__device__ __forceinline__ unsigned long long load_relaxed_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ unsigned long long load_acquire_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void store_relaxed_u64(unsigned long long* p, unsigned long long v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

/* The two halves of grid_sync, for a CTA that has work to do between its
   arrival and the point where it needs the others' arrivals: grid_arrive
   after a __syncthreads (the release covers every write of the CTA before
   it), grid_wait before the next reads of other CTAs' data.  grid_wait with
   a seed slot (NetDev::seed64) also fetches the population's softmax seed
   for the tick it opens: the barrier thread loads the slot beside every poll
   of the arrival counter, so the value is usually in hand when the barrier
   completes; a slot whose tag is not `tag` yet is read again after the
   completing acquire, which orders it after the publisher's store (made
   before the publisher's release arrival).  *s_seed gets the float. */
__device__ __forceinline__ void grid_arrive(unsigned int* bar) {
  if (threadIdx.x == 0) atomic_add_release(bar, 1u);
}

__device__ __forceinline__ bool grid_wait(unsigned int* bar, unsigned int target, int* err, int* s_ok,
                                          const unsigned long long* seed, unsigned int tag, float* s_seed) {
  if (threadIdx.x == 0) {
    unsigned long long t0 = globaltimer_ns();
    int ok = 1;
    unsigned long long sv = 0;
    for (;;) {
      if (seed) sv = load_relaxed_u64(seed);
      if (load_acquire(bar) >= target) break;
      if (*(volatile int*)err) {
        ok = 0;
        break;
      }
      if (globaltimer_ns() - t0 > kBarrierNs) {
        atomicOr(err, kErrBarrier);
        ok = 0;
        break;
      }
      __nanosleep(20);
    }
    if (ok && seed) {
      if ((unsigned int)(sv >> 32) != tag) sv = load_acquire_u64(seed);
      if ((unsigned int)(sv >> 32) != tag) {
        atomicOr(err, kErrSeed);
        ok = 0;
      }
      *s_seed = __uint_as_float((unsigned int)sv);
    }
    *s_ok = ok;
  }
  __syncthreads();
  return *s_ok != 0;
}

/* Failure-detection self-test: every CTA enters grid_sync with a target one
   arrival above the grid size, which nothing provides, so each wait runs out
   after limit_ns, sets kErrBarrier in *err and returns. */
__global__ void barrier_probe_kernel(unsigned int* bar, int* err, unsigned long long limit_ns) {
  __shared__ int s_ok;
  grid_sync(bar, gridDim.x + 1u, err, &s_ok, limit_ns);
}

/* Deferred column updates, Proj.cpp:481-536, of the MCUs that spiked in the
   tick at `simstep`.  Units [beg, *tail) of the ring half go round robin to
   the CTAs of the grid (unit b + i*G to CTA b); the calling group (kGroup
   threads, named barrier bar_id) does this CTA's units, kHelpUnits at a time,
   then signals each unit's owner CTA with a release add on col_done[owner].
   The descriptors of the first units are loaded beside the tail count (one
   round trip for both; a descriptor beyond the tail is never used), and the
   projection and decay constants come from the CTA's shared copies when the
   unit's projection is one of them.  A unit's slots were published by their
   owner after its row updates of that tick, so every cell sees the row update
   first, as in gsbn (rows, then columns). */
constexpr int kCellsPerUnit = kColUnit / kGroup;          /* cells of one unit per thread */
constexpr int kHelpUnits = kCellsPerUnit >= 2 ? 1 : 2;    /* units per pass */

template <int kF64>
__device__ __forceinline__ void help_columns(const NetDev* __restrict__ net, const RunParams* __restrict__ rp,
                                             const int4* __restrict__ ring, unsigned beg,
                                             const unsigned int* tail, int simstep, unsigned int* col_done,
                                             int gtid, int bar_id, unsigned int* s_end, const int* s_inp,
                                             const ProjDev* s_proj, const TabRef* s_tab, int n_in) {
  const unsigned G = gridDim.x;
  const unsigned cap = (unsigned)net->col_cap;
  const float prn = rp->prn;
  PROBE_DECL;
  int4 d[kHelpUnits];
#pragma unroll
  for (int u = 0; u < kHelpUnits; ++u) d[u] = __ldcg(ring + (beg + blockIdx.x + (unsigned)u * G) % cap);
  if (gtid == 0) *s_end = __ldcg(tail);
  group_sync(bar_id);
  const unsigned n = *s_end - beg;
  for (unsigned u0 = blockIdx.x; u0 < n; u0 += kHelpUnits * G) {
    if (u0 != blockIdx.x) {
#pragma unroll
      for (int u = 0; u < kHelpUnits; ++u)
        if (u0 + u * G < n) d[u] = __ldcg(ring + (beg + u0 + (unsigned)u * G) % cap);
    }
    size_t index[kHelpUnits][kCellsPerUnit];
    int tv[kHelpUnits][kCellsPerUnit];
    float4 cv[kHelpUnits][kCellsPerUnit];
    bool ok[kHelpUnits][kCellsPerUnit];
    const ProjDev* Jp[kHelpUnits];
    const TabRef* Tp[kHelpUnits];
#pragma unroll
    for (int u = 0; u < kHelpUnits; ++u) {
      const bool valid = u0 + u * G < n;
      Jp[u] = nullptr;
      Tp[u] = nullptr;
      if (valid) {
        for (int q = 0; q < n_in; ++q)
          if (s_inp[q] == d[u].y) {
            Jp[u] = &s_proj[q];
            Tp[u] = &s_tab[q];
          }
        if (!Jp[u]) {
          Jp[u] = &net->projs[d[u].y];
          Tp[u] = &rp->tabs[d[u].y];
        }
      }
#pragma unroll
      for (int c = 0; c < kCellsPerUnit; ++c) {
        const int r = c * kGroup + gtid;
        ok[u][c] = false;
        if (valid && r < (d[u].w >> 16)) {
          const ProjDev& J = *Jp[u];
          const int row = d[u].z + r;
          index[u][c] = (size_t)row * J.M + (d[u].w & 0xffff);
          ok[u][c] = J.ii[row] >= 0;
          tv[u][c] = __ldcg(J.tij + index[u][c]);
          cv[u][c] = __ldcg(J.cell + index[u][c]);
        }
      }
    }
    PROBE(3); /* B slot 19 */
    float4 tA[kHelpUnits][kCellsPerUnit], tB[kHelpUnits][kCellsPerUnit];
    double2 tR0[kHelpUnits][kCellsPerUnit], tR1[kHelpUnits][kCellsPerUnit];
#pragma unroll
    for (int u = 0; u < kHelpUnits; ++u)
#pragma unroll
      for (int c = 0; c < kCellsPerUnit; ++c) {
        if (!ok[u][c]) continue;
        const TabRef& T = *Tp[u];
        const int pdt = simstep - tv[u][c];
        if (pdt > 0 && pdt < T.len) {
          tA[u][c] = T.tab[(size_t)pdt * 4 + 0];
          tB[u][c] = T.tab[(size_t)pdt * 4 + 1];
          tR0[u][c] = T.rtab[(size_t)pdt * 4 + 0];
          tR1[u][c] = T.rtab[(size_t)pdt * 4 + 1];
        }
      }
#pragma unroll
    for (int u = 0; u < kHelpUnits; ++u)
#pragma unroll
      for (int c = 0; c < kCellsPerUnit; ++c) {
        if (!ok[u][c]) continue;
        const ProjDev& J = *Jp[u];
        const int pdt = simstep - tv[u][c];
        float4 c4 = cv[u][c];
        if (pdt <= 0) {
          c4.w += J.kftj;
        } else {
          float4 A = tA[u][c], B = tB[u][c];
          double2 R0 = tR0[u][c], R1 = tR1[u][c];
          if (pdt >= Tp[u]->len) {
            const Coef k = make_coef(J.taupdt * prn, J.ke, J.kzi, J.kzj, kF64);
            if (kF64)
              table_pair(k.kp, k.ke, k.kzi, k.kzj, pdt, 0, A, B, 1);
            else
              cell_factors(k.kp, k.ke, k.kzi, k.kzj, pdt, A, B);
            recip_part(A, B, 0, R0, R1);
          }
          c4 = cell_step_nl(c4, Tp[u], A, B, R0, R1);
          c4.w = c4.w + J.kftj;
        }
        J.cell[index[u][c]] = c4;
        J.tij[index[u][c]] = simstep;
      }
    PROBE(4); /* B slot 20 */
    group_sync(bar_id);
    PROBE(5); /* B slot 21 */
    if (gtid == 0)
#pragma unroll
      for (int u = 0; u < kHelpUnits; ++u)
        if (u0 + u * G < n) atomic_add_release(&col_done[d[u].x], 1u);
  }
}

/* Ticks it0 .. it0+n_ticks-1 of the run for this CTA's (population, HCU). */
/* kF64: the trace-decay form, fixed at compile time so the default
   instance carries no trace of the other (0: gsbn's closed form in float,
   1: FP64-built propagators, see fp64_entry).  kDefer: column updates
   deferred and spread over the grid (the persistent launch with its unit
   ring) or done by the CTA itself in the tick (one launch per tick); each
   instance holds only its own form. */
template <int kF64, int kDefer>
__global__ void __launch_bounds__(kBlock, kMinBlocks) tick_kernel(const NetDev* __restrict__ net_g,
                                                         const RunParams* __restrict__ rp_g, int it0, int n_ticks,
                                                         unsigned int* bar) {
  extern __shared__ __align__(16) float sm[];
  /* the network descriptor and the run's parameters, read every tick: shared
     copies, so that no read of them waits on an L1 miss behind the cell
     traffic of the tick */
  __shared__ NetDev s_net;
  __shared__ RunParams s_rp;
  if (threadIdx.x == 0) {
    s_net = *net_g;
    s_rp = *rp_g;
  }
  __syncthreads();
  const NetDev* __restrict__ net = &s_net;
  const RunParams* __restrict__ rp = &s_rp;
  __shared__ int s_warpA[kGroupWarps];
  __shared__ float s_red[kGroupWarps];
  __shared__ int s_totalA;
  __shared__ float s_dsup0;
  __shared__ float s_wm;
  __shared__ float s_vsum;
  __shared__ int s_flag9;
  __shared__ int s_nspk;
  __shared__ int s_ok;
  __shared__ unsigned int s_hend, s_upos, s_exp_total, s_last_end[2];
  /* cell updates of the launch, added to NetDev::counters once at its end */
  __shared__ unsigned long long s_rows_acc, s_cols_acc;
  __shared__ int s_nspkp[2];
  __shared__ int s_dq[kDQ * kGroupWarps];

  /* this CTA's population and incoming projections, their decay tables and
     the spike buffers it feeds, copied to shared memory once per launch: every
     tick reads them many times, in chains of dependent loads */
  __shared__ PopDev s_pop;
  __shared__ ProjDev s_proj[kMaxIn];
  __shared__ TabRef s_tab[kMaxIn];
  __shared__ int s_inp[kMaxIn];
  __shared__ int8_t* s_siout[kMaxIn][2];

  const int P = net->cta_pop[blockIdx.x];
  const int h = net->cta_hcu[blockIdx.x];
  if (threadIdx.x == 0) s_pop = net->pops[P];
  __syncthreads();
  if (threadIdx.x < kMaxIn && threadIdx.x < s_pop.n_in) {
    const int p = s_pop.in_proj[threadIdx.x];
    s_inp[threadIdx.x] = p;
    s_proj[threadIdx.x] = net->projs[p];
    s_tab[threadIdx.x] = rp->tabs[p];
  }
  if (threadIdx.x < kMaxIn && threadIdx.x < s_pop.n_out) {
    const ProjDev& O = net->projs[s_pop.out_proj[threadIdx.x]];
    s_siout[threadIdx.x][0] = O.si[0];
    s_siout[threadIdx.x][1] = O.si[1];
  }
  __syncthreads();
  const PopDev& pop = s_pop;
  const int M = pop.M, n = pop.n;
  const int n_in = pop.n_in;
  const int tid = threadIdx.x;
  const bool groupA = tid < kGroup;
  const int gtid = groupA ? tid : tid - kGroup;
  const float prn = rp->prn;
  /* deferred columns (persistent launch): bar[1..2] unit counters by tick
     parity, bar[4 + cta] units done for each CTA */
  constexpr int defer = kDefer;
  unsigned int* const col_tail = bar + 1;
  unsigned int* const col_done = bar + 4;

  /* the shared-memory layout lives in shared memory itself: indexed by
     projection at run time, a register copy would sit in local memory, whose
     per-thread frames (x 512 threads) do not fit in L1 next to this kernel's
     shared memory, and every read would be an L2 round trip */
  __shared__ TickLayout s_L;
  __shared__ int s_C[kMaxIn];
  if (tid_is_zero()) {
    int c[kMaxIn];
#pragma unroll
    for (int q = 0; q < kMaxIn; ++q) c[q] = q < n_in ? s_proj[q].C : 0;
#pragma unroll
    for (int q = 0; q < kMaxIn; ++q) s_C[q] = c[q];
    tick_layout(M, n_in, c, s_L);
  }
  __syncthreads();
  const TickLayout& L = s_L;
  const int* Cq = s_C;

  float* w_dsup = sm + L.w_dsup;
  float* w_act = sm + L.w_act;
  int* w_spkl = (int*)(sm + L.w_spkl);
  float* w_pi = sm + L.w_pi;
  float* w_w = sm + L.w_w;
  int8_t* w_spk = (int8_t*)(sm + L.w_spk);
  int* w_spkp = (int*)(sm + L.w_spkp);
  int8_t* w_skip = (int8_t*)(sm + L.w_skip);
  float* w_lgc = sm + L.w_lg;
  float* st_dsup = sm + L.st_dsup;
  float* st_act = sm + L.st_act;
  int* st_cnt = (int*)(sm + L.st_cnt);

  /* ---- load the resident state (buffers written by the previous tick) ---- */
  const int cur0 = (rp->k0 + it0) & 1;
  {
    const int prev0 = cur0 ^ 1;
    for (int j = tid; j < M; j += kBlock) {
      int idx = h * M + j;
      st_dsup[j] = pop.dsup[prev0][idx];
      st_act[j] = pop.act[idx];
      st_cnt[j] = pop.counter[idx];
      w_spk[j] = pop.spike[idx];
    }
    for (int q = 0; q < n_in; ++q) {
      const ProjDev& J = s_proj[q];
      QView V = qview(sm, L, q, M, J.C);
      const size_t eoff = (size_t)J.proj_in_pop * n;
      for (int j = tid; j < M; j += kBlock) {
        int idx = h * M + j;
        V.pj[j] = J.pj[idx];
        V.ej[j] = J.ej[idx];
        V.zj[j] = J.zj[idx];
        V.epsc[j] = pop.epsc[prev0][eoff + idx];
        V.bj[j] = pop.bj[prev0][eoff + idx];
      }
      for (int s = tid; s < J.C; s += kBlock) {
        int r = h * J.C + s;
        V.ii[s] = J.ii[r];
        V.di[s] = J.di[r];
        V.qi[s] = J.qi[r];
        V.list[cur0 * J.C + s] = J.list[r];
      }
      for (int w = tid; w < V.W; w += kBlock) V.bits[cur0 * V.W + w] = 0u;
      if (tid == 0) V.nlist[cur0] = J.list_cnt[h];
    }
    /* the run's stimulus of this HCU (constant within the launch) */
    for (int j = tid; j < M; j += kBlock) w_lgc[j] = rp->lginp[pop.mcu_start + h * M + j];
    if (tid == 0) {
      s_rows_acc = 0;
      s_cols_acc = 0;
      s_exp_total = 0;
      s_last_end[0] = s_last_end[1] = 0;
      s_nspkp[0] = s_nspkp[1] = 0;
      s_wm = rp->wmask[pop.hcu_start + h];
    }
  }
  __syncthreads();
  for (int q = 0; q < n_in; ++q) {
    const ProjDev& J = s_proj[q];
    QView V = qview(sm, L, q, M, J.C);
    for (int e = tid; e < V.nlist[cur0]; e += kBlock) {
      int s = V.list[cur0 * J.C + e] - h * J.C;
      atomicOr(&V.bits[cur0 * V.W + (s >> 5)], 1u << (s & 31));
    }
  }
  if (n_in > 0) {
    const ProjDev& J = s_proj[0];
    QView V = qview(sm, L, 0, M, J.C);
    int nr = V.nlist[cur0] < row_chunk_rows(M) ? V.nlist[cur0] : row_chunk_rows(M);
    stage_rows(J, V.list + cur0 * J.C, 0, nr, M, rp->simstep0 + it0, s_tab[0].tab, s_tab[0].rtab, s_tab[0].len, sm,
               L, tid, kBlock);
  }

  PROBE_BEGIN();
  PROBE_DECL;
  for (int it = it0; it < it0 + n_ticks; ++it) {
    if (it > it0) {
      /* this CTA arrived at the end of the previous tick (grid_arrive) */
      if (!grid_wait(bar, (unsigned int)(it - it0) * gridDim.x, net->err, &s_ok,
                     (defer && h != 0) ? net->seed64 + 2 * P + ((rp->serial0 + (unsigned int)(it - it0)) & 1u) : nullptr,
                     rp->serial0 + (unsigned int)(it - it0),
                     &s_dsup0))
        return;
    } else {
      __syncthreads();
    }
    PROBE(0);
    PROBE_TICK();
    const int simstep = rp->simstep0 + it;
    const int kk = rp->k0 + it;
    const int cur = kk & 1, prev = cur ^ 1, nxt = cur ^ 1;

    if (groupA) {
      /* ================= group A: population, j-traces, rows ============= */
      /* column units this CTA published up to the previous tick (group B adds
         this tick's only after the spike hand-over below) */
      const unsigned int exp_done = s_exp_total;
      /* population update, Pop.cpp:229-323 */
      const float* lginp = rp->lginp + pop.mcu_start;
      const float* wmask = rp->wmask + pop.hcu_start;
      for (int j = gtid; j < M; j += kGroup) {
        float wsup = 0.0f;
        for (int m = 0; m < pop.dim_proj; m++) {
          const float* b = sm + L.st_q[m];
          wsup += b[4 * M + j] + b[3 * M + j];   /* bj + epsc */
        }
        int idx = h * M + j;
        float noise = 0.0f;
        if (pop.snoise != 0.0f)
          noise = pop.snoise * dev_normal01(pop.rng_seed, pop.rng_pop, (uint32_t)simstep, (uint32_t)idx);
        float sup = pop.lgbias + pop.igain * w_lgc[j] + noise;
        sup += (pop.wgain * s_wm) * wsup;
        float d = st_dsup[j];
        w_dsup[j] = d + (sup - d) * pop.taumdt;
      }
      PROBE(1);
      /* the softmax max of every HCU is seeded with the population's first
         MCU (Pop.cpp:270), published by HCU 0's CTA in the previous tick */
      /* in a launch's first tick (or without the deferred-column form) from
         global memory; later the barrier brought it (grid_wait) */
      const int tseed = (M < kGroup) ? kGroup - 1 : 0;
      if (gtid == tseed && h != 0 && (it == it0 || !defer)) {
        float wsup = 0.0f;
        int offset = 0;
        for (int m = 0; m < pop.dim_proj; m++) {
          wsup += __ldcg(pop.bj[prev] + offset) + __ldcg(pop.epsc[prev] + offset);
          offset += n;
        }
        float noise = 0.0f;
        if (pop.snoise != 0.0f) noise = pop.snoise * dev_normal01(pop.rng_seed, pop.rng_pop, (uint32_t)simstep, 0u);
        float sup = pop.lgbias + pop.igain * lginp[0] + noise;
        sup += (pop.wgain * wmask[0]) * wsup;
        float d = __ldcg(pop.dsup[prev]);
        s_dsup0 = d + (sup - d) * pop.taumdt;
      }
      group_sync(kBarA);
      const float seed0 = (h == 0) ? w_dsup[0] : s_dsup0;
      float tmax = seed0;
      for (int j = gtid; j < M; j += kGroup) tmax = (w_dsup[j] > tmax) ? w_dsup[j] : tmax;
      const float maxdsup = group_max(tmax, gtid, kBarA, s_red);
      PROBE(10);
      const float maxact = bx_expf(pop.wtagain * maxdsup);
      for (int j = gtid; j < M; j += kGroup) {
        float a = bx_expf(pop.wtagain * (w_dsup[j] - maxdsup));
        if (maxact < 1.0f) a *= maxact;
        w_act[j] = a;
      }
      group_sync(kBarA);
      PROBE(11);
      if (gtid == 0) {
        /* serial, in MCU order (Pop.cpp:281-293) */
        float vsum = 0.0f;
        int m = 0;
        if (M >= 8) {
          float a[8];
#pragma unroll
          for (int u = 0; u < 8; ++u) a[u] = w_act[u];
          for (m = 8; m + 8 <= M; m += 8) {
            float b[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) b[u] = w_act[m + u];
#pragma unroll
            for (int u = 0; u < 8; ++u) vsum += a[u];
#pragma unroll
            for (int u = 0; u < 8; ++u) a[u] = b[u];
          }
#pragma unroll
          for (int u = 0; u < 8; ++u) vsum += a[u];
        }
        for (; m < M; m++) vsum += w_act[m];
        s_vsum = vsum;
      }
      group_sync(kBarA);
      PROBE(2);
      const float vsum = s_vsum;
      const float pr = net->poisson_hz * net->dt;
      for (int j = gtid; j < M; j += kGroup) {
        int idx = h * M + j;
        float a = w_act[j];
        if (vsum > 1.0f) a /= vsum;
        st_act[j] = a;
        st_dsup[j] = w_dsup[j];
        float u = bx_uniform01(pop.rng_seed, pop.rng_pop, (uint32_t)simstep, (uint32_t)idx);
        int8_t spk = (int8_t)(u < a * pop.maxfqdt);
        if (net->poisson_hz > 0.0f) {
          float up = bx_uniform01_poisson(pop.rng_seed, pop.rng_pop, (uint32_t)simstep, (uint32_t)idx);
          if (up < pr) spk = 1;
        }
        st_cnt[j] += spk;
        w_spk[j] = spk;
      }
      PROBE(12);
      if (h == 0 && gtid == 0) pop.dsup[cur][0] = w_dsup[0];
      /* external spike replay overrides the sampled spikes (Pop.cpp:389-409) */
      if (pop.ext) {
        group_sync(kBarA);
        for (int j = gtid; j < M; j += kGroup) w_spk[j] = 0;
        group_sync(kBarA);
        if (simstep >= pop.ext_t0 && simstep < pop.ext_t1) {
          int b0 = pop.ext_off[simstep - pop.ext_t0], b1 = pop.ext_off[simstep - pop.ext_t0 + 1];
          for (int e = b0 + gtid; e < b1; e += kGroup) {
            int v = pop.ext_idx[e];
            if (v >= h * M && v < h * M + M) w_spk[v - h * M] = 1;
          }
        }
      }
      group_sync(kBarA);
      /* ordered list of this HCU's spiking MCUs; publish */
      int nspk = 0;
      for (int base = 0; base < M; base += kGroup) {
        int j = base + gtid;
        bool f = (j < M) && w_spk[j] > 0;
        int tot;
        int pos = group_prefix(f, gtid, kBarA, s_warpA, &s_totalA, &tot);
        if (f) w_spkl[nspk + pos] = j;
        nspk += tot;
      }
      if (gtid == 0) s_nspk = nspk;
      {
        uint32_t* log = pop.spk_log + (size_t)it * pop.log_words;
        for (int j = gtid; j < M; j += kGroup) {
          int idx = h * M + j;
          int8_t sv = w_spk[j];
          if (sv) atomicOr(&log[idx >> 5], 1u << (idx & 31));
          for (int q = 0; q < pop.n_out; ++q) {
            int8_t* si = q < kMaxIn ? s_siout[q][cur] : net->projs[pop.out_proj[q]].si[cur];
            si[idx] = sv;
          }
        }
      }
      /* hand the spike list to group B */
      asm volatile("bar.arrive %0, %1;" ::"r"(kBarSpikes), "r"(kBlock) : "memory");
      PROBE(3);

      for (int q = 0; q < n_in; ++q) {
        const int p = s_inp[q];
        const ProjDev& J = s_proj[q];
        const int C = J.C;
        QView V = qview(sm, L, q, M, C);
        const float kp = J.taupdt * prn;
        const Coef k = make_coef(kp, J.ke, J.kzi, J.kzj, kF64);
        const float4* tab = s_tab[q].tab;
        const double2* rtab = s_tab[q].rtab;
        const int tlen = s_tab[q].len;
        const size_t eoff = (size_t)J.proj_in_pop * n;

        /* j-traces and bias, Proj.cpp:310-363 */
        for (int j = gtid; j < M; j += kGroup) {
          float pj = V.pj[j], ej = V.ej[j], zj = V.zj[j];
          float e = V.epsc[j];
          e *= (1 - J.kepsc);
          pj += (ej - pj) * kp;
          ej += (zj - ej) * k.ke;
          zj *= (1 - J.kzj);
          if (w_spk[j] > 0) zj += J.kftj;
          if (kp != 0.0f) V.bj[j] = J.bgain * bx_logf(pj + J.eps);
          V.pj[j] = pj;
          V.ej[j] = ej;
          V.zj[j] = zj;
          V.epsc[j] = e;
        }
        if (gtid == 0) {
          s_flag9 = 0;
          if (h == 0) pop.bj[cur][eoff] = V.bj[0];
        }
        group_sync(kBarA);
        PROBE(4);
        if (defer && q == 0 && it > it0) {
          /* the previous tick's columns of this HCU, done by the grid, must be
             in place before its rows; then refresh the staged cells they hit */
          if (gtid == 0) {
            const unsigned long long t0 = globaltimer_ns();
            while (load_acquire(col_done + blockIdx.x) < exp_done) {
              if (*(volatile int*)net->err) break;
              if (globaltimer_ns() - t0 > kBarrierNs) {
                atomicOr(net->err, kErrColumns);
                break;
              }
              __nanosleep(20);
            }
          }
          group_sync(kBarA);
          const int np = s_nspkp[prev];
          const int nr0 = V.nlist[cur] < row_chunk_rows(M) ? V.nlist[cur] : row_chunk_rows(M);
          if (np > 0 && nr0 > 0) {
            float4* fcv = (float4*)(sm + L.stg_cv);
            float4* fcA = (float4*)(sm + L.stg_cA);
            float4* fcB = (float4*)(sm + L.stg_cB);
            double2* fcR = (double2*)(sm + L.stg_cR);
            int* ftv = (int*)(sm + L.stg_tv);
            const int* frow = (const int*)(sm + L.stg_row);
            for (int c = gtid; c < nr0 * np; c += kGroup) {
              const int rr = c / np;
              const int j = w_spkp[prev * M + (c - rr * np)];
              const size_t index = (size_t)frow[rr] * M + j;
              const int tv = __ldcg(J.tij + index);
              const float4 c4 = __ldcg(J.cell + index);
              const int pdt = simstep - tv;
              float4 A = make_float4(0, 0, 0, 0), B = A;
              double2 R0 = make_double2(0, 0), R1 = R0;
              if (pdt > 0 && pdt < tlen) {
                A = tab[(size_t)pdt * 4 + 0];
                B = tab[(size_t)pdt * 4 + 1];
                R0 = rtab[(size_t)pdt * 4 + 0];
                R1 = rtab[(size_t)pdt * 4 + 1];
              }
              ftv[rr * M + j] = tv;
              fcv[rr * M + j] = c4;
              fcA[rr * M + j] = A;
              fcB[rr * M + j] = B;
              fcR[2 * (rr * M + j)] = R0;
              fcR[2 * (rr * M + j) + 1] = R1;
            }
            group_sync(kBarA);
          }
        }

        PROBE(5);
        /* row updates of this HCU's active rows, ascending, Proj.cpp:365-479 */
        const int nrow = V.nlist[cur];
        const int* list = V.list + cur * C;
        const int rch = row_chunk_rows(M);
        const float4* stg_rtr = (const float4*)(sm + L.stg_rtr);
        const float4* stg_rA = (const float4*)(sm + L.stg_rA);
        const float4* stg_rB = (const float4*)(sm + L.stg_rB);
        const float4* stg_cv = (const float4*)(sm + L.stg_cv);
        const float4* stg_cA = (const float4*)(sm + L.stg_cA);
        const float4* stg_cB = (const float4*)(sm + L.stg_cB);
        const double2* stg_rR = (const double2*)(sm + L.stg_rR);
        const double2* stg_cR = (const double2*)(sm + L.stg_cR);
        const int* stg_row = (const int*)(sm + L.stg_row);
        const int* stg_ti = (const int*)(sm + L.stg_ti);
        const int* stg_tv = (const int*)(sm + L.stg_tv);
        const float* stg_wv = sm + L.stg_wv;
        for (int base = 0; base < nrow; base += rch) {
          const int nr = (nrow - base) < rch ? (nrow - base) : rch;
          if (!(q == 0 && base == 0)) {
            stage_rows(J, list, base, nr, M, simstep, tab, rtab, tlen, sm, L, gtid, kGroup);
            group_sync(kBarA);
          }
          /* row traces (threads from the top of the group) beside the cell
             decays (from the bottom): a cell's decay does not need its row's
             new traces, only its weight does */
          for (int t = kGroup - 1 - gtid; t < nr; t += kGroup) {
            int r = stg_row[t];
            if (r == 9) s_flag9 = 1;
            float4 tr = stg_rtr[t];
            int pdt = simstep - stg_ti[t];
            if (pdt <= 0) {
              J.zi[r] = tr.z + J.kfti;
              J.ti[r] = simstep;
              w_pi[t] = tr.x;
            } else {
              float pi = tr.x, ei = tr.y, zi = tr.z;
              float4 A = stg_rA[t], B = stg_rB[t];
              double2 R0 = stg_rR[2 * t], R1 = stg_rR[2 * t + 1];
              if (pdt >= tlen) {
                load_entry(tab, tlen, k, pdt, 2, A, B);
                recip_part(A, B, 2, R0, R1);
              }
              {
                const float4 rt = row_step_nl(make_float4(pi, ei, zi, 0.0f), &s_tab[q], A, B, R0, R1);
                pi = rt.x;
                ei = rt.y;
                zi = rt.z;
              }
              zi = zi + J.kfti;
              J.pi[r] = pi;
              J.ei[r] = ei;
              J.zi[r] = zi;
              J.ti[r] = simstep;
              w_pi[t] = pi;
            }
          }
          for (int c = gtid; c < nr * M; c += kGroup) {
            int rr = c / M;
            int j = c - rr * M;
            size_t index = (size_t)stg_row[rr] * M + j;
            int pdt = simstep - stg_tv[c];
            float4 cv = stg_cv[c];
            if (pdt <= 0) {
              cv.z += J.kfti;
              J.cell[index] = cv;
              J.tij[index] = simstep;
              w_skip[c] = 1;
            } else {
              float4 A = stg_cA[c], B = stg_cB[c];
              double2 R0 = stg_cR[2 * c], R1 = stg_cR[2 * c + 1];
              if (pdt >= tlen) {
                load_entry(tab, tlen, k, pdt, 0, A, B);
                recip_part(A, B, 0, R0, R1);
              }
              cv = cell_step_nl(cv, &s_tab[q], A, B, R0, R1);
              cv.z = cv.z + J.kfti;
              J.cell[index] = cv;
              J.tij[index] = simstep;
              w_w[c] = cv.x; /* the new pij, for the weight below */
              w_skip[c] = 0;
            }
          }
          group_sync(kBarA);
          /* weights of the decayed cells, Proj.cpp:458-462 */
          for (int c = gtid; c < nr * M; c += kGroup) {
            if (w_skip[c]) continue;
            int rr = c / M;
            int j = c - rr * M;
            float w;
            if (kp != 0.0f) {
              w = J.wgain * bx_logf((w_w[c] + J.eps2) / ((w_pi[rr] + J.eps) * (V.pj[j] + J.eps)));
              J.wij[(size_t)stg_row[rr] * M + j] = w;
            } else {
              w = stg_wv[c];
            }
            w_w[c] = w;
          }
          group_sync(kBarA);
          for (int j = gtid; j < M; j += kGroup) {
            float e = V.epsc[j];
            for (int rr = 0; rr < nr; ++rr)
              if (!w_skip[rr * M + j]) e += w_w[rr * M + j];
            V.epsc[j] = e;
          }
          group_sync(kBarA);
        }
        PROBE(6);
        if (gtid == 0) {
          if (h == 0) pop.epsc[cur][eoff] = V.epsc[0];
          /* debug flags of ProcSpkRec (ssi/ssj contain index 9) */
          uint32_t f = 0;
          if (s_flag9) f |= 1;
          if (h == 9 / M && 9 < n && w_spk[9 - h * M] > 0) f |= 2;
          if (f) atomicOr(&net->ss_log[(size_t)it * net->n_projs + p], f);
          s_rows_acc += (unsigned long long)nrow * M;
        }
      }
      /* HCU 0 publishes the next tick's softmax seed, dsup of MCU 0 after
         that tick's support step (NetDev::seed64): its terms are final now
         (the deferred columns leave epsc and bj alone), and this thread's
         barrier arrival releases the store */
      if (defer && h == 0 && gtid == 0 && it + 1 < it0 + n_ticks) {
        float wsup = 0.0f;
        for (int m = 0; m < pop.dim_proj; m++) {
          const float* b = sm + L.st_q[m];
          wsup += b[4 * M] + b[3 * M];   /* bj + epsc of MCU 0 */
        }
        float noise = 0.0f;
        if (pop.snoise != 0.0f) noise = pop.snoise * dev_normal01(pop.rng_seed, pop.rng_pop, (uint32_t)(simstep + 1), 0u);
        float sup = pop.lgbias + pop.igain * w_lgc[0] + noise;
        sup += (pop.wgain * s_wm) * wsup;
        const float d = st_dsup[0];
        const float next = d + (sup - d) * pop.taumdt;
        const unsigned int tag = rp->serial0 + (unsigned int)(it + 1 - it0);
        store_relaxed_u64(net->seed64 + 2 * P + (tag & 1u), ((unsigned long long)tag << 32) | __float_as_uint(next));
      }
      /* rows done: group B may now update column cells of active rows */
      if (!defer) asm volatile("bar.arrive %0, %1;" ::"r"(kBarRows), "r"(kBlock) : "memory");
      PROBE(7);
    } else {
      /* ================= group B: delay queue, columns =================== */
      /* the delay queue's first spike flags (first projection, first chunk of
         slots), loaded now so that their round trip overlaps the column work;
         one byte per chunk, packed in one register */
      uint32_t dq_pre = 0;
      if (n_in > 0) {
        const ProjDev& J0 = s_proj[0];
        const int* ii0 = qview(sm, L, 0, M, J0.C).ii;
        const int8_t* si0 = J0.si[prev];
#pragma unroll
        for (int u = 0; u < kDQ; ++u) {
          const int s = u * kGroup + gtid;
          if (s < J0.C) {
            const int src = ii0[s];
            if (src >= 0 && src < J0.Ns) dq_pre |= (uint32_t)(uint8_t)__ldcg(si0 + src) << (8 * u);
          }
        }
      }
      if (defer) {
        /* the grid's column units of the previous tick, this CTA's share */
        help_columns<kF64>(net, rp, net->col_ring + (size_t)prev * net->col_cap, s_last_end[prev], col_tail + prev,
                           simstep - 1, col_done, gtid, kBarB, &s_hend, s_inp, s_proj, s_tab, n_in);
        if (gtid == 0) s_last_end[prev] = s_hend;
      }
      PROBE(10);
      for (int q = 0; q < n_in; ++q) {
        const ProjDev& J = s_proj[q];
        const int C = J.C;
        QView V = qview(sm, L, q, M, C);
        /* delay queue of this HCU's slots and ordered compaction of the next
           tick's active rows, Proj.cpp:621-630, 645-664 */
        const int8_t* si = J.si[prev];
        int* nlist = V.list + nxt * C;
        uint32_t* nbits = V.bits + nxt * V.W;
        /* kDQ chunks of kGroup slots at a time: their spike flags are
           loaded together, then compacted with one shared-memory scan */
        const int lane = gtid & 31, warp = gtid >> 5;
        int cnt = 0;
        for (int s0 = 0; s0 < C; s0 += kDQ * kGroup) {
          int8_t sv[kDQ];
#pragma unroll
          for (int u = 0; u < kDQ; ++u) {
            const int s = s0 + u * kGroup + gtid;
            sv[u] = 0;
            if (q == 0 && s0 == 0) {
              sv[u] = (int8_t)(dq_pre >> (8 * u));
            } else if (s < C) {
              const int src = V.ii[s];
              if (src >= 0 && src < J.Ns) sv[u] = __ldcg(si + src);
            }
          }
          unsigned mb[kDQ];
#pragma unroll
          for (int u = 0; u < kDQ; ++u) {
            const int s = s0 + u * kGroup + gtid;
            bool act = false;
            if (s < C) {
              const int src = V.ii[s];
              if (src >= 0) {
                if (src >= J.Ns) {
                  atomicOr(net->err, kErrIndex);
                } else {
                  int qv = V.qi[s];
                  act = (qv & 0x01) != 0;
                  qv >>= 1;
                  if (sv[u] > 0) qv |= (0x01 << (V.di[s] - 1));
                  V.qi[s] = qv;
                }
              }
            }
            mb[u] = __ballot_sync(0xffffffffu, act);
            if (lane == 0) {
              s_dq[u * kGroupWarps + warp] = __popc(mb[u]);
              if (s < C) nbits[s >> 5] = mb[u];
            }
          }
          PROBE(1); /* B slot 17 */
          group_sync(kBarB);
          PROBE(2); /* B slot 18 */
          /* slots in ascending order: chunk by chunk, warp by warp, lane by lane */
          int run = 0;
#pragma unroll
          for (int u = 0; u < kDQ; ++u) {
            int before = 0, tot = 0;
            for (int w = 0; w < kGroupWarps; ++w) {
              const int c = s_dq[u * kGroupWarps + w];
              tot += c;
              before += (w < warp) ? c : 0;
            }
            if ((mb[u] >> lane) & 1u)
              nlist[cnt + run + before + __popc(mb[u] & ((1u << lane) - 1u))] = h * C + s0 + u * kGroup + gtid;
            run += tot;
          }
          cnt += run;
          group_sync(kBarB);
        }
        if (gtid == 0) V.nlist[nxt] = cnt;
      }
      PROBE(11);
      /* wait for group A's spike list */
      asm volatile("bar.sync %0, %1;" ::"r"(kBarSpikes), "r"(kBlock) : "memory");
      PROBE(12);
      const int nspk = s_nspk;
      if (defer) {
        /* publish this tick's column units; the grid does them next tick */
        for (int i = gtid; i < nspk; i += kGroup) w_spkp[cur * M + i] = w_spkl[i];
        auto parts = [&](int q) { return (Cq[q] + kColUnit - 1) / kColUnit; };
        int nunits = 0;
        for (int q = 0; q < n_in; ++q) nunits += nspk * parts(q);
        if (gtid == 0) {
          s_nspkp[cur] = nspk;
          if (nunits > 0) {
            s_upos = atomicAdd(col_tail + cur, (unsigned int)nunits);
            s_exp_total += (unsigned int)nunits;
            for (int q = 0; q < n_in; ++q) s_cols_acc += (unsigned long long)nspk * Cq[q];
          }
        }
        group_sync(kBarB);
        if (nunits > 0) {
          const unsigned int pos = s_upos, cap = (unsigned int)net->col_cap;
          int4* ring = net->col_ring + (size_t)cur * net->col_cap;
          for (int u = gtid; u < nunits; u += kGroup) {
            int q = 0, uu = u;
            while (uu >= nspk * parts(q)) {
              uu -= nspk * parts(q);
              ++q;
            }
            const int i = uu / parts(q), part = uu - i * parts(q);
            const int C = Cq[q];
            const int rows = min(kColUnit, C - part * kColUnit);
            ring[(pos + (unsigned int)u) % cap] =
                make_int4((int)blockIdx.x, s_inp[q], h * C + part * kColUnit, w_spkl[i] | (rows << 16));
          }
        }
      } else
      /* column updates of this HCU's spiking MCUs, Proj.cpp:481-536.  Pass
         0: slots whose row is not active this tick; pass 1, after group A's
         row updates: the cells of active rows.  One code site for both, loads
         of a batch issued before its compute. */
      for (int pass = 0; pass < 2; ++pass) {
        if (pass == 1) asm volatile("bar.sync %0, %1;" ::"r"(kBarRows), "r"(kBlock) : "memory");
        if (nspk == 0) continue;
        for (int q = 0; q < n_in; ++q) {
          const ProjDev& J = s_proj[q];
          const int C = J.C;
          QView V = qview(sm, L, q, M, C);
          const float kp = J.taupdt * prn;
          const Coef k = make_coef(kp, J.ke, J.kzi, J.kzj, kF64);
          const float4* tab = s_tab[q].tab;
          const double2* rtab = s_tab[q].rtab;
            const int tlen = s_tab[q].len;
          const uint32_t* cbits = V.bits + cur * V.W;
          const int* clist = V.list + cur * C;
          const int ncol = (pass == 0) ? nspk * C : V.nlist[cur] * nspk;
          for (int b0 = 0; b0 < ncol; b0 += kColU * kGroup) {
            size_t index[kColU];
            int tv[kColU];
            float4 cv[kColU];
            bool ok[kColU];
#pragma unroll
            for (int u = 0; u < kColU; ++u) {
              int c = b0 + u * kGroup + gtid;
              ok[u] = false;
              if (c < ncol) {
                int s, j;
                if (pass == 0) {
                  int qq = c / C;
                  s = c - qq * C;
                  j = w_spkl[qq];
                  ok[u] = V.ii[s] >= 0 && !((cbits[s >> 5] >> (s & 31)) & 1u);
                } else {
                  int rr = c / nspk;
                  s = clist[rr] - h * C;
                  j = w_spkl[c - rr * nspk];
                  ok[u] = V.ii[s] >= 0;
                }
                index[u] = (size_t)(h * C + s) * M + j;
              }
              if (ok[u]) {
                tv[u] = J.tij[index[u]];
                cv[u] = J.cell[index[u]];
              }
            }
            /* decay-table entries of the whole batch, then the compute */
            float4 tA[kColU], tB[kColU];
            double2 tR0[kColU], tR1[kColU];
#pragma unroll
            for (int u = 0; u < kColU; ++u) {
              int pdt = simstep - tv[u];
              if (ok[u] && pdt > 0 && pdt < tlen) {
                tA[u] = tab[(size_t)pdt * 4 + 0];
                tB[u] = tab[(size_t)pdt * 4 + 1];
                tR0[u] = rtab[(size_t)pdt * 4 + 0];
                tR1[u] = rtab[(size_t)pdt * 4 + 1];
              }
            }
#pragma unroll
            for (int u = 0; u < kColU; ++u) {
              if (!ok[u]) continue;
              int pdt = simstep - tv[u];
              float4 c4 = cv[u];
              if (pdt <= 0) {
                c4.w += J.kftj;
              } else {
                float4 A = tA[u], B = tB[u];
                double2 R0 = tR0[u], R1 = tR1[u];
                if (pdt >= tlen) {
                  if (k.fp64)
                    table_pair(k.kp, k.ke, k.kzi, k.kzj, pdt, 0, A, B, 1);
                  else
                    cell_factors(k.kp, k.ke, k.kzi, k.kzj, pdt, A, B);
                  recip_part(A, B, 0, R0, R1);
                }
                c4 = cell_step_nl(c4, &s_tab[q], A, B, R0, R1);
                c4.w = c4.w + J.kftj;
              }
              J.cell[index[u]] = c4;
              J.tij[index[u]] = simstep;
            }
          }
          if (pass == 0 && gtid == 0) s_cols_acc += (unsigned long long)nspk * C;
        }
      }
    }
    PROBE(13);
    __syncthreads();
    PROBE(8);
    /* every write of this tick is done: arrive now, and stage the next tick's
       first row chunk while the others arrive (cells of that chunk that the
       grid's column units of this tick change are refreshed after the
       column wait) */
    if (it + 1 < it0 + n_ticks) grid_arrive(bar);

    if (it + 1 < it0 + n_ticks && n_in > 0) {
      const ProjDev& J = s_proj[0];
      QView V = qview(sm, L, 0, M, J.C);
      int nr = V.nlist[nxt] < row_chunk_rows(M) ? V.nlist[nxt] : row_chunk_rows(M);
      stage_rows(J, V.list + nxt * J.C, 0, nr, M, simstep + 1, s_tab[0].tab, s_tab[0].rtab, s_tab[0].len, sm, L,
                 tid, kBlock);
    }
    PROBE(9);
  }

  /* ---- the last tick's deferred columns -------------------------------- */
  if (defer) {
    if (!grid_sync(bar, (unsigned int)n_ticks * gridDim.x, net->err, &s_ok)) return;
    if (!groupA) {
      const int lastp = (rp->k0 + it0 + n_ticks - 1) & 1;
      help_columns<kF64>(net, rp, net->col_ring + (size_t)lastp * net->col_cap, s_last_end[lastp], col_tail + lastp,
                         rp->simstep0 + it0 + n_ticks - 1, col_done, gtid, kBarB, &s_hend, s_inp, s_proj, s_tab,
                         n_in);
    }
  }

  /* ---- write the resident state back (buffers of the last tick) --------- */
  PROBE_FLUSH();
  __syncthreads();
  if (tid == 0) {
    if (s_rows_acc) atomicAdd(&net->counters[0], s_rows_acc);
    if (s_cols_acc) atomicAdd(&net->counters[1], s_cols_acc);
  }
  {
    const int last = (rp->k0 + it0 + n_ticks - 1) & 1;
    const int next = last ^ 1;
    for (int j = tid; j < M; j += kBlock) {
      int idx = h * M + j;
      pop.dsup[last][idx] = st_dsup[j];
      pop.act[idx] = st_act[j];
      pop.counter[idx] = st_cnt[j];
      pop.spike[idx] = w_spk[j];
    }
    for (int q = 0; q < n_in; ++q) {
      const ProjDev& J = s_proj[q];
      QView V = qview(sm, L, q, M, J.C);
      const size_t eoff = (size_t)J.proj_in_pop * n;
      for (int j = tid; j < M; j += kBlock) {
        int idx = h * M + j;
        J.pj[idx] = V.pj[j];
        J.ej[idx] = V.ej[j];
        J.zj[idx] = V.zj[j];
        pop.epsc[last][eoff + idx] = V.epsc[j];
        pop.bj[last][eoff + idx] = V.bj[j];
      }
      for (int s = tid; s < J.C; s += kBlock) {
        int r = h * J.C + s;
        J.qi[r] = V.qi[s];
        J.list[r] = V.list[next * J.C + s];
      }
      if (tid == 0) J.list_cnt[h] = V.nlist[next];
    }
  }
}

/* dynamic shared memory of tick_kernel for the largest population */
inline size_t tick_smem_bytes_for(int M, int n_in, const int* C) {
  TickLayout L;
  tick_layout(M, n_in, C, L);
  return (size_t)L.total * 4;
}

}  // namespace BCPNN_TICK_NS
}  // namespace bcpnn
