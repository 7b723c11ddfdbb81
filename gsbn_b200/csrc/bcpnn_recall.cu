/*
 * bcpnn_recall.cu -- replicate recall engine (include/bcpnn_recall.h).
 *
 * Two launches per tick on two streams, side by side: the population update
 * of tick t (recall_pop_kernel: support from epsc(t-1), softmax/WTA, Philox
 * spikes, writing dsup(t), the BF16 spike row S(t) and the recall counters)
 * and the contraction with its epilogue epsc(t) = epsc(t-1) * (1 - kepsc) +
 * S(t-3) . W.  The contraction comes in two forms, chosen at create time:
 *
 * BF16 (recall_tick_kernel), persistent, CTA tile = 128 replicates x 256
 * destination MCUs, the K loop over the N source MCUs in stages of 64:
 *   warp 0      TMA producer: S(t-3) tile [128 x 64] and W^T tile [256 x 64]
 *               (BF16, 128-byte swizzle) into a 4-stage shared-memory ring,
 *               one mbarrier per stage with the transaction byte count;
 *   warp 1      allocates 512 TMEM columns (two accumulators); one elected
 *               thread issues tcgen05.mma.cta_group::1.kind::f16 (M=128,
 *               N=256, K=16, FP32 accumulate) per 16-wide K step and
 *               tcgen05.commit to free each stage and, at the end, to signal
 *               the accumulator;
 *   warps 2..5  epilogue, one replicate row per thread (TMEM lane = row):
 *               tcgen05.ld of the accumulator and the epsc update.
 *
 * FP32 (recall_fp32_kernel): the same contraction on the FP32 pipes with W
 * kept in FP32 -- a register-tiled SIMT product (CTA tile 128 x 128, 8 x 8
 * outputs per thread, K stages of 16 double-buffered in shared memory) with
 * the same epilogue expression.  It exists to measure the tensor-core form
 * against the same engine at full precision.
 *
 * Every mbarrier wait is bounded (1 s of %globaltimer); a wait that runs out
 * sets an error bit and the CTA leaves its loops, waits (bounded) for its own
 * outstanding copies and MMAs, frees TMEM and returns.  No cluster multicast.
 */
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "bcpnn_numerics.h"
#include "bcpnn_recall.h"

namespace bcpnn_recall_dev {

constexpr int kTileM = 128, kTileN = 256, kTileK = 64, kStages = 4, kUmmaK = 16;
constexpr int kThreads = 192;
constexpr uint32_t kBytesA = kTileM * kTileK * 2; /* 16 KB */
constexpr uint32_t kBytesB = kTileN * kTileK * 2; /* 32 KB */
constexpr uint32_t kStageBytes = kBytesA + kBytesB;
constexpr uint32_t kTmemCols = 512; /* two 128 x 256 FP32 accumulators */
constexpr int kEpiThreads = 128;
constexpr int kErrWait = 4;
constexpr int kErrAlign = 8; /* a self-check found a misaligned or out-of-range access (skipped) */
constexpr unsigned long long kWaitNs = 1000000000ull;
/* dynamic shared memory: ring (1024-aligned) + barriers + TMEM address */
constexpr size_t kSmemBytes = 1024 + kStages * kStageBytes + 256;

struct Params {
  const float* dsup_prev;
  float* dsup_cur;
  const float* epsc_prev;
  float* epsc_cur;
  uint16_t* s_out; /* BF16 [R][N] spikes of this tick */
  uint8_t* counts; /* [R][N] */
  int count_on;
  const float* bj;
  const int32_t* lgidx; /* [R][H] */
  const float* wmask;   /* [R][H] */
  float lg_hit, lg_miss;
  int N, H, R;
  float taumdt, maxfqdt, wtagain, igain, wgain, lgbias, snoise, one_m_kepsc, pr;
  uint32_t seed_base;
  int simstep;
  int poisson;
  int* err;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long gtimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

/* bounded wait; false when it ran out or another thread reported an error */
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* err) {
  if (mbar_try_wait(bar, parity)) return true;
  unsigned long long t0 = gtimer();
  while (!mbar_try_wait(bar, parity)) {
    if (*(volatile int*)err) return false;
    if (gtimer() - t0 > kWaitNs) {
      atomicOr(err, kErrWait);
      return false;
    }
  }
  return true;
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];"
      ::"r"(smem_u32(dst)), "l"((uint64_t)map), "r"(smem_u32(bar)), "r"(x), "r"(y)
      : "memory");
}

/* shared-memory matrix descriptor: K-major operand, 128-byte swizzle, 8-row
   core groups 1024 bytes apart, descriptor version 1 (sm_100) */
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFF);
  d |= (uint64_t)1 << 16;                /* leading byte offset (unused for swizzled K-major) */
  d |= (uint64_t)(1024 >> 4) << 32;      /* stride byte offset */
  d |= (uint64_t)1 << 46;                /* version */
  d |= (uint64_t)2 << 61;                /* SWIZZLE_128B */
  return d;
}

/* instruction descriptor: D F32, A BF16, B BF16, both K-major, N=256, M=128 */
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kTileN >> 3) << 17) |
                            ((uint32_t)(kTileM >> 4) << 24);

__device__ __forceinline__ void umma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
      ::"r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(kIdesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

/* 32 consecutive FP32 accumulator columns of this thread's lane */
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

/* population update of tick `simstep` for MCU 0 of the population (the
   softmax max seed of every HCU, Pop.cpp:270) */
__device__ __forceinline__ float dsup_mcu0(const Params& p, int row, uint32_t seed) {
  const size_t base = (size_t)row * p.N;
  float wsup = 0.0f;
  wsup += p.bj[0] + p.epsc_prev[base];
  float noise = 0.0f;
  if (p.snoise != 0.0f) noise = p.snoise * bx_normal01(seed, 0u, (uint32_t)p.simstep, 0u);
  float lginp = (p.lgidx[(size_t)row * p.H] == 0) ? p.lg_hit : p.lg_miss;
  float sup = p.lgbias + p.igain * lginp + noise;
  sup += (p.wgain * p.wmask[(size_t)row * p.H]) * wsup;
  float d = p.dsup_prev[base];
  return d + (sup - d) * p.taumdt;
}

/* Population update of tick `simstep` (Pop.cpp:229-323) for one quarter of
   one HCU of one replicate: thread tid = (replicate * H + HCU) * 4 + q holds
   MCUs q*Q .. q*Q+Q-1 of the HCU (Q = M/4), so four consecutive lanes hold
   the four quarters of an HCU.  The HCU maximum is a shuffle max (exact); the
   activity sum keeps gsbn's serial MCU order by passing the running sum from
   lane to lane; one Philox call per four MCUs and stream.  Its own kernel,
   run beside the contraction on a second stream: a CTA of the contraction
   leaves room on its SM for three of its CTAs. */
template <int M>
__global__ void __launch_bounds__(256) recall_pop_kernel(Params p) {
  constexpr int Q = M / 4;
  const int lane = threadIdx.x & 31;
  const int tid = blockIdx.x * 256 + threadIdx.x;
  const int g = tid >> 2, q = tid & 3;
  const int h = g % p.H, r = g / p.H;
  const uint32_t seed = p.seed_base + (uint32_t)r;
  const size_t row = (size_t)r * p.N;
  const int c0 = h * M + q * Q;
  /* self-check: every vector access below is in bounds and aligned */
  {
    const size_t n = (size_t)p.R * p.N;
    const bool bad = r >= p.R || row + c0 + Q > n || ((row + c0) & 3) != 0 || (c0 + Q) > p.N ||
                     (reinterpret_cast<uintptr_t>(p.dsup_prev) & 15) || (reinterpret_cast<uintptr_t>(p.dsup_cur) & 15) ||
                     (reinterpret_cast<uintptr_t>(p.epsc_prev) & 15) || (reinterpret_cast<uintptr_t>(p.bj) & 15) ||
                     (reinterpret_cast<uintptr_t>(p.s_out) & 15) || (reinterpret_cast<uintptr_t>(p.counts) & 15);
    /* the warp leaves together: the shuffles below take all 32 lanes */
    if (__any_sync(0xffffffffu, bad)) {
      if (bad && atomicOr(p.err, kErrAlign) == 0) p.err[1] = tid;
      return;
    }
  }
  const float seed0 = dsup_mcu0(p, r, seed);
  const int lg = p.lgidx[(size_t)r * p.H + h];
  const float wm = p.wgain * p.wmask[(size_t)r * p.H + h];
  float d[Q];
#pragma unroll
  for (int m = 0; m < Q; m += 4) {
    float4 dp = *reinterpret_cast<const float4*>(p.dsup_prev + row + c0 + m);
    float4 ep = *reinterpret_cast<const float4*>(p.epsc_prev + row + c0 + m);
    float4 bb = *reinterpret_cast<const float4*>(p.bj + c0 + m);
    float dpv[4] = {dp.x, dp.y, dp.z, dp.w}, epv[4] = {ep.x, ep.y, ep.z, ep.w}, bjv[4] = {bb.x, bb.y, bb.z, bb.w};
#pragma unroll
    for (int k = 0; k < 4; k++) {
      float wsup = 0.0f;
      wsup += bjv[k] + epv[k];
      float noise = 0.0f;
      if (p.snoise != 0.0f) noise = p.snoise * bx_normal01(seed, 0u, (uint32_t)p.simstep, (uint32_t)(c0 + m + k));
      float lginp = (lg == q * Q + m + k) ? p.lg_hit : p.lg_miss;
      float sup = p.lgbias + p.igain * lginp + noise;
      sup += wm * wsup;
      d[m + k] = dpv[k] + (sup - dpv[k]) * p.taumdt;
    }
  }
  float mx = seed0; /* the new dsup of population MCU 0 (also d[0] of HCU 0's first quarter) */
#pragma unroll
  for (int m = 0; m < Q; m++) mx = (d[m] > mx) ? d[m] : mx;
  mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, 1));
  mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, 2));
  const float maxact = bx_expf(p.wtagain * mx);
  float a[Q];
#pragma unroll
  for (int m = 0; m < Q; m++) {
    a[m] = bx_expf(p.wtagain * (d[m] - mx));
    if (maxact < 1.0f) a[m] *= maxact;
  }
  float vs = 0.0f;
#pragma unroll
  for (int s = 0; s < 4; s++) {
    if (q == s) {
#pragma unroll
      for (int m = 0; m < Q; m++) vs += a[m];
    }
    vs = __shfl_sync(0xffffffffu, vs, (lane & ~3) | s);
  }
  uint32_t bits = 0u;
#pragma unroll
  for (int m = 0; m < Q; m += 4) {
    bx_u32x4 cu;
    cu.v[0] = (uint32_t)(c0 + m) >> 2;
    cu.v[1] = (uint32_t)p.simstep;
    cu.v[2] = 0u;
    cu.v[3] = 0u;
    const bx_u32x4 ou = bx_philox4x32_10(cu, seed, 0u * 16u + BX_STREAM_UNIFORM);
    bx_u32x4 op;
    if (p.poisson) op = bx_philox4x32_10(cu, seed, 0u * 16u + BX_STREAM_POISSON);
#pragma unroll
    for (int k = 0; k < 4; k++) {
      float act = a[m + k];
      if (vs > 1.0f) act /= vs;
      bool spk = bx_u01(ou.v[k]) < act * p.maxfqdt;
      if (p.poisson && bx_u01(op.v[k]) < p.pr) spk = true;
      if (spk) bits |= 1u << (m + k);
    }
  }
#pragma unroll
  for (int m = 0; m < Q; m += 4)
    *reinterpret_cast<float4*>(p.dsup_cur + row + c0 + m) = make_float4(d[m], d[m + 1], d[m + 2], d[m + 3]);
  /* BF16 1.0 = 0x3F80; four MCUs per 8-byte store (Q is a multiple of 4) */
#pragma unroll
  for (int m = 0; m < Q; m += 4) {
    uint32_t w[2];
#pragma unroll
    for (int k = 0; k < 2; k++)
      w[k] = (((bits >> (m + 2 * k)) & 1u) ? 0x3F80u : 0u) | ((((bits >> (m + 2 * k + 1)) & 1u) ? 0x3F80u : 0u) << 16);
    *reinterpret_cast<uint2*>(p.s_out + row + c0 + m) = make_uint2(w[0], w[1]);
  }
  if (p.count_on) {
#pragma unroll
    for (int m = 0; m < Q; m += 4) {
      uint32_t* c = reinterpret_cast<uint32_t*>(p.counts + row + c0 + m);
      uint32_t add = 0;
#pragma unroll
      for (int k = 0; k < 4; k++) add |= ((bits >> (m + k)) & 1u) << (8 * k);
      *c = *c + add; /* no carry between bytes: at most 255 counted ticks between clears */
    }
  }
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

/* Persistent contraction + epsc epilogue: one CTA per SM walks the output
   tiles t = blockIdx.x, blockIdx.x + gridDim.x, ... (tile t = M-tile t / nN,
   N-tile t % nN).  The stage ring runs on across tiles; two TMEM accumulators
   of 256 columns alternate, so the epilogue of one tile overlaps the MMAs of
   the next (acc_full: MMA -> epilogue, acc_empty: epilogue -> MMA). */
__global__ void __launch_bounds__(kThreads, 1)
    recall_tick_kernel(const __grid_constant__ CUtensorMap map_s, const __grid_constant__ CUtensorMap map_w,
                       Params p) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* ring = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  uint64_t* full = reinterpret_cast<uint64_t*>(ring + kStages * kStageBytes);
  uint64_t* empty = full + kStages;
  uint64_t* acc_full = empty + kStages;   /* [2] */
  uint64_t* acc_empty = acc_full + 2;     /* [2] */
  uint64_t* mma_done = acc_empty + 2;
  uint32_t* s_tmem = reinterpret_cast<uint32_t*>(mma_done + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nN = p.N / kTileN, nM = p.R / kTileM, n_tiles = nN * nM;
  const int kIters = p.N / kTileK;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int j = 0; j < 2; j++) {
      mbar_init(&acc_full[j], 1);
      mbar_init(&acc_empty[j], kEpiThreads);
    }
    mbar_init(mma_done, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(s_tmem)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *s_tmem;
  /* self-check of the set-up every access below relies on: ring and barrier
     alignment, the accumulators' TMEM columns, whole tiles */
  const bool setup_ok = (smem_u32(ring) & 1023u) == 0 && (smem_u32(full) & 7u) == 0 && (tmem >> 16) == 0 &&
                        (tmem & 0xFFFFu) + kTmemCols <= 512u && p.N % kTileN == 0 && p.R % kTileM == 0 &&
                        (reinterpret_cast<uintptr_t>(p.epsc_prev) & 15) == 0 &&
                        (reinterpret_cast<uintptr_t>(p.epsc_cur) & 15) == 0;
  if (!setup_ok && threadIdx.x == 0 && atomicOr(p.err, kErrAlign) == 0) p.err[1] = -1 - (int)blockIdx.x;

  if (setup_ok && warp == 0) {
    /* ---------------- TMA producer ---------------- */
    if (lane == 0) {
      long long it = 0;
      bool ok = true;
      for (int t = blockIdx.x; t < n_tiles && ok; t += gridDim.x) {
        const int m0 = (t / nN) * kTileM, n0 = (t % nN) * kTileN;
        for (int k = 0; k < kIters; k++, it++) {
          const int s = (int)(it % kStages);
          if (!mbar_wait(&empty[s], (uint32_t)(((it / kStages) & 1) ^ 1), p.err)) {
            ok = false;
            break;
          }
          uint8_t* a = ring + s * kStageBytes;
          mbar_expect_tx(&full[s], kStageBytes);
          tma_load_2d(a, &map_s, &full[s], k * kTileK, m0);
          tma_load_2d(a + kBytesA, &map_w, &full[s], k * kTileK, n0);
        }
      }
      /* leave no copy in flight: the last use of every slot completes */
      for (long long j = (it > kStages ? it - kStages : 0); j < it; j++) {
        unsigned long long t0 = gtimer();
        while (!mbar_try_wait(&full[j % kStages], (uint32_t)((j / kStages) & 1)) && gtimer() - t0 < kWaitNs) {
        }
      }
    }
  } else if (setup_ok && warp == 1) {
    /* ---------------- MMA issuer ---------------- */
    if (lane == 0) {
      long long it = 0;
      bool ok = true;
      int li = 0;
      for (int t = blockIdx.x; t < n_tiles && ok; t += gridDim.x, li++) {
        const int j = li & 1;
        if (!mbar_wait(&acc_empty[j], (uint32_t)(((li >> 1) & 1) ^ 1), p.err)) break;
        tc_fence_after();
        const uint32_t acc = tmem + (uint32_t)(j * kTileN);
        for (int k = 0; k < kIters; k++, it++) {
          const int s = (int)(it % kStages);
          if (!mbar_wait(&full[s], (uint32_t)((it / kStages) & 1), p.err)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t a = smem_u32(ring + s * kStageBytes);
          const uint32_t b = a + kBytesA;
#pragma unroll
          for (int kk = 0; kk < kTileK / kUmmaK; kk++) {
            /* +32 bytes along K inside the 128-byte swizzled row */
            umma(acc, smem_desc(a + kk * 32), smem_desc(b + kk * 32), (k > 0 || kk > 0) ? 1u : 0u);
          }
          umma_commit(&empty[s]);
        }
        if (ok) umma_commit(&acc_full[j]);
      }
    }
  } else if (setup_ok) {
    /* ---------------- epilogue: one replicate row per thread ---------------- */
    const int q = warp & 3; /* TMEM lane quarter this warp may access */
    int li = 0;
    for (int t = blockIdx.x; t < n_tiles; t += gridDim.x, li++) {
      const int j = li & 1;
      const int m0 = (t / nN) * kTileM, n0 = (t % nN) * kTileN;
      /* warp-uniform: tcgen05.ld is .sync.aligned */
      const bool ok = __all_sync(0xffffffffu, mbar_wait(&acc_full[j], (uint32_t)((li >> 1) & 1), p.err) ? 1 : 0) != 0;
      if (!ok) break;
      tc_fence_after();
      const int row = m0 + q * 32 + lane;
      const size_t base = (size_t)row * p.N + n0;
      for (int c = 0; c < kTileN; c += 32) {
        float acc[32];
        tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(j * kTileN + c), acc);
#pragma unroll
        for (int i = 0; i < 32; i += 4) {
          float4 e = *reinterpret_cast<const float4*>(p.epsc_prev + base + c + i);
          float4 o;
          o.x = e.x * p.one_m_kepsc + acc[i];
          o.y = e.y * p.one_m_kepsc + acc[i + 1];
          o.z = e.z * p.one_m_kepsc + acc[i + 2];
          o.w = e.w * p.one_m_kepsc + acc[i + 3];
          *reinterpret_cast<float4*>(p.epsc_cur + base + c + i) = o;
        }
      }
      tc_fence_before();
      mbar_arrive(&acc_empty[j]);
    }
  }
  /* every tcgen05 operation of this CTA completes before TMEM is freed: the
     MMA thread's last commit (all MMAs it issued) is waited for, bounded */
  if (warp == 1 && lane == 0) {
    umma_commit(mma_done);
    unsigned long long t0 = gtimer();
    while (!mbar_try_wait(mma_done, 0) && gtimer() - t0 < kWaitNs) {
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 1)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
}

constexpr int kF32BM = 128, kF32BN = 128, kF32BK = 16, kF32Threads = 256;

/* FP32 SIMT contraction with the epsc epilogue of recall_tick_kernel:
   epsc(t)[r][j] = epsc(t-1)[r][j] * (1 - kepsc) + sum_i S(t-3)[r][i] * W[i][j]
   with W in FP32 ([source i][destination j], row-major) and S the BF16 0/1
   spike ring (its value is exact: the bits shifted into an FP32 word).

   One CTA per 128 x 128 output tile (blockIdx.x = M-tile * (N/128) + N-tile);
   thread (ty, tx) = (tid / 16, tid % 16) owns rows {ty*4 .. +3, 64 + ty*4 ..
   +3} and columns {tx*4 .. +3, 64 + tx*4 .. +3} of the tile, 64 FP32
   accumulators.  K stages of 16: S as [k][row] and W as [k][col] in shared
   memory, two buffers, the next stage's global loads held in registers while
   the current one is multiplied, one barrier per stage. */
__global__ void __launch_bounds__(kF32Threads, 2)
    recall_fp32_kernel(const uint16_t* __restrict__ s, const float* __restrict__ w, Params p) {
  __shared__ __align__(16) float As[2][kF32BK][kF32BM];
  __shared__ __align__(16) float Bs[2][kF32BK][kF32BN];
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const int nN = p.N / kF32BN, nM = p.R / kF32BM;
  const int m0 = ((int)blockIdx.x / nN) * kF32BM, n0 = ((int)blockIdx.x % nN) * kF32BN;
  /* self-check: whole tiles, the tile inside the arrays, 16-byte alignment of
     every vector access */
  {
    const bool bad = p.N % kF32BN != 0 || p.R % kF32BM != 0 || (int)blockIdx.x >= nN * nM ||
                     (reinterpret_cast<uintptr_t>(s) & 15) || (reinterpret_cast<uintptr_t>(w) & 15) ||
                     (reinterpret_cast<uintptr_t>(p.epsc_prev) & 15) ||
                     (reinterpret_cast<uintptr_t>(p.epsc_cur) & 15);
    if (bad) {
      if (tid == 0 && atomicOr(p.err, kErrAlign) == 0) p.err[1] = -1 - (int)blockIdx.x;
      return;
    }
  }
  /* S stage: row a_row, eight BF16 at a_k (one 16-byte load); W stage: row
     b_k, eight floats at b_n (two 16-byte loads) */
  const int a_row = tid & 127, a_k = (tid >> 7) * 8;
  const int b_k = tid >> 4, b_n = (tid & 15) * 8;
  const uint16_t* ag = s + (size_t)(m0 + a_row) * p.N + a_k;
  const float* bg = w + (size_t)b_k * p.N + n0 + b_n;
  const size_t b_step = (size_t)kF32BK * p.N;
  uint4 ra = __ldg(reinterpret_cast<const uint4*>(ag));
  float4 rb0 = __ldg(reinterpret_cast<const float4*>(bg));
  float4 rb1 = __ldg(reinterpret_cast<const float4*>(bg + 4));
  float acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; i++)
#pragma unroll
    for (int j = 0; j < 8; j++) acc[i][j] = 0.0f;

  auto stage = [&](int buf) {
    const uint32_t u[4] = {ra.x, ra.y, ra.z, ra.w};
#pragma unroll
    for (int j = 0; j < 4; j++) {
      As[buf][a_k + 2 * j][a_row] = __uint_as_float(u[j] << 16);
      As[buf][a_k + 2 * j + 1][a_row] = __uint_as_float(u[j] & 0xFFFF0000u);
    }
    *reinterpret_cast<float4*>(&Bs[buf][b_k][b_n]) = rb0;
    *reinterpret_cast<float4*>(&Bs[buf][b_k][b_n + 4]) = rb1;
  };
  stage(0);
  __syncthreads();
  const int kTiles = p.N / kF32BK;
  for (int kt = 0; kt < kTiles; kt++) {
    const int buf = kt & 1;
    if (kt + 1 < kTiles) {
      ra = __ldg(reinterpret_cast<const uint4*>(ag + (size_t)(kt + 1) * kF32BK));
      const float* b = bg + (size_t)(kt + 1) * b_step;
      rb0 = __ldg(reinterpret_cast<const float4*>(b));
      rb1 = __ldg(reinterpret_cast<const float4*>(b + 4));
    }
#pragma unroll
    for (int k = 0; k < kF32BK; k++) {
      const float4 a0 = *reinterpret_cast<const float4*>(&As[buf][k][ty * 4]);
      const float4 a1 = *reinterpret_cast<const float4*>(&As[buf][k][64 + ty * 4]);
      const float4 b0 = *reinterpret_cast<const float4*>(&Bs[buf][k][tx * 4]);
      const float4 b1 = *reinterpret_cast<const float4*>(&Bs[buf][k][64 + tx * 4]);
      const float av[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
      const float bv[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
      for (int i = 0; i < 8; i++)
#pragma unroll
        for (int j = 0; j < 8; j++) acc[i][j] = fmaf(av[i], bv[j], acc[i][j]);
    }
    /* the other buffer was last read in stage kt-1, before the barrier
       that ended it */
    if (kt + 1 < kTiles) stage(buf ^ 1);
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 8; i++) {
    const int row = m0 + (i < 4 ? ty * 4 + i : 64 + ty * 4 + (i - 4));
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const size_t o = (size_t)row * p.N + n0 + h * 64 + tx * 4;
      const float4 e = *reinterpret_cast<const float4*>(p.epsc_prev + o);
      float4 v;
      v.x = e.x * p.one_m_kepsc + acc[i][h * 4 + 0];
      v.y = e.y * p.one_m_kepsc + acc[i][h * 4 + 1];
      v.z = e.z * p.one_m_kepsc + acc[i][h * 4 + 2];
      v.w = e.w * p.one_m_kepsc + acc[i][h * 4 + 3];
      *reinterpret_cast<float4*>(p.epsc_cur + o) = v;
    }
  }
}

__global__ void broadcast_spikes_kernel(uint16_t* s, int R, int N, const int8_t* row) {
  size_t n = (size_t)R * N;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    s[i] = row[i % N] ? 0x3F80u : 0u;
}

__global__ void broadcast_f32_kernel(float* dst, int R, int N, const float* row) {
  size_t n = (size_t)R * N;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    dst[i] = row[i % N];
}

}  // namespace bcpnn_recall_dev

using namespace bcpnn_recall_dev;

struct bcpnn_recall {
  bcpnn_recall_desc d;
  int N = 0;
  cudaStream_t stream = nullptr;      /* contraction + epsc; the handle's stream */
  cudaStream_t pop_stream = nullptr;  /* population update, concurrent with it */
  cudaEvent_t ev_pop = nullptr, ev_gemm = nullptr;
  float* dsup[2] = {nullptr, nullptr};
  float* epsc[2] = {nullptr, nullptr};
  uint16_t* s[4] = {nullptr, nullptr, nullptr, nullptr}; /* spike ring, by tick mod 4 */
  uint16_t* wt = nullptr; /* W^T BF16 [N][N] (BF16 contraction) */
  float* wf = nullptr;    /* W FP32 [N][N], [source][destination] (FP32 contraction) */
  uint8_t* counts = nullptr;
  float* bj = nullptr;
  int32_t* lgidx = nullptr;
  float* wmask = nullptr;
  int* err = nullptr;
  float lg_hit = 0.f, lg_miss = 0.f;
  bool loaded = false, cued = false;
  long long kk = 0; /* ticks run since load */
  int counted = 0;   /* counted ticks since the counters were cleared */
  CUtensorMap map_s[4];
  CUtensorMap map_w;
  uint64_t launches = 0;
  int sms = 148;
  /* in-place timing of the contraction launches (bcpnn_recall_timing) */
  bool timing = false;
  std::vector<cudaEvent_t> tev;
  double contraction_ms = 0.0;
  uint64_t contraction_launches = 0;
  std::string last_error;
  std::vector<void*> allocs;
};

namespace {

int fail(bcpnn_recall* r, int code, const std::string& msg) {
  if (r) r->last_error = msg;
  return code;
}

#define RCU(call)                                                                             \
  do {                                                                                        \
    cudaError_t e_ = (call);                                                                  \
    if (e_ != cudaSuccess)                                                                    \
      return fail(r, BCPNN_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));     \
  } while (0)

typedef CUresult (*EncodeTiled)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

int encode_map(bcpnn_recall* r, CUtensorMap* map, void* base, int rows, int cols, int box_rows) {
  static EncodeTiled fn = nullptr;
  if (!fn) {
    cudaDriverEntryPointQueryResult q;
    void* p = nullptr;
    RCU(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
    if (q != cudaDriverEntryPointSuccess || !p) return fail(r, BCPNN_ERR_CUDA, "cuTensorMapEncodeTiled not available");
    fn = (EncodeTiled)p;
  }
  cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)cols * 2};
  cuuint32_t box[2] = {(cuuint32_t)kTileK, (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult e = fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, base, dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (e != CUDA_SUCCESS) return fail(r, BCPNN_ERR_CUDA, "cuTensorMapEncodeTiled failed: " + std::to_string((int)e));
  return BCPNN_OK;
}

template <typename T>
int dalloc(bcpnn_recall* r, T** p, size_t count) {
  *p = nullptr;
  RCU(cudaMalloc((void**)p, (count ? count : 1) * sizeof(T)));
  r->allocs.push_back((void*)*p);
  return BCPNN_OK;
}

uint16_t to_bf16(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  if ((u & 0x7F800000u) == 0x7F800000u) return (uint16_t)((u >> 16) | ((u & 0xFFFFu) ? 0x40u : 0u));
  u += 0x7FFFu + ((u >> 16) & 1u); /* round to nearest even */
  return (uint16_t)(u >> 16);
}

int check_err(bcpnn_recall* r) {
  int e[2] = {0, 0};
  RCU(cudaMemcpyAsync(e, r->err, sizeof(e), cudaMemcpyDeviceToHost, r->stream));
  RCU(cudaStreamSynchronize(r->stream));
  if (e[0]) {
    RCU(cudaMemsetAsync(r->err, 0, sizeof(e), r->stream));
    std::string why;
    if (e[0] & kErrWait) why += " an mbarrier wait timed out;";
    if (e[0] & kErrAlign) why += " a self-check skipped a misaligned or out-of-range access (thread " + std::to_string(e[1]) + ");";
    return fail(r, BCPNN_ERR_DEVICE, "recall kernel reported error word " + std::to_string(e[0]) + ":" + why);
  }
  return BCPNN_OK;
}

int mod4(long long v) { return (int)(v & 3); }

}  // namespace

extern "C" {

int bcpnn_recall_create(const bcpnn_recall_desc* d, bcpnn_recall** out) {
  if (!d || !out) return BCPNN_ERR_INVALID;
  *out = nullptr;
  const int H = d->hcu_num, M = d->mcu_num, R = d->replicates;
  if (H < 1 || M < 1 || R < kTileM || R % kTileM) return BCPNN_ERR_INVALID;
  const long long N = (long long)H * M;
  if (N % kTileN || kTileN % M || (M != 16 && M != 32 && M != 64) || N > 65536) return BCPNN_ERR_INVALID;
  if (!(d->dt > 0.f) || !(d->pop.taum > 0.f) || d->poisson_noise_hz < 0.f) return BCPNN_ERR_INVALID;
  if (d->contraction != BCPNN_RECALL_BF16 && d->contraction != BCPNN_RECALL_FP32) return BCPNN_ERR_INVALID;
  const bool fp32 = d->contraction == BCPNN_RECALL_FP32;
  bcpnn_recall* r = new bcpnn_recall();
  r->d = *d;
  r->N = (int)N;
  auto bad = [&](int rc) {
    bcpnn_recall_destroy(r);
    return rc;
  };
  if (cudaSetDevice(d->device) != cudaSuccess) return bad(BCPNN_ERR_CUDA);
  int major = 0, minor = 0;
  cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, d->device);
  cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, d->device);
  if (major != 10 || minor != 0) return bad(BCPNN_ERR_DEVICE);
  cudaDeviceGetAttribute(&r->sms, cudaDevAttrMultiProcessorCount, d->device);
  if (r->sms < 1) r->sms = 1;
  /* the contraction's stream first in the block scheduler's order: its CTAs
     (one per SM) take their SMs before the population update fills the rest */
  int prio_low = 0, prio_high = 0;
  cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high);
  if (cudaStreamCreateWithPriority(&r->stream, cudaStreamNonBlocking, prio_high) != cudaSuccess)
    return bad(BCPNN_ERR_CUDA);
  size_t RN = (size_t)R * N;
  int rc = BCPNN_OK;
  for (int i = 0; i < 2 && !rc; i++) rc = dalloc(r, &r->dsup[i], RN);
  for (int i = 0; i < 2 && !rc; i++) rc = dalloc(r, &r->epsc[i], RN);
  for (int i = 0; i < 4 && !rc; i++) rc = dalloc(r, &r->s[i], RN);
  if (!rc && !fp32) rc = dalloc(r, &r->wt, (size_t)N * N);
  if (!rc && fp32) rc = dalloc(r, &r->wf, (size_t)N * N);
  if (!rc) rc = dalloc(r, &r->counts, RN);
  if (!rc) rc = dalloc(r, &r->bj, (size_t)N);
  if (!rc) rc = dalloc(r, &r->lgidx, (size_t)R * H);
  if (!rc) rc = dalloc(r, &r->wmask, (size_t)R * H);
  if (!rc) rc = dalloc(r, &r->err, 2);
  if (rc) return bad(rc);
  if (cudaMemset(r->err, 0, 2 * sizeof(int)) != cudaSuccess || cudaMemset(r->counts, 0, RN) != cudaSuccess)
    return bad(BCPNN_ERR_CUDA);
  if (!fp32) {
    for (int i = 0; i < 4 && !rc; i++) rc = encode_map(r, &r->map_s[i], r->s[i], R, (int)N, kTileM);
    if (!rc) rc = encode_map(r, &r->map_w, r->wt, (int)N, (int)N, kTileN);
    if (rc) return bad(rc);
    if (cudaFuncSetAttribute(recall_tick_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBytes) !=
        cudaSuccess)
      return bad(BCPNN_ERR_CUDA);
  }
  if (cudaStreamCreateWithPriority(&r->pop_stream, cudaStreamNonBlocking, prio_low) != cudaSuccess ||
      cudaEventCreateWithFlags(&r->ev_pop, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&r->ev_gemm, cudaEventDisableTiming) != cudaSuccess)
    return bad(BCPNN_ERR_CUDA);
  *out = r;
  return BCPNN_OK;
}

int bcpnn_recall_destroy(bcpnn_recall* r) {
  if (!r) return BCPNN_ERR_INVALID;
  cudaSetDevice(r->d.device);
  if (r->stream) cudaStreamSynchronize(r->stream);
  if (r->pop_stream) cudaStreamSynchronize(r->pop_stream);
  for (void* p : r->allocs) cudaFree(p);
  for (cudaEvent_t e : r->tev) cudaEventDestroy(e);
  if (r->ev_pop) cudaEventDestroy(r->ev_pop);
  if (r->ev_gemm) cudaEventDestroy(r->ev_gemm);
  if (r->pop_stream) cudaStreamDestroy(r->pop_stream);
  if (r->stream) cudaStreamDestroy(r->stream);
  delete r;
  return BCPNN_OK;
}

int bcpnn_recall_load(bcpnn_recall* r, const float* w, const float* bj, const float* epsc, const float* dsup,
                      const int8_t* spikes_tm3, const int8_t* spikes_tm2, const int8_t* spikes_tm1) {
  if (!r) return BCPNN_ERR_INVALID;
  if (!w || !bj || !epsc || !dsup || !spikes_tm3 || !spikes_tm2 || !spikes_tm1)
    return fail(r, BCPNN_ERR_INVALID, "null buffer");
  const int N = r->N, R = r->d.replicates;
  RCU(cudaSetDevice(r->d.device));
  if (r->wf) {
    /* FP32 contraction: W as given, [source][destination] */
    RCU(cudaMemcpy(r->wf, w, (size_t)N * N * 4, cudaMemcpyHostToDevice));
  } else {
    /* W^T in BF16: row j = destination MCU, K-contiguous over source MCUs */
    std::vector<uint16_t> wt((size_t)N * N);
    for (int i = 0; i < N; i++)
      for (int j = 0; j < N; j++) wt[(size_t)j * N + i] = to_bf16(w[(size_t)i * N + j]);
    RCU(cudaMemcpy(r->wt, wt.data(), wt.size() * 2, cudaMemcpyHostToDevice));
  }
  RCU(cudaMemcpy(r->bj, bj, (size_t)N * 4, cudaMemcpyHostToDevice));
  float* row_f = nullptr;
  int8_t* row_s = nullptr;
  RCU(cudaMalloc((void**)&row_f, (size_t)N * 4));
  cudaError_t e = cudaMalloc((void**)&row_s, (size_t)N * 3);
  if (e != cudaSuccess) {
    cudaFree(row_f);
    return fail(r, BCPNN_ERR_CUDA, std::string("recall load: ") + cudaGetErrorString(e));
  }
  r->kk = 0;
  const int prev = 1; /* parity buffer read by the next tick (kk = 0) */
  e = cudaMemcpy(row_f, epsc, (size_t)N * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    broadcast_f32_kernel<<<592, 256, 0, r->stream>>>(r->epsc[prev], R, N, row_f);
    e = cudaStreamSynchronize(r->stream);
  }
  if (e == cudaSuccess) e = cudaMemcpy(row_f, dsup, (size_t)N * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    broadcast_f32_kernel<<<592, 256, 0, r->stream>>>(r->dsup[prev], R, N, row_f);
    e = cudaStreamSynchronize(r->stream);
  }
  if (e == cudaSuccess) e = cudaMemcpy(row_s, spikes_tm3, (size_t)N, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(row_s + N, spikes_tm2, (size_t)N, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(row_s + 2 * N, spikes_tm1, (size_t)N, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    for (int k = 0; k < 3; k++)
      broadcast_spikes_kernel<<<592, 256, 0, r->stream>>>(r->s[mod4(k - 3)], R, N, row_s + (size_t)k * N);
    e = cudaStreamSynchronize(r->stream);
  }
  cudaFree(row_f);
  cudaFree(row_s);
  if (e != cudaSuccess) return fail(r, BCPNN_ERR_CUDA, std::string("recall load: ") + cudaGetErrorString(e));
  r->launches += 5;
  r->loaded = true;
  return BCPNN_OK;
}

int bcpnn_recall_set_cues(bcpnn_recall* r, const int32_t* lgidx, float eps, const float* wmask) {
  if (!r) return BCPNN_ERR_INVALID;
  if (!lgidx || !wmask) return fail(r, BCPNN_ERR_INVALID, "null buffer");
  const size_t n = (size_t)r->d.replicates * r->d.hcu_num;
  RCU(cudaSetDevice(r->d.device));
  RCU(cudaMemcpyAsync(r->lgidx, lgidx, n * 4, cudaMemcpyHostToDevice, r->stream));
  RCU(cudaMemcpyAsync(r->wmask, wmask, n * 4, cudaMemcpyHostToDevice, r->stream));
  RCU(cudaStreamSynchronize(r->stream));
  r->lg_hit = bx_extgen_logf(1 + eps);
  r->lg_miss = bx_extgen_logf(0 + eps);
  r->cued = true;
  return BCPNN_OK;
}

int bcpnn_recall_clear_counts(bcpnn_recall* r) {
  if (!r) return BCPNN_ERR_INVALID;
  RCU(cudaSetDevice(r->d.device));
  RCU(cudaMemsetAsync(r->counts, 0, (size_t)r->d.replicates * r->N, r->stream));
  r->counted = 0;
  return BCPNN_OK;
}

int bcpnn_recall_run(bcpnn_recall* r, int32_t first, int32_t n_ticks, int32_t count_first, int32_t count_last) {
  if (!r) return BCPNN_ERR_INVALID;
  if (!r->loaded || !r->cued) return fail(r, BCPNN_ERR_STATE, "bcpnn_recall_run before load and set_cues");
  if (n_ticks < 0 || first < 0 || (long long)first + n_ticks > 0x7fffffffLL)
    return fail(r, BCPNN_ERR_INVALID, "bad tick range");
  int counted = 0;
  for (int t = first; t < first + n_ticks; t++) counted += (t >= count_first && t <= count_last);
  if (r->counted + counted > 255)
    return fail(r, BCPNN_ERR_INVALID, "more than 255 counted ticks since the last clear (uint8 counters)");
  RCU(cudaSetDevice(r->d.device));
  const bcpnn_recall_desc& d = r->d;
  Params p;
  p.counts = r->counts;
  p.bj = r->bj;
  p.lgidx = r->lgidx;
  p.wmask = r->wmask;
  p.lg_hit = r->lg_hit;
  p.lg_miss = r->lg_miss;
  p.N = r->N;
  p.H = d.hcu_num;
  p.R = d.replicates;
  p.taumdt = d.dt / d.pop.taum;   /* Pop.cpp:34 */
  p.maxfqdt = d.pop.maxfq * d.dt; /* Pop.cpp:36 */
  p.wtagain = d.pop.wtagain;
  p.igain = d.pop.igain;
  p.wgain = d.pop.wgain;
  p.lgbias = d.pop.lgbias;
  p.snoise = d.pop.snoise;
  p.one_m_kepsc = 1.0f - d.kepsc;
  p.pr = d.poisson_noise_hz * d.dt;
  p.poisson = d.poisson_noise_hz > 0.f;
  p.seed_base = d.seed_base;
  p.err = r->err;
  const int n_tiles = (r->N / kTileN) * (d.replicates / kTileM);
  const int grid = n_tiles < r->sms ? n_tiles : r->sms;
  const int f32_tiles = (r->N / kF32BN) * (d.replicates / kF32BM);
  const int pop_blocks = (int)((size_t)d.replicates * d.hcu_num * 4 / 256);
  /* Tick kk: the population update needs epsc(kk-1) and dsup(kk-1); the
     contraction needs S(kk-3) and epsc(kk-1).  So both wait only for tick
     kk-1 and run side by side: pop(kk) after gemm(kk-1) (it also must not
     overwrite S(kk) = S(kk-4) while gemm(kk-1) reads it), gemm(kk) after
     pop(kk-1) (which last read the epsc buffer gemm(kk) writes). */
  if (r->timing) {
    while (r->tev.size() < 2 * (size_t)n_ticks) {
      cudaEvent_t e;
      RCU(cudaEventCreate(&e));
      r->tev.push_back(e);
    }
  }
  RCU(cudaEventRecord(r->ev_gemm, r->stream));
  RCU(cudaStreamWaitEvent(r->pop_stream, r->ev_gemm, 0));
  for (int i = 0; i < n_ticks; i++) {
    const long long kk = r->kk + i;
    const int cur = (int)(kk & 1), prev = cur ^ 1;
    p.dsup_prev = r->dsup[prev];
    p.dsup_cur = r->dsup[cur];
    p.epsc_prev = r->epsc[prev];
    p.epsc_cur = r->epsc[cur];
    p.s_out = r->s[mod4(kk)];
    p.simstep = first + i;
    p.count_on = (first + i >= count_first && first + i <= count_last) ? 1 : 0;
    if (d.mcu_num == 16) recall_pop_kernel<16><<<pop_blocks, 256, 0, r->pop_stream>>>(p);
    if (d.mcu_num == 32) recall_pop_kernel<32><<<pop_blocks, 256, 0, r->pop_stream>>>(p);
    if (d.mcu_num == 64) recall_pop_kernel<64><<<pop_blocks, 256, 0, r->pop_stream>>>(p);
    RCU(cudaGetLastError());
    if (r->timing) RCU(cudaEventRecord(r->tev[2 * i], r->stream));
    if (r->wf)
      recall_fp32_kernel<<<f32_tiles, kF32Threads, 0, r->stream>>>(r->s[mod4(kk - 3)], r->wf, p);
    else
      recall_tick_kernel<<<grid, kThreads, kSmemBytes, r->stream>>>(r->map_s[mod4(kk - 3)], r->map_w, p);
    RCU(cudaGetLastError());
    if (r->timing) RCU(cudaEventRecord(r->tev[2 * i + 1], r->stream));
    /* both kernels of tick kk are queued: each stream waits for the other's
       kernel of this tick before its kernel of tick kk+1 */
    RCU(cudaEventRecord(r->ev_pop, r->pop_stream));
    RCU(cudaEventRecord(r->ev_gemm, r->stream));
    RCU(cudaStreamWaitEvent(r->stream, r->ev_pop, 0));
    RCU(cudaStreamWaitEvent(r->pop_stream, r->ev_gemm, 0));
  }
  r->kk += n_ticks;
  r->counted += counted;
  r->launches += 2 * (uint64_t)n_ticks;
  int rc = check_err(r); /* synchronises the stream: every timing event has completed */
  if (rc == BCPNN_OK && r->timing) {
    for (int i = 0; i < n_ticks; i++) {
      float ms = 0.f;
      RCU(cudaEventElapsedTime(&ms, r->tev[2 * i], r->tev[2 * i + 1]));
      r->contraction_ms += ms;
    }
    r->contraction_launches += (uint64_t)n_ticks;
  }
  return rc;
}

static int resolve_rows(bcpnn_recall* r, const char* name, int32_t row0, int32_t n_rows, size_t bytes, void** base,
                        size_t* elem, int* kind) {
  if (!name) return fail(r, BCPNN_ERR_INVALID, "null name");
  const int R = r->d.replicates;
  if (row0 < 0 || n_rows < 0 || row0 + (long long)n_rows > R) return fail(r, BCPNN_ERR_INVALID, "rows out of range");
  std::string s(name);
  const long long last = r->kk - 1; /* last tick run */
  *kind = 0;
  if (s == "dsup") {
    *base = r->dsup[(int)(last & 1) & 1];
    *elem = 4;
  } else if (s == "epsc") {
    *base = r->epsc[(int)(last & 1) & 1];
    *elem = 4;
  } else if (s == "counts") {
    *base = r->counts;
    *elem = 1;
  } else if (s == "spike" || s == "spike_tm1") {
    *base = r->s[mod4(last)];
    *elem = 2;
    *kind = 1;
  } else if (s == "spike_tm2") {
    *base = r->s[mod4(last - 1)];
    *elem = 2;
    *kind = 1;
  } else if (s == "spike_tm3") {
    *base = r->s[mod4(last - 2)];
    *elem = 2;
    *kind = 1;
  } else {
    return fail(r, BCPNN_ERR_NOT_FOUND, "unknown recall array " + s);
  }
  size_t want = (size_t)n_rows * r->N * (*kind ? 1 : *elem);
  if (bytes != want) return fail(r, BCPNN_ERR_SIZE, "buffer size does not match rows x N");
  return BCPNN_OK;
}

int bcpnn_recall_read(bcpnn_recall* r, const char* name, int32_t row0, int32_t n_rows, void* host, size_t bytes) {
  if (!r || !host) return BCPNN_ERR_INVALID;
  void* base;
  size_t elem;
  int kind;
  int rc = resolve_rows(r, name, row0, n_rows, bytes, &base, &elem, &kind);
  if (rc) return rc;
  RCU(cudaSetDevice(r->d.device));
  const size_t off = (size_t)row0 * r->N * elem, n = (size_t)n_rows * r->N;
  if (kind == 1) {
    std::vector<uint16_t> tmp(n);
    RCU(cudaMemcpyAsync(tmp.data(), (uint8_t*)base + off, n * 2, cudaMemcpyDeviceToHost, r->stream));
    RCU(cudaStreamSynchronize(r->stream));
    int8_t* o = (int8_t*)host;
    for (size_t i = 0; i < n; i++) o[i] = tmp[i] ? 1 : 0;
  } else {
    RCU(cudaMemcpyAsync(host, (uint8_t*)base + off, n * elem, cudaMemcpyDeviceToHost, r->stream));
    RCU(cudaStreamSynchronize(r->stream));
  }
  return BCPNN_OK;
}

int bcpnn_recall_write(bcpnn_recall* r, const char* name, int32_t row0, int32_t n_rows, const void* host,
                       size_t bytes) {
  if (!r || !host) return BCPNN_ERR_INVALID;
  if (name && std::string(name) == "counts") return fail(r, BCPNN_ERR_INVALID, "counts are cleared, not written");
  void* base;
  size_t elem;
  int kind;
  int rc = resolve_rows(r, name, row0, n_rows, bytes, &base, &elem, &kind);
  if (rc) return rc;
  RCU(cudaSetDevice(r->d.device));
  const size_t off = (size_t)row0 * r->N * elem, n = (size_t)n_rows * r->N;
  if (kind == 1) {
    std::vector<uint16_t> tmp(n);
    const int8_t* in = (const int8_t*)host;
    for (size_t i = 0; i < n; i++) tmp[i] = in[i] ? 0x3F80u : 0u;
    RCU(cudaMemcpyAsync((uint8_t*)base + off, tmp.data(), n * 2, cudaMemcpyHostToDevice, r->stream));
    RCU(cudaStreamSynchronize(r->stream));
  } else {
    RCU(cudaMemcpyAsync((uint8_t*)base + off, host, n * elem, cudaMemcpyHostToDevice, r->stream));
    RCU(cudaStreamSynchronize(r->stream));
  }
  return BCPNN_OK;
}

int bcpnn_recall_get_stream(const bcpnn_recall* r, void** stream) {
  if (!r || !stream) return BCPNN_ERR_INVALID;
  *stream = (void*)r->stream;
  return BCPNN_OK;
}

int bcpnn_recall_launches(const bcpnn_recall* r, uint64_t* out) {
  if (!r || !out) return BCPNN_ERR_INVALID;
  *out = r->launches;
  return BCPNN_OK;
}

int bcpnn_recall_timing(bcpnn_recall* r, int32_t on) {
  if (!r) return BCPNN_ERR_INVALID;
  r->timing = on != 0;
  r->contraction_ms = 0.0;
  r->contraction_launches = 0;
  return BCPNN_OK;
}

int bcpnn_recall_contraction_time(const bcpnn_recall* r, double* total_ms, uint64_t* n_launches) {
  if (!r || !total_ms || !n_launches) return BCPNN_ERR_INVALID;
  *total_ms = r->contraction_ms;
  *n_launches = r->contraction_launches;
  return BCPNN_OK;
}

const char* bcpnn_recall_last_error(const bcpnn_recall* r) { return r ? r->last_error.c_str() : ""; }

}  // extern "C"
