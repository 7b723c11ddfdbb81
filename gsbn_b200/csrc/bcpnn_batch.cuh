/*
 * bcpnn_batch.cuh -- the batch engine (include/bcpnn_batch.h): many
 * independent single-population networks advanced together by one persistent
 * sm_100a kernel per run.  Compiled in the translation unit of the C ABI
 * (bcpnn_capi.cu includes it), which also holds the device functions of
 * bcpnn_device.cuh it shares.
 *
 * Per tick and per (member, HCU) item, one warp does what gsbn's ProcUpdLazy
 * does for that HCU (ProcUpdLazy.cpp:88-124), in gsbn's order and with its
 * expression trees:
 *   - the delay queue (Proj.cpp:645-664) as arrivals: the previous tick's
 *     spikes of the item's MCUs set, for every slot they feed, the bit of the
 *     destination HCU's arrival ring at the tick the row turns active
 *     (spike at T -> row update at T + 2 + delay, gsbn's exchange -> queue ->
 *     compaction latency);
 *   - population update (Pop.cpp:229-323): support, softmax with the maximum
 *     seeded by the member's MCU 0 (Pop.cpp:270, recomputed by every item from
 *     the previous tick's double-buffered values), spikes from the member's
 *     Philox stream;
 *   - j-traces and bias (Proj.cpp:310-363);
 *   - the active rows in ascending slot order with weights and the ordered
 *     epsc sum (Proj.cpp:365-479, 667-720);
 *   - column units for the tick's spikes (Proj.cpp:481-536), done in phase B
 *     by every warp of the grid after a grid barrier (rows before columns).
 * A second grid barrier ends the tick.  The decay closed forms, tables and the
 * exact reciprocal division are those of the single-network kernels
 * (bcpnn_device.cuh), so every float matches the oracle bit for bit.
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <new>
#include <string>
#include <vector>

#include "bcpnn_batch.h"
#include "bcpnn_device.cuh"

namespace bcpnn {
namespace batch {

constexpr int kRing = 64;     /* arrival ring length in executed ticks (delays <= 31 need < 64) */
constexpr int kMaxM = 64;     /* MCUs per HCU: two per lane */
constexpr int kUnit = 64;     /* slots of one column unit: two per lane */
constexpr int kListCap = 64;  /* active rows gathered per pass of a warp */
constexpr int kCellsPerPass = 64; /* row cells decayed per pass of a warp: two per lane */
constexpr int kCPL = kCellsPerPass / 32; /* cells per lane and pass */
constexpr int kMaxW = 4;      /* arrival words per lane of an HCU: C <= 4096 slots */
/* per-warp shared scratch, in floats: the member's and its tables'
   descriptors, then the item's buffers */
constexpr int kOffMember = 0;
constexpr int kOffTab = 96;
constexpr int kOffAct = 160;
constexpr int kOffPj = kOffAct + kMaxM;
constexpr int kOffPi = kOffPj + kMaxM;
constexpr int kOffList = kOffPi + kListCap;
constexpr int kOffW = kOffList + kListCap;
constexpr int kOffSkip = kOffW + kCellsPerPass;
constexpr int kWarpScratch = kOffSkip + kCellsPerPass / 4;
constexpr unsigned long long kBarrierNs = 2000000000ull;

struct Member {
  int H, M, C, n;
  uint32_t rng_seed;
  float taumdt, wtagain, maxfqdt, igain, wgain, lgbias, snoise;
  float taupdt, ke, kzi, kzj, kepsc, kfti, kftj, eps, eps2, pwgain, bgain;
  float lg_hit, lg_miss;
  float* dsup[2];
  float* act;
  float* epsc[2];
  float* bj[2];
  int8_t* spike;
  int* counter;
  float *pj, *ej, *zj;
  int *ii, *di;
  float *pi, *ei, *zi;
  int* ti;
  float4* cell;
  int* tij;
  float* wij;
  uint32_t* ring; /* [H][kRing][W] */
  int W;
  const int* fo_off;   /* [n + 1] fan-out of each source MCU (CSR) */
  const int* fo_row;   /* destination row h*C + s */
  const int8_t* fo_di; /* its delay */
  const int32_t* lgidx; /* [lg_rows][H] */
  const float* wmask;   /* [wm_rows][H] */
  int lg_rows, wm_rows;
  uint32_t* log; /* [max_ticks][log_words] */
  int log_words;
};

struct Dev {
  int n_members;
  const Member* m;
  const int2* items;     /* (member, hcu) */
  const int* warp_off;   /* [n_warps + 1] */
  const int* warp_items; /* item ids, by warp */
  int n_warps;
  int4* units;           /* [2][unit_cap]: (member, first row, mcu | rows << 16, 0) */
  int unit_cap;
  unsigned int* unit_cnt; /* [2] by tick parity */
  unsigned long long* counters;
  int* err;
  float poisson_hz, dt;
};

struct Run {
  int simstep0, k0, n_ticks;
  float prn, old_prn;
  int lg_row, wm_row;
  const TabRef* tabs; /* [n_members] */
};

__device__ __forceinline__ unsigned long long gtimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void red_release(unsigned int* p, unsigned int v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ unsigned int ld_acquire(const unsigned int* p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

/* bounded grid barrier of the cooperative launch (arrivals counter `bar`,
   zero at launch, must reach `target`); false when it gave up */
__device__ __forceinline__ bool grid_sync(unsigned int* bar, unsigned int target, int* err, int* s_ok) {
  __syncthreads();
  if (threadIdx.x == 0) {
    red_release(bar, 1u);
    const unsigned long long t0 = gtimer();
    int ok = 1;
    while (ld_acquire(bar) < target) {
      if (*(volatile int*)err) {
        ok = 0;
        break;
      }
      if (gtimer() - t0 > kBarrierNs) {
        atomicOr(err, kErrBarrier);
        ok = 0;
        break;
      }
      __nanosleep(32);
    }
    *s_ok = ok;
  }
  __syncthreads();
  return *s_ok != 0;
}

/* the decays with the reciprocal form inline (no call, so no registers saved
   around one) and the exact fallback out of line, which is rare */
__device__ __forceinline__ float4 cell_step_in(float4 c, const TabRef* __restrict__ T, float4 A, float4 B, double2 R0,
                                               double2 R1) {
  float4 f = c;
  if (cell_decay_fast(f, T->k, T->rk, A, B, R0, R1)) return f;
  return cell_step_nl(c, T, A, B, R0, R1);
}

__device__ __forceinline__ float4 row_step_in(float4 r, const TabRef* __restrict__ T, float4 A, float4 B, double2 R0,
                                              double2 R1) {
  float4 f = r;
  if (row_decay_fast(f, T->k, T->rk, A, B, R0, R1)) return f;
  return row_step_nl(r, T, A, B, R0, R1);
}

__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const float w = __shfl_xor_sync(0xffffffffu, v, o);
    v = (w > v) ? w : v;
  }
  return v;
}

/* Active rows ros[0..nr) (ascending slots of HCU h) of member B at tick
   simstep: row traces, cells, weights, ordered epsc sum into e[2] (MCUs lane,
   lane + 32).  kp as the tick's prn gives it.  The loads of the row traces
   and of the first cells go out together, then their table entries. */
template <int kCP>
__device__ __noinline__ void rows_pass(const Member& B, const TabRef* __restrict__ T, int h, const int* ros, int nr,
                                       int simstep, float kp, float* ws_pi, const float* ws_pj, float* ws_w,
                                       int8_t* ws_skip, float e[2], int lane) {
  static_assert(kCP == 1 || kCP == kCPL, "one or kCPL cells per lane and pass");
  const int M = B.M, C = B.C;
  const Coef& k = T->k;
  const int tlen = T->len;
  const int ncell = nr * M;
  /* row traces, Proj.cpp:397-416 (one lane per row; at most kListCap rows),
     kCP rows of a lane at a time */
#pragma unroll 1
  for (int v0 = 0; v0 < 2; v0 += kCP) {
    int ti[kCP], row[kCP];
    float4 tr[kCP];
#pragma unroll
    for (int v = 0; v < kCP; ++v) {
      const int r = lane + 32 * (v0 + v);
      if (r < nr) {
        row[v] = h * C + ros[r];
        ti[v] = B.ti[row[v]];
        tr[v] = make_float4(B.pi[row[v]], B.ei[row[v]], B.zi[row[v]], 0.0f);
      }
    }
    float4 A[kCP], Bt[kCP];
    double2 R0[kCP], R1[kCP];
#pragma unroll
    for (int v = 0; v < kCP; ++v) {
      const int pdt = simstep - ti[v];
      if (lane + 32 * (v0 + v) < nr && pdt > 0 && pdt < tlen) {
        A[v] = T->tab[(size_t)pdt * 4 + 2];
        Bt[v] = T->tab[(size_t)pdt * 4 + 3];
        R0[v] = T->rtab[(size_t)pdt * 4 + 2];
        R1[v] = T->rtab[(size_t)pdt * 4 + 3];
      }
    }
#pragma unroll
    for (int v = 0; v < kCP; ++v) {
      const int r = lane + 32 * (v0 + v);
      if (r >= nr) continue;
      const int pdt = simstep - ti[v];
      if (pdt <= 0) {
        B.zi[row[v]] = tr[v].z + B.kfti;
        B.ti[row[v]] = simstep;
        ws_pi[r] = tr[v].x;
      } else {
        if (pdt >= tlen) {
          load_entry(T->tab, tlen, k, pdt, 2, A[v], Bt[v]);
          recip_part(A[v], Bt[v], 2, R0[v], R1[v]);
        }
        const float4 rt = row_step_in(tr[v], T, A[v], Bt[v], R0[v], R1[v]);
        B.pi[row[v]] = rt.x;
        B.ei[row[v]] = rt.y;
        B.zi[row[v]] = rt.z + B.kfti;
        B.ti[row[v]] = simstep;
        ws_pi[r] = rt.x;
      }
    }
  }
  __syncwarp();
  /* cells, Proj.cpp:418-478, 32*kCP at a time, kCP per lane */
  constexpr int kPass = 32 * kCP;
  for (int b0 = 0; b0 < ncell; b0 += kPass) {
    int tv[kCP];
    float4 cv[kCP];
    float wv[kCP];
    size_t index[kCP];
    bool ok[kCP];
#pragma unroll
    for (int u = 0; u < kCP; ++u) {
      const int c = b0 + u * 32 + lane;
      ok[u] = c < ncell;
      if (ok[u]) {
        const int r = c / M, j = c - r * M;
        index[u] = (size_t)(h * C + ros[r]) * M + j;
        /* other warps' column units of the previous tick wrote these */
        tv[u] = __ldcg(B.tij + index[u]);
        cv[u] = __ldcg(B.cell + index[u]);
        wv[u] = B.wij[index[u]];
      }
    }
    float4 tA[kCP], tB[kCP];
    double2 tR0[kCP], tR1[kCP];
#pragma unroll
    for (int u = 0; u < kCP; ++u) {
      const int pdt = simstep - tv[u];
      if (ok[u] && pdt > 0 && pdt < tlen) {
        tA[u] = T->tab[(size_t)pdt * 4 + 0];
        tB[u] = T->tab[(size_t)pdt * 4 + 1];
        tR0[u] = T->rtab[(size_t)pdt * 4 + 0];
        tR1[u] = T->rtab[(size_t)pdt * 4 + 1];
      }
    }
#pragma unroll
    for (int u = 0; u < kCP; ++u) {
      if (!ok[u]) continue;
      const int c = b0 + u * 32 + lane;
      const int r = c / M, j = c - r * M;
      const int pdt = simstep - tv[u];
      float4 q = cv[u];
      if (pdt <= 0) {
        q.z += B.kfti;
        B.cell[index[u]] = q;
        B.tij[index[u]] = simstep;
        ws_skip[c - b0] = 1;
      } else {
        float4 A = tA[u], Bt = tB[u];
        double2 R0 = tR0[u], R1 = tR1[u];
        if (pdt >= tlen) {
          load_entry(T->tab, tlen, k, pdt, 0, A, Bt);
          recip_part(A, Bt, 0, R0, R1);
        }
        q = cell_step_in(q, T, A, Bt, R0, R1);
        q.z = q.z + B.kfti;
        B.cell[index[u]] = q;
        B.tij[index[u]] = simstep;
        float w;
        if (kp != 0.0f) {
          w = B.pwgain * dev_logf(div_rn(q.x + B.eps2, (ws_pi[r] + B.eps) * (ws_pj[j] + B.eps)));
          B.wij[index[u]] = w;
        } else {
          w = wv[u];
        }
        ws_w[c - b0] = w;
        ws_skip[c - b0] = 0;
      }
    }
    __syncwarp();
    /* epsc[j] += w over the rows in ascending order (Proj.cpp:466-477) */
#pragma unroll
    for (int jj = 0; jj < 2; ++jj) {
      const int j = lane + 32 * jj;
      if (j >= M) continue;
      for (int c = (b0 / M) * M + j; c < min(ncell, b0 + kPass); c += M) {
        if (c < b0) continue;
        if (!ws_skip[c - b0]) e[jj] += ws_w[c - b0];
      }
    }
    __syncwarp();
  }
}

/* gather the active slots of HCU h (the arrival-ring words `words`, already
   loaded: word g*32 + lane in words[g]) into ascending passes of at most
   kListCap rows; every pass runs rows_pass.  Returns the number of rows. */
template <int kCP>
__device__ __forceinline__ int item_rows(const Member& B, const TabRef* __restrict__ T, int h, int simstep, float kp,
                                         const uint32_t words[kMaxW], int* ws_list, float* ws_pi, const float* ws_pj,
                                         float* ws_w, int8_t* ws_skip, float e[2], int lane) {
  int nl = 0, total_rows = 0;
#pragma unroll
  for (int g = 0; g < kMaxW; ++g) {
    if (g * 32 >= B.W) break;
    const uint32_t word = words[g];
    const int cnt = __popc(word);
    int incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    const int excl = incl - cnt;
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    total_rows += total;
    for (int done = 0; done < total;) {
      const int room = kListCap - nl;
      const int take = min(room, total - done);
      uint32_t wbits = word;
      int p = excl;
      while (wbits) {
        const int b = __ffs(wbits) - 1;
        wbits &= wbits - 1;
        if (p >= done && p < done + take) ws_list[nl + p - done] = (g * 32 + lane) * 32 + b;
        ++p;
      }
      __syncwarp();
      nl += take;
      done += take;
      if (nl == kListCap) {
        rows_pass<kCP>(B, T, h, ws_list, nl, simstep, kp, ws_pi, ws_pj, ws_w, ws_skip, e, lane);
        nl = 0;
      }
    }
  }
  if (nl) rows_pass<kCP>(B, T, h, ws_list, nl, simstep, kp, ws_pi, ws_pj, ws_w, ws_skip, e, lane);
  return total_rows;
}

/* one tick of one (member, HCU) item, phase A, by one warp.  The member's
   and its tables' descriptors are copied to the warp's shared scratch first;
   then every load the tick needs that depends on nothing else goes out
   together (previous-tick state of the HCU's MCUs, stimulus, the softmax
   seed's terms, the HCU's arrival words of this tick). */
template <int kCP>
__device__ __forceinline__ void item_tick(const Dev& D, const Run& R, int n, int h, int it, float* ws,
                                       unsigned long long& rows_acc, unsigned long long& cols_acc) {
  const int lane = threadIdx.x & 31;
  {
    const uint32_t* src = (const uint32_t*)&D.m[n];
    uint32_t* dst = (uint32_t*)(ws + kOffMember);
    for (int k = lane; k < (int)(sizeof(Member) / 4); k += 32) dst[k] = src[k];
    const uint32_t* tsrc = (const uint32_t*)&R.tabs[n];
    uint32_t* tdst = (uint32_t*)(ws + kOffTab);
    for (int k = lane; k < (int)(sizeof(TabRef) / 4); k += 32) tdst[k] = tsrc[k];
  }
  __syncwarp();
  const Member& B = *(const Member*)(ws + kOffMember);
  const TabRef* T = (const TabRef*)(ws + kOffTab);
  const int M = B.M, C = B.C, H = B.H, base = h * M;
  const int simstep = R.simstep0 + it, kk = R.k0 + it;
  const int cur = kk & 1, prev = cur ^ 1;
  float* ws_act = ws + kOffAct;
  float* ws_pj = ws + kOffPj;
  float* ws_pi = ws + kOffPi;
  int* ws_list = (int*)(ws + kOffList);
  float* ws_w = ws + kOffW;
  int8_t* ws_skip = (int8_t*)(ws + kOffSkip);

  /* every independent load of the tick at once */
  const int lgrow = min(R.lg_row, B.lg_rows - 1), wmrow = min(R.wm_row, B.wm_rows - 1);
  const int want = B.lgidx[(size_t)lgrow * H + h];
  const float wm = B.wmask[(size_t)wmrow * H + h];
  float dsp[2], bjp[2], esp[2], pjv[2], ejv[2], zjv[2];
#pragma unroll
  for (int jj = 0; jj < 2; ++jj) {
    const int j = lane + 32 * jj;
    if (j < M) {
      const int idx = base + j;
      dsp[jj] = B.dsup[prev][idx];
      bjp[jj] = B.bj[prev][idx];
      esp[jj] = B.epsc[prev][idx];
      pjv[jj] = B.pj[idx];
      ejv[jj] = B.ej[idx];
      zjv[jj] = B.zj[idx];
    }
  }
  float sd = 0.0f, sb = 0.0f, se = 0.0f, sw = 0.0f;
  int sl = 0;
  if (h != 0 && lane == 0) {
    /* HCU 0's item wrote these in the previous tick, on another SM */
    sd = __ldcg(B.dsup[prev]);
    sb = __ldcg(B.bj[prev]);
    se = __ldcg(B.epsc[prev]);
    sl = B.lgidx[(size_t)lgrow * H];
    sw = B.wmask[(size_t)wmrow * H];
  }
  uint32_t words[kMaxW];
  uint32_t* rw = B.ring + ((size_t)h * kRing + (unsigned)kk % kRing) * B.W;
#pragma unroll
  for (int g = 0; g < kMaxW; ++g) {
    words[g] = 0u;
    if (g * 32 + lane < B.W) words[g] = __ldcg(rw + g * 32 + lane);
  }
#pragma unroll
  for (int g = 0; g < kMaxW; ++g)
    if (words[g]) rw[g * 32 + lane] = 0u;

  /* population update, Pop.cpp:229-323 */
  float dn[2];
#pragma unroll
  for (int jj = 0; jj < 2; ++jj) {
    const int j = lane + 32 * jj;
    dn[jj] = 0.0f;
    if (j < M) {
      const int idx = base + j;
      float wsup = 0.0f;
      wsup += bjp[jj] + esp[jj];
      float noise = 0.0f;
      if (B.snoise != 0.0f) noise = B.snoise * dev_normal01(B.rng_seed, 0u, (uint32_t)simstep, (uint32_t)idx);
      float sup = B.lgbias + B.igain * (want == j ? B.lg_hit : B.lg_miss) + noise;
      sup += (B.wgain * wm) * wsup;
      dn[jj] = dsp[jj] + (sup - dsp[jj]) * B.taumdt;
    }
  }
  /* the softmax maximum is seeded with the member's MCU 0 (Pop.cpp:270) */
  float seed0;
  if (h == 0) {
    seed0 = __shfl_sync(0xffffffffu, dn[0], 0);
  } else {
    float s0 = 0.0f;
    if (lane == 0) {
      float wsup = 0.0f;
      wsup += sb + se;
      float noise = 0.0f;
      if (B.snoise != 0.0f) noise = B.snoise * dev_normal01(B.rng_seed, 0u, (uint32_t)simstep, 0u);
      float sup = B.lgbias + B.igain * (sl == 0 ? B.lg_hit : B.lg_miss) + noise;
      sup += (B.wgain * sw) * wsup;
      s0 = sd + (sup - sd) * B.taumdt;
    }
    seed0 = __shfl_sync(0xffffffffu, s0, 0);
  }
  float tmax = seed0;
#pragma unroll
  for (int jj = 0; jj < 2; ++jj)
    if (lane + 32 * jj < M) tmax = (dn[jj] > tmax) ? dn[jj] : tmax;
  const float maxdsup = warp_max(tmax);
  const float maxact = dev_expf(B.wtagain * maxdsup);
  float a[2];
#pragma unroll
  for (int jj = 0; jj < 2; ++jj) {
    const int j = lane + 32 * jj;
    a[jj] = 0.0f;
    if (j < M) {
      a[jj] = dev_expf(B.wtagain * (dn[jj] - maxdsup));
      if (maxact < 1.0f) a[jj] *= maxact;
      ws_act[j] = a[jj];
    }
  }
  __syncwarp();
  float vs = 0.0f;
  if (lane == 0) {
    float v = 0.0f; /* serial, in MCU order (Pop.cpp:281-293) */
    for (int j = 0; j < M; ++j) v += ws_act[j];
    vs = v;
  }
  const float vsum = __shfl_sync(0xffffffffu, vs, 0);
  const float pr = D.poisson_hz * D.dt;
  int8_t spk[2];
  uint32_t* log = B.log + (size_t)it * B.log_words;
#pragma unroll
  for (int jj = 0; jj < 2; ++jj) {
    const int j = lane + 32 * jj;
    spk[jj] = 0;
    if (j < M) {
      const int idx = base + j;
      float av = a[jj];
      if (vsum > 1.0f) av /= vsum;
      const float u = bx_uniform01(B.rng_seed, 0u, (uint32_t)simstep, (uint32_t)idx);
      int8_t sv = (int8_t)(u < av * B.maxfqdt);
      if (D.poisson_hz > 0.0f) {
        const float up = bx_uniform01_poisson(B.rng_seed, 0u, (uint32_t)simstep, (uint32_t)idx);
        if (up < pr) sv = 1;
      }
      spk[jj] = sv;
      B.counter[idx] += sv;
      B.spike[idx] = sv;
      B.act[idx] = av;
      B.dsup[cur][idx] = dn[jj];
      if (sv) atomicOr(&log[idx >> 5], 1u << (idx & 31));
    }
  }

  /* j-traces and bias, Proj.cpp:310-363 */
  const float kp = B.taupdt * R.prn;
  float e[2];
#pragma unroll
  for (int jj = 0; jj < 2; ++jj) {
    const int j = lane + 32 * jj;
    e[jj] = 0.0f;
    if (j < M) {
      const int idx = base + j;
      float pj = pjv[jj], ej = ejv[jj], zj = zjv[jj];
      float ev = esp[jj];
      ev *= (1 - B.kepsc);
      pj += (ej - pj) * kp;
      ej += (zj - ej) * B.ke;
      zj *= (1 - B.kzj);
      if (spk[jj] > 0) zj += B.kftj;
      B.bj[cur][idx] = (kp != 0.0f) ? B.bgain * dev_logf(pj + B.eps) : bjp[jj];
      B.pj[idx] = pj;
      B.ej[idx] = ej;
      B.zj[idx] = zj;
      ws_pj[j] = pj;
      e[jj] = ev;
    }
  }
  __syncwarp();

  /* the active rows of this tick, ascending (Proj.cpp:365-479, 667-720) */
  const int nrows = item_rows<kCP>(B, T, h, simstep, kp, words, ws_list, ws_pi, ws_pj, ws_w, ws_skip, e, lane);
#pragma unroll
  for (int jj = 0; jj < 2; ++jj) {
    const int j = lane + 32 * jj;
    if (j < M) B.epsc[cur][base + j] = e[jj];
  }

  /* units of phase B for this tick's spikes: per spike, its column in
     slot pieces (Proj.cpp:481-536) and its fan-out (the delay queue of the
     next tick, as arrivals); one counter add for all of them */
  const unsigned m0 = __ballot_sync(0xffffffffu, spk[0] > 0), m1 = __ballot_sync(0xffffffffu, spk[1] > 0);
  const int nspk = __popc(m0) + __popc(m1);
  if (nspk > 0) {
    const int parts = (C + kUnit - 1) / kUnit + 1;
    unsigned int pos = 0;
    if (lane == 0) pos = atomicAdd(D.unit_cnt + cur, (unsigned int)(parts * nspk));
    pos = __shfl_sync(0xffffffffu, pos, 0);
    if (pos + (unsigned)(parts * nspk) > (unsigned)D.unit_cap) {
      if (lane == 0) atomicOr(D.err, kErrIndex);
    } else {
      int4* units = D.units + (size_t)cur * D.unit_cap;
      for (int k = lane; k < parts * nspk; k += 32) {
        const int i = k / parts, p = k - i * parts;
        /* the i-th spiking MCU, in MCU order */
        unsigned mm = m0;
        int j = 0, left = i;
        if (left >= __popc(m0)) {
          left -= __popc(m0);
          mm = m1;
          j = 32;
        }
        for (; left > 0; --left) mm &= mm - 1;
        j += __ffs(mm) - 1;
        if (p < parts - 1) {
          const int rows = min(kUnit, C - p * kUnit);
          units[pos + k] = make_int4(n, h * C + p * kUnit, j | (rows << 16), 0);
        } else {
          units[pos + k] = make_int4(n, base + j, 0, 1); /* fan-out of MCU base + j */
        }
      }
    }
  }
  if (lane == 0) {
    rows_acc += (unsigned long long)nrows * M;
    cols_acc += (unsigned long long)nspk * C;
  }
}

/* a unit of phase B.  w == 0: column unit, slots [row0, row0 + rows) of
   member n's column j (Proj.cpp:481-536); every cell of the tick's active
   rows already has tij = simstep (rows ran in phase A), so it only gains
   kftj.  w == 1: the fan-out of source MCU y, whose spike of this tick turns
   each slot it feeds active at kk + 2 + delay (the delay queue, as events). */
template <int kV>
__device__ __noinline__ void column_unit(const Dev& D, const Run& R, int4 u, int simstep, int kk) {
  const Member& B = D.m[u.x];
  const int lane = threadIdx.x & 31;
  if (u.w == 1) {
    const int src = u.y, C = B.C;
    const int e0 = B.fo_off[src], e1 = B.fo_off[src + 1];
    for (int e = e0 + lane; e < e1; e += 32) {
      const int row = B.fo_row[e];
      const int hd = row / C, s = row - hd * C;
      const unsigned slot = (unsigned)(kk + 2 + B.fo_di[e]) % kRing;
      atomicOr(B.ring + ((size_t)hd * kRing + slot) * B.W + (s >> 5), 1u << (s & 31));
    }
    return;
  }
  const TabRef* T = &R.tabs[u.x];
  const int row0 = u.y, j = u.z & 0xffff, rows = u.z >> 16, M = B.M;
  const int tlen = T->len;
  /* kV of the lane's kUnit/32 cells at a time: their loads issued together */
#pragma unroll 1
  for (int v0 = 0; v0 < kUnit / 32; v0 += kV) {
    size_t index[kV];
    int tv[kV];
    float4 cv[kV];
    bool ok[kV];
#pragma unroll
    for (int v = 0; v < kV; ++v) {
      const int s = (v0 + v) * 32 + lane;
      ok[v] = false;
      if (s < rows) {
        const int row = row0 + s;
        index[v] = (size_t)row * M + j;
        ok[v] = B.ii[row] >= 0;
        /* the owner's rows of this tick (phase A, another SM) wrote these */
        tv[v] = __ldcg(B.tij + index[v]);
        cv[v] = __ldcg(B.cell + index[v]);
      }
    }
    float4 tA[kV], tB[kV];
    double2 tR0[kV], tR1[kV];
#pragma unroll
    for (int v = 0; v < kV; ++v) {
      const int pdt = simstep - tv[v];
      if (ok[v] && pdt > 0 && pdt < tlen) {
        tA[v] = T->tab[(size_t)pdt * 4 + 0];
        tB[v] = T->tab[(size_t)pdt * 4 + 1];
        tR0[v] = T->rtab[(size_t)pdt * 4 + 0];
        tR1[v] = T->rtab[(size_t)pdt * 4 + 1];
      }
    }
#pragma unroll
    for (int v = 0; v < kV; ++v) {
      if (!ok[v]) continue;
      const int pdt = simstep - tv[v];
      float4 q = cv[v];
      if (pdt <= 0) {
        q.w += B.kftj;
      } else {
        float4 A = tA[v], Bt = tB[v];
        double2 R0 = tR0[v], R1 = tR1[v];
        if (pdt >= tlen) {
          load_entry(T->tab, tlen, T->k, pdt, 0, A, Bt);
          recip_part(A, Bt, 0, R0, R1);
        }
        q = cell_step_in(q, T, A, Bt, R0, R1);
        q.w = q.w + B.kftj;
      }
      B.cell[index[v]] = q;
      B.tij[index[v]] = simstep;
    }
  }
}

/* kThreads 512: 16 warps per SM, 128 registers a thread (the column decays
   then keep some values in local memory); 384: 12 warps with 168 registers;
   256: 8 warps per SM with room for every value in registers.  The tuner
   times them all. */
template <int kThreads>
__global__ void __launch_bounds__(kThreads, 1) batch_kernel(const Dev* __restrict__ dg, const Run* __restrict__ rg,
                                                           unsigned int* bar) {
  extern __shared__ __align__(16) float wsm[];
  __shared__ Dev D;
  __shared__ Run R;
  __shared__ int s_ok;
  if (threadIdx.x == 0) {
    D = *dg;
    R = *rg;
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wpc = blockDim.x >> 5;
  const int gwarp = blockIdx.x * wpc + warp;
  const int nw = gridDim.x * wpc;
  float* ws = wsm + (size_t)warp * kWarpScratch;
  unsigned long long rows_acc = 0, cols_acc = 0;
  unsigned int arrivals = 0;
  const int i0 = gwarp < D.n_warps ? D.warp_off[gwarp] : 0;
  const int i1 = gwarp < D.n_warps ? D.warp_off[gwarp + 1] : 0;
#ifdef BCPNN_PHASE_PROBE
  /* per CTA: [0] phase A cycles summed over warps and ticks, [1] the slowest
     warp's, summed over ticks, [2], [3] the same for phase B, [4], [5] the
     waits of the two barriers (thread 0), [6] ticks, [7] units done, [8]
     items done */
  if (threadIdx.x < kProbeSlots) g_probe_smem[threadIdx.x] = 0;
  __shared__ unsigned long long s_pmax[2];
  __syncthreads();
#endif
  for (int it = 0; it < R.n_ticks; ++it) {
    const int simstep = R.simstep0 + it, kk = R.k0 + it;
#ifdef BCPNN_PHASE_PROBE
    long long pt0 = clock64();
    if (threadIdx.x == 0) s_pmax[0] = s_pmax[1] = 0;
    __syncthreads();
#endif
    for (int e = i0; e < i1; ++e) {
      const int2 item = D.items[D.warp_items[e]];
      item_tick<(kThreads >= 384) ? 1 : kCPL>(D, R, item.x, item.y, it, ws, rows_acc, cols_acc);
    }
#ifdef BCPNN_PHASE_PROBE
    if (lane == 0) {
      const unsigned long long d = (unsigned long long)(clock64() - pt0);
      atomicAdd(&g_probe_smem[0], d);
      atomicMax(&s_pmax[0], d);
      atomicAdd(&g_probe_smem[8], (unsigned long long)(i1 - i0));
    }
    long long pt1 = clock64();
#endif
    arrivals += gridDim.x;
    if (!grid_sync(bar, arrivals, D.err, &s_ok)) return;
#ifdef BCPNN_PHASE_PROBE
    if (threadIdx.x == 0) g_probe_smem[4] += (unsigned long long)(clock64() - pt1);
    long long pt2 = clock64();
#endif
    /* phase B: the tick's column units over every warp of the grid */
    /* a counter past the ring's capacity (reported in phase A) is clamped */
    const unsigned int nu = min(__ldcg(D.unit_cnt + (kk & 1)), (unsigned int)D.unit_cap);
    const int4* units = D.units + (size_t)(kk & 1) * D.unit_cap;
    for (unsigned int u = gwarp; u < nu; u += nw)
      column_unit<(kThreads >= 384) ? 1 : kUnit / 32>(D, R, __ldcg(units + u), simstep, kk);
#ifdef BCPNN_PHASE_PROBE
    if (lane == 0) {
      const unsigned long long d = (unsigned long long)(clock64() - pt2);
      atomicAdd(&g_probe_smem[2], d);
      atomicMax(&s_pmax[1], d);
      if (gwarp < (int)nu) atomicAdd(&g_probe_smem[7], (unsigned long long)((nu - gwarp + nw - 1) / nw));
    }
    long long pt3 = clock64();
#endif
    /* the other parity's counter is free again (its units were done in the
       previous tick's phase B); the next tick appends to it */
    if (blockIdx.x == 0 && threadIdx.x == 0) D.unit_cnt[(kk + 1) & 1] = 0u;
    arrivals += gridDim.x;
    if (!grid_sync(bar, arrivals, D.err, &s_ok)) return;
#ifdef BCPNN_PHASE_PROBE
    if (threadIdx.x == 0) {
      g_probe_smem[5] += (unsigned long long)(clock64() - pt3);
      g_probe_smem[1] += s_pmax[0];
      g_probe_smem[3] += s_pmax[1];
      g_probe_smem[6] += 1;
    }
#endif
  }
#ifdef BCPNN_PHASE_PROBE
  __syncthreads();
  if (threadIdx.x < kProbeSlots && blockIdx.x < kProbeCtas)
    atomicAdd(&g_phase_probe[blockIdx.x * kProbeSlots + threadIdx.x], g_probe_smem[threadIdx.x]);
#endif
  if (lane == 0) {
    if (rows_acc) atomicAdd(&D.counters[0], rows_acc);
    if (cols_acc) atomicAdd(&D.counters[1], cols_acc);
  }
}

/* all-cells catch-up at a change of prn (Proj.cpp:209-308, 538-588) over
   every member: rows first (their pi feed the weights), then cells; flat
   indices, the member found in a prefix table */
__device__ __forceinline__ int find_member(const unsigned long long* off, int n, unsigned long long x) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (off[mid] <= x) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

__global__ void batch_all_rows_kernel(const Dev* __restrict__ dg, const Run* __restrict__ rg,
                                      const unsigned long long* row_off, unsigned long long total) {
  const Dev& D = *dg;
  const Run& R = *rg;
  const int simstep = R.simstep0 - 1;
  for (unsigned long long x = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; x < total;
       x += (unsigned long long)gridDim.x * blockDim.x) {
    const int n = find_member(row_off, D.n_members, x);
    const Member& B = D.m[n];
    const TabRef& T = R.tabs[n];
    const int r = (int)(x - row_off[n]);
    const int pdt = simstep - B.ti[r];
    if (pdt > 0) {
      const Coef k = make_coef(B.taupdt * R.old_prn, B.ke, B.kzi, B.kzj, 0);
      float pi = B.pi[r], ei = B.ei[r], zi = B.zi[r];
      float4 A, Bt;
      load_entry(T.tab_old, T.old_len, k, pdt, 2, A, Bt);
      row_decay(pi, ei, zi, k, A, Bt);
      B.pi[r] = pi;
      B.ei[r] = ei;
      B.zi[r] = zi;
      B.ti[r] = simstep;
    }
  }
}

__global__ void batch_all_cells_kernel(const Dev* __restrict__ dg, const Run* __restrict__ rg,
                                       const unsigned long long* cell_off, unsigned long long total) {
  const Dev& D = *dg;
  const Run& R = *rg;
  const int simstep = R.simstep0 - 1;
  for (unsigned long long x = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; x < total;
       x += (unsigned long long)gridDim.x * blockDim.x) {
    const int n = find_member(cell_off, D.n_members, x);
    const Member& B = D.m[n];
    const TabRef& T = R.tabs[n];
    const size_t c = (size_t)(x - cell_off[n]);
    const int pdt = simstep - B.tij[c];
    if (pdt <= 0) {
      B.tij[c] = simstep;
    } else {
      const float kp = B.taupdt * R.old_prn;
      const Coef k = make_coef(kp, B.ke, B.kzi, B.kzj, 0);
      float4 q = B.cell[c];
      float4 A, Bt;
      load_entry(T.tab_old, T.old_len, k, pdt, 0, A, Bt);
      cell_decay(q.x, q.y, q.z, q.w, k, A, Bt);
      B.cell[c] = q;
      B.tij[c] = simstep;
      if (kp != 0.0f) {
        const int r = (int)(c / B.M);
        const int j = (int)(c - (size_t)r * B.M);
        const int h = r / B.C;
        B.wij[c] = B.pwgain * dev_logf((q.x + B.eps2) / ((B.pi[r] + B.eps) * (B.pj[h * B.M + j] + B.eps)));
      }
    }
  }
}

template <typename T>
__global__ void bfill_kernel(T* p, size_t n, T v) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) p[i] = v;
}

}  // namespace batch
}  // namespace bcpnn

/* ======================================================================== */
/* host side                                                                 */
/* ======================================================================== */

using namespace bcpnn;
using namespace bcpnn::batch;

namespace {

struct TSlot {
  float4* ptr = nullptr;
  double2* rptr = nullptr;
  int len = 0;
};

struct MemberHost {
  bcpnn_batch_member d;
  int H, M, C, n;
  bool conn = false, stim = false;
  std::vector<int32_t> ii, di; /* host copy (state reads of ii/di, fan-out) */
};

}  // namespace

struct bcpnn_batch {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::vector<void*> allocs;
  std::vector<MemberHost> mh;
  std::vector<Member> hm;
  Member* d_m = nullptr;
  Dev h{};
  Dev* d_dev = nullptr;
  Run rp{};
  Run* d_run = nullptr;
  std::vector<TabRef> tabs;
  TabRef* d_tabs = nullptr;
  std::map<std::vector<uint32_t>, TSlot> tcache;
  std::vector<int2> items;
  int2* d_items = nullptr;
  int* d_warp_off = nullptr;
  int* d_warp_items = nullptr;
  int threads = 512, grid = 0, n_warps = 0;
  size_t smem = 0;
  int lpt[3] = {64, 4, 1};
  unsigned int* bar = nullptr;
  unsigned long long* d_row_off = nullptr;
  unsigned long long* d_cell_off = nullptr;
  unsigned long long total_rows = 0, total_cells = 0;
  int max_ticks = 0, last_ticks = 0;
  int64_t k_total = 0;
  uint64_t launches = 0;
  int lg_row = 0, wm_row = 0;
  unsigned long long all_cells = 0;
  std::string err;
  ~bcpnn_batch() {
    if (device >= 0) cudaSetDevice(device);
    for (auto& kv : tcache)
      if (kv.second.ptr) cudaFree(kv.second.ptr);
    for (void* p : allocs) cudaFree(p);
    if (d_warp_off) cudaFree(d_warp_off);
    if (d_warp_items) cudaFree(d_warp_items);
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace {

int bfail(bcpnn_batch* b, int code, const std::string& msg) {
  if (b) b->err = msg;
  return code;
}

#define BCU(call)                                                                              \
  do {                                                                                         \
    cudaError_t e_ = (call);                                                                   \
    if (e_ != cudaSuccess) return bfail(b, BCPNN_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

template <typename T>
int balloc(bcpnn_batch* b, T** p, size_t count) {
  *p = nullptr;
  if (count == 0) count = 1;
  BCU(cudaMalloc((void**)p, count * sizeof(T)));
  b->allocs.push_back((void*)*p);
  return BCPNN_OK;
}

int bgrid(size_t n) { return (int)std::max<size_t>(1, std::min<size_t>((n + 255) / 256, 148 * 16)); }

template <typename T>
int bset(bcpnn_batch* b, T* p, size_t n, T v) {
  if (!n) return BCPNN_OK;
  bfill_kernel<T><<<bgrid(n), 256, 0, b->stream>>>(p, n, v);
  BCU(cudaGetLastError());
  b->launches++;
  return BCPNN_OK;
}

int bzero(bcpnn_batch* b, void* p, size_t bytes) {
  if (bytes) BCU(cudaMemsetAsync(p, 0, bytes, b->stream));
  return BCPNN_OK;
}

bool finite_pos(float x) { return x > 0.0f && x <= 3.4028234663852886e38f; }

/* gsbn's initial values of one member (Pop.cpp:59-65, Proj.cpp:88-105) */
int reset_member(bcpnn_batch* b, int n) {
  const MemberHost& Mh = b->mh[n];
  Member& B = b->hm[n];
  const size_t N = B.n, R = (size_t)B.H * B.C, cells = R * B.M;
  int rc;
  for (int p = 0; p < 2; ++p) {
    if ((rc = bset(b, B.dsup[p], N, (float)bx_log_d(1.0 / B.M)))) return rc;
    if ((rc = bzero(b, B.epsc[p], N * sizeof(float)))) return rc;
    if ((rc = bzero(b, B.bj[p], N * sizeof(float)))) return rc;
  }
  if ((rc = bset(b, B.act, N, (float)(1.0 / B.M)))) return rc;
  if ((rc = bzero(b, B.spike, N))) return rc;
  if ((rc = bzero(b, B.counter, N * sizeof(int)))) return rc;
  if ((rc = bset(b, B.pj, N, (float)(1.0 / B.M)))) return rc;
  if ((rc = bzero(b, B.ej, N * sizeof(float)))) return rc;
  if ((rc = bzero(b, B.zj, N * sizeof(float)))) return rc;
  if ((rc = bset(b, B.pi, R, (float)(1.0 / B.C)))) return rc;
  if ((rc = bzero(b, B.ei, R * sizeof(float)))) return rc;
  if ((rc = bzero(b, B.zi, R * sizeof(float)))) return rc;
  if ((rc = bzero(b, B.ti, R * sizeof(int)))) return rc;
  if ((rc = bset(b, B.cell, cells, make_float4((float)(1.0 / B.C / B.M), 0.0f, 0.0f, 0.0f)))) return rc;
  if ((rc = bzero(b, B.tij, cells * sizeof(int)))) return rc;
  if ((rc = bzero(b, B.wij, cells * sizeof(float)))) return rc;
  if ((rc = bzero(b, B.ring, (size_t)B.H * kRing * B.W * sizeof(uint32_t)))) return rc;
  (void)Mh;
  return BCPNN_OK;
}

/* decay tables for (kp, ke, kzi, kzj), shared by every member with those
   constants; grown to `need` entries */
int table_for(bcpnn_batch* b, float kp, float ke, float kzi, float kzj, int need, TSlot** out) {
  std::vector<uint32_t> key = {bx_fbits(kp), bx_fbits(ke), bx_fbits(kzi), bx_fbits(kzj)};
  TSlot& T = b->tcache[key];
  if (T.len < need) {
    int cap = 1024;
    while (cap < need) cap *= 2;
    if (T.ptr) BCU(cudaFree(T.ptr));
    T.ptr = nullptr;
    BCU(cudaMalloc((void**)&T.ptr, (size_t)cap * 4 * (sizeof(float4) + sizeof(double2))));
    T.rptr = (double2*)(T.ptr + (size_t)cap * 4);
    build_table_kernel<<<bgrid(cap), 256, 0, b->stream>>>(T.ptr, T.rptr, cap, kp, ke, kzi, kzj);
    BCU(cudaGetLastError());
    b->launches++;
    T.len = cap;
  }
  *out = &T;
  return BCPNN_OK;
}

/* the batch kernel instance of a CTA size (256, 384 or 512 threads) */
const void* kernel_for(int threads) {
  switch (threads) {
    case 256:
      return (const void*)batch_kernel<256>;
    case 384:
      return (const void*)batch_kernel<384>;
    default:
      return (const void*)batch_kernel<512>;
  }
}

/* longest-processing-time assignment of the items to the warps of the grid */
int schedule_items(bcpnn_batch* b) {
  const int wpc = b->threads / 32;
  const size_t smem = (size_t)wpc * kWarpScratch * sizeof(float);
  int per_sm = 0;
  const void* fn = kernel_for(b->threads);
  BCU(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  BCU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, b->threads, smem));
  int sms = 0;
  BCU(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device));
  if (per_sm < 1) return bfail(b, BCPNN_ERR_STATE, "batch kernel does not fit on an SM");
  b->grid = per_sm * sms;
  b->smem = smem;
  b->n_warps = b->grid * wpc;
  std::vector<std::pair<long long, int>> order;
  for (size_t i = 0; i < b->items.size(); ++i) {
    const Member& B = b->hm[b->items[i].x];
    const long long cost = (long long)b->lpt[0] + (long long)b->lpt[1] * B.M + (long long)b->lpt[2] * ((B.C + 31) / 32);
    order.push_back({-cost, (int)i});
  }
  std::sort(order.begin(), order.end());
  /* min-heap of (load, warp) */
  std::vector<std::pair<long long, int>> heap;
  for (int w = 0; w < b->n_warps; ++w) heap.push_back({0, w});
  std::make_heap(heap.begin(), heap.end(), std::greater<std::pair<long long, int>>());
  std::vector<std::vector<int>> per(b->n_warps);
  for (auto& o : order) {
    std::pop_heap(heap.begin(), heap.end(), std::greater<std::pair<long long, int>>());
    auto& top = heap.back();
    per[top.second].push_back(o.second);
    top.first += -o.first;
    std::push_heap(heap.begin(), heap.end(), std::greater<std::pair<long long, int>>());
  }
  std::vector<int> off(b->n_warps + 1, 0), flat;
  for (int w = 0; w < b->n_warps; ++w) {
    /* a warp's items in member order, HCU order (neighbouring state) */
    std::sort(per[w].begin(), per[w].end());
    off[w + 1] = off[w] + (int)per[w].size();
    flat.insert(flat.end(), per[w].begin(), per[w].end());
  }
  if (b->d_warp_off) cudaFree(b->d_warp_off);
  if (b->d_warp_items) cudaFree(b->d_warp_items);
  b->d_warp_off = nullptr;
  b->d_warp_items = nullptr;
  BCU(cudaMalloc((void**)&b->d_warp_off, off.size() * sizeof(int)));
  BCU(cudaMalloc((void**)&b->d_warp_items, std::max<size_t>(1, flat.size()) * sizeof(int)));
  BCU(cudaMemcpy(b->d_warp_off, off.data(), off.size() * sizeof(int), cudaMemcpyHostToDevice));
  if (!flat.empty()) BCU(cudaMemcpy(b->d_warp_items, flat.data(), flat.size() * sizeof(int), cudaMemcpyHostToDevice));
  b->h.warp_off = b->d_warp_off;
  b->h.warp_items = b->d_warp_items;
  b->h.n_warps = b->n_warps;
  BCU(cudaMemcpy(b->d_dev, &b->h, sizeof(Dev), cudaMemcpyHostToDevice));
  return BCPNN_OK;
}

int check_device_error(bcpnn_batch* b) {
  int e = 0;
  BCU(cudaMemcpy(&e, b->h.err, sizeof(int), cudaMemcpyDeviceToHost));
  if (e) {
    std::string why;
    if (e & kErrBarrier) why += " a grid barrier wait of the batch kernel timed out;";
    if (e & kErrIndex) why += " the column-unit ring overflowed;";
    return bfail(b, BCPNN_ERR_DEVICE, "batch kernel reported error word " + std::to_string(e) + ":" + why);
  }
  return BCPNN_OK;
}

}  // namespace

extern "C" {

int bcpnn_batch_create(const bcpnn_batch_desc* desc, bcpnn_batch** out) {
  if (!out) return BCPNN_ERR_INVALID;
  *out = nullptr;
  if (!desc || desc->n_members <= 0 || !desc->members || !finite_pos(desc->dt) || desc->max_ticks_per_run <= 0 ||
      (desc->threads != 0 && desc->threads != 256 && desc->threads != 384 && desc->threads != 512) ||
      !(desc->poisson_noise_hz >= 0.0f && desc->poisson_noise_hz <= 3.4028234663852886e38f))
    return BCPNN_ERR_INVALID;
  for (int i = 0; i < desc->n_members; ++i) {
    const bcpnn_batch_member& m = desc->members[i];
    const bcpnn_proj_desc& q = m.proj;
    if (m.pop.hcu_num <= 0 || m.pop.mcu_num <= 0 || m.pop.mcu_num > kMaxM || !finite_pos(m.pop.taum) ||
        q.src_pop != 0 || q.dest_pop != 0 || !(q.slot_num >= 1.0f && q.slot_num < 2147483648.0f) ||
        !finite_pos(q.tauzi) || !finite_pos(q.tauzj) || !finite_pos(q.taue) || !finite_pos(q.taup) ||
        !finite_pos(q.maxfq) || !(q.tauepsc <= 3.4028234663852886e38f) ||
        (long long)m.pop.hcu_num * m.pop.mcu_num > (1ll << 24))
      return BCPNN_ERR_INVALID;
    const long long C = std::min<long long>((long long)m.pop.hcu_num * m.pop.mcu_num, (long long)q.slot_num);
    if (C > 65535 || (long long)m.pop.hcu_num * C * m.pop.mcu_num > (1ll << 31)) return BCPNN_ERR_INVALID;
  }
  bcpnn_batch* b = new (std::nothrow) bcpnn_batch();
  if (!b) return BCPNN_ERR_INVALID;
  *out = b;
  b->device = desc->device;
  b->max_ticks = desc->max_ticks_per_run;
  b->threads = desc->threads ? desc->threads : 512;
  if (desc->lpt_weights[0] || desc->lpt_weights[1] || desc->lpt_weights[2])
    for (int k = 0; k < 3; ++k) b->lpt[k] = desc->lpt_weights[k];
  BCU(cudaSetDevice(b->device));
  BCU(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
  const float dt = desc->dt;
  const int N = desc->n_members;
  b->mh.resize(N);
  b->hm.resize(N);
  std::vector<unsigned long long> row_off(N + 1, 0), cell_off(N + 1, 0);
  size_t unit_cap = 0;
  int rc;
  for (int i = 0; i < N; ++i) {
    MemberHost& Mh = b->mh[i];
    Mh.d = desc->members[i];
    const bcpnn_pop_desc& P = Mh.d.pop;
    const bcpnn_proj_desc& Q = Mh.d.proj;
    Mh.H = P.hcu_num;
    Mh.M = P.mcu_num;
    Mh.n = Mh.H * Mh.M;
    Mh.C = (int)std::min<long long>((long long)Mh.n, (long long)(int)Q.slot_num);
    Member& B = b->hm[i];
    std::memset(&B, 0, sizeof(B));
    B.H = Mh.H;
    B.M = Mh.M;
    B.C = Mh.C;
    B.n = Mh.n;
    B.rng_seed = Mh.d.seed;
    /* ProcUpdLazy/Pop.cpp:35-44, Proj.cpp:38-52, in float */
    B.taumdt = dt / P.taum;
    B.wtagain = P.wtagain;
    B.maxfqdt = P.maxfq * dt;
    B.igain = P.igain;
    B.wgain = P.wgain;
    B.lgbias = P.lgbias;
    B.snoise = P.snoise;
    B.kzi = dt / Q.tauzi;
    B.kzj = dt / Q.tauzj;
    B.ke = dt / Q.taue;
    B.taupdt = dt / Q.taup;
    B.eps = dt / Q.taup;
    B.eps2 = (dt / Q.taup) * (dt / Q.taup);
    B.kfti = 1 / (Q.maxfq * Q.tauzi);
    B.kftj = 1 / (Q.maxfq * Q.tauzj);
    B.bgain = Q.bgain;
    B.pwgain = Q.wgain;
    B.kepsc = Q.tauepsc > 0 ? dt / Q.tauepsc : B.kzi;
    const size_t n = B.n, R = (size_t)B.H * B.C, cells = R * B.M;
    B.W = (B.C + 31) / 32;
    B.log_words = (B.n + 31) / 32;
    for (int p = 0; p < 2; ++p) {
      if ((rc = balloc(b, &B.dsup[p], n)) || (rc = balloc(b, &B.epsc[p], n)) || (rc = balloc(b, &B.bj[p], n)))
        return rc;
    }
    if ((rc = balloc(b, &B.act, n)) || (rc = balloc(b, &B.spike, n)) || (rc = balloc(b, &B.counter, n)) ||
        (rc = balloc(b, &B.pj, n)) || (rc = balloc(b, &B.ej, n)) || (rc = balloc(b, &B.zj, n)) ||
        (rc = balloc(b, &B.ii, R)) || (rc = balloc(b, &B.di, R)) || (rc = balloc(b, &B.pi, R)) ||
        (rc = balloc(b, &B.ei, R)) || (rc = balloc(b, &B.zi, R)) || (rc = balloc(b, &B.ti, R)) ||
        (rc = balloc(b, &B.cell, cells)) || (rc = balloc(b, &B.tij, cells)) || (rc = balloc(b, &B.wij, cells)) ||
        (rc = balloc(b, &B.ring, (size_t)B.H * kRing * B.W)) ||
        (rc = balloc(b, &B.log, (size_t)b->max_ticks * B.log_words)))
      return rc;
    int* fo_off = nullptr;
    if ((rc = balloc(b, &fo_off, n + 1)) || (rc = bzero(b, fo_off, (n + 1) * sizeof(int)))) return rc;
    B.fo_off = fo_off;
    if ((rc = bset(b, B.ii, R, -1)) || (rc = bzero(b, B.di, R * sizeof(int)))) return rc;
    Mh.ii.assign(R, -1);
    Mh.di.assign(R, 0);
    if ((rc = reset_member(b, i))) return rc;
    row_off[i + 1] = row_off[i] + R;
    cell_off[i + 1] = cell_off[i] + cells;
    unit_cap += (size_t)B.n * ((B.C + kUnit - 1) / kUnit + 1); /* column pieces + the fan-out */
    for (int hh = 0; hh < B.H; ++hh) b->items.push_back(make_int2(i, hh));
  }
  b->total_rows = row_off[N];
  b->total_cells = cell_off[N];
  if ((rc = balloc(b, &b->d_row_off, N + 1)) || (rc = balloc(b, &b->d_cell_off, N + 1))) return rc;
  BCU(cudaMemcpy(b->d_row_off, row_off.data(), (N + 1) * sizeof(unsigned long long), cudaMemcpyHostToDevice));
  BCU(cudaMemcpy(b->d_cell_off, cell_off.data(), (N + 1) * sizeof(unsigned long long), cudaMemcpyHostToDevice));
  if ((rc = balloc(b, &b->d_items, b->items.size()))) return rc;
  BCU(cudaMemcpy(b->d_items, b->items.data(), b->items.size() * sizeof(int2), cudaMemcpyHostToDevice));
  if ((rc = balloc(b, &b->d_m, (size_t)N)) || (rc = balloc(b, &b->d_dev, 1)) || (rc = balloc(b, &b->d_run, 1)) ||
      (rc = balloc(b, &b->d_tabs, (size_t)N)))
    return rc;
  b->tabs.assign(N, TabRef());
  Dev& D = b->h;
  D.n_members = N;
  D.m = b->d_m;
  D.items = b->d_items;
  D.poisson_hz = desc->poisson_noise_hz;
  D.dt = dt;
  if (unit_cap > (size_t)0x7fffffff) return bfail(b, BCPNN_ERR_INVALID, "batch too large for the column-unit ring");
  D.unit_cap = (int)std::max<size_t>(1, unit_cap);
  if ((rc = balloc(b, &D.units, 2 * (size_t)D.unit_cap)) || (rc = balloc(b, &D.unit_cnt, 2)) ||
      (rc = balloc(b, &D.counters, 3)) || (rc = balloc(b, &D.err, 1)) || (rc = balloc(b, &b->bar, 1)))
    return rc;
  if ((rc = bzero(b, D.counters, 3 * sizeof(unsigned long long))) || (rc = bzero(b, D.err, sizeof(int))))
    return rc;
  BCU(cudaStreamSynchronize(b->stream));
  if ((rc = schedule_items(b))) return rc;
  return BCPNN_OK;
}

int bcpnn_batch_destroy(bcpnn_batch* b) {
  if (!b) return BCPNN_ERR_INVALID;
  delete b;
  return BCPNN_OK;
}

int bcpnn_batch_set_conn(bcpnn_batch* b, int32_t member, const int32_t* ii, const int32_t* di, size_t n) {
  if (!b) return BCPNN_ERR_INVALID;
  if (member < 0 || member >= (int)b->mh.size() || !ii || !di)
    return bfail(b, BCPNN_ERR_INVALID, "bcpnn_batch_set_conn: bad arguments");
  MemberHost& Mh = b->mh[member];
  Member& B = b->hm[member];
  const size_t R = (size_t)B.H * B.C;
  if (n != R) return bfail(b, BCPNN_ERR_SIZE, "bcpnn_batch_set_conn: n != H * C");
  std::vector<int> cnt(B.n + 1, 0);
  for (size_t r = 0; r < R; ++r) {
    if (ii[r] >= B.n || ii[r] < -1) return bfail(b, BCPNN_ERR_INVALID, "bcpnn_batch_set_conn: source index out of range");
    if (ii[r] >= 0) {
      if (di[r] < 1 || di[r] > 31) return bfail(b, BCPNN_ERR_INVALID, "bcpnn_batch_set_conn: delay outside 1..31");
      cnt[ii[r] + 1]++;
    }
  }
  for (int k = 0; k < B.n; ++k) cnt[k + 1] += cnt[k];
  const int nfo = cnt[B.n];
  std::vector<int> row(std::max(1, nfo));
  std::vector<int8_t> dl(std::max(1, nfo));
  std::vector<int> fill(cnt.begin(), cnt.end() - 1);
  for (size_t r = 0; r < R; ++r)
    if (ii[r] >= 0) {
      const int e = fill[ii[r]]++;
      row[e] = (int)r;
      dl[e] = (int8_t)di[r];
    }
  int* fo_row = nullptr;
  int8_t* fo_di = nullptr;
  int rc;
  if ((rc = balloc(b, &fo_row, row.size())) || (rc = balloc(b, &fo_di, dl.size()))) return rc;
  BCU(cudaMemcpy(fo_row, row.data(), row.size() * sizeof(int), cudaMemcpyHostToDevice));
  BCU(cudaMemcpy(fo_di, dl.data(), dl.size(), cudaMemcpyHostToDevice));
  BCU(cudaMemcpy((void*)B.fo_off, cnt.data(), cnt.size() * sizeof(int), cudaMemcpyHostToDevice));
  BCU(cudaMemcpy(B.ii, ii, R * sizeof(int), cudaMemcpyHostToDevice));
  BCU(cudaMemcpy(B.di, di, R * sizeof(int), cudaMemcpyHostToDevice));
  B.fo_row = fo_row;
  B.fo_di = fo_di;
  Mh.ii.assign(ii, ii + R);
  Mh.di.assign(di, di + R);
  Mh.conn = true;
  return BCPNN_OK;
}

int bcpnn_batch_upload_stimuli_idx(bcpnn_batch* b, int32_t member, int32_t n_lgidx_rows, const int32_t* lgidx_rows,
                                   float eps, int32_t n_wmask_rows, const float* wmask_rows) {
  if (!b) return BCPNN_ERR_INVALID;
  if (member < 0 || member >= (int)b->mh.size() || n_lgidx_rows <= 0 || n_wmask_rows <= 0 || !lgidx_rows ||
      !wmask_rows)
    return bfail(b, BCPNN_ERR_INVALID, "bcpnn_batch_upload_stimuli_idx: bad arguments");
  Member& B = b->hm[member];
  int32_t* lg = nullptr;
  float* wm = nullptr;
  int rc;
  if ((rc = balloc(b, &lg, (size_t)n_lgidx_rows * B.H)) || (rc = balloc(b, &wm, (size_t)n_wmask_rows * B.H)))
    return rc;
  BCU(cudaMemcpy(lg, lgidx_rows, (size_t)n_lgidx_rows * B.H * sizeof(int32_t), cudaMemcpyHostToDevice));
  BCU(cudaMemcpy(wm, wmask_rows, (size_t)n_wmask_rows * B.H * sizeof(float), cudaMemcpyHostToDevice));
  B.lgidx = lg;
  B.wmask = wm;
  B.lg_rows = n_lgidx_rows;
  B.wm_rows = n_wmask_rows;
  /* ProcExtGen's values, with the host's float log as gsbn computes them */
  B.lg_hit = bx_extgen_logf(1 + eps);
  B.lg_miss = bx_extgen_logf(0 + eps);
  b->mh[member].stim = true;
  return BCPNN_OK;
}

int bcpnn_batch_use_stimulus(bcpnn_batch* b, int32_t lgidx_row, int32_t wmask_row) {
  if (!b) return BCPNN_ERR_INVALID;
  for (size_t i = 0; i < b->hm.size(); ++i)
    if (!b->mh[i].stim || lgidx_row < 0 || lgidx_row >= b->hm[i].lg_rows || wmask_row < 0 ||
        wmask_row >= b->hm[i].wm_rows)
      return bfail(b, BCPNN_ERR_INVALID, "bcpnn_batch_use_stimulus: row outside member " + std::to_string(i) +
                                             "'s tables (or no tables)");
  b->lg_row = lgidx_row;
  b->wm_row = wmask_row;
  return BCPNN_OK;
}

int bcpnn_batch_reset(bcpnn_batch* b) {
  if (!b) return BCPNN_ERR_INVALID;
  BCU(cudaSetDevice(b->device));
  for (size_t i = 0; i < b->hm.size(); ++i) {
    int rc = reset_member(b, (int)i);
    if (rc) return rc;
  }
  b->k_total = 0;
  return BCPNN_OK;
}

int bcpnn_batch_run(bcpnn_batch* b, int32_t first_simstep, int32_t n_ticks, float prn, float old_prn) {
  if (!b) return BCPNN_ERR_INVALID;
  if (n_ticks <= 0 || n_ticks > b->max_ticks)
    return bfail(b, BCPNN_ERR_INVALID, "bcpnn_batch_run: n_ticks outside [1, max_ticks_per_run]");
  if (first_simstep < 1 || (int64_t)first_simstep + n_ticks > (1 << 24))
    return bfail(b, BCPNN_ERR_INVALID, "bcpnn_batch_run: simstep outside [1, 2^24)");
  if (!(std::fabs(prn) <= 3.4028234663852886e38f) || !(std::fabs(old_prn) <= 3.4028234663852886e38f))
    return bfail(b, BCPNN_ERR_INVALID, "bcpnn_batch_run: prn and old_prn must be finite");
  for (size_t i = 0; i < b->mh.size(); ++i)
    if (!b->mh[i].conn || !b->mh[i].stim)
      return bfail(b, BCPNN_ERR_STATE, "bcpnn_batch_run: member " + std::to_string(i) + " has no connectivity or stimulus");
  BCU(cudaSetDevice(b->device));
  const bool with_all = old_prn != prn;
  const int need = first_simstep + n_ticks + 1;
  for (size_t i = 0; i < b->hm.size(); ++i) {
    const Member& B = b->hm[i];
    TSlot* T = nullptr;
    int rc;
    if ((rc = table_for(b, B.taupdt * prn, B.ke, B.kzi, B.kzj, need, &T))) return rc;
    TabRef& R = b->tabs[i];
    R.tab = T->ptr;
    R.rtab = T->rptr;
    R.len = T->len;
    R.k = make_coef(B.taupdt * prn, B.ke, B.kzi, B.kzj, 0);
    const float kp = B.taupdt * prn;
    R.rk.Dekp = 1.0 / (double)(B.ke - kp);
    R.rk.D2 = 1.0 / (double)((B.kzi - kp) + B.kzj);
    R.rk.D3 = 1.0 / (double)((B.kzi - B.ke) + B.kzj);
    R.rk.Dpzi = 1.0 / (double)(kp - B.kzi);
    R.rk.Dezi = 1.0 / (double)(B.ke - B.kzi);
    R.tab_old = nullptr;
    R.old_len = 0;
    if (with_all) {
      TSlot* To = nullptr;
      if ((rc = table_for(b, B.taupdt * old_prn, B.ke, B.kzi, B.kzj, first_simstep + 1, &To))) return rc;
      R.tab_old = To->ptr;
      R.old_len = To->len;
    }
  }
  Run& r = b->rp;
  r.simstep0 = first_simstep;
  r.k0 = (int)(b->k_total & 0x7fffffff);
  r.n_ticks = n_ticks;
  r.prn = prn;
  r.old_prn = old_prn;
  r.lg_row = b->lg_row;
  r.wm_row = b->wm_row;
  r.tabs = b->d_tabs;
  BCU(cudaMemcpyAsync(b->d_m, b->hm.data(), b->hm.size() * sizeof(Member), cudaMemcpyHostToDevice, b->stream));
  BCU(cudaMemcpyAsync(b->d_tabs, b->tabs.data(), b->tabs.size() * sizeof(TabRef), cudaMemcpyHostToDevice, b->stream));
  BCU(cudaMemcpyAsync(b->d_run, &r, sizeof(Run), cudaMemcpyHostToDevice, b->stream));
  for (size_t i = 0; i < b->hm.size(); ++i)
    BCU(cudaMemsetAsync(b->hm[i].log, 0, (size_t)n_ticks * b->hm[i].log_words * sizeof(uint32_t), b->stream));
  BCU(cudaMemsetAsync(b->bar, 0, sizeof(unsigned int), b->stream));
  BCU(cudaMemsetAsync(b->h.unit_cnt, 0, 2 * sizeof(unsigned int), b->stream));
  if (with_all) {
    batch_all_rows_kernel<<<bgrid(b->total_rows), 256, 0, b->stream>>>(b->d_dev, b->d_run, b->d_row_off, b->total_rows);
    BCU(cudaGetLastError());
    batch_all_cells_kernel<<<bgrid(b->total_cells), 256, 0, b->stream>>>(b->d_dev, b->d_run, b->d_cell_off,
                                                                         b->total_cells);
    BCU(cudaGetLastError());
    b->launches += 2;
    b->all_cells += b->total_cells; /* Proj.cpp:538-588 visits every cell */
  }
  void* args[] = {(void*)&b->d_dev, (void*)&b->d_run, (void*)&b->bar};
  const void* fn = kernel_for(b->threads);
  BCU(cudaLaunchCooperativeKernel(fn, dim3(b->grid), dim3(b->threads), args, b->smem, b->stream));
  b->launches++;
  b->k_total += n_ticks;
  b->last_ticks = n_ticks;
  return BCPNN_OK;
}

}  // extern "C"

namespace {

struct BView {
  int type;        /* BCPNN_F32 / I32 / I8 */
  size_t count;
  int kind;        /* 0 plain device array, 1 cell field, 2 qi, 3 .siq */
  const void* ptr;
  int field;
};

bool resolve_batch(bcpnn_batch* b, int member, const char* cname, BView* v) {
  if (!cname) return false;
  std::string name(cname);
  const size_t us = name.rfind('_');
  if (us == std::string::npos || name.substr(us + 1) != "0") return false;
  const std::string base = name.substr(0, us);
  const Member& B = b->hm[member];
  const int last = (int)((b->k_total - 1) & 1);
  const size_t n = B.n, R = (size_t)B.H * B.C, cells = R * B.M;
  auto plain = [&](const void* p, int type, size_t count) {
    v->kind = 0;
    v->ptr = p;
    v->type = type;
    v->count = count;
    return true;
  };
  if (base == "dsup") return plain(B.dsup[last], BCPNN_F32, n);
  if (base == "epsc") return plain(B.epsc[last], BCPNN_F32, n);
  if (base == "bj") return plain(B.bj[last], BCPNN_F32, n);
  if (base == "act") return plain(B.act, BCPNN_F32, n);
  if (base == "spike" || base == "si") return plain(B.spike, BCPNN_I8, n); /* exchange: si = the last spikes */
  if (base == ".counter") return plain(B.counter, BCPNN_I32, n);
  if (base == "pj") return plain(B.pj, BCPNN_F32, n);
  if (base == "ej") return plain(B.ej, BCPNN_F32, n);
  if (base == "zj") return plain(B.zj, BCPNN_F32, n);
  if (base == "ii") return plain(B.ii, BCPNN_I32, R);
  if (base == "di") return plain(B.di, BCPNN_I32, R);
  if (base == "pi") return plain(B.pi, BCPNN_F32, R);
  if (base == "ei") return plain(B.ei, BCPNN_F32, R);
  if (base == "zi") return plain(B.zi, BCPNN_F32, R);
  if (base == "ti") return plain(B.ti, BCPNN_I32, R);
  if (base == "tij") return plain(B.tij, BCPNN_I32, cells);
  if (base == "wij") return plain(B.wij, BCPNN_F32, cells);
  const char* fields[4] = {"pij", "eij", "zi2", "zj2"};
  for (int f = 0; f < 4; ++f)
    if (base == fields[f]) {
      v->kind = 1;
      v->ptr = B.cell;
      v->field = f;
      v->type = BCPNN_F32;
      v->count = cells;
      return true;
    }
  if (base == "qi") {
    v->kind = 2;
    v->type = BCPNN_I32;
    v->count = R;
    return true;
  }
  if (base == ".siq") {
    v->kind = 3;
    v->type = BCPNN_I8;
    v->count = R;
    return true;
  }
  return false;
}

size_t tsize(int type) { return type == BCPNN_I8 ? 1 : 4; }

}  // namespace

extern "C" {

int bcpnn_batch_sync(bcpnn_batch* b) {
  if (!b) return BCPNN_ERR_INVALID;
  BCU(cudaSetDevice(b->device));
  BCU(cudaStreamSynchronize(b->stream));
  return check_device_error(b);
}

int bcpnn_batch_get_stream(const bcpnn_batch* b, void** stream) {
  if (!b || !stream) return BCPNN_ERR_INVALID;
  *stream = (void*)b->stream;
  return BCPNN_OK;
}

int bcpnn_batch_state_info(bcpnn_batch* b, int32_t member, const char* name, int32_t* type, size_t* count) {
  if (!b) return BCPNN_ERR_INVALID;
  if (member < 0 || member >= (int)b->hm.size()) return bfail(b, BCPNN_ERR_INVALID, "bcpnn_batch_state_info: no such member");
  BView v;
  if (!resolve_batch(b, member, name, &v)) return bfail(b, BCPNN_ERR_NOT_FOUND, "bcpnn_batch_state_info: unknown vector");
  if (type) *type = v.type;
  if (count) *count = v.count;
  return BCPNN_OK;
}

int bcpnn_batch_read_state(bcpnn_batch* b, int32_t member, const char* name, void* host, size_t bytes) {
  if (!b) return BCPNN_ERR_INVALID;
  if (member < 0 || member >= (int)b->hm.size() || !host)
    return bfail(b, BCPNN_ERR_INVALID, "bcpnn_batch_read_state: bad arguments");
  BView v;
  if (!resolve_batch(b, member, name, &v)) return bfail(b, BCPNN_ERR_NOT_FOUND, "bcpnn_batch_read_state: unknown vector");
  if (bytes != v.count * tsize(v.type)) return bfail(b, BCPNN_ERR_SIZE, "bcpnn_batch_read_state: size mismatch");
  BCU(cudaSetDevice(b->device));
  BCU(cudaStreamSynchronize(b->stream));
  const Member& B = b->hm[member];
  try {
    if (v.kind == 0) {
      BCU(cudaMemcpy(host, v.ptr, bytes, cudaMemcpyDeviceToHost));
    } else if (v.kind == 1) {
      std::vector<float4> c(v.count);
      BCU(cudaMemcpy(c.data(), v.ptr, v.count * sizeof(float4), cudaMemcpyDeviceToHost));
      float* o = (float*)host;
      for (size_t i = 0; i < v.count; ++i) o[i] = (&c[i].x)[v.field];
    } else {
      /* gsbn's delay queue from the arrival ring: at the end of executed tick
         K, qi bit k of a slot is its row turning active at K + 2 + k, .siq its
         row turning active at K + 1.  The ring already holds the arrivals of
         the spikes of K (phase B of K), which gsbn queues only at K + 1 (they
         are in si): a slot's bit at K + 2 + k comes from its source's spike at
         K + k - delay, so bit k = delay is left out when the source spiked at
         K. */
      const size_t words = (size_t)B.H * kRing * B.W;
      std::vector<uint32_t> ring(words);
      std::vector<int8_t> last_spk(B.n);
      BCU(cudaMemcpy(ring.data(), B.ring, words * sizeof(uint32_t), cudaMemcpyDeviceToHost));
      BCU(cudaMemcpy(last_spk.data(), B.spike, (size_t)B.n, cudaMemcpyDeviceToHost));
      const MemberHost& Mh = b->mh[member];
      const int64_t K = b->k_total - 1;
      for (int h = 0; h < B.H; ++h)
        for (int s = 0; s < B.C; ++s) {
          auto bit = [&](int64_t tick) {
            const size_t slot = (size_t)(((tick % kRing) + kRing) % kRing);
            return (ring[((size_t)h * kRing + slot) * B.W + (s >> 5)] >> (s & 31)) & 1u;
          };
          const size_t r = (size_t)h * B.C + s;
          if (v.kind == 2) {
            int32_t q = 0;
            if (b->k_total > 0) {
              for (int k = 0; k < 31; ++k) q |= (int32_t)(bit(K + 2 + k) << k);
              const int src = Mh.ii[r];
              if (src >= 0 && last_spk[src] > 0 && Mh.di[r] <= 30) q &= ~(int32_t)(1u << Mh.di[r]);
            }
            ((int32_t*)host)[r] = q;
          } else {
            ((int8_t*)host)[r] = b->k_total > 0 ? (int8_t)bit(K + 1) : 0;
          }
        }
    }
  } catch (const std::bad_alloc&) {
    return bfail(b, BCPNN_ERR_INVALID, "bcpnn_batch_read_state: no host memory");
  }
  return BCPNN_OK;
}

int bcpnn_batch_get_spike_log(bcpnn_batch* b, int32_t member, uint32_t* out, size_t n_words) {
  if (!b) return BCPNN_ERR_INVALID;
  if (member < 0 || member >= (int)b->hm.size() || !out)
    return bfail(b, BCPNN_ERR_INVALID, "bcpnn_batch_get_spike_log: bad arguments");
  const Member& B = b->hm[member];
  if (n_words != (size_t)b->last_ticks * B.log_words)
    return bfail(b, BCPNN_ERR_SIZE, "bcpnn_batch_get_spike_log: n_words != last run ticks * words");
  BCU(cudaSetDevice(b->device));
  BCU(cudaStreamSynchronize(b->stream));
  BCU(cudaMemcpy(out, B.log, n_words * sizeof(uint32_t), cudaMemcpyDeviceToHost));
  return check_device_error(b);
}

int bcpnn_batch_counters(bcpnn_batch* b, uint64_t out[3]) {
  if (!b || !out) return BCPNN_ERR_INVALID;
  unsigned long long c[3];
  BCU(cudaSetDevice(b->device));
  BCU(cudaStreamSynchronize(b->stream));
  BCU(cudaMemcpy(c, b->h.counters, sizeof(c), cudaMemcpyDeviceToHost));
  out[0] = c[0];
  out[1] = c[1];
  out[2] = b->all_cells;
  return BCPNN_OK;
}

int bcpnn_batch_kernel_launches(const bcpnn_batch* b, uint64_t* out) {
  if (!b || !out) return BCPNN_ERR_INVALID;
  *out = b->launches;
  return BCPNN_OK;
}

int bcpnn_batch_tune(bcpnn_batch* b, int32_t probe_ticks, int32_t lgidx_train, int32_t wmask_train,
                     int32_t lgidx_recall, int32_t wmask_recall, int32_t out[4], float* us_per_tick) {
  if (!b || !out || !us_per_tick) return BCPNN_ERR_INVALID;
  if (probe_ticks <= 0 || probe_ticks > b->max_ticks)
    return bfail(b, BCPNN_ERR_INVALID, "bcpnn_batch_tune: probe_ticks outside [1, max_ticks_per_run]");
  struct Cand {
    int threads, w0, w1, w2;
  };
  /* launch shapes: CTA size (512, 384: one CTA of 16 or 12 warps per SM; 256:
     8-warp CTAs) and the cost model of the warp schedule (per item: a fixed
     part, per MCU, per 32 slots) */
  const Cand cands[] = {{512, 64, 4, 1}, {512, 16, 4, 4}, {512, 128, 2, 1}, {512, 32, 8, 2},
                        {384, 64, 4, 1}, {384, 16, 4, 4}, {384, 128, 2, 1}, {384, 32, 8, 2},
                        {256, 64, 4, 1}, {256, 16, 4, 4}, {256, 128, 2, 1}, {256, 32, 8, 2}};
  const int old_threads = b->threads;
  int old_w[3] = {b->lpt[0], b->lpt[1], b->lpt[2]};
  float best = 1e30f;
  int bi = -1;
  cudaEvent_t e0, e1;
  BCU(cudaEventCreate(&e0));
  BCU(cudaEventCreate(&e1));
  int rc = BCPNN_OK;
  for (int c = 0; c < (int)(sizeof(cands) / sizeof(cands[0])); ++c) {
    b->threads = cands[c].threads;
    b->lpt[0] = cands[c].w0;
    b->lpt[1] = cands[c].w1;
    b->lpt[2] = cands[c].w2;
    if ((rc = schedule_items(b)) || (rc = bcpnn_batch_reset(b))) break;
    float ms = 0.0f, t = 0.0f;
    /* training ticks, then recall ticks after the catch-up */
    if ((rc = bcpnn_batch_use_stimulus(b, lgidx_train, wmask_train))) break;
    cudaEventRecord(e0, b->stream);
    if ((rc = bcpnn_batch_run(b, 1, probe_ticks, 1.0f, 0.0f))) break;
    if ((rc = bcpnn_batch_use_stimulus(b, lgidx_recall, wmask_recall))) break;
    if ((rc = bcpnn_batch_run(b, 1 + probe_ticks, probe_ticks, 0.0f, 1.0f))) break;
    cudaEventRecord(e1, b->stream);
    if ((rc = bcpnn_batch_sync(b))) break;
    cudaEventElapsedTime(&t, e0, e1);
    ms = t;
    if (ms < best) {
      best = ms;
      bi = c;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) {
    b->threads = old_threads;
    for (int k = 0; k < 3; ++k) b->lpt[k] = old_w[k];
    schedule_items(b);
    return rc;
  }
  b->threads = cands[bi].threads;
  b->lpt[0] = cands[bi].w0;
  b->lpt[1] = cands[bi].w1;
  b->lpt[2] = cands[bi].w2;
  if ((rc = schedule_items(b)) || (rc = bcpnn_batch_reset(b))) return rc;
  out[0] = cands[bi].threads;
  out[1] = cands[bi].w0;
  out[2] = cands[bi].w1;
  out[3] = cands[bi].w2;
  *us_per_tick = best * 1000.0f / (2.0f * probe_ticks);
  return BCPNN_OK;
}

const char* bcpnn_batch_last_error(const bcpnn_batch* b) { return b ? b->err.c_str() : "null handle"; }

int bcpnn_batch_phase_probe(bcpnn_batch* b, uint64_t* out, int32_t max_ctas, int32_t* n_ctas, int32_t reset) {
  if (!b) return BCPNN_ERR_INVALID;
#ifdef BCPNN_PHASE_PROBE
  if (!n_ctas || (max_ctas > 0 && !out)) return bfail(b, BCPNN_ERR_INVALID, "bcpnn_batch_phase_probe: null buffer");
  const int n = std::min(b->grid, kProbeCtas);
  *n_ctas = n;
  BCU(cudaSetDevice(b->device));
  BCU(cudaStreamSynchronize(b->stream));
  if (max_ctas > 0) BCU(cudaMemcpyFromSymbol(out, g_phase_probe, (size_t)std::min(n, (int)max_ctas) * kProbeSlots * 8));
  if (reset) {
    static const uint64_t zeros[kProbeCtas * kProbeSlots] = {};
    BCU(cudaMemcpyToSymbol(g_phase_probe, zeros, sizeof(zeros)));
  }
  return BCPNN_OK;
#else
  (void)out; (void)max_ctas; (void)reset;
  if (n_ctas) *n_ctas = 0;
  return bfail(b, BCPNN_ERR_STATE, "bcpnn_batch_phase_probe: this library was built without BCPNN_PHASE_PROBE");
#endif
}

}  // extern "C"
