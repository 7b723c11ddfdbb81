/*
 * bcpnn_device.cuh -- sm_100a kernels of the plain FP32 ProcUpdLazy path.
 *
 * Compiled with -fmad=false: every float expression below is evaluated with
 * the same IEEE operations, in the same order, as gsbn's CPU path
 * (src/gsbn/procedures/ProcUpdLazy/Pop.cpp, Proj.cpp), so the results are
 * bit-identical to a CPU replay that uses the same exp/log definitions
 * (include/bcpnn_numerics.h).
 *
 * Execution model (one network, one GPU):
 *   - tick_kernel: one CTA per (population, destination HCU).  A tick of gsbn
 *     touches, for destination HCU h, only state that belongs to h (its MCUs,
 *     its slots, its cells), except the delayed presynaptic spikes read by the
 *     delay queue, which come from the previous tick.  So one CTA does, for HCU
 *     h: support/softmax/spike sampling (Pop.cpp:229-323), the j-trace step of
 *     every incoming projection (Proj.cpp:310-363), the row updates of h's
 *     active rows with ordered epsc accumulation (Proj.cpp:365-479, 667-720),
 *     the column updates of h's spiking MCUs (Proj.cpp:481-536, 722-760) and
 *     the delay queue of h's slots with ascending warp-ballot compaction of
 *     the next tick's active rows (Proj.cpp:621-664).  The kernel boundary is
 *     the only grid-wide synchronisation per tick.
 *   - Values read across CTAs inside a tick (the population's MCU-0 support
 *     that seeds every HCU's softmax max, Pop.cpp:270; si) are double
 *     buffered by tick parity: a tick reads buffer prev and writes buffer cur.
 *   - all_rows_kernel / all_cells_kernel: the all-cells catch-up at a change
 *     of prn (Proj.cpp:209-308, 538-588), a streaming pass over every row and
 *     every cell.
 *   - The closed-form decay factors depend on the elapsed ticks pdt only; they
 *     are tabulated per projection and per kp by build_table_kernel with the
 *     same float expressions the reference evaluates inline, so a table
 *     lookup returns the very bits an inline evaluation would.
 */
#ifndef BCPNN_DEVICE_CUH
#define BCPNN_DEVICE_CUH

#include <cuda_runtime.h>
#include <stdint.h>

#include "bcpnn_numerics.h"

namespace bcpnn {

constexpr int kBlock = 256;         /* threads of tick_kernel                  */
constexpr int kMaxProj = 64;        /* projections per network                 */
constexpr int kRowChunkCells = 4096;/* row-phase cells staged in shared memory */

/* error bits of NetDev::err */
constexpr int kErrIndex = 1;        /* ii out of the source population range   */

struct PopDev {
  int H, M, n, hcu_start, mcu_start, dim_proj, id;
  float taumdt, wtagain, maxfqdt, igain, wgain, lgbias, snoise;
  float* dsup[2];   /* [n], by tick parity                                  */
  float* act;       /* [n]                                                  */
  float* epsc[2];   /* [dim_proj][n], by tick parity                        */
  float* bj[2];     /* [dim_proj][n], by tick parity                        */
  int8_t* spike;    /* [n] spikes of the last tick (spike_<pop>)            */
  int* counter;     /* [n] .counter_<pop>                                   */
  uint32_t* spk_log;/* [max_ticks][log_words]                               */
  int log_words;
  int n_in;         /* projections whose destination is this population    */
  const int* in_proj;
  int n_out;        /* projections whose si this population feeds          */
  const int* out_proj;
  int ext;          /* external spike replay                                */
  const int* ext_off; /* [ext_t1 - ext_t0 + 1] offsets by simstep - ext_t0 */
  const int* ext_idx;
  int ext_t0, ext_t1;
};

struct ProjDev {
  int src, dest, H, M, C, Ns, proj_in_pop;
  float taupdt, ke, kzi, kzj, kepsc, kfti, kftj, eps, eps2, wgain, bgain;
  int* ii; int* di; int* qi;            /* [H*C] */
  float* pi; float* ei; float* zi;      /* [H*C] */
  int* ti;                              /* [H*C] */
  float* pj; float* ej; float* zj;      /* [H*M] */
  float4* cell;                         /* [H*C*M] (pij, eij, zi2, zj2) */
  int* tij;                             /* [H*C*M] */
  float* wij;                           /* [H*C*M] */
  int8_t* si[2];                        /* [Ns], by tick parity */
  int* list;                            /* [H*C] active rows, per HCU segment */
  int* list_cnt;                        /* [H] */
};

struct NetDev {
  int n_pops, n_projs;
  float dt, poisson_hz;
  uint32_t seed;
  PopDev pops[16];
  ProjDev projs[kMaxProj];
  const int* cta_pop;   /* CTA -> population */
  const int* cta_hcu;   /* CTA -> HCU        */
  float* lginp;         /* [total MCUs] host-set stimulus */
  float* wmask;         /* [total HCUs] */
  uint32_t* ss_log;     /* [max_ticks][n_projs] debug flags of ProcSpkRec */
  unsigned long long* counters; /* row cells, col cells, all cells */
  int* err;
};

/* Decay table entry for one elapsed-tick count d: four float4
   [0] cell: Ep, Epe, Epzz, Ep*D3
   [1] cell: Ee, (Ezi*Ezj)*D3, Emzi, Emzj
   [2] row:  Ep, Epe, Epzi, Ep*(ke-kzi)
   [3] row:  Ee, Eezi, Ee*(ke-kzi), Emzi
   with a = kp*d, b = ke*d, c = kzi*d, e = kzj*d (float products),
   Ep = exp(a), Epe = exp(a-b), Epzz = exp((a-c)-e), Ee = exp(b),
   Ezi = exp(c), Ezj = exp(e), Emzi = exp(-kzi*d), Emzj = exp(-kzj*d),
   Epzi = exp(a-c), Eezi = exp(b-c), D3 = (kzi-ke)+kzj.                     */
struct RunParams {
  int simstep0;   /* simstep of the first tick of the run */
  int k0;         /* ticks executed before the run (parity base) */
  int n_ticks;
  float prn, old_prn;
  const float* lginp;   /* stimulus of the run: [total MCUs] */
  const float* wmask;   /* [total HCUs] */
  const float4* tab[kMaxProj];      /* kp = taupdt*prn     */
  const float4* tab_old[kMaxProj];  /* kp = taupdt*old_prn */
  int tab_len[kMaxProj];
  int tab_old_len[kMaxProj];
};

/* constants of the closed form for one kp */
struct Coef {
  float kp, ke, kzi, kzj, kekp, Dekp, Dpzi, Dezi, D2, D3;
};

__device__ __forceinline__ Coef make_coef(float kp, float ke, float kzi, float kzj) {
  Coef k;
  k.kp = kp; k.ke = ke; k.kzi = kzi; k.kzj = kzj;
  k.kekp = ke * kp;
  k.Dekp = ke - kp;
  k.Dpzi = kp - kzi;
  k.Dezi = ke - kzi;
  k.D2 = (kzi - kp) + kzj;
  k.D3 = (kzi - ke) + kzj;
  return k;
}

/* table entry computed inline (used to build tables and for an elapsed time
   beyond the table) */
__device__ __forceinline__ void table_entry(float kp, float ke, float kzi, float kzj, int d, float4 out[4]) {
  float fd = (float)d;
  float a = kp * fd, b = ke * fd, c = kzi * fd, e = kzj * fd;
  float D3 = (kzi - ke) + kzj;
  float Dezi = ke - kzi;
  float Ep = bx_expf(a);
  float Epe = bx_expf(a - b);
  float Epzz = bx_expf((a - c) - e);
  float Ee = bx_expf(b);
  float Ezi = bx_expf(c);
  float Ezj = bx_expf(e);
  float Emzi = bx_expf(-kzi * fd);
  float Emzj = bx_expf(-kzj * fd);
  float Epzi = bx_expf(a - c);
  float Eezi = bx_expf(b - c);
  out[0] = make_float4(Ep, Epe, Epzz, Ep * D3);
  out[1] = make_float4(Ee, (Ezi * Ezj) * D3, Emzi, Emzj);
  out[2] = make_float4(Ep, Epe, Epzi, Ep * Dezi);
  out[3] = make_float4(Ee, Eezi, Ee * Dezi, Emzi);
}

__device__ __forceinline__ void load_entry(const float4* tab, int len, const Coef& k, int d, int part,
                                           float4& A, float4& B) {
  if (d < len) {
    A = tab[(size_t)d * 4 + part];
    B = tab[(size_t)d * 4 + part + 1];
  } else {
    float4 t[4];
    table_entry(k.kp, k.ke, k.kzi, k.kzj, d, t);
    A = t[part];
    B = t[part + 1];
  }
}

/* Closed-form decay of one cell over pdt ticks, Proj.cpp:435-443 (row),
   :519-527 (column), :269-277 (all).  A = entry[0], B = entry[1]. */
__device__ __forceinline__ void cell_decay(float& pij, float& eij, float& zi2, float& zj2, const Coef& k,
                                           float4 A, float4 B) {
  float U = (((eij * k.kp) * k.kzi - (eij * k.ke) * k.kp) + (eij * k.kp) * k.kzj) + (k.kekp * zi2) * zj2;
  float V = (k.kekp * zi2) * zj2;
  float pn = (pij + (U / k.Dekp - V / k.D2) / k.D3) / A.x - ((A.y * U) / k.Dekp - (V * A.z) / k.D2) / A.w;
  float W = (k.ke * zi2) * zj2;
  float en = (eij + W / k.D3) / B.x - W / B.y;
  pij = pn;
  eij = en;
  zi2 = zi2 * B.z;
  zj2 = zj2 * B.w;
}

/* Closed-form decay of the row traces, Proj.cpp:409-415 (row), :241-247
   (all).  A = entry[2], B = entry[3]. */
__device__ __forceinline__ void row_decay(float& pi, float& ei, float& zi, const Coef& k, float4 A, float4 B) {
  float X = ((ei * k.kp) * k.kzi - (ei * k.ke) * k.kp) + k.kekp * zi;
  float Y = k.kekp * zi;
  float pn = (pi - (X / k.Dekp + Y / k.Dpzi) / k.Dezi) / A.x + ((A.y * X) / k.Dekp + (Y * A.z) / k.Dpzi) / A.w;
  float KZ = k.ke * zi;
  float en = (ei - KZ / k.Dezi) / B.x + (KZ * B.y) / B.z;
  pi = pn;
  ei = en;
  zi = zi * B.w;
}

/* ------------------------------------------------------------------------ */

__global__ void build_table_kernel(float4* tab, int len, float kp, float ke, float kzi, float kzj) {
  for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < len; d += gridDim.x * blockDim.x) {
    float4 t[4];
    table_entry(kp, ke, kzi, kzj, d, t);
    tab[(size_t)d * 4 + 0] = t[0];
    tab[(size_t)d * 4 + 1] = t[1];
    tab[(size_t)d * 4 + 2] = t[2];
    tab[(size_t)d * 4 + 3] = t[3];
  }
}

/* All-cells catch-up, row part (Proj.cpp:234-254): every row with
   pdt = simstep-1-ti > 0. */
__global__ void all_rows_kernel(const NetDev* __restrict__ net, const RunParams* __restrict__ rp, int p) {
  const ProjDev& J = net->projs[p];
  int simstep = rp->simstep0 - 1;
  float kp = J.taupdt * rp->old_prn;
  Coef k = make_coef(kp, J.ke, J.kzi, J.kzj);
  const float4* tab = rp->tab_old[p];
  int len = rp->tab_old_len[p];
  int R = J.H * J.C;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < R; r += gridDim.x * blockDim.x) {
    int pdt = simstep - J.ti[r];
    if (pdt > 0) {
      float pi = J.pi[r], ei = J.ei[r], zi = J.zi[r];
      float4 A, B;
      load_entry(tab, len, k, pdt, 2, A, B);
      row_decay(pi, ei, zi, k, A, B);
      J.pi[r] = pi;
      J.ei[r] = ei;
      J.zi[r] = zi;
      J.ti[r] = simstep;
    }
  }
}

/* All-cells catch-up, cell part (Proj.cpp:256-307).  Runs after
   all_rows_kernel so w_ij sees the updated pi. */
__global__ void all_cells_kernel(const NetDev* __restrict__ net, const RunParams* __restrict__ rp, int p) {
  const ProjDev& J = net->projs[p];
  int simstep = rp->simstep0 - 1;
  float kp = J.taupdt * rp->old_prn;
  Coef k = make_coef(kp, J.ke, J.kzi, J.kzj);
  const float4* tab = rp->tab_old[p];
  int len = rp->tab_old_len[p];
  size_t ncell = (size_t)J.H * J.C * J.M;
  for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < ncell; c += (size_t)gridDim.x * blockDim.x) {
    int pdt = simstep - J.tij[c];
    if (pdt <= 0) {
      J.tij[c] = simstep;
    } else {
      float4 q = J.cell[c];
      float4 A, B;
      load_entry(tab, len, k, pdt, 0, A, B);
      cell_decay(q.x, q.y, q.z, q.w, k, A, B);
      J.cell[c] = q;
      J.tij[c] = simstep;
      if (kp != 0.0f) {
        int r = (int)(c / J.M);
        int j = (int)(c - (size_t)r * J.M);
        int h = r / J.C;
        float pi = J.pi[r];
        float pj = J.pj[h * J.M + j];
        J.wij[c] = J.wgain * bx_logf((q.x + J.eps2) / ((pi + J.eps) * (pj + J.eps)));
      }
    }
  }
}

/* ------------------------------------------------------------------------ */
/* block helpers                                                              */
/* ------------------------------------------------------------------------ */

/* Ordered compaction of one flag per thread over a block of kBlock threads:
   returns the position of this thread's item among the set flags and writes
   the total to *total (shared). */
__device__ __forceinline__ int block_prefix(bool flag, int* s_warp, int* total) {
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned m = __ballot_sync(0xffffffffu, flag);
  int before = __popc(m & ((1u << lane) - 1u));
  if (lane == 0) s_warp[warp] = __popc(m);
  __syncthreads();
  if (threadIdx.x == 0) {
    int acc = 0;
    for (int w = 0; w < kBlock / 32; ++w) {
      int c = s_warp[w];
      s_warp[w] = acc;
      acc += c;
    }
    *total = acc;
  }
  __syncthreads();
  int pos = s_warp[warp] + before;
  return pos;
}

__device__ __forceinline__ float block_max(float v, float* s_red) {
  for (int o = 16; o > 0; o >>= 1) {
    float w = __shfl_xor_sync(0xffffffffu, v, o);
    v = (w > v) ? w : v;
  }
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) s_red[warp] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    float m = s_red[0];
    for (int w = 1; w < kBlock / 32; ++w) m = (s_red[w] > m) ? s_red[w] : m;
    s_red[0] = m;
  }
  __syncthreads();
  float r = s_red[0];
  __syncthreads();
  return r;
}

/* ------------------------------------------------------------------------ */
/* one tick for one (population, destination HCU)                             */
/* ------------------------------------------------------------------------ */

/* dynamic shared memory layout (floats unless noted):
   s_dsup[M] s_act[M] s_epsc[M] s_pj[M] s_w[kRowChunkCells] s_pi[kRowChunkCells]
   s_spkl[M] (int) s_spk[M] (int8) s_skip[kRowChunkCells] (int8)            */
__host__ __device__ inline size_t tick_smem_bytes(int max_m) {
  return (size_t)4 * max_m * 4 + (size_t)kRowChunkCells * 8 + (size_t)max_m * 4 + (size_t)max_m +
         (size_t)kRowChunkCells + 64;
}

__global__ void __launch_bounds__(kBlock) tick_kernel(const NetDev* __restrict__ net,
                                                      const RunParams* __restrict__ rp, int it, int max_m) {
  extern __shared__ float smem[];
  __shared__ int s_warp[kBlock / 32];
  __shared__ float s_red[kBlock / 32];
  __shared__ int s_total;
  __shared__ float s_dsup0;
  __shared__ float s_vsum;
  __shared__ int s_nspk;
  __shared__ int s_cnt;
  __shared__ int s_flag9;

  const int P = net->cta_pop[blockIdx.x];
  const int h = net->cta_hcu[blockIdx.x];
  const PopDev& pop = net->pops[P];
  const int M = pop.M, n = pop.n;
  const int simstep = rp->simstep0 + it;
  const int kk = rp->k0 + it;
  const int cur = kk & 1, prev = cur ^ 1;
  const float prn = rp->prn;
  const int tid = threadIdx.x;

  float* s_dsup = smem;
  float* s_act = s_dsup + max_m;
  float* s_epsc = s_act + max_m;
  float* s_pj = s_epsc + max_m;
  float* s_w = s_pj + max_m;
  float* s_pi = s_w + kRowChunkCells;
  int* s_spkl = (int*)(s_pi + kRowChunkCells);
  int8_t* s_spk = (int8_t*)(s_spkl + max_m);
  int8_t* s_skip = s_spk + max_m;

  /* ---- population update, Pop.cpp:229-323 -------------------------------- */
  const float* lginp = rp->lginp + pop.mcu_start;
  const float* wmask = rp->wmask + pop.hcu_start;
  const float* epsc_prev = pop.epsc[prev];
  const float* bj_prev = pop.bj[prev];
  const float* dsup_prev = pop.dsup[prev];

  /* support of MCU `idx` of HCU `hh` (update_sup_kernel_1_cpu) */
  auto support = [&](int hh, int idx) -> float {
    float wsup = 0.0f;
    int offset = 0;
    for (int m = 0; m < pop.dim_proj; m++) {
      wsup += bj_prev[offset + idx] + epsc_prev[offset + idx];
      offset += n;
    }
    float noise = 0.0f;
    if (pop.snoise != 0.0f) noise = pop.snoise * bx_normal01(net->seed, (uint32_t)P, (uint32_t)simstep, (uint32_t)idx);
    float sup = pop.lgbias + pop.igain * lginp[idx] + noise;
    sup += (pop.wgain * wmask[hh]) * wsup;
    float d = dsup_prev[idx];
    return d + (sup - d) * pop.taumdt;
  };

  for (int j = tid; j < M; j += kBlock) s_dsup[j] = support(h, h * M + j);
  if (tid == 0) s_dsup0 = (h == 0) ? -1.0f : support(0, 0);
  __syncthreads();
  if (h == 0 && tid == 0) s_dsup0 = s_dsup[0];
  __syncthreads();
  /* max seeded with the population's first MCU (Pop.cpp:270) */
  float tmax = s_dsup0;
  for (int j = tid; j < M; j += kBlock) tmax = (s_dsup[j] > tmax) ? s_dsup[j] : tmax;
  const float maxdsup = block_max(tmax, s_red);
  const float maxact = bx_expf(pop.wtagain * maxdsup);
  for (int j = tid; j < M; j += kBlock) {
    float a = bx_expf(pop.wtagain * (s_dsup[j] - maxdsup));
    if (maxact < 1.0f) a *= maxact;
    s_act[j] = a;
  }
  __syncthreads();
  if (tid == 0) {
    float vsum = 0.0f;
    for (int m = 0; m < M; m++) vsum += s_act[m];  /* serial, in MCU order */
    s_vsum = vsum;
  }
  __syncthreads();
  const float vsum = s_vsum;
  const float pr = net->poisson_hz * net->dt;
  for (int j = tid; j < M; j += kBlock) {
    int idx = h * M + j;
    float a = s_act[j];
    if (vsum > 1.0f) a /= vsum;
    pop.act[idx] = a;
    pop.dsup[cur][idx] = s_dsup[j];
    float u = bx_uniform01(net->seed, (uint32_t)P, (uint32_t)simstep, (uint32_t)idx);
    int8_t spk = (int8_t)(u < a * pop.maxfqdt);
    if (net->poisson_hz > 0.0f) {
      float up = bx_uniform01_poisson(net->seed, (uint32_t)P, (uint32_t)simstep, (uint32_t)idx);
      if (up < pr) spk = 1;
    }
    pop.counter[idx] += spk;
    s_spk[j] = spk;
  }
  /* external spike replay overrides the sampled spikes (Pop.cpp:389-409) */
  if (pop.ext) {
    __syncthreads();
    for (int j = tid; j < M; j += kBlock) s_spk[j] = 0;
    __syncthreads();
    if (simstep >= pop.ext_t0 && simstep < pop.ext_t1) {
      int b0 = pop.ext_off[simstep - pop.ext_t0], b1 = pop.ext_off[simstep - pop.ext_t0 + 1];
      for (int e = b0 + tid; e < b1; e += kBlock) {
        int v = pop.ext_idx[e];
        if (v >= h * M && v < h * M + M) s_spk[v - h * M] = 1;
      }
    }
  }
  __syncthreads();
  /* publish spikes; ordered list of this HCU's spiking MCUs */
  if (tid == 0) s_nspk = 0;
  for (int base = 0; base < M; base += kBlock) {
    int j = base + tid;
    bool f = (j < M) && s_spk[j] > 0;
    int pos = block_prefix(f, s_warp, &s_total);
    if (f) s_spkl[s_nspk + pos] = j;
    __syncthreads();
    if (tid == 0) s_nspk += s_total;
    __syncthreads();
  }
  uint32_t* log = pop.spk_log + (size_t)it * pop.log_words;
  for (int j = tid; j < M; j += kBlock) {
    int idx = h * M + j;
    int8_t s = s_spk[j];
    pop.spike[idx] = s;
    if (s) atomicOr(&log[idx >> 5], 1u << (idx & 31));
    for (int q = 0; q < pop.n_out; ++q) net->projs[pop.out_proj[q]].si[cur][idx] = s;
  }
  const int nspk = s_nspk;

  /* ---- incoming projections ------------------------------------------------ */
  for (int q = 0; q < pop.n_in; ++q) {
    const int p = pop.in_proj[q];
    const ProjDev& J = net->projs[p];
    const int C = J.C;
    const float kp = J.taupdt * prn;
    const Coef k = make_coef(kp, J.ke, J.kzi, J.kzj);
    const float4* tab = rp->tab[p];
    const int tlen = rp->tab_len[p];
    const size_t eoff = (size_t)J.proj_in_pop * n;

    /* j-traces and bias, Proj.cpp:310-363 */
    for (int j = tid; j < M; j += kBlock) {
      int idx = h * M + j;
      float pj = J.pj[idx], ej = J.ej[idx], zj = J.zj[idx];
      float e = pop.epsc[prev][eoff + idx];
      e *= (1 - J.kepsc);
      pj += (ej - pj) * kp;
      ej += (zj - ej) * k.ke;
      zj *= (1 - J.kzj);
      if (s_spk[j] > 0) zj += J.kftj;
      float b = pop.bj[prev][eoff + idx];
      if (kp != 0.0f) b = J.bgain * bx_logf(pj + J.eps);
      pop.bj[cur][eoff + idx] = b;
      J.pj[idx] = pj;
      J.ej[idx] = ej;
      J.zj[idx] = zj;
      s_epsc[j] = e;
      s_pj[j] = pj;
    }
    if (tid == 0) s_flag9 = 0;
    __syncthreads();

    /* row updates of this HCU's active rows, ascending, Proj.cpp:365-479 */
    const int nrow = J.list_cnt[h];
    const int* rows = J.list + (size_t)h * C;
    const int rch = (kRowChunkCells / M) > 0 ? (kRowChunkCells / M) : 1;
    for (int base = 0; base < nrow; base += rch) {
      const int nr = (nrow - base) < rch ? (nrow - base) : rch;
      for (int t = tid; t < nr; t += kBlock) {
        int r = rows[base + t];
        if (r == 9) s_flag9 = 1;
        int pdt = simstep - J.ti[r];
        if (pdt <= 0) {
          J.zi[r] += J.kfti;
          J.ti[r] = simstep;
          s_pi[t] = J.pi[r];
        } else {
          float pi = J.pi[r], ei = J.ei[r], zi = J.zi[r];
          float4 A, B;
          load_entry(tab, tlen, k, pdt, 2, A, B);
          row_decay(pi, ei, zi, k, A, B);
          zi = zi + J.kfti;
          J.pi[r] = pi;
          J.ei[r] = ei;
          J.zi[r] = zi;
          J.ti[r] = simstep;
          s_pi[t] = pi;
        }
      }
      __syncthreads();
      for (int c = tid; c < nr * M; c += kBlock) {
        int rr = c / M;
        int j = c - rr * M;
        int r = rows[base + rr];
        size_t index = (size_t)r * M + j;
        int pdt = simstep - J.tij[index];
        float4 cv = J.cell[index];
        if (pdt <= 0) {
          cv.z += J.kfti;
          J.cell[index] = cv;
          J.tij[index] = simstep;
          s_skip[c] = 1;
        } else {
          float4 A, B;
          load_entry(tab, tlen, k, pdt, 0, A, B);
          cell_decay(cv.x, cv.y, cv.z, cv.w, k, A, B);
          cv.z = cv.z + J.kfti;
          J.cell[index] = cv;
          J.tij[index] = simstep;
          float w;
          if (kp != 0.0f) {
            w = J.wgain * bx_logf((cv.x + J.eps2) / ((s_pi[rr] + J.eps) * (s_pj[j] + J.eps)));
            J.wij[index] = w;
          } else {
            w = J.wij[index];
          }
          s_w[c] = w;
          s_skip[c] = 0;
        }
      }
      __syncthreads();
      for (int j = tid; j < M; j += kBlock) {
        float e = s_epsc[j];
        for (int rr = 0; rr < nr; ++rr)
          if (!s_skip[rr * M + j]) e += s_w[rr * M + j];
        s_epsc[j] = e;
      }
      __syncthreads();
    }
    for (int j = tid; j < M; j += kBlock) pop.epsc[cur][eoff + h * M + j] = s_epsc[j];

    /* column updates of this HCU's spiking MCUs, Proj.cpp:481-536 */
    for (int c = tid; c < nspk * C; c += kBlock) {
      int qq = c / C;
      int s = c - qq * C;
      int j = s_spkl[qq];
      int r = h * C + s;
      if (J.ii[r] < 0) continue;
      size_t index = (size_t)r * M + j;
      int pdt = simstep - J.tij[index];
      float4 cv = J.cell[index];
      if (pdt <= 0) {
        cv.w += J.kftj;
      } else {
        float4 A, B;
        load_entry(tab, tlen, k, pdt, 0, A, B);
        cell_decay(cv.x, cv.y, cv.z, cv.w, k, A, B);
        cv.w = cv.w + J.kftj;
      }
      J.cell[index] = cv;
      J.tij[index] = simstep;
    }

    /* delay queue of this HCU's slots and ordered compaction of the next
       tick's active rows, Proj.cpp:621-630, 645-664 */
    if (tid == 0) s_cnt = 0;
    __syncthreads();
    const int8_t* si = J.si[prev];
    for (int base = 0; base < C; base += kBlock) {
      int s = base + tid;
      bool act = false;
      int r = h * C + s;
      if (s < C) {
        int src = J.ii[r];
        if (src >= 0) {
          if (src >= J.Ns) {
            atomicOr(net->err, kErrIndex);
          } else {
            int qv = J.qi[r];
            act = (qv & 0x01) != 0;
            qv >>= 1;
            if (si[src] > 0) qv |= (0x01 << (J.di[r] - 1));
            J.qi[r] = qv;
          }
        }
      }
      int pos = block_prefix(act, s_warp, &s_total);
      if (act) J.list[(size_t)h * C + s_cnt + pos] = r;
      __syncthreads();
      if (tid == 0) s_cnt += s_total;
      __syncthreads();
    }
    if (tid == 0) {
      J.list_cnt[h] = s_cnt;
      /* debug flags of ProcSpkRec (ssi/ssj contain index 9) */
      uint8_t f = 0;
      if (s_flag9) f |= 1;
      if (h == 9 / M && 9 < n && s_spk[9 - h * M] > 0) f |= 2;
      if (f) atomicOr(&net->ss_log[(size_t)it * net->n_projs + p], (uint32_t)f);
      atomicAdd(&net->counters[0], (unsigned long long)nrow * M);
      atomicAdd(&net->counters[1], (unsigned long long)nspk * C);
    }
    __syncthreads();
  }
}

/* fill kernels used to (re)initialise the state on the device */
template <typename T>
__global__ void fill_kernel(T* p, size_t n, T v) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) p[i] = v;
}

/* gather / scatter of one float of the (pij, eij, zi2, zj2) cells */
__global__ void cell_gather_kernel(const float4* cell, size_t n, int field, float* out) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    float4 v = cell[i];
    out[i] = field == 0 ? v.x : field == 1 ? v.y : field == 2 ? v.z : v.w;
  }
}

__global__ void cell_scatter_kernel(float4* cell, size_t n, int field, const float* in) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    float4 v = cell[i];
    float x = in[i];
    if (field == 0) v.x = x; else if (field == 1) v.y = x; else if (field == 2) v.z = x; else v.w = x;
    cell[i] = v;
  }
}

}  // namespace bcpnn

#endif /* BCPNN_DEVICE_CUH */
