/*
 * bcpnn_multi.cuh -- the ProcUpdMulti variant of the update
 * (src/gsbn/procedures/ProcUpdMulti.cpp:94-125, ProcUpdMulti/Pop.cpp,
 * ProcUpdMulti/Proj.cpp).  What differs from ProcUpdLazy:
 *   - population: adaptation current `ada` subtracted from the support and
 *     relaxed towards adgain*act (Pop.cpp:222-311), a constant 6.9*wmask in
 *     double (Pop.cpp:246), the soft-WTA maximum seeded with the HCU's own
 *     first MCU (Pop.cpp:263), spikes kept in a ring of `spike buffer size`
 *     ticks (Pop.cpp:320-329);
 *   - projections: no column updates.  A cell has no zi2/tij of its own; it
 *     starts from its row's zi and ti and, when its row is active, replays
 *     the postsynaptic spikes still in the ring since then (each one: decay
 *     to that tick, zj2 += kftj), decays to now and adds kftj for a spike
 *     now (Proj.cpp:364-488); the row's zi gains kfti only when time passed
 *     (Proj.cpp:685-693); every active cell adds its weight to epsc.
 * The closed forms are gsbn's (same expressions as ProcUpdLazy), evaluated
 * with the shared decay tables and the exact division of bcpnn_device.cuh.
 *
 * Launch forms: one persistent cooperative launch per run, with each HCU's
 * state resident in shared memory (res_tick_loop) or in global memory
 * (tick_loop, for spike rings longer than 32 ticks or states too large for
 * shared memory); or, when the grid cannot be co-resident, one launch of
 * pop_kernel per tick over every (population, HCU) and one of proj_kernel
 * per projection over its destination HCUs (512 threads).  all_kernel does
 * the catch-up at a change of prn.  Per-tick buffers follow the ProcUpdLazy
 * path's tick parity (dsup, epsc, bj, si), so state reads and the spike log
 * work unchanged.
 */
#ifndef BCPNN_MULTI_CUH
#define BCPNN_MULTI_CUH

#include "bcpnn_device.cuh"

namespace bcpnn {
namespace multi {

constexpr int kPopThreads = 128;
constexpr int kProjThreads = kBlock; /* 512: block_prefix works over kBlock threads */
constexpr int kRowCells = 1024;      /* cells of one row chunk in shared memory */

__host__ __device__ inline int row_chunk(int M) { return M >= kRowCells ? 1 : kRowCells / M; }

/* phase probe of the persistent launch (BCPNN_PHASE_PROBE): thread 0 adds
   the cycles since its previous mark to slot `slot` of its CTA's counters:
   0 barrier wait, 1 support, 2 softmax maximum and exponentials, 3 softmax
   sum, 4 spikes, 5 j-traces and row list (in the resident launch after the
   staging of the tick's first row chunk), 6 row traces and cell replays (of
   a staged chunk: its spike now and the cell writes), 7 weights, 8 epsc
   sums, 9 delay queue, 10 (resident launch) wait for the delay-queue warps,
   11 (resident launch) the next tick's uniforms, 12 (resident launch, the
   first delay-queue thread) its wait at the grid barrier; kProbeTicks
   counts the ticks.  In the resident launch slot 0 holds no barrier wait
   (only the delay-queue warps wait there). */
#ifdef BCPNN_PHASE_PROBE
#define MPROBE(slot)                                                   \
  do {                                                                 \
    if (threadIdx.x == 0) {                                            \
      const long long t_ = clock64();                                  \
      g_probe_smem[slot] += (unsigned long long)(t_ - *probe_t);       \
      *probe_t = t_;                                                   \
    }                                                                  \
  } while (0)
#else
#define MPROBE(slot) do {} while (0)
#endif

/* dynamic shared memory of proj_kernel, in bytes */
__host__ __device__ inline size_t proj_smem_bytes(int M, int C) {
  return (size_t)(M + C + kRowCells + 3 * row_chunk(M)) * 4;
}

/* the decay-table pair of `part` for d elapsed ticks (d < len from the table,
   else computed) */
__device__ __forceinline__ void entry(const float4* tab, int len, const Coef& k, int d, int part, float4& A,
                                      float4& B) {
  load_entry(tab, len, k, d, part, A, B);
}

/* Population update, ProcUpdMulti/Pop.cpp:222-311 and fill_spike 403-421.
   dynamic shared memory: 2*M floats. */
__device__ __forceinline__ void pop_hcu(const NetDev* __restrict__ net, const RunParams* __restrict__ rp, int it, int P,
                                        int h, float* sm, float* s_vsum_p, long long* probe_t,
                                        uint32_t* s_hist = nullptr) {
  (void)probe_t;
  float& s_vsum = *s_vsum_p;
  __shared__ float s_red[32];
  const PopDev& pop = net->pops[P];
  const int M = pop.M, n = pop.n;
  const int simstep = rp->simstep0 + it, kk = rp->k0 + it;
  const int cur = kk & 1, prev = cur ^ 1;
  float* s_dsup = sm;
  float* s_act = sm + M;
  int8_t* s_spk = (int8_t*)(sm + 2 * M);
  const float wm = rp->wmask[pop.hcu_start + h];
  const float* lginp = rp->lginp + pop.mcu_start;

  /* update_sup_kernel_1_cpu, Pop.cpp:222-253 */
  for (int j = threadIdx.x; j < M; j += blockDim.x) {
    const int idx = h * M + j;
    float wsup = 0.0f;
    int offset = 0;
    for (int m = 0; m < pop.dim_proj; ++m) {
      wsup += pop.bj[prev][offset + idx] + pop.epsc[prev][offset + idx];
      offset += n;
    }
    float noise = 0.0f;
    if (pop.snoise != 0.0f)
      noise = pop.snoise * dev_normal01(pop.rng_seed, pop.rng_pop, (uint32_t)simstep, (uint32_t)idx);
    float sup = pop.lgbias + pop.igain * lginp[idx] + noise;
    sup += (pop.wgain * wm) * wsup;
    sup -= wm * pop.ada[idx];
    sup = (float)((double)sup + 6.9 * (double)wm); /* a double constant in gsbn */
    const float d = pop.dsup[prev][idx];
    const float nd = d + (sup - d) * pop.taumdt;
    pop.dsup[cur][idx] = nd;
    s_dsup[j] = nd;
  }
  __syncthreads();
  MPROBE(1);
  /* update_sup_kernel_2_cpu, Pop.cpp:255-286: the maximum (order does not
     matter) and the exponentials in parallel, the sum serial in MCU order */
  {
    float mx = s_dsup[0];
    for (int m = threadIdx.x; m < M; m += blockDim.x) mx = s_dsup[m] > mx ? s_dsup[m] : mx;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const float w = __shfl_xor_sync(0xffffffffu, mx, o);
      mx = w > mx ? w : mx;
    }
    if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = mx;
    __syncthreads();
    mx = s_red[0];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) mx = s_red[w] > mx ? s_red[w] : mx;
    const float maxact = bx_expf(pop.wtagain * mx);
    for (int m = threadIdx.x; m < M; m += blockDim.x) {
      float a = bx_expf(pop.wtagain * (s_dsup[m] - mx));
      if (maxact < 1.0f) a *= maxact;
      s_act[m] = a;
    }
    __syncthreads();
    MPROBE(2);
    if (threadIdx.x == 0) {
      float vsum = 0.0f;
      for (int m = 0; m < M; ++m) vsum += s_act[m];
      s_vsum = vsum;
    }
    __syncthreads();
    MPROBE(3);
  }
  /* update_sup_kernel_3_cpu, Pop.cpp:288-311 */
  const float vsum = s_vsum;
  const float pr = net->poisson_hz * net->dt;
  for (int j = threadIdx.x; j < M; j += blockDim.x) {
    const int idx = h * M + j;
    float a = s_act[j];
    if (vsum > 1.0f) a /= vsum;
    pop.act[idx] = a;
    const float u = bx_uniform01(pop.rng_seed, pop.rng_pop, (uint32_t)simstep, (uint32_t)idx);
    int8_t spk = (int8_t)(u < a * pop.maxfqdt);
    if (net->poisson_hz > 0.0f) {
      const float up = bx_uniform01_poisson(pop.rng_seed, pop.rng_pop, (uint32_t)simstep, (uint32_t)idx);
      if (up < pr) spk = 1;
    }
    pop.counter[idx] += spk;
    pop.ada[idx] += (pop.adgain * a - pop.ada[idx]) * pop.tauadt;
    s_spk[j] = spk;
  }
  /* fill_spike, Pop.cpp:403-421: replayed spikes replace the sampled ones */
  if (pop.ext) {
    __syncthreads();
    for (int j = threadIdx.x; j < M; j += blockDim.x) s_spk[j] = 0;
    __syncthreads();
    if (simstep >= pop.ext_t0 && simstep < pop.ext_t1) {
      const int b0 = pop.ext_off[simstep - pop.ext_t0], b1 = pop.ext_off[simstep - pop.ext_t0 + 1];
      for (int e = b0 + threadIdx.x; e < b1; e += blockDim.x) {
        const int v = pop.ext_idx[e];
        if (v >= h * M && v < h * M + M) s_spk[v - h * M] = 1;
      }
    }
  }
  __syncthreads();
  int8_t* ring = pop.ring + (size_t)(simstep % pop.ring_len) * n;
  uint32_t* log = pop.spk_log + (size_t)it * pop.log_words;
  for (int j = threadIdx.x; j < M; j += blockDim.x) {
    const int idx = h * M + j;
    const int8_t sv = s_spk[j];
    ring[idx] = sv;
    if (s_hist) s_hist[j] = (s_hist[j] << 1) | (sv > 0 ? 1u : 0u);
    pop.spike[idx] = sv;
    if (sv) atomicOr(&log[idx >> 5], 1u << (idx & 31));
    for (int q = 0; q < pop.n_out; ++q) net->projs[pop.out_proj[q]].si[cur][idx] = sv;
  }
  MPROBE(4);
}

__global__ void pop_kernel(const NetDev* __restrict__ net, const RunParams* __restrict__ rp, int it) {
  extern __shared__ __align__(16) float sm[];
  __shared__ float s_vsum;
  long long probe_t = 0;
  pop_hcu(net, rp, it, net->cta_pop[blockIdx.x], net->cta_hcu[blockIdx.x], sm, &s_vsum, &probe_t);
}

/* One closed-form decay of a cell over pdt ticks.  With the run's TabRef of
   this kp (T non-null: the tick path, whose kp the TabRef's coefficients
   and reciprocal table were made for) the divisions are multiplications by
   the tabulated double reciprocals with the exact fallback (cell_step_nl,
   bit-identical to cell_decay); without it (the catch-up at a change of prn,
   with the old kp) cell_decay itself. */
__device__ __forceinline__ void decay_cell(float& pij, float& eij, float& zi2, float& zj2, const Coef& k,
                                           const float4* tab, int tlen, const TabRef* T, int pdt) {
  float4 A, Bv;
  if (T) {
    double2 R0, R1;
    if (pdt < tlen) {
      A = tab[(size_t)pdt * 4];
      Bv = tab[(size_t)pdt * 4 + 1];
      R0 = T->rtab[(size_t)pdt * 4];
      R1 = T->rtab[(size_t)pdt * 4 + 1];
    } else {
      table_pair(k.kp, k.ke, k.kzi, k.kzj, pdt, 0, A, Bv, k.fp64);
      recip_part(A, Bv, 0, R0, R1);
    }
    const float4 c = cell_step_nl(make_float4(pij, eij, zi2, zj2), T, A, Bv, R0, R1);
    pij = c.x;
    eij = c.y;
    zi2 = c.z;
    zj2 = c.w;
    return;
  }
  entry(tab, tlen, k, pdt, 0, A, Bv);
  cell_decay(pij, eij, zi2, zj2, k, A, Bv);
}

/* One cell of an active row (update_row_kernel_cpu, Proj.cpp:409-488, after
   the row traces): replay of the postsynaptic spikes in the ring, decay to
   simstep, kftj for a spike now.  tij/zi2 start from the row's ti/zi.  T as
   for decay_cell. */
__device__ __forceinline__ void replay_cell(float4& c4, int tij, float zi2, int simstep, int last_exclusive,
                                            const int8_t* __restrict__ ring, int B, int n, int mcu, const Coef& k,
                                            const float4* tab, int tlen, const TabRef* T, float kftj,
                                            bool final_decay_always) {
  float pij = c4.x, eij = c4.y, zj2 = c4.w;
  int now = tij;
  if (simstep - now >= B) now = simstep - B + 1;
  while (now < simstep) {
    ++now;
    if ((!last_exclusive || now < simstep) && ring[(size_t)(now % B) * n + mcu] > 0) {
      const int pdt = now - tij;
      if (pdt > 0) {
        decay_cell(pij, eij, zi2, zj2, k, tab, tlen, T, pdt);
        zj2 = zj2 + kftj;
        tij = now;
      }
    }
  }
  const int pdt = simstep - tij;
  if (final_decay_always || pdt > 0) {
    float zi2_unused = zi2;
    decay_cell(pij, eij, zi2_unused, zj2, k, tab, tlen, T, pdt);
  }
  c4 = make_float4(pij, eij, zi2, zj2);
}

/* replay_cell of the tick path (last tick exclusive, final decay always)
   with the postsynaptic spikes of the last 32 ticks as a mask: bit b of
   `hist` is the spike of this cell's MCU at tick simstep - b, as the ring
   holds it (ring length B <= 32).  The ticks visited and the decays done are
   those of replay_cell's loop over the ring: the ticks after
   max(tij, simstep - B + 1) and before simstep, ascending. */
__device__ __forceinline__ void replay_cell_hist(float4& c4, int tij, float zi2, int simstep, uint32_t hist, int B,
                                                 const Coef& k, const float4* tab, int tlen, const TabRef* T,
                                                 float kftj) {
  float pij = c4.x, eij = c4.y, zj2 = c4.w;
  const int lo = (simstep - tij >= B) ? simstep - B + 1 : tij;
  const int span = simstep - lo; /* ticks lo+1 .. simstep are bits span-1 .. 0 */
  uint32_t m = span > 1 ? (hist & (0xffffffffu >> (32 - span))) & ~1u : 0u;
  /* the final decay runs from the last replayed tick (the lowest set bit b:
     tick simstep - b) or from tij; its table entries are loaded before the
     replays, beside the cell's own load */
  const int pdt_f = m ? __ffs(m) - 1 : simstep - tij;
  const bool tab_f = (unsigned)pdt_f < (unsigned)tlen;
  float4 Af = make_float4(0, 0, 0, 0), Bf = Af;
  double2 R0f = make_double2(0, 0), R1f = R0f;
  if (tab_f) {
    Af = tab[(size_t)pdt_f * 4];
    Bf = tab[(size_t)pdt_f * 4 + 1];
    R0f = T->rtab[(size_t)pdt_f * 4];
    R1f = T->rtab[(size_t)pdt_f * 4 + 1];
  }
  while (m) {
    const int b = 31 - __clz(m);
    m &= ~(1u << b);
    const int now = simstep - b;
    decay_cell(pij, eij, zi2, zj2, k, tab, tlen, T, now - tij);
    zj2 = zj2 + kftj;
    tij = now;
  }
  if (!tab_f) {
    table_pair(k.kp, k.ke, k.kzi, k.kzj, pdt_f, 0, Af, Bf, k.fp64);
    recip_part(Af, Bf, 0, R0f, R1f);
  }
  const float4 c = cell_step_nl(make_float4(pij, eij, zi2, zj2), T, Af, Bf, R0f, R1f);
  c4 = make_float4(c.x, c.y, zi2, c.w); /* the cell keeps the zi2 of its last replay */
}

/* One tick of projection p for one destination HCU: update_jxx_cpu,
   update_ssi_cpu, update_row_cpu and update_que_cpu (Proj.cpp:557-706). */
struct ProjShared {
  int warp[kWarps], total, flag9;
};

__device__ __forceinline__ void proj_hcu(const NetDev* __restrict__ net, const RunParams* __restrict__ rp, int it,
                                         int p, int h, float* sm, ProjShared* ps, long long* probe_t,
                                         const uint32_t* s_hist = nullptr) {
  (void)probe_t;
  int* s_warp = ps->warp;
  int& s_total = ps->total;
  int& s_flag9 = ps->flag9;
  const ProjDev& J = net->projs[p];
  const PopDev& pop = net->pops[J.dest];
  const int M = J.M, C = J.C, n = pop.n, B = pop.ring_len;
  const int simstep = rp->simstep0 + it, kk = rp->k0 + it;
  const int cur = kk & 1, prev = cur ^ 1;
  const float kp = J.taupdt * rp->prn;
  const Coef k = make_coef(kp, J.ke, J.kzi, J.kzj);
  const float4* tab = rp->tabs[p].tab;
  const int tlen = rp->tabs[p].len;
  const TabRef* T = &rp->tabs[p]; /* coefficients and reciprocals of this kp */
  const size_t eoff = (size_t)J.proj_in_pop * n;
  const int8_t* sj = pop.ring + (size_t)(simstep % B) * n;
  const int rch = row_chunk(M);
  float* s_epsc = sm;
  int* s_list = (int*)(sm + M);
  float* s_w = sm + M + C;
  float* s_pi = s_w + kRowCells;
  int* s_ti = (int*)(s_pi + rch);
  float* s_zi = (float*)(s_ti + rch);
  const int tid = threadIdx.x;

  /* update_jxx_kernel_cpu, Proj.cpp:321-362 */
  for (int j = tid; j < M; j += blockDim.x) {
    const int idx = h * M + j;
    float pj = J.pj[idx], ej = J.ej[idx], zj = J.zj[idx];
    float e = pop.epsc[prev][eoff + idx];
    e *= (1 - J.kepsc);
    pj += (ej - pj) * kp;
    ej += (zj - ej) * k.ke;
    zj *= (1 - J.kzj);
    if (sj[idx] > 0) zj += J.kftj;
    pop.bj[cur][eoff + idx] = (kp != 0.0f) ? J.bgain * bx_logf(pj + J.eps) : pop.bj[prev][eoff + idx];
    J.pj[idx] = pj;
    J.ej[idx] = ej;
    J.zj[idx] = zj;
    s_epsc[j] = e;
  }
  /* the active rows of this tick (the previous tick's delay queue), ascending */
  const int nrow = J.list_cnt[h];
  for (int i = tid; i < nrow; i += blockDim.x) s_list[i] = J.list[h * C + i];
  if (tid == 0) s_flag9 = 0;
  __syncthreads();
  MPROBE(5);

  /* update_row_cpu, Proj.cpp:638-706 */
  for (int base = 0; base < nrow; base += rch) {
    const int nr = (nrow - base) < rch ? (nrow - base) : rch;
    for (int t = tid; t < nr; t += blockDim.x) {
      const int r = s_list[base + t];
      s_ti[t] = J.ti[r];
      s_zi[t] = J.zi[r];
      if (r == 9) s_flag9 = 1;
    }
    __syncthreads();
    /* row traces (from the top thread down) beside the cells (from thread 0 up) */
    for (int t = blockDim.x - 1 - tid; t < nr; t += blockDim.x) {
      const int r = s_list[base + t];
      const int pdt = simstep - s_ti[t];
      float pi = J.pi[r];
      if (pdt > 0) {
        float ei = J.ei[r], zi = s_zi[t];
        float4 A, Bv;
        double2 R0, R1;
        if (pdt < tlen) {
          A = tab[(size_t)pdt * 4 + 2];
          Bv = tab[(size_t)pdt * 4 + 3];
          R0 = T->rtab[(size_t)pdt * 4 + 2];
          R1 = T->rtab[(size_t)pdt * 4 + 3];
        } else {
          table_pair(k.kp, k.ke, k.kzi, k.kzj, pdt, 2, A, Bv, k.fp64);
          recip_part(A, Bv, 2, R0, R1);
        }
        /* zi becomes zi*exp(-kzi*pdt) */
        const float4 rv = row_step_nl(make_float4(pi, ei, zi, 0.0f), T, A, Bv, R0, R1);
        pi = rv.x;
        ei = rv.y;
        zi = rv.z;
        J.pi[r] = pi;
        J.ei[r] = ei;
        J.zi[r] = zi + J.kfti;
      }
      J.ti[r] = simstep;
      s_pi[t] = pi;
    }
    for (int c = tid; c < nr * M; c += blockDim.x) {
      const int rr = c / M, j = c - rr * M;
      const size_t index = (size_t)s_list[base + rr] * M + j;
      float4 c4 = J.cell[index];
      if (s_hist) {
        const uint32_t hist = s_hist[j];
        replay_cell_hist(c4, s_ti[rr], s_zi[rr], simstep, hist, B, k, tab, tlen, T, J.kftj);
        if (hist & 1u) c4.w += J.kftj;
      } else {
        replay_cell(c4, s_ti[rr], s_zi[rr], simstep, 1, pop.ring, B, n, h * M + j, k, tab, tlen, T, J.kftj, true);
        if (sj[h * M + j] > 0) c4.w += J.kftj;
      }
      J.cell[index] = c4;
      s_w[c] = c4.x;
    }
    __syncthreads();
    MPROBE(6);
    for (int c = tid; c < nr * M; c += blockDim.x) {
      const int rr = c / M, j = c - rr * M;
      const size_t index = (size_t)s_list[base + rr] * M + j;
      float w;
      if (kp != 0.0f) {
        w = J.wgain * bx_logf((s_w[c] + J.eps2) / ((s_pi[rr] + J.eps) * (J.pj[h * M + j] + J.eps)));
        J.wij[index] = w;
      } else {
        w = J.wij[index];
      }
      s_w[c] = w;
    }
    __syncthreads();
    MPROBE(7);
    for (int j = tid; j < M; j += blockDim.x) {
      float e = s_epsc[j];
      for (int rr = 0; rr < nr; ++rr) e += s_w[rr * M + j];
      s_epsc[j] = e;
    }
    __syncthreads();
    MPROBE(8);
  }
  for (int j = tid; j < M; j += blockDim.x) pop.epsc[cur][eoff + h * M + j] = s_epsc[j];

  /* update_que_cpu, Proj.cpp:620-636, and the next tick's active rows
     (update_ssi_cpu, :580-588), ascending */
  const int8_t* si = J.si[prev];
  int cnt = 0;
  /* kQB chunks of blockDim slots at a time: their table loads, then their
     source-spike loads, are issued together, and the chunks' compactions
     follow in slot order */
  constexpr int kQB = 4;
  for (int s0 = 0; s0 < C; s0 += kQB * (int)blockDim.x) {
    int src[kQB], qv[kQB], dv[kQB];
    bool act[kQB];
#pragma unroll
    for (int u = 0; u < kQB; ++u) {
      const int s = s0 + u * (int)blockDim.x + tid;
      src[u] = -1;
      qv[u] = 0;
      dv[u] = 1;
      if (s < C) {
        src[u] = J.ii[h * C + s];
        if (src[u] >= 0) {
          qv[u] = J.qi[h * C + s];
          dv[u] = J.di[h * C + s];
        }
      }
    }
#pragma unroll
    for (int u = 0; u < kQB; ++u) {
      const int s = s0 + u * (int)blockDim.x + tid;
      act[u] = false;
      if (src[u] >= 0) {
        if (src[u] >= J.Ns) {
          atomicOr(net->err, kErrIndex);
        } else {
          int q = qv[u];
          act[u] = (q & 0x01) != 0;
          q >>= 1;
          if (si[src[u]] > 0) q |= (0x01 << (dv[u] - 1));
          J.qi[h * C + s] = q;
        }
      }
    }
#pragma unroll
    for (int u = 0; u < kQB; ++u) {
      if (s0 + u * (int)blockDim.x >= C) break;
      int tot;
      const int pos = block_prefix(act[u], s_warp, &s_total, &tot);
      if (act[u]) J.list[h * C + cnt + pos] = h * C + s0 + u * (int)blockDim.x + tid;
      cnt += tot;
    }
  }
  if (tid == 0) {
    J.list_cnt[h] = cnt;
    uint32_t f = 0;
    if (s_flag9) f |= 1;
    if (h == 9 / M && 9 < n && sj[9] > 0) f |= 2;
    if (f) atomicOr(&net->ss_log[(size_t)it * net->n_projs + p], f);
    atomicAdd(&net->counters[0], (unsigned long long)nrow * M);
  }
  MPROBE(9);
}

__global__ void __launch_bounds__(kProjThreads, 1) proj_kernel(const NetDev* __restrict__ net,
                                                              const RunParams* __restrict__ rp, int it, int p) {
  extern __shared__ __align__(16) float sm[];
  __shared__ ProjShared ps;
  long long probe_t = 0;
  proj_hcu(net, rp, it, p, blockIdx.x, sm, &ps, &probe_t);
}

/* Persistent form: one cooperative launch per run, one CTA per (population,
   HCU).  A tick of ProcUpdMulti needs from other HCUs only the source spikes
   of the previous tick (si, the exchange), so one CTA does its HCU's
   population update and then its rows of every incoming projection, and one
   grid barrier separates the ticks.  The bodies are those of pop_kernel and
   proj_kernel.  bar: the grid-barrier arrival counter, zero at launch. */
template <typename GridSync>
__device__ __forceinline__ void tick_loop(const NetDev* __restrict__ net, const RunParams* __restrict__ rp, int it0,
                                          int n_ticks, GridSync sync) {
  extern __shared__ __align__(16) float sm[];
  __shared__ float s_vsum;
  __shared__ ProjShared ps;
  const int P = net->cta_pop[blockIdx.x];
  const int h = net->cta_hcu[blockIdx.x];
  const PopDev& pop = net->pops[P];
#ifdef BCPNN_PHASE_PROBE
  if (threadIdx.x < kProbeSlots) g_probe_smem[threadIdx.x] = 0;
  __syncthreads();
#endif
#ifdef BCPNN_PHASE_PROBE
  long long probe_clock = clock64();
#else
  long long probe_clock = 0;
#endif
  long long* probe_t = &probe_clock;
  /* the HCU's spikes of the last 32 ticks, one mask per MCU (ring length
     <= 32): bit b of s_hist[j] is the ring's entry for tick s - 1 - b before
     the first tick s of this launch, and the entry for tick s - b once tick
     s has sampled its spikes */
  __shared__ uint32_t s_hist_buf[kProjThreads];
  uint32_t* s_hist = nullptr;
  if (pop.ring_len <= 32 && pop.M <= kProjThreads) {
    s_hist = s_hist_buf;
    const int B = pop.ring_len, M = pop.M, s0 = rp->simstep0 + it0;
    for (int j = threadIdx.x; j < M; j += blockDim.x) {
      uint32_t m = 0;
      for (int b = 0; b < B - 1; ++b) {
        const int t = s0 - 1 - b;
        if (t >= 0 && pop.ring[(size_t)(t % B) * pop.n + h * M + j] > 0) m |= 1u << b;
      }
      s_hist[j] = m;
    }
    __syncthreads();
  }
  for (int it = it0; it < it0 + n_ticks; ++it) {
    if (it > it0 && !sync(it - it0)) break;
    MPROBE(0);
#ifdef BCPNN_PHASE_PROBE
    if (threadIdx.x == 0) g_probe_smem[kProbeTicks] += 1;
#endif
    pop_hcu(net, rp, it, P, h, sm, &s_vsum, probe_t, s_hist);
    __syncthreads();
    for (int q = 0; q < pop.n_in; ++q) {
      proj_hcu(net, rp, it, pop.in_proj[q], h, sm, &ps, probe_t, s_hist);
      __syncthreads();
    }
  }
#ifdef BCPNN_PHASE_PROBE
  __syncthreads();
  if (threadIdx.x < kProbeSlots && blockIdx.x < kProbeCtas)
    atomicAdd(&g_phase_probe[blockIdx.x * kProbeSlots + threadIdx.x], g_probe_smem[threadIdx.x]);
#endif
}

/* ---- resident persistent launch ----------------------------------------

   The same tick as tick_loop, with the HCU's state kept in shared memory for
   the whole launch: the population's dsup, ada, act, counter and stimulus
   row; per incoming projection pj, ej, zj, epsc, bj, the slot tables ii, di,
   qi, the row traces pi, ei, zi, ti and the active-row list (by tick
   parity).  They are loaded at launch and written back after the last tick,
   epsc/bj/dsup into the buffer of the last tick's parity, which is where the
   next run and the state reads look.  What other CTAs read stays in global
   memory every tick: the source spikes si of the exchange, the ring, the
   spike vector and the spike log; the cells (pij, eij, zi2, zj2) and wij
   stay in global memory.

   The delay queue of a tick reads only the previous tick's source spikes and
   qi, so its 4 warps (threads 384-511) compute the next tick's active rows
   while the other 12 warps (the population group) do the population update
   and then the tick's projections.
   The previous tick's source spikes are the only data of other CTAs a tick
   reads, and only the delay queue reads them: the population group arrives
   at the grid barrier once it has written this tick's source spikes and
   goes on with the tick's rows (listed by the previous tick's queue), while
   the delay-queue warps wait for the previous tick's arrivals and run the
   queue; the groups join before the staging.  CTAs may run ticks apart, so
   the source spikes live in four buffers by tick (tick mod 4).  Right after
   its arrival the population group stages the tick's first row chunk of
   projection 0 (row traces, cell replays and decays); at the end of a tick
   the CTA draws the next tick's sampling uniforms. */
constexpr int kResQueueWarps = 4;
constexpr int kResPopThreads = kProjThreads - 32 * kResQueueWarps; /* 384 */
constexpr int kBarPop = 1, kBarQueue = 2;

__device__ __forceinline__ void named_sync(int id, int n) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory");
}

/* word offsets of the resident layout in dynamic shared memory */
struct ResLayout {
  int stc;                                 /* [kRowCells] float4: staged cells */
  int dsup, ada, act, cnt, lg, hist, u, up, spk; /* population, [M] (spk: bytes) */
  int w, rpi, rti, rzi;                   /* row-chunk scratch            */
  int qmask;                              /* delay-queue ballots          */
  int q[kMaxIn];                          /* incoming projection blocks   */
  int total;
};

/* one projection block: pj ej zj epsc bj [M]; ii di qi pi ei zi ti [C];
   list [2][C] */
__host__ __device__ inline int res_qwords(int M, int C) { return 5 * M + 9 * C; }

__host__ __device__ inline void res_layout(int M, int n_in, const int* C, ResLayout& L) {
  int o = 0;
  L.stc = o; o += 4 * kRowCells;
  const int M4 = (M + 3) & ~3; /* population arrays start on 16-byte boundaries */
  L.dsup = o; o += M4;
  L.ada = o; o += M4;
  L.act = o; o += M4;
  L.cnt = o; o += M4;
  L.lg = o; o += M4;
  L.hist = o; o += M4;
  L.u = o; o += M4;
  L.up = o; o += M4;
  L.spk = o; o += (M + 3) / 4;
  const int rch = row_chunk(M);
  L.w = o; o += kRowCells;
  L.rpi = o; o += rch;
  L.rti = o; o += rch;
  L.rzi = o; o += rch;
  int cmax = 0;
  for (int q = 0; q < n_in; ++q) cmax = C[q] > cmax ? C[q] : cmax;
  L.qmask = o; o += (cmax + 31) / 32;
  for (int q = 0; q < kMaxIn; ++q) {
    L.q[q] = o;
    if (q < n_in) o += res_qwords(M, C[q]);
  }
  L.total = o;
}

/* dynamic shared memory of the resident launch for one population, bytes */
__host__ __device__ inline size_t res_smem_bytes(int M, int n_in, const int* C) {
  ResLayout L;
  res_layout(M, n_in, C, L);
  return (size_t)L.total * 4;
}

struct ResQ {
  float *pj, *ej, *zj, *epsc, *bj;
  int *ii, *di, *qi;
  float *pi, *ei, *zi;
  int *ti, *list;
};

__device__ __forceinline__ ResQ res_q(float* sm, const ResLayout& L, int q, int M, int C) {
  ResQ v;
  float* b = sm + L.q[q];
  v.pj = b;
  v.ej = b + M;
  v.zj = b + 2 * M;
  v.epsc = b + 3 * M;
  v.bj = b + 4 * M;
  int* ib = (int*)(b + 5 * M);
  v.ii = ib;
  v.di = ib + C;
  v.qi = ib + 2 * C;
  v.pi = (float*)(ib + 3 * C);
  v.ei = (float*)(ib + 4 * C);
  v.zi = (float*)(ib + 5 * C);
  v.ti = ib + 6 * C;
  v.list = ib + 7 * C;
  return v;
}

/* uniforms of one tick's spike sampling for the HCU's MCUs (they depend on
   the tick and the MCU only), drawn ahead by threads tid, tid + nth, ... */
__device__ __forceinline__ void res_draw(const PopDev& pop, bool poisson, int simstep, int h, float* r_u, float* r_up,
                                         int tid, int nth) {
  for (int j = tid; j < pop.M; j += nth) {
    const uint32_t idx = (uint32_t)(h * pop.M + j);
    r_u[j] = bx_uniform01(pop.rng_seed, pop.rng_pop, (uint32_t)simstep, idx);
    r_up[j] = poisson ? bx_uniform01_poisson(pop.rng_seed, pop.rng_pop, (uint32_t)simstep, idx) : 1.0f;
  }
}

/* the grid barrier of the resident launch, split: a CTA arrives (release
   add) once its tick's source spikes are written and its delay queue has
   read the previous tick's; only the delay-queue warps wait (acquire poll,
   bounded) before they read the source spikes of the previous tick */
__device__ __forceinline__ void mp_arrive(unsigned int* bar) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(bar), "r"(1u) : "memory");
}

constexpr int kErrBarrierWait = 2; /* the error bit of a grid-barrier wait that ran out of time */

__device__ __forceinline__ bool mp_poll(const unsigned int* bar, unsigned int target, int* err) {
  unsigned long long t0, t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
  for (;;) {
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(bar) : "memory");
    if (v >= target) return true;
    if (*(volatile int*)err) return false;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    if (t - t0 > 2000000000ull) {
      atomicOr(err, kErrBarrierWait);
      return false;
    }
    __nanosleep(20);
  }
}

/* bar: four arrival counters (by tick mod 4), zero at launch */
__device__ __forceinline__ void res_tick_loop(const NetDev* __restrict__ net, const RunParams* __restrict__ rp,
                                              int it0, int n_ticks, unsigned int* bar) {
  extern __shared__ __align__(16) float sm[];
  /* descriptors, copied once per launch: every tick reads them in chains */
  __shared__ PopDev s_pop;
  __shared__ ProjDev s_proj[kMaxIn];
  __shared__ TabRef s_tab[kMaxIn];
  __shared__ int s_inp[kMaxIn];
  __shared__ int8_t* s_siout[kMaxIn][2];
  __shared__ ResLayout s_L;
  __shared__ int s_nlist[kMaxIn][2];
  __shared__ int s_qcnt[kResQueueWarps];
  __shared__ float s_red[32];
  __shared__ float s_vsum, s_wm;
  __shared__ int s_flag9;
  __shared__ int s_staged; /* rows of projection 0's first chunk staged for this tick, or -1 */
  __shared__ int s_qok;    /* the delay-queue warps' barrier wait succeeded */

  const int tid = threadIdx.x;
  const int P = net->cta_pop[blockIdx.x];
  const int h = net->cta_hcu[blockIdx.x];
  if (tid == 0) s_pop = net->pops[P];
  __syncthreads();
  if (tid < kMaxIn && tid < s_pop.n_in) {
    const int p = s_pop.in_proj[tid];
    s_inp[tid] = p;
    s_proj[tid] = net->projs[p];
    s_tab[tid] = rp->tabs[p];
  }
  if (tid < kMaxIn && tid < s_pop.n_out) {
    const ProjDev& O = net->projs[s_pop.out_proj[tid]];
    s_siout[tid][0] = O.si[0];
    s_siout[tid][1] = O.si[1];
  }
  __syncthreads();
  const PopDev& pop = s_pop;
  const int M = pop.M, n = pop.n, n_in = pop.n_in, B = pop.ring_len;
  if (tid == 0) {
    int c[kMaxIn];
#pragma unroll
    for (int q = 0; q < kMaxIn; ++q) c[q] = q < n_in ? s_proj[q].C : 0;
    res_layout(M, n_in, c, s_L);
    s_wm = rp->wmask[pop.hcu_start + h];
  }
  __syncthreads();
  const ResLayout& L = s_L;
  float* r_dsup = sm + L.dsup;
  float* r_ada = sm + L.ada;
  float* r_act = sm + L.act;
  int* r_cnt = (int*)(sm + L.cnt);
  float* r_lg = sm + L.lg;
  uint32_t* r_hist = (uint32_t*)(sm + L.hist);
  float* r_u = sm + L.u;
  float* r_up = sm + L.up;
  int8_t* r_spk = (int8_t*)(sm + L.spk);
  const bool poisson = net->poisson_hz > 0.0f;
  float4* st_c4 = (float4*)(sm + L.stc);
  float* s_w = sm + L.w;
  float* s_pi = sm + L.rpi;
  int* s_ti = (int*)(sm + L.rti);
  float* s_zi = sm + L.rzi;
  uint32_t* s_qmask = (uint32_t*)(sm + L.qmask);
  const int rch = row_chunk(M);

  /* ---- load the resident state: buffers of the tick before the launch ---- */
  {
    const int prev0 = ((rp->k0 + it0) & 1) ^ 1;
    const int s0 = rp->simstep0 + it0;
    for (int j = tid; j < M; j += blockDim.x) {
      const int idx = h * M + j;
      r_dsup[j] = pop.dsup[prev0][idx];
      r_ada[j] = pop.ada[idx];
      r_act[j] = pop.act[idx];
      r_cnt[j] = pop.counter[idx];
      r_lg[j] = rp->lginp[pop.mcu_start + idx];
      /* bit b: the ring's entry for tick s0 - 1 - b (ring length <= 32) */
      uint32_t m = 0;
      for (int b = 0; b < B - 1; ++b) {
        const int t = s0 - 1 - b;
        if (t >= 0 && pop.ring[(size_t)(t % B) * n + idx] > 0) m |= 1u << b;
      }
      r_hist[j] = m;
    }
    for (int q = 0; q < n_in; ++q) {
      const ProjDev& J = s_proj[q];
      const int C = J.C;
      const ResQ V = res_q(sm, L, q, M, C);
      const size_t eoff = (size_t)J.proj_in_pop * n;
      for (int j = tid; j < M; j += blockDim.x) {
        const int idx = h * M + j;
        V.pj[j] = J.pj[idx];
        V.ej[j] = J.ej[idx];
        V.zj[j] = J.zj[idx];
        V.epsc[j] = pop.epsc[prev0][eoff + idx];
        V.bj[j] = pop.bj[prev0][eoff + idx];
      }
      for (int s = tid; s < C; s += blockDim.x) {
        const int r = h * C + s;
        V.ii[s] = J.ii[r];
        V.di[s] = J.di[r];
        V.qi[s] = J.qi[r];
        V.pi[s] = J.pi[r];
        V.ei[s] = J.ei[r];
        V.zi[s] = J.zi[r];
        V.ti[s] = J.ti[r];
      }
      const int cnt = J.list_cnt[h];
      for (int e = tid; e < cnt; e += blockDim.x) V.list[e] = J.list[h * C + e] - h * C;
      if (tid == 0) s_nlist[q][0] = cnt;
    }
    res_draw(pop, poisson, s0, h, r_u, r_up, tid, blockDim.x);
    if (tid == 0) {
      s_staged = -1;
      s_qok = 1;
    }
  }
  __syncthreads();
#ifdef BCPNN_PHASE_PROBE
  if (tid < kProbeSlots) g_probe_smem[tid] = 0;
  __syncthreads();
  long long probe_clock = clock64();
  long long* probe_t = &probe_clock;
#endif

  int it = it0;
  for (; it < it0 + n_ticks; ++it) {
    MPROBE(0);
#ifdef BCPNN_PHASE_PROBE
    if (tid == 0) g_probe_smem[kProbeTicks] += 1;
#endif
    const int simstep = rp->simstep0 + it, kk = rp->k0 + it;
    const int lp = (it - it0) & 1; /* list parity: this tick's rows */

    if (tid < kResPopThreads) {
      /* ---- population update (ProcUpdMulti/Pop.cpp:222-311, 403-421) ---- */
      constexpr int G = kResPopThreads;
      const float wm = s_wm;
      for (int j = tid; j < M; j += G) {
        float wsup = 0.0f;
        for (int m = 0; m < n_in; ++m) {
          const float* b = sm + L.q[m];
          wsup += b[4 * M + j] + b[3 * M + j]; /* bj + epsc of the previous tick */
        }
        float noise = 0.0f;
        if (pop.snoise != 0.0f)
          noise = pop.snoise * dev_normal01(pop.rng_seed, pop.rng_pop, (uint32_t)simstep, (uint32_t)(h * M + j));
        float sup = pop.lgbias + pop.igain * r_lg[j] + noise;
        sup += (pop.wgain * wm) * wsup;
        sup -= wm * r_ada[j];
        sup = (float)((double)sup + 6.9 * (double)wm); /* a double constant in gsbn */
        const float d = r_dsup[j];
        r_dsup[j] = d + (sup - d) * pop.taumdt;
      }
      named_sync(kBarPop, G);
      MPROBE(1);
      /* the maximum (order does not matter) and the exponentials in
         parallel, the sum serial in MCU order */
      float mx = r_dsup[0];
      for (int m = tid; m < M; m += G) mx = r_dsup[m] > mx ? r_dsup[m] : mx;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const float w = __shfl_xor_sync(0xffffffffu, mx, o);
        mx = w > mx ? w : mx;
      }
      if ((tid & 31) == 0) s_red[tid >> 5] = mx;
      named_sync(kBarPop, G);
      mx = s_red[0];
      for (int w = 1; w < G / 32; ++w) mx = s_red[w] > mx ? s_red[w] : mx;
      const float maxact = bx_expf(pop.wtagain * mx);
      for (int m = tid; m < M; m += G) {
        float a = bx_expf(pop.wtagain * (r_dsup[m] - mx));
        if (maxact < 1.0f) a *= maxact;
        r_act[m] = a;
      }
      named_sync(kBarPop, G);
      MPROBE(2);
      if (tid == 0) {
        float vsum = 0.0f;
        const float4* a4 = (const float4*)r_act;
        int m = 0;
#pragma unroll 4
        for (; m + 4 <= M; m += 4) {
          const float4 v = a4[m >> 2];
          vsum += v.x;
          vsum += v.y;
          vsum += v.z;
          vsum += v.w;
        }
        for (; m < M; ++m) vsum += r_act[m];
        s_vsum = vsum;
      }
      named_sync(kBarPop, G);
      MPROBE(3);
      const float vsum = s_vsum;
      const float pr = net->poisson_hz * net->dt;
      for (int j = tid; j < M; j += G) {
        float a = r_act[j];
        if (vsum > 1.0f) a /= vsum;
        r_act[j] = a;
        int8_t spk = (int8_t)(r_u[j] < a * pop.maxfqdt); /* uniforms drawn before the tick */
        if (poisson && r_up[j] < pr) spk = 1;
        r_cnt[j] += spk;
        r_ada[j] += (pop.adgain * a - r_ada[j]) * pop.tauadt;
        r_spk[j] = spk;
      }
      if (pop.ext) { /* fill_spike: replayed spikes replace the sampled ones */
        named_sync(kBarPop, G);
        for (int j = tid; j < M; j += G) r_spk[j] = 0;
        named_sync(kBarPop, G);
        if (simstep >= pop.ext_t0 && simstep < pop.ext_t1) {
          const int b0 = pop.ext_off[simstep - pop.ext_t0], b1 = pop.ext_off[simstep - pop.ext_t0 + 1];
          for (int e = b0 + tid; e < b1; e += G) {
            const int v = pop.ext_idx[e];
            if (v >= h * M && v < h * M + M) r_spk[v - h * M] = 1;
          }
        }
      }
      named_sync(kBarPop, G);
      int8_t* ring = pop.ring + (size_t)(simstep % B) * n;
      uint32_t* log = pop.spk_log + (size_t)it * pop.log_words;
      for (int j = tid; j < M; j += G) {
        const int idx = h * M + j;
        const int8_t sv = r_spk[j];
        ring[idx] = sv;
        r_hist[j] = (r_hist[j] << 1) | (sv > 0 ? 1u : 0u);
        pop.spike[idx] = sv;
        if (sv) atomicOr(&log[idx >> 5], 1u << (idx & 31));
        /* source spikes in four buffers by tick (kk mod 4): a CTA may write
           tick u's while others still read ticks u-3 .. u-1 */
        for (int q = 0; q < pop.n_out; ++q) {
          int8_t* si = (q < kMaxIn ? s_siout[q][0] : net->projs[pop.out_proj[q]].si[0]) + (size_t)(kk & 3) * n;
          si[idx] = sv;
        }
      }
      MPROBE(4);
      /* this tick's source spikes are written: the group's arrival */
      named_sync(kBarPop, G);
      if (tid == 0 && it + 1 < it0 + n_ticks) mp_arrive(bar + ((it - it0) & 3));
      /* stage this tick's first row chunk of projection 0 (listed by the
         previous tick's queue) after the arrival: row traces, and the
         cells' replays and decays to this tick; the rows phase adds a spike
         now and writes the cells */
      if (n_in > 0) {
        const ProjDev& J = s_proj[0];
        const TabRef* T = &s_tab[0];
        const int C = J.C;
        const ResQ V = res_q(sm, L, 0, M, C);
        const float kp = J.taupdt * rp->prn;
        const Coef k = make_coef(kp, J.ke, J.kzi, J.kzj);
        const float4* tab = T->tab;
        const int tlen = T->len;
        const int ts = simstep;
        const int* nl = V.list + lp * C;
        const int nrow1 = s_nlist[0][lp];
        const int nr = nrow1 < rch ? nrow1 : rch;
        for (int t = tid; t < nr; t += G) {
          const int sl = nl[t];
          s_ti[t] = V.ti[sl];
          s_zi[t] = V.zi[sl];
        }
        named_sync(kBarPop, G);
        for (int t = G - 1 - tid; t < nr; t += G) {
          const int sl = nl[t];
          const int pdt = ts - s_ti[t];
          float pi = V.pi[sl];
          if (pdt > 0) {
            float4 A, Bv;
            double2 R0, R1;
            if (pdt < tlen) {
              A = tab[(size_t)pdt * 4 + 2];
              Bv = tab[(size_t)pdt * 4 + 3];
              R0 = T->rtab[(size_t)pdt * 4 + 2];
              R1 = T->rtab[(size_t)pdt * 4 + 3];
            } else {
              table_pair(k.kp, k.ke, k.kzi, k.kzj, pdt, 2, A, Bv, k.fp64);
              recip_part(A, Bv, 2, R0, R1);
            }
            /* zi becomes zi*exp(-kzi*pdt) */
            const float4 rv = row_step_nl(make_float4(pi, V.ei[sl], s_zi[t], 0.0f), T, A, Bv, R0, R1);
            pi = rv.x;
            V.pi[sl] = rv.x;
            V.ei[sl] = rv.y;
            V.zi[sl] = rv.z + J.kfti;
          }
          V.ti[sl] = ts;
          s_pi[t] = pi;
        }
        for (int c = tid; c < nr * M; c += G) {
          const int rr = c / M, j = c - rr * M;
          float4 c4 = J.cell[(size_t)(h * C + nl[rr]) * M + j];
          /* bit b of the history is tick ts - b; bit 0 (a spike now) is
             not replayed */
          replay_cell_hist(c4, s_ti[rr], s_zi[rr], ts, r_hist[j], B, k, tab, tlen, T, J.kftj);
          st_c4[c] = c4;
        }
        if (tid == 0) s_staged = nr;
      }

        /* ---- projections (update_jxx_cpu, update_row_cpu, Proj.cpp:557-706),
           by the population group while the delay-queue warps run on: the
           rows of this tick come from the previous tick's queue ---- */
      for (int q = 0; q < n_in; ++q) {
        const ProjDev& J = s_proj[q];
        const TabRef* T = &s_tab[q]; /* coefficients and reciprocals of this kp */
        const int C = J.C;
        const ResQ V = res_q(sm, L, q, M, C);
        const float kp = J.taupdt * rp->prn;
        const Coef k = make_coef(kp, J.ke, J.kzi, J.kzj);
        const float4* tab = T->tab;
        const int tlen = T->len;
        for (int j = tid; j < M; j += G) {
          float pj = V.pj[j], ej = V.ej[j], zj = V.zj[j];
          float e = V.epsc[j];
          e *= (1 - J.kepsc);
          pj += (ej - pj) * kp;
          ej += (zj - ej) * k.ke;
          zj *= (1 - J.kzj);
          if (r_hist[j] & 1u) zj += J.kftj;
          if (kp != 0.0f) V.bj[j] = J.bgain * bx_logf(pj + J.eps);
          V.pj[j] = pj;
          V.ej[j] = ej;
          V.zj[j] = zj;
          V.epsc[j] = e;
        }
        const int nrow = s_nlist[q][lp];
        const int* list = V.list + lp * C;
        if (tid == 0) s_flag9 = 0;
        named_sync(kBarPop, G);
        MPROBE(5);
        for (int base = 0; base < nrow; base += rch) {
          const int nr = (nrow - base) < rch ? (nrow - base) : rch;
          if (q == 0 && base == 0 && s_staged == nr) {
            /* staged after this tick's barrier arrival: the row traces
               are up to date, the cells replayed and decayed to this tick;
               what is left is a spike now */
            for (int t = tid; t < nr; t += G)
              if (h * C + list[t] == 9) s_flag9 = 1;
            for (int c = tid; c < nr * M; c += G) {
              const int rr = c / M, j = c - rr * M;
              const size_t index = (size_t)(h * C + list[rr]) * M + j;
              float4 c4 = st_c4[c];
              if (r_hist[j] & 1u) c4.w += J.kftj;
              J.cell[index] = c4;
              s_w[c] = c4.x;
            }
            named_sync(kBarPop, G);
            MPROBE(6);
          } else {
          for (int t = tid; t < nr; t += G) {
            const int sl = list[base + t];
            s_ti[t] = V.ti[sl];
            s_zi[t] = V.zi[sl];
            if (h * C + sl == 9) s_flag9 = 1;
          }
          named_sync(kBarPop, G);
          /* row traces (from the top thread down) beside the cells (from
             thread 0 up) */
          for (int t = G - 1 - tid; t < nr; t += G) {
            const int sl = list[base + t];
            const int pdt = simstep - s_ti[t];
            float pi = V.pi[sl];
            if (pdt > 0) {
              float4 A, Bv;
              double2 R0, R1;
              if (pdt < tlen) {
                A = tab[(size_t)pdt * 4 + 2];
                Bv = tab[(size_t)pdt * 4 + 3];
                R0 = T->rtab[(size_t)pdt * 4 + 2];
                R1 = T->rtab[(size_t)pdt * 4 + 3];
              } else {
                table_pair(k.kp, k.ke, k.kzi, k.kzj, pdt, 2, A, Bv, k.fp64);
                recip_part(A, Bv, 2, R0, R1);
              }
              /* zi becomes zi*exp(-kzi*pdt) */
              const float4 rv = row_step_nl(make_float4(pi, V.ei[sl], s_zi[t], 0.0f), T, A, Bv, R0, R1);
              pi = rv.x;
              V.pi[sl] = rv.x;
              V.ei[sl] = rv.y;
              V.zi[sl] = rv.z + J.kfti;
            }
            V.ti[sl] = simstep;
            s_pi[t] = pi;
          }
          for (int c = tid; c < nr * M; c += G) {
            const int rr = c / M, j = c - rr * M;
            const size_t index = (size_t)(h * C + list[base + rr]) * M + j;
            float4 c4 = J.cell[index];
            const uint32_t hist = r_hist[j];
            replay_cell_hist(c4, s_ti[rr], s_zi[rr], simstep, hist, B, k, tab, tlen, T, J.kftj);
            if (hist & 1u) c4.w += J.kftj;
            J.cell[index] = c4;
            s_w[c] = c4.x;
          }
          named_sync(kBarPop, G);
          MPROBE(6);
          }
          for (int c = tid; c < nr * M; c += G) {
            const int rr = c / M, j = c - rr * M;
            const size_t index = (size_t)(h * C + list[base + rr]) * M + j;
            float w;
            if (kp != 0.0f) {
              w = J.wgain * bx_logf((s_w[c] + J.eps2) / ((s_pi[rr] + J.eps) * (V.pj[j] + J.eps)));
              J.wij[index] = w;
            } else {
              w = J.wij[index];
            }
            s_w[c] = w;
          }
          named_sync(kBarPop, G);
          MPROBE(7);
          for (int j = tid; j < M; j += G) {
            float e = V.epsc[j];
            for (int rr = 0; rr < nr; ++rr) e += s_w[rr * M + j];
            V.epsc[j] = e;
          }
          named_sync(kBarPop, G);
          MPROBE(8);
        }
        if (tid == 0) {
          uint32_t f = 0;
          if (s_flag9) f |= 1;
          if (h == 9 / M && 9 < n && (r_hist[9 - h * M] & 1u)) f |= 2;
          if (f) atomicOr(&net->ss_log[(size_t)it * net->n_projs + s_inp[q]], f);
          atomicAdd(&net->counters[0], (unsigned long long)nrow * M);
        }
      }
    } else {
      /* ---- delay queue (update_que_cpu, Proj.cpp:620-636) and the next
         tick's active rows (update_ssi_cpu, :580-588), ascending ---- */
      const int qt = tid - kResPopThreads, qw = qt >> 5, lane = tid & 31;
      const int nq = lp ^ 1;
      /* the previous tick's source spikes are complete once every CTA has
         arrived for it (the launch's first tick reads the last launch's) */
      if (it > it0) {
#ifdef BCPNN_PHASE_PROBE
        const long long qclk = clock64();
#endif
        /* one arrival per CTA and tick, its population group's (source
           spikes written), on the counter of the tick's slot (tick mod 4).
           A CTA arrives for tick u only once tick u - 2 is complete, so
           while tick t - 1 is incomplete no arrival for a tick above t
           exists, and the slot's count for t - 1 is CTAs x its ticks so
           far.  Tick u - 2 complete also means every CTA's queue has read
           the spikes of tick u - 4 or earlier: four buffers suffice */
        const int tp = it - 1 - it0;
        if (qt == 0 && !mp_poll(bar + (tp & 3), gridDim.x * (unsigned int)((tp >> 2) + 1), net->err)) s_qok = 0;
#ifdef BCPNN_PHASE_PROBE
        if (qt == 0) g_probe_smem[12] += (unsigned long long)(clock64() - qclk);
#endif
        named_sync(kBarQueue, 32 * kResQueueWarps);
      }
      for (int q = 0; q < n_in && s_qok; ++q) {
        const ProjDev& J = s_proj[q];
        const int C = J.C, Ns = J.Ns;
        const ResQ V = res_q(sm, L, q, M, C);
        const int8_t* si = J.si[0] + (size_t)((kk + 3) & 3) * Ns;
        const int ng = (C + 31) >> 5; /* groups of 32 slots; warp qw takes a contiguous range */
        const int per = (ng + kResQueueWarps - 1) / kResQueueWarps;
        const int g0 = qw * per, g1 = min(ng, g0 + per);
        int cnt = 0;
        for (int gb = g0; gb < g1; gb += 8) {
          int src[8], qv[8], dv[8];
          int8_t sv[8];
#pragma unroll
          for (int u = 0; u < 8; ++u) {
            const int s = (gb + u) * 32 + lane;
            src[u] = -1;
            qv[u] = 0;
            dv[u] = 1;
            if (gb + u < g1 && s < C) {
              src[u] = V.ii[s];
              qv[u] = V.qi[s];
              dv[u] = V.di[s];
            }
          }
#pragma unroll
          for (int u = 0; u < 8; ++u) sv[u] = (src[u] >= 0 && src[u] < Ns) ? si[src[u]] : (int8_t)0;
#pragma unroll
          for (int u = 0; u < 8; ++u) {
            if (gb + u >= g1) break; /* warp-uniform */
            bool act = false;
            if (src[u] >= 0) {
              if (src[u] >= Ns) {
                atomicOr(net->err, kErrIndex);
              } else {
                int v = qv[u];
                act = (v & 0x01) != 0;
                v >>= 1;
                if (sv[u] > 0) v |= (0x01 << (dv[u] - 1));
                V.qi[(gb + u) * 32 + lane] = v;
              }
            }
            const unsigned mb = __ballot_sync(0xffffffffu, act);
            if (lane == 0) s_qmask[gb + u] = mb;
            cnt += __popc(mb);
          }
        }
        if (lane == 0) s_qcnt[qw] = cnt;
        named_sync(kBarQueue, 32 * kResQueueWarps);
        int base = 0;
        for (int w = 0; w < qw; ++w) base += s_qcnt[w];
        int* out = V.list + nq * C;
        for (int g = g0; g < g1; ++g) {
          const uint32_t mb = s_qmask[g];
          if ((mb >> lane) & 1u) out[base + __popc(mb & ((1u << lane) - 1u))] = g * 32 + lane;
          base += __popc(mb);
        }
        if (qw == kResQueueWarps - 1 && lane == 0) s_nlist[q][nq] = base;
        named_sync(kBarQueue, 32 * kResQueueWarps); /* s_qmask and s_qcnt are reused; the list is complete */
        /* the cells of the next tick's rows, into L2 ahead of their loads */
        const int nnext = s_nlist[q][nq];
        const int lines = (M * 16 + 127) / 128 + 1; /* a row's cells, not 128-byte aligned */
        for (int e = qt; e < nnext * lines; e += 32 * kResQueueWarps) {
          const int rr = e / lines, ln = e - rr * lines;
          const char* row = (const char*)(J.cell + (size_t)(h * C + out[rr]) * M);
          const char* end = row + (size_t)M * 16;
          const char* a = (const char*)((uintptr_t)row & ~(uintptr_t)127) + (size_t)ln * 128;
          if (a < end) asm volatile("prefetch.global.L2 [%0];" ::"l"(a));
        }
      }
    }
    __syncthreads();
    MPROBE(10);
    if (!s_qok) break;

    /* the next tick's uniforms (they depend on tick and MCU only) */
    if (it + 1 < it0 + n_ticks) {
      {
        const int j = (tid + kProjThreads / 2) & (kProjThreads - 1);
        if (j < M) {
          const uint32_t idx = (uint32_t)(h * M + j);
          r_u[j] = bx_uniform01(pop.rng_seed, pop.rng_pop, (uint32_t)(simstep + 1), idx);
          r_up[j] = poisson ? bx_uniform01_poisson(pop.rng_seed, pop.rng_pop, (uint32_t)(simstep + 1), idx) : 1.0f;
        }
      }
      MPROBE(11);
      /* the next tick's population update reads the uniforms drawn here */
      __syncthreads();
    }
  }

  /* ---- write the resident state back: the last tick's buffers ---- */
  __syncthreads();
  if (it > it0) {
    const int last = it - 1;
    const int curL = (rp->k0 + last) & 1;
    const int lpn = ((last - it0) & 1) ^ 1; /* the list the next tick reads */
    for (int j = tid; j < M; j += blockDim.x) {
      const int idx = h * M + j;
      pop.dsup[curL][idx] = r_dsup[j];
      pop.ada[idx] = r_ada[j];
      pop.act[idx] = r_act[j];
      pop.counter[idx] = r_cnt[j];
    }
    for (int q = 0; q < n_in; ++q) {
      const ProjDev& J = s_proj[q];
      const int C = J.C;
      const ResQ V = res_q(sm, L, q, M, C);
      const size_t eoff = (size_t)J.proj_in_pop * n;
      for (int j = tid; j < M; j += blockDim.x) {
        const int idx = h * M + j;
        J.pj[idx] = V.pj[j];
        J.ej[idx] = V.ej[j];
        J.zj[idx] = V.zj[j];
        pop.epsc[curL][eoff + idx] = V.epsc[j];
        pop.bj[curL][eoff + idx] = V.bj[j];
      }
      for (int s = tid; s < C; s += blockDim.x) {
        const int r = h * C + s;
        J.qi[r] = V.qi[s];
        J.pi[r] = V.pi[s];
        J.ei[r] = V.ei[s];
        J.zi[r] = V.zi[s];
        J.ti[r] = V.ti[s];
      }
      const int cnt = s_nlist[q][lpn];
      for (int e = tid; e < cnt; e += blockDim.x) J.list[h * C + e] = h * C + V.list[lpn * C + e];
      if (tid == 0) J.list_cnt[h] = cnt;
    }
  }
#ifdef BCPNN_PHASE_PROBE
  __syncthreads();
  if (tid < kProbeSlots && blockIdx.x < kProbeCtas)
    atomicAdd(&g_phase_probe[blockIdx.x * kProbeSlots + tid], g_probe_smem[tid]);
#endif
}

/* update_all_cpu (Proj.cpp:490-555) for projection p at a change of prn:
   every row and its cells caught up to simstep0-1 with kp = taupdt*old_prn,
   replaying the ring up to and including that tick.  One warp per row. */
__global__ void all_kernel(const NetDev* __restrict__ net, const RunParams* __restrict__ rp, int p) {
  const ProjDev& J = net->projs[p];
  const PopDev& pop = net->pops[J.dest];
  const int M = J.M, C = J.C, n = pop.n, B = pop.ring_len;
  const int simstep = rp->simstep0 - 1;
  const float kp = J.taupdt * rp->old_prn;
  const Coef k = make_coef(kp, J.ke, J.kzi, J.kzj);
  const float4* tab = rp->tabs[p].tab_old;
  const int tlen = rp->tabs[p].old_len;
  const int lane = threadIdx.x & 31;
  const int R = J.H * C;
  if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&net->counters[2], (unsigned long long)R * M);
  for (int r = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); r < R; r += (gridDim.x * blockDim.x) >> 5) {
    const int ti = J.ti[r];
    const float zi = J.zi[r];
    const int h = r / C;
    const int pdt = simstep - ti;
    float4 rA = make_float4(0, 0, 0, 0), rB = rA;
    if (pdt > 0) entry(tab, tlen, k, pdt, 2, rA, rB);
    if (lane == 0 && pdt > 0) {
      float pi = J.pi[r], ei = J.ei[r], z = zi;
      row_decay(pi, ei, z, k, rA, rB);
      J.pi[r] = pi;
      J.ei[r] = ei;
    }
    __syncwarp();
    const float pi_new = J.pi[r];
    for (int j = lane; j < M; j += 32) {
      const size_t index = (size_t)r * M + j;
      float4 c4 = J.cell[index];
      replay_cell(c4, ti, zi, simstep, 0, pop.ring, B, n, h * M + j, k, tab, tlen, nullptr, J.kftj, false);
      J.cell[index] = c4;
      if (kp != 0.0f)
        J.wij[index] = J.wgain * bx_logf((c4.x + J.eps2) / ((pi_new + J.eps) * (J.pj[h * M + j] + J.eps)));
    }
    __syncwarp();
    if (lane == 0) {
      if (pdt > 0) J.zi[r] = zi * rB.w;
      J.ti[r] = simstep;
    }
    __syncwarp();
  }
}

}  // namespace multi
}  // namespace bcpnn

#endif /* BCPNN_MULTI_CUH */
