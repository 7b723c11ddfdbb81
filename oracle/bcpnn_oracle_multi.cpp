/*
 * bcpnn_oracle_multi.cpp -- TEST INFRASTRUCTURE, NOT PART OF THE PRODUCT.
 *
 * A C++ restatement of gsbn's ProcUpdMulti (the row-only update that replays
 * a ring of postsynaptic spikes), float32 scalar arithmetic, the same
 * expression trees as the Python restatement oracle/multi.py (which the tests
 * hold it to bit for bit) and as the reference text (paths relative to the
 * gsbn source tree):
 *
 *   ProcUpdMulti::update_cpu   src/gsbn/procedures/ProcUpdMulti.cpp:94-125
 *   Pop::init_new              ProcUpdMulti/Pop.cpp:6-110 (dsup, act, ada, spike ring)
 *   update_sup_kernel_1..3     ProcUpdMulti/Pop.cpp:222-401
 *   Proj::init_new             ProcUpdMulti/Proj.cpp:6-108
 *   update_all_kernel_cpu      ProcUpdMulti/Proj.cpp:210-319, update_all_cpu 490-555
 *   update_jxx_kernel_cpu      ProcUpdMulti/Proj.cpp:321-362, update_jxx_cpu 557-583
 *   update_row_kernel_cpu      ProcUpdMulti/Proj.cpp:364-488, update_row_cpu 638-706
 *   update_que_cpu             ProcUpdMulti/Proj.cpp:620-636 (ssi: 585-594)
 *   ProcExchangeSpike          src/gsbn/procedures/ProcExchangeSpike.cpp:94-139
 *
 * It exists for speed: the Python restatement is sized for 10x10 networks,
 * this one runs the 100x100 workload and is the CPU baseline of the
 * ProcUpdMulti measurement.  Deviations from the reference are those of the
 * ProcUpdLazy oracle: Philox streams for the uniform and normal draws, the
 * shared bit-exact exp/log (bx_expf/bx_logf).  Parity against a gsbn binary
 * is unpinned (the reference cannot be built here).
 *
 * Built into oracle/_build/libbcpnn_oracle.so with bcpnn_oracle.cpp
 * (oracle/Makefile: -O2 -ffp-contract=off, no fast-math), so every float
 * operation below is one correctly rounded IEEE operation.
 */
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "bcpnn_numerics.h"

namespace oracle_multi {

static inline float E(float x) { return bx_expf(x); }
static inline float L(float x) { return bx_logf(x); }

struct Pop {
  int H, M, n, hcu_start, mcu_start, dim_proj = 0;
  float taumdt, wtagain, maxfqdt, igain, wgain, lgbias, snoise, tauadt, adgain;
  std::vector<float> dsup, act, ada, epsc, bj;
  std::vector<int8_t> ring, spike;  // ring: [B][n]
  std::vector<int> counter;
};

struct Proj {
  int src, dest, H, M, C, proj_in_pop;
  float kzi, kzj, ke, taupdt, eps, eps2, kfti, kftj, bgain, wgain, kepsc;
  std::vector<int> ii, di, qi, ti;
  std::vector<int8_t> siq, si;
  std::vector<float> pi, ei, zi, pj, ej, zj, pij, eij, zj2, wij;
};

struct Net {
  float dt;
  uint32_t seed;
  int B;
  std::vector<Pop> pops;
  std::vector<Proj> projs;
  std::vector<float> lginp, wmask;
  uint64_t row_cells = 0, all_cells = 0;
};

/* Pop::init_new (ProcUpdMulti/Pop.cpp:6-110) and Proj::init_new
   (ProcUpdMulti/Proj.cpp:6-108): coefficients and initial values.  pop_f per
   population: taum, wtagain, maxfq, igain, wgain, lgbias, snoise, taua,
   adgain; proj_f per projection: tauzi, tauzj, taue, taup, maxfq, bgain,
   wgain, tauepsc (<= 0: absent), slot_num. */
static Net* build(float dt, uint32_t seed, int B, int n_pops, const int* dims, const float* pop_f, int n_projs,
                  const int* proj_i, const float* proj_f) {
  Net* net = new Net();
  net->dt = dt;
  net->seed = seed;
  net->B = B;
  int hcu = 0, mcu = 0;
  for (int k = 0; k < n_pops; ++k) {
    const float* f = pop_f + 9 * k;
    Pop p;
    p.H = dims[2 * k];
    p.M = dims[2 * k + 1];
    p.n = p.H * p.M;
    p.hcu_start = hcu;
    p.mcu_start = mcu;
    p.taumdt = dt / f[0];
    p.wtagain = f[1];
    p.maxfqdt = f[2] * dt;
    p.igain = f[3];
    p.wgain = f[4];
    p.lgbias = f[5];
    p.snoise = f[6];
    p.tauadt = dt / f[7];
    p.adgain = f[8];
    p.dsup.assign(p.n, (float)bx_log_d(1.0 / p.M));
    p.act.assign(p.n, (float)(1.0 / p.M));
    p.ada.assign(p.n, 0.0f);
    p.ring.assign((size_t)B * p.n, 0);
    p.spike.assign(p.n, 0);
    p.counter.assign(p.n, 0);
    net->pops.push_back(p);
    hcu += p.H;
    mcu += p.n;
  }
  for (int q = 0; q < n_projs; ++q) {
    const float* f = proj_f + 9 * q;
    Proj J;
    J.src = proj_i[2 * q];
    J.dest = proj_i[2 * q + 1];
    Pop& P = net->pops[J.dest];
    const Pop& S = net->pops[J.src];
    float tauzi = f[0], tauzj = f[1], taue = f[2], taup = f[3], maxfq = f[4], tauepsc = f[7];
    J.H = P.H;
    J.M = P.M;
    J.C = S.n < (int)f[8] ? S.n : (int)f[8];
    J.proj_in_pop = P.dim_proj;
    J.kzi = dt / tauzi;
    J.kzj = dt / tauzj;
    J.ke = dt / taue;
    J.taupdt = dt / taup;
    J.eps = dt / taup;
    J.eps2 = J.eps * J.eps;
    J.kfti = 1.0f / (maxfq * tauzi);
    J.kftj = 1.0f / (maxfq * tauzj);
    J.bgain = f[5];
    J.wgain = f[6];
    J.kepsc = tauepsc > 0 ? dt / tauepsc : dt / tauzi;
    size_t R = (size_t)J.H * J.C;
    J.ii.assign(R, -1);
    J.di.assign(R, 0);
    J.qi.assign(R, 0);
    J.ti.assign(R, 0);
    J.siq.assign(R, 0);
    J.pi.assign(R, (float)(1.0 / J.C));
    J.ei.assign(R, 0.0f);
    J.zi.assign(R, 0.0f);
    J.pj.assign(P.n, (float)(1.0 / P.M));
    J.ej.assign(P.n, 0.0f);
    J.zj.assign(P.n, 0.0f);
    J.pij.assign(R * J.M, (float)(1.0 / J.C / P.M));
    J.eij.assign(R * J.M, 0.0f);
    J.zj2.assign(R * J.M, 0.0f);
    J.wij.assign(R * J.M, 0.0f);
    J.si.assign(S.n, 0);
    P.dim_proj += 1;
    net->projs.push_back(J);
  }
  for (Pop& P : net->pops) {
    int d = P.dim_proj > 0 ? P.dim_proj : 1;
    P.epsc.assign((size_t)d * P.n, 0.0f);
    P.bj.assign((size_t)d * P.n, 0.0f);
  }
  return net;
}

/* update_sup_kernel_1..3 (ProcUpdMulti/Pop.cpp:222-401): support with the
   adaptation current and the constant 6.9*wmask added in double, the soft
   WTA seeded with the HCU's own first MCU, spikes into the ring. */
static void pop_update(Net& net, int k, Pop& P, int t) {
  const int H = P.H, M = P.M;
  std::vector<int8_t> spk(P.n, 0);
  for (int i = 0; i < H; ++i) {
    float wm = net.wmask[P.hcu_start + i];
    for (int j = 0; j < M; ++j) {
      int idx = i * M + j;
      float wsup = 0.0f;
      size_t off = 0;
      for (int d = 0; d < P.dim_proj; ++d) {
        wsup = wsup + (P.bj[off + idx] + P.epsc[off + idx]);
        off += P.n;
      }
      float noise = P.snoise != 0 ? P.snoise * bx_normal01(net.seed, (uint32_t)k, (uint32_t)t, (uint32_t)idx) : 0.0f;
      float sup = (P.lgbias + P.igain * net.lginp[P.mcu_start + idx]) + noise;
      sup = sup + (P.wgain * wm) * wsup;
      sup = sup - wm * P.ada[idx];
      sup = (float)((double)sup + 6.9 * (double)wm);
      float d = P.dsup[idx];
      P.dsup[idx] = d + (sup - d) * P.taumdt;
    }
    int base = i * M;
    float mx = P.dsup[base];
    for (int m = 0; m < M; ++m)
      if (P.dsup[base + m] > mx) mx = P.dsup[base + m];
    float maxact = E(P.wtagain * mx);
    float vsum = 0.0f;
    for (int m = 0; m < M; ++m) {
      float a = E(P.wtagain * (P.dsup[base + m] - mx));
      if (maxact < 1) a = a * maxact;
      vsum = vsum + a;
      P.act[base + m] = a;
    }
    if (vsum > 1)
      for (int m = 0; m < M; ++m) P.act[base + m] = P.act[base + m] / vsum;
    for (int j = 0; j < M; ++j) {
      int idx = base + j;
      float u = bx_uniform01(net.seed, (uint32_t)k, (uint32_t)t, (uint32_t)idx);
      int8_t s = u < P.act[idx] * P.maxfqdt ? 1 : 0;
      spk[idx] = s;
      P.counter[idx] += s;
      P.ada[idx] = P.ada[idx] + ((P.adgain * P.act[idx]) - P.ada[idx]) * P.tauadt;
    }
  }
  std::memcpy(&P.ring[(size_t)(t % net.B) * P.n], spk.data(), P.n);
  P.spike = spk;
}

/* closed-form row traces, ProcUpdMulti/Proj.cpp:244-251 */
static void row_traces(float& pi, float& ei, float zi, int pdt, float kp, float ke, float kzi) {
  float fd = (float)pdt;
  float a = kp * fd;
  float x = (((ei * kp) * kzi) - ((ei * ke) * kp)) + ((ke * kp) * zi);
  float t1 = x / (ke - kp);
  float t2 = ((ke * kp) * zi) / (kp - kzi);
  float pn = (pi - (t1 + t2) / (ke - kzi)) / E(a);
  float u1 = (E(a - ke * fd) * x) / (ke - kp);
  float u2 = (((ke * kp) * zi) * E(a - kzi * fd)) / (kp - kzi);
  pn = pn + (u1 + u2) / (E(a) * (ke - kzi));
  float b = ke * fd;
  float en = (ei - (ke * zi) / (ke - kzi)) / E(b) + ((ke * zi) * E(b - kzi * fd)) / (E(b) * (ke - kzi));
  pi = pn;
  ei = en;
}

/* closed-form cell traces, ProcUpdMulti/Proj.cpp:268-275 */
static void cell(float& pij, float& eij, float zi2, float zj2, int pdt, float kp, float ke, float kzi, float kzj) {
  float fd = (float)pdt;
  float a = kp * fd;
  float zz = ((ke * kp) * zi2) * zj2;
  float x = ((((eij * kp) * kzi) - ((eij * ke) * kp)) + ((eij * kp) * kzj)) + zz;
  float d2 = (kzi - kp) + kzj;
  float d3 = (kzi - ke) + kzj;
  float pn = (pij + ((x / (ke - kp)) - (zz / d2)) / d3) / E(a);
  float v1 = (E(a - ke * fd) * x) / (ke - kp);
  float v2 = (zz * E((a - kzi * fd) - kzj * fd)) / d2;
  pn = pn - (v1 - v2) / (E(a) * d3);
  float w = (ke * zi2) * zj2;
  float en = ((eij + w / d3) / E(ke * fd)) - (w / ((E(kzi * fd) * E(kzj * fd)) * d3));
  pij = pn;
  eij = en;
}

/* the cell loop of update_row/update_all_kernel_cpu: replay the ring's
   postsynaptic spikes after tij (the newest B ticks at most) into one cell;
   `exclusive` leaves out a spike at simstep itself */
static void replay(const Net& net, const Proj& J, const Pop& P, int row, int j, int& tij, float& zi2, int simstep,
                   float kp, bool exclusive, float& pij, float& eij, float& zj2) {
  size_t idx = (size_t)row * J.M + j;
  pij = J.pij[idx];
  eij = J.eij[idx];
  zj2 = J.zj2[idx];
  int mcu = (row / J.C) * J.M + j;
  int now = tij;
  if (simstep - now >= net.B) now = simstep - net.B + 1;
  while (now < simstep) {
    now += 1;
    if (P.ring[(size_t)(now % net.B) * P.n + mcu] > 0 && (!exclusive || now < simstep)) {
      int pdt = now - tij;
      if (pdt > 0) {
        cell(pij, eij, zi2, zj2, pdt, kp, J.ke, J.kzi, J.kzj);
        zi2 = zi2 * E(-J.kzi * (float)pdt);
        zj2 = zj2 * E(-J.kzj * (float)pdt) + J.kftj;
        tij = now;
      }
    }
  }
}

/* update_all_cpu with simstep-1 (ProcUpdMulti/Proj.cpp:490-555, kernel
   210-319): every row and cell brought to the previous tick at a change of
   prn, with the old prn. */
static void proj_all(Net& net, Proj& J, int simstep, float old_prn) {
  const Pop& P = net.pops[J.dest];
  int t = simstep - 1;
  float kp = J.taupdt * old_prn;
  int R = J.H * J.C;
  for (int i = 0; i < R; ++i) {
    int ti = J.ti[i];
    float zi = J.zi[i];
    int pdt = t - ti;
    if (pdt > 0) row_traces(J.pi[i], J.ei[i], zi, pdt, kp, J.ke, J.kzi);
    for (int j = 0; j < J.M; ++j) {
      int tij = ti;
      float zi2 = zi, pij, eij, zj2;
      replay(net, J, P, i, j, tij, zi2, t, kp, false, pij, eij, zj2);
      int pdt2 = t - tij;
      if (pdt2 > 0) {
        cell(pij, eij, zi2, zj2, pdt2, kp, J.ke, J.kzi, J.kzj);
        zj2 = zj2 * E(-J.kzj * (float)pdt2);
      }
      size_t idx = (size_t)i * J.M + j;
      J.pij[idx] = pij;
      J.eij[idx] = eij;
      J.zj2[idx] = zj2;
      if (kp != 0) {
        float pj = J.pj[(i / J.C) * J.M + j];
        J.wij[idx] = J.wgain * L((pij + J.eps2) / ((J.pi[i] + J.eps) * (pj + J.eps)));
      }
    }
    if (pdt > 0) J.zi[i] = zi * E(-J.kzi * (float)pdt);
    J.ti[i] = t;
  }
  net.all_cells += (uint64_t)R * J.M;
}

/* update_jxx, update_ssi, update_row and update_que of one projection
   (ProcUpdMulti/Proj.cpp:557-583, 585-594, 638-706, 620-636) */
static void proj_update(Net& net, Proj& J, int simstep, float prn) {
  Pop& P = net.pops[J.dest];
  const int M = J.M, C = J.C, n = P.n;
  float kp = J.taupdt * prn;
  size_t eoff = (size_t)J.proj_in_pop * n;
  const int8_t* sj = &P.ring[(size_t)(simstep % net.B) * n];
  for (int idx = 0; idx < n; ++idx) {
    P.epsc[eoff + idx] = P.epsc[eoff + idx] * (1.0f - J.kepsc);
    float pj = J.pj[idx], ej = J.ej[idx], zj = J.zj[idx];
    pj = pj + (ej - pj) * kp;
    ej = ej + (zj - ej) * J.ke;
    zj = zj * (1.0f - J.kzj);
    if (sj[idx] > 0) zj = zj + J.kftj;
    if (kp != 0) P.bj[eoff + idx] = J.bgain * L(pj + J.eps);
    J.pj[idx] = pj;
    J.ej[idx] = ej;
    J.zj[idx] = zj;
  }
  int R = J.H * C;
  uint64_t rows = 0;
  for (int row = 0; row < R; ++row) {
    if (J.siq[row] <= 0) continue;
    ++rows;
    int ti = J.ti[row];
    float zi = J.zi[row];
    int pdt = simstep - ti;
    if (pdt > 0) row_traces(J.pi[row], J.ei[row], zi, pdt, kp, J.ke, J.kzi);
    int h = row / C;
    for (int j = 0; j < M; ++j) {
      int tij = ti;
      float zi2 = zi, pij, eij, zj2;
      replay(net, J, P, row, j, tij, zi2, simstep, kp, true, pij, eij, zj2);
      int pdt2 = simstep - tij;
      cell(pij, eij, zi2, zj2, pdt2, kp, J.ke, J.kzi, J.kzj);
      zj2 = zj2 * E(-J.kzj * (float)pdt2);
      if (sj[h * M + j] > 0) zj2 = zj2 + J.kftj;
      size_t idx = (size_t)row * M + j;
      J.pij[idx] = pij;
      J.eij[idx] = eij;
      J.zj2[idx] = zj2;
      float w;
      if (kp != 0) {
        float pj = J.pj[h * M + j];
        w = J.wgain * L((pij + J.eps2) / ((J.pi[row] + J.eps) * (pj + J.eps)));
        J.wij[idx] = w;
      } else {
        w = J.wij[idx];
      }
      P.epsc[eoff + h * M + j] = P.epsc[eoff + h * M + j] + w;
    }
    if (pdt > 0) J.zi[row] = zi * E(-J.kzi * (float)pdt) + J.kfti;
    J.ti[row] = simstep;
  }
  net.row_cells += rows * M;
  for (int r = 0; r < R; ++r) {
    if (J.ii[r] < 0) continue;
    J.siq[r] = (int8_t)(J.qi[r] & 1);
    J.qi[r] >>= 1;
    if (J.si[J.ii[r]] > 0) J.qi[r] |= 1 << (J.di[r] - 1);
  }
}

/* ProcUpdMulti::update_cpu (ProcUpdMulti.cpp:94-125) for ticks first ..
   first+n-1, then ProcExchangeSpike (si <- the source population's spikes);
   logs: per population [n][words] spike bits, concatenated, or null. */
static void run(Net& net, int first, int n, float prn, float old_prn, uint32_t* logs) {
  std::vector<size_t> log_off(net.pops.size());
  size_t off = 0;
  for (size_t q = 0; q < net.pops.size(); ++q) {
    log_off[q] = off;
    off += (size_t)n * ((net.pops[q].n + 31) / 32);
  }
  if (logs) std::memset(logs, 0, off * sizeof(uint32_t));
  for (int k = 0; k < n; ++k) {
    int t = first + k;
    for (size_t q = 0; q < net.pops.size(); ++q) {
      Pop& P = net.pops[q];
      pop_update(net, (int)q, P, t);
      if (logs) {
        uint32_t* row = logs + log_off[q] + (size_t)k * ((P.n + 31) / 32);
        for (int i = 0; i < P.n; ++i)
          if (P.spike[i]) row[i >> 5] |= 1u << (i & 31);
      }
    }
    for (Proj& J : net.projs) {
      if (k == 0 && prn != old_prn) proj_all(net, J, t, old_prn);
      proj_update(net, J, t, prn);
    }
    for (Proj& J : net.projs) J.si = net.pops[J.src].spike;
  }
}

/* named state vector: kind 0 f32, 1 i32, 2 i8 */
static void* find(Net* net, const std::string& name, int* kind, size_t* count) {
  size_t us = name.rfind('_');
  if (us == std::string::npos) return nullptr;
  std::string base = name.substr(0, us);
  int k = std::atoi(name.c_str() + us + 1);
  if (base == "dsup" || base == "act" || base == "ada" || base == "epsc" || base == "bj" || base == "spike" ||
      base == ".counter") {
    if (k < 0 || k >= (int)net->pops.size()) return nullptr;
    Pop& P = net->pops[k];
    if (base == "spike") { *kind = 2; *count = P.spike.size(); return P.spike.data(); }
    if (base == ".counter") { *kind = 1; *count = P.counter.size(); return P.counter.data(); }
    std::vector<float>& v = base == "dsup" ? P.dsup : base == "act" ? P.act : base == "ada" ? P.ada
                          : base == "epsc" ? P.epsc : P.bj;
    *kind = 0;
    *count = v.size();
    return v.data();
  }
  if (k < 0 || k >= (int)net->projs.size()) return nullptr;
  Proj& J = net->projs[k];
  std::vector<int>* vi = base == "ii" ? &J.ii : base == "di" ? &J.di : base == "qi" ? &J.qi
                       : base == "ti" ? &J.ti : nullptr;
  if (vi) { *kind = 1; *count = vi->size(); return vi->data(); }
  std::vector<int8_t>* v8 = (base == "siq" || base == ".siq") ? &J.siq : base == "si" ? &J.si : nullptr;
  if (v8) { *kind = 2; *count = v8->size(); return v8->data(); }
  std::vector<float>* vf = base == "pi" ? &J.pi : base == "ei" ? &J.ei : base == "zi" ? &J.zi
                         : base == "pj" ? &J.pj : base == "ej" ? &J.ej : base == "zj" ? &J.zj
                         : base == "pij" ? &J.pij : base == "eij" ? &J.eij : base == "zj2" ? &J.zj2
                         : base == "wij" ? &J.wij : nullptr;
  if (vf) { *kind = 0; *count = vf->size(); return vf->data(); }
  return nullptr;
}

}  // namespace oracle_multi

using oracle_multi::Net;

extern "C" {

void* oracle_multi_create(float dt, uint32_t seed, int spike_buffer, int n_pops, const int* pop_dims,
                          const float* pop_f, int n_projs, const int* proj_i, const float* proj_f) {
  if (spike_buffer < 1 || n_pops < 1) return nullptr;
  return oracle_multi::build(dt, seed, spike_buffer, n_pops, pop_dims, pop_f, n_projs, proj_i, proj_f);
}

void oracle_multi_destroy(void* h) { delete (Net*)h; }

/* lginp over all MCUs of all populations, wmask_row over all HCUs */
int oracle_multi_set_stimulus(void* h, const float* lginp, const float* wmask_row) {
  Net* net = (Net*)h;
  int mcus = 0, hcus = 0;
  for (auto& P : net->pops) { mcus += P.n; hcus += P.H; }
  net->lginp.assign(lginp, lginp + mcus);
  net->wmask.assign(wmask_row, wmask_row + hcus);
  return 0;
}

int oracle_multi_run(void* h, int first, int n, float prn, float old_prn, uint32_t* logs) {
  Net* net = (Net*)h;
  if (net->lginp.empty() || n < 0) return -1;
  oracle_multi::run(*net, first, n, prn, old_prn, logs);
  return 0;
}

long long oracle_multi_state_info(void* h, const char* name, int* kind) {
  size_t count = 0;
  if (!oracle_multi::find((Net*)h, name, kind, &count)) return -1;
  return (long long)count;
}

int oracle_multi_read_state(void* h, const char* name, void* out, size_t bytes) {
  int kind = 0;
  size_t count = 0;
  void* p = oracle_multi::find((Net*)h, name, &kind, &count);
  if (!p) return -1;
  size_t esz = kind == 2 ? 1 : 4;
  if (bytes != count * esz) return -2;
  if (bytes) std::memcpy(out, p, bytes);
  return 0;
}

int oracle_multi_write_state(void* h, const char* name, const void* in, size_t bytes) {
  int kind = 0;
  size_t count = 0;
  void* p = oracle_multi::find((Net*)h, name, &kind, &count);
  if (!p) return -1;
  size_t esz = kind == 2 ? 1 : 4;
  if (bytes != count * esz) return -2;
  if (bytes) std::memcpy(p, in, bytes);
  return 0;
}

/* cells brought to the current tick: active-row cells and all-cells sweeps
   (the counters the device keeps for this variant) */
void oracle_multi_counters(void* h, unsigned long long* out2) {
  Net* net = (Net*)h;
  out2[0] = net->row_cells;
  out2[1] = net->all_cells;
}

}  // extern "C"
