/*
 * bcpnn_oracle.cpp -- TEST INFRASTRUCTURE, NOT PART OF THE PRODUCT.
 *
 * A CPU restatement of gsbn's ProcUpdLazy hot path (population update,
 * lazy-update projection kernels, delay queue, spike compaction) and of the
 * single-rank semantics of ProcExchangeSpike.  It follows the reference loop
 * order and expression trees one for one; each function cites the reference
 * file:line it restates (paths relative to the gsbn source tree).  Only
 * tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg load it, and
 * only as the checker or the timed CPU baseline.
 *
 * Deliberate deviations from the reference, all selectable:
 *   - RNG: gsbn's Random (std::default_random_engine / cuRAND seeded from
 *     std::random_device, src/gsbn/Random.cpp:5-13) is replaced by the
 *     Philox4x32-10 stream map of include/bcpnn_numerics.h.
 *   - math: MATH_LIBM calls std::exp/std::log on the value type exactly like
 *     the reference (float -> glibc expf/logf); MATH_SHARED calls the shared
 *     bx_expf/bx_logf so the GPU kernels can match bit for bit.
 *   - value type: float (the reference) or double (the FP64 oracle used to
 *     state the error of the BF16/FP32 extensions).
 *   - poisson-noise-hz: project-defined input noise (absent from gsbn): an
 *     independent Bernoulli(f dt) spike per MCU per tick OR-ed into the sampled
 *     spike before the counter and the projections see it.
 *
 * Parity status: the reference cannot be built in this environment (its
 * sources need protoc-generated gsbn.pb.h, libprotobuf and MPI), and its RNG
 * is unseedable, so no reference output exists to compare against.  The
 * restatement is pinned on the reference's own fixtures (prototxt, stimulus
 * file and connection maps decode identically), on the published Philox
 * known-answer vectors, and on analytical identities of the closed-form trace
 * solution; numeric parity against a reference binary is unpinned.
 *
 * Build: oracle/Makefile (g++ -O2 -ffp-contract=off, no fast-math, no OpenMP),
 * output oracle/_build/libbcpnn_oracle.so.
 */
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <type_traits>
#include <vector>

#include "bcpnn_numerics.h"

#ifdef BCPNN_ORACLE_REF
/* gsbn's own kernels (ProcUpdLazy/Proj.cpp:209-536, ProcUpdLazy/Pop.cpp:
   229-323), compiled from the gsbn sources by oracle/extract_ref_kernels.sh.
   In math mode MATH_REF the oracle's loops call these instead of its own
   restatement, so the arithmetic is the reference's, unmodified. */
namespace gsbn {
namespace proc_upd_lazy {
void update_all_kernel_cpu(int i, int j, int dim_conn, int dim_mcu, float* ptr_pi, float* ptr_ei, float* ptr_zi,
                           int* ptr_ti, const float* ptr_pj, float* ptr_pij, float* ptr_eij, float* ptr_zi2,
                           float* ptr_zj2, int* ptr_tij, float* ptr_wij, int simstep, float kp, float ke, float kzi,
                           float kzj, float wgain, float eps, float eps2);
void update_jxx_kernel_cpu(int idx, const int8_t* ptr_sj, float* ptr_pj, float* ptr_ej, float* ptr_zj,
                           float* ptr_bj, float* ptr_epsc, float kp, float ke, float kzj, float kzi, float kepsc,
                           float kftj, float bgain, float eps);
void update_row_kernel_cpu(int i, int j, int dim_conn, int dim_mcu, const int* ptr_ssi, float* ptr_pi,
                           float* ptr_ei, float* ptr_zi, int* ptr_ti, const float* ptr_pj, float* ptr_pij,
                           float* ptr_eij, float* ptr_zi2, float* ptr_zj2, int* ptr_tij, float* ptr_wij,
                           float* ptr_epsc, int simstep, float kp, float ke, float kzi, float kzj, float kfti,
                           float wgain, float eps, float eps2);
void update_col_kernel_cpu(int i, int j, int dim_conn, int dim_mcu, const int* ptr_ii, const int* ptr_ssj,
                           float* ptr_pij, float* ptr_eij, float* ptr_zi2, float* ptr_zj2, int* ptr_tij,
                           int simstep, float kp, float ke, float kzi, float kzj, float kftj);
void update_sup_kernel_1_cpu(int i, int j, int dim_proj, int dim_hcu, int dim_mcu, const float* ptr_epsc,
                             const float* ptr_bj, const float* ptr_lginp, const float* ptr_wmask,
                             const float* ptr_rnd_normal, const float* ptr_ada, float* ptr_dsup, float wgain,
                             float lgbias, float igain, float taumdt);
void update_sup_kernel_2_cpu(int i, int dim_mcu, const float* ptr_dsup, float* ptr_act, float wtagain);
void update_sup_kernel_3_cpu(int i, int j, int dim_mcu, const float* ptr_act, const float* ptr_rnd_uniform01,
                             int8_t* ptr_spk, int* ptr_counter, float* ptr_ada, float maxfqdt, float adgain,
                             float ka);
}  // namespace proc_upd_lazy
}  // namespace gsbn
namespace ref = gsbn::proc_upd_lazy;
static constexpr bool kHaveRef = true;
#else
static constexpr bool kHaveRef = false;
#endif


namespace oracle {

enum { MATH_LIBM = 0, MATH_SHARED = 1, MATH_REF = 2 };


/* exp/log as the reference calls them (on the value type), or the shared
   definition. */
template <typename T> struct Fn;
template <> struct Fn<float> {
  static float exp(int mode, float x) { return mode == MATH_SHARED ? bx_expf(x) : std::exp(x); }
  static float log(int mode, float x) { return mode == MATH_SHARED ? bx_logf(x) : std::log(x); }
};
template <> struct Fn<double> {
  static double exp(int, double x) { return std::exp(x); }
  static double log(int, double x) { return std::log(x); }
};

/* log(double) used by Pop::init_new for dsup = log(1.0/M) (Pop.cpp:59). */
static double log_double(int mode, double x) {
  return mode == MATH_SHARED ? bx_log_d(x) : std::log(x);
}

template <typename T> struct Pop;
template <typename T> struct Proj;

/* ProcUpdLazy/Pop.hpp:12-83 (state only). */
template <typename T> struct Pop {
  int id = 0, dim_proj = 0, dim_hcu = 0, dim_mcu = 0, hcu_start = 0, mcu_start = 0;
  T taumdt, wtagain, maxfqdt, igain, wgain, lgbias, snoise;
  std::vector<T> dsup, act, epsc, bj, rnd_uniform01, rnd_normal;
  std::vector<int8_t> spike;
  std::vector<int> counter;
  bool flag_ext_spike = false;
  std::map<int, std::vector<int>> ext_spikes;
};

/* ProcUpdLazy/Proj.hpp:103-200 (state only). */
template <typename T> struct Proj {
  int id = 0, proj_in_pop = 0, dim_conn = 0, dim_hcu = 0, dim_mcu = 0;
  Pop<T>* src = nullptr;
  Pop<T>* dest = nullptr;
  T taupdt, tauedt, tauzidt, tauzjdt, tauepscdt, eps, eps2, kfti, kftj, wgain, bgain;
  std::vector<int> ii, qi, di, ti, tij, ssi, ssj;
  std::vector<int8_t> siq, si;
  std::vector<T> pi, ei, zi, pj, ej, zj, pij, eij, zi2, zj2, wij;
};

struct PopDesc { int hcu_num, mcu_num; float taum, wtagain, maxfq, igain, wgain, lgbias, snoise; };
struct ProjDesc {
  int src_pop, dest_pop;
  float tauzi, tauzj, taue, taup, maxfq, bgain, wgain, tauepsc; /* tauepsc <= 0: absent */
  float slot_num;
};

struct Counters { uint64_t row_cells = 0, col_cells = 0, all_cells = 0; };

template <typename T> struct Net {
  int math = MATH_SHARED;
  float dt = 0.001f;
  uint32_t seed = 0;
  float poisson_hz = 0.0f;
  std::vector<Pop<T>*> pops;
  std::vector<Proj<T>*> projs;
  std::vector<T> lginp;      /* .lginp row 0, total MCUs    */
  std::vector<T> wmask_row;  /* .wmask row wmask-idx, total HCUs */
  std::vector<int8_t> shared_buffer; /* ProcExchangeSpike::_shared_buffer */
  Counters cnt;
  ~Net() { for (auto p : pops) delete p; for (auto p : projs) delete p; }
};

/* Pop::init_new, ProcUpdLazy/Pop.cpp:8-65 (+ ProcUpdLazy.cpp:19-29 for the
   running hcu/mcu offsets). */
template <typename T>
void pop_init(Net<T>& net, const PopDesc& d, int* hcu_cnt, int* mcu_cnt) {
  Pop<T>* p = new Pop<T>();
  p->id = (int)net.pops.size();
  net.pops.push_back(p);
  p->dim_proj = 0;
  p->dim_hcu = d.hcu_num;
  p->dim_mcu = d.mcu_num;
  p->hcu_start = *hcu_cnt;
  p->mcu_start = *mcu_cnt;
  *hcu_cnt += p->dim_hcu;
  *mcu_cnt += p->dim_hcu * p->dim_mcu;
  T dt = (T)net.dt;
  p->taumdt = dt / (T)d.taum;
  p->wtagain = (T)d.wtagain;
  p->maxfqdt = (T)d.maxfq * dt;
  p->igain = (T)d.igain;
  p->wgain = (T)d.wgain;
  p->lgbias = (T)d.lgbias;
  p->snoise = (T)d.snoise;
  int n = p->dim_hcu * p->dim_mcu;
  p->dsup.assign(n, (T)log_double(net.math, 1.0 / p->dim_mcu));
  p->act.assign(n, (T)(1.0 / p->dim_mcu));
  p->spike.assign(n, 0);
  p->rnd_uniform01.assign(n, 0);
  p->rnd_normal.assign(n, 0);
  p->counter.assign(n, 0);
}

/* Proj::init_new, ProcUpdLazy/Proj.cpp:6-107. */
template <typename T>
void proj_init(Net<T>& net, const ProjDesc& d) {
  Proj<T>* j = new Proj<T>();
  j->id = (int)net.projs.size();
  net.projs.push_back(j);
  j->src = net.pops[d.src_pop];
  j->dest = net.pops[d.dest_pop];
  Pop<T>* p = j->dest;
  j->dim_hcu = p->dim_hcu;
  j->dim_mcu = p->dim_mcu;
  j->dim_conn = j->src->dim_hcu * j->src->dim_mcu;
  int slot_num = (int)d.slot_num;  /* float field read into int, Proj.cpp:23 */
  if (j->dim_conn > slot_num) j->dim_conn = slot_num;
  j->proj_in_pop = p->dim_proj;
  p->dim_proj++;
  T dt = (T)net.dt;
  j->tauzidt = dt / (T)d.tauzi;
  j->tauzjdt = dt / (T)d.tauzj;
  j->tauedt = dt / (T)d.taue;
  j->taupdt = dt / (T)d.taup;
  j->eps = dt / (T)d.taup;
  j->eps2 = (dt / (T)d.taup) * (dt / (T)d.taup);
  j->kfti = 1 / ((T)d.maxfq * (T)d.tauzi);
  j->kftj = 1 / ((T)d.maxfq * (T)d.tauzj);
  j->bgain = (T)d.bgain;
  j->wgain = (T)d.wgain;
  j->tauepscdt = d.tauepsc > 0 ? dt / (T)d.tauepsc : j->tauzidt;
  int nm = p->dim_proj * p->dim_hcu * p->dim_mcu;
  p->epsc.resize(nm, 0);
  p->bj.resize(nm, 0);
  int R = j->dim_hcu * j->dim_conn;
  int HM = j->dim_hcu * j->dim_mcu;
  size_t cells = (size_t)R * j->dim_mcu;
  j->ii.assign(R, -1);
  j->qi.assign(R, 0);
  j->di.assign(R, 0);
  j->pi.assign(R, (T)(1.0 / j->dim_conn));
  j->ei.assign(R, 0);
  j->zi.assign(R, 0);
  j->ti.assign(R, 0);
  j->siq.assign(R, 0);
  j->pj.assign(HM, (T)(1.0 / j->dim_mcu));
  j->ej.assign(HM, 0);
  j->zj.assign(HM, 0);
  j->pij.assign(cells, (T)(1.0 / j->dim_conn / j->dim_mcu));
  j->eij.assign(cells, 0);
  j->zi2.assign(cells, 0);
  j->zj2.assign(cells, 0);
  j->tij.assign(cells, 0);
  j->wij.assign(cells, 0);
  j->si.assign(j->src->dim_hcu * j->src->dim_mcu, 0);
}

/* Pop::update_rnd_cpu, Pop.cpp:220-227, with Random replaced by Philox. */
template <typename T>
void pop_update_rnd(Net<T>& net, Pop<T>* p, int simstep) {
  int size = p->dim_hcu * p->dim_mcu;
  for (int i = 0; i < size; i++) {
    p->rnd_uniform01[i] = (T)bx_uniform01(net.seed, (uint32_t)p->id, (uint32_t)simstep, (uint32_t)i);
    if (p->snoise != 0) {
      p->rnd_normal[i] = p->snoise * (T)bx_normal01(net.seed, (uint32_t)p->id, (uint32_t)simstep, (uint32_t)i);
    } else {
      p->rnd_normal[i] = 0;
    }
  }
}

/* update_sup_kernel_1_cpu, Pop.cpp:229-261. */
template <typename T>
void sup_kernel_1(int i, int j, int dim_proj, int dim_hcu, int dim_mcu, const T* ptr_epsc,
                  const T* ptr_bj, const T* ptr_lginp, const T* ptr_wmask, const T* ptr_rnd_normal,
                  T* ptr_dsup, T wgain, T lgbias, T igain, T taumdt) {
  int idx = i * dim_mcu + j;
  T wsup = 0;
  int offset = 0;
  int mcu_num_in_pop = dim_hcu * dim_mcu;
  for (int m = 0; m < dim_proj; m++) {
    wsup += ptr_bj[offset + idx] + ptr_epsc[offset + idx];
    offset += mcu_num_in_pop;
  }
  T sup = lgbias + igain * ptr_lginp[idx] + ptr_rnd_normal[idx];
  sup += (wgain * ptr_wmask[i]) * wsup;
  T dsup = ptr_dsup[idx];
  ptr_dsup[idx] += (sup - dsup) * taumdt;
}

/* update_sup_kernel_2_cpu, Pop.cpp:263-303.  The running max is seeded with
   dsup[0] of the population (Pop.cpp:270), not of HCU i. */
template <typename T>
void sup_kernel_2(int mode, int i, int dim_mcu, const T* ptr_dsup, T* ptr_act, T wtagain) {
  T maxdsup = ptr_dsup[0];
  for (int m = 0; m < dim_mcu; m++) {
    int idx = i * dim_mcu + m;
    T dsup = ptr_dsup[idx];
    if (dsup > maxdsup) maxdsup = dsup;
  }
  T maxact = Fn<T>::exp(mode, wtagain * maxdsup);
  T vsum = 0;
  for (int m = 0; m < dim_mcu; m++) {
    int idx = i * dim_mcu + m;
    T dsup = ptr_dsup[idx];
    T act = Fn<T>::exp(mode, wtagain * (dsup - maxdsup));
    if (maxact < 1) act *= maxact;
    vsum += act;
    ptr_act[idx] = act;
  }
  if (vsum > 1) {
    for (int m = 0; m < dim_mcu; m++) {
      int idx = i * dim_mcu + m;
      ptr_act[idx] /= vsum;
    }
  }
}

/* update_sup_kernel_3_cpu, Pop.cpp:305-323 (+ the project-defined Poisson
   input noise, OR-ed in before the counter). */
template <typename T>
void sup_kernel_3(Net<T>& net, Pop<T>* p, int simstep, int i, int j) {
  int idx = i * p->dim_mcu + j;
  int8_t spk = int8_t(p->rnd_uniform01[idx] < p->act[idx] * p->maxfqdt);
  if (net.poisson_hz > 0.0f) {
    float pr = net.poisson_hz * net.dt;
    float u = bx_uniform01_poisson(net.seed, (uint32_t)p->id, (uint32_t)simstep, (uint32_t)idx);
    if (u < pr) spk = 1;
  }
  p->spike[idx] = spk;
  p->counter[idx] += spk;
}

/* Pop::update_sup_cpu, Pop.cpp:325-387. */
template <typename T>
void pop_update_sup(Net<T>& net, Pop<T>* p, int simstep) {
  const T* ptr_wmask = net.wmask_row.data() + p->hcu_start;
  const T* ptr_lginp = net.lginp.data() + p->mcu_start;
#ifdef BCPNN_ORACLE_REF
  if constexpr (std::is_same<T, float>::value) {
    if (net.math == MATH_REF) {
      /* Pop::update_sup_cpu's loop (Pop.cpp:343-386) over gsbn's kernels;
         the adaptation pointer is unused there (its lines are commented out,
         Pop.cpp:258,322).  The project-defined Poisson input noise is OR-ed
         in afterwards with the same effect on spike and counter. */
      for (int i = 0; i < p->dim_hcu; i++) {
        for (int j = 0; j < p->dim_mcu; j++)
          ref::update_sup_kernel_1_cpu(i, j, p->dim_proj, p->dim_hcu, p->dim_mcu, p->epsc.data(), p->bj.data(),
                                       ptr_lginp, ptr_wmask, p->rnd_normal.data(), nullptr, p->dsup.data(),
                                       p->wgain, p->lgbias, p->igain, p->taumdt);
        ref::update_sup_kernel_2_cpu(i, p->dim_mcu, p->dsup.data(), p->act.data(), p->wtagain);
        for (int j = 0; j < p->dim_mcu; j++) {
          ref::update_sup_kernel_3_cpu(i, j, p->dim_mcu, p->act.data(), p->rnd_uniform01.data(), p->spike.data(),
                                       p->counter.data(), nullptr, p->maxfqdt, 0.0f, 0.0f);
          if (net.poisson_hz > 0.0f) {
            int idx = i * p->dim_mcu + j;
            float u = bx_uniform01_poisson(net.seed, (uint32_t)p->id, (uint32_t)simstep, (uint32_t)idx);
            if (u < net.poisson_hz * net.dt && p->spike[idx] == 0) {
              p->spike[idx] = 1;
              p->counter[idx] += 1;
            }
          }
        }
      }
      return;
    }
  }
#endif
  for (int i = 0; i < p->dim_hcu; i++) {
    for (int j = 0; j < p->dim_mcu; j++) {
      sup_kernel_1<T>(i, j, p->dim_proj, p->dim_hcu, p->dim_mcu, p->epsc.data(), p->bj.data(), ptr_lginp,
                      ptr_wmask, p->rnd_normal.data(), p->dsup.data(), p->wgain, p->lgbias, p->igain,
                      p->taumdt);
    }
    sup_kernel_2<T>(net.math, i, p->dim_mcu, p->dsup.data(), p->act.data(), p->wtagain);
    for (int j = 0; j < p->dim_mcu; j++) sup_kernel_3<T>(net, p, simstep, i, j);
  }
}

/* Pop::fill_spike, Pop.cpp:389-409: with an external spike file every tick
   is overwritten (a tick missing from the file gives an all-zero vector). */
template <typename T>
void pop_fill_spike(Pop<T>* p, int simstep) {
  if (!p->flag_ext_spike) return;
  std::vector<int> spk = p->ext_spikes[simstep];
  for (int i = 0; i < p->dim_hcu * p->dim_mcu; i++) p->spike[i] = 0;
  for (size_t i = 0; i < spk.size(); i++) p->spike[spk[i]] = 1;
}

/* update_all_kernel_cpu, Proj.cpp:209-308. */
template <typename T>
void all_kernel(int mode, int i, int j, int dim_conn, int dim_mcu, T* ptr_pi, T* ptr_ei, T* ptr_zi,
                int* ptr_ti, const T* ptr_pj, T* ptr_pij, T* ptr_eij, T* ptr_zi2, T* ptr_zj2, int* ptr_tij,
                T* ptr_wij, int simstep, T kp, T ke, T kzi, T kzj, T wgain, T eps, T eps2) {
  if (j == 0) {
    T pi = ptr_pi[i];
    T zi = ptr_zi[i];
    int ti = ptr_ti[i];
    int pdt = simstep - ti;
    if (pdt > 0) {
      T ei = ptr_ei[i];
      pi = (pi - ((ei * kp * kzi - ei * ke * kp + ke * kp * zi) / (ke - kp) + (ke * kp * zi) / (kp - kzi)) /
                     (ke - kzi)) / Fn<T>::exp(mode, kp * pdt) +
           ((Fn<T>::exp(mode, kp * pdt - ke * pdt) * (ei * kp * kzi - ei * ke * kp + ke * kp * zi)) / (ke - kp) +
            (ke * kp * zi * Fn<T>::exp(mode, kp * pdt - kzi * pdt)) / (kp - kzi)) /
               (Fn<T>::exp(mode, kp * pdt) * (ke - kzi));
      ei = (ei - (ke * zi) / (ke - kzi)) / Fn<T>::exp(mode, ke * pdt) +
           (ke * zi * Fn<T>::exp(mode, ke * pdt - kzi * pdt)) / (Fn<T>::exp(mode, ke * pdt) * (ke - kzi));
      zi = zi * Fn<T>::exp(mode, -kzi * pdt);
      ti = simstep;
      ptr_pi[i] = pi;
      ptr_ei[i] = ei;
      ptr_zi[i] = zi;
      ptr_ti[i] = ti;
    }
  }
  int index = i * dim_mcu + j;
  int tij = ptr_tij[index];
  T zi2 = ptr_zi2[index];
  int pdt = simstep - tij;
  if (pdt <= 0) {
    ptr_tij[index] = simstep;
  } else {
    T pij = ptr_pij[index];
    T eij = ptr_eij[index];
    T zj2 = ptr_zj2[index];
    pij = (pij + ((eij * kp * kzi - eij * ke * kp + eij * kp * kzj + ke * kp * zi2 * zj2) / (ke - kp) -
                  (ke * kp * zi2 * zj2) / (kzi - kp + kzj)) / (kzi - ke + kzj)) / Fn<T>::exp(mode, kp * pdt) -
          ((Fn<T>::exp(mode, kp * pdt - ke * pdt) *
            (eij * kp * kzi - eij * ke * kp + eij * kp * kzj + ke * kp * zi2 * zj2)) / (ke - kp) -
           (ke * kp * zi2 * zj2 * Fn<T>::exp(mode, kp * pdt - kzi * pdt - kzj * pdt)) / (kzi - kp + kzj)) /
              (Fn<T>::exp(mode, kp * pdt) * (kzi - ke + kzj));
    eij = (eij + (ke * zi2 * zj2) / (kzi - ke + kzj)) / Fn<T>::exp(mode, ke * pdt) -
          (ke * zi2 * zj2) / (Fn<T>::exp(mode, kzi * pdt) * Fn<T>::exp(mode, kzj * pdt) * (kzi - ke + kzj));
    zi2 = zi2 * Fn<T>::exp(mode, -kzi * pdt);
    zj2 = zj2 * Fn<T>::exp(mode, -kzj * pdt);
    tij = simstep;
    ptr_pij[index] = pij;
    ptr_eij[index] = eij;
    ptr_zi2[index] = zi2;
    ptr_zj2[index] = zj2;
    ptr_tij[index] = tij;
    if (kp) {
      T pi = ptr_pi[i];
      T pj = ptr_pj[i / dim_conn * dim_mcu + j];
      T wij = wgain * Fn<T>::log(mode, (pij + eps2) / ((pi + eps) * (pj + eps)));
      ptr_wij[index] = wij;
    }
  }
}

/* update_jxx_kernel_cpu, Proj.cpp:310-363. */
template <typename T>
void jxx_kernel(int mode, int idx, const int8_t* ptr_sj, T* ptr_pj, T* ptr_ej, T* ptr_zj, T* ptr_bj,
                T* ptr_epsc, T kp, T ke, T kzj, T kepsc, T kftj, T bgain, T eps) {
  T pj = ptr_pj[idx];
  T ej = ptr_ej[idx];
  T zj = ptr_zj[idx];
  int sj = ptr_sj[idx];
  ptr_epsc[idx] *= (1 - kepsc);
  pj += (ej - pj) * kp;
  ej += (zj - ej) * ke;
  zj *= (1 - kzj);
  if (sj > 0) zj += kftj;
  if (kp) {
    T bj = bgain * Fn<T>::log(mode, pj + eps);
    ptr_bj[idx] = bj;
  }
  ptr_pj[idx] = pj;
  ptr_ej[idx] = ej;
  ptr_zj[idx] = zj;
}

/* update_row_kernel_cpu, Proj.cpp:365-479. */
template <typename T>
void row_kernel(int mode, int i, int j, int dim_conn, int dim_mcu, const int* ptr_ssi, T* ptr_pi, T* ptr_ei,
                T* ptr_zi, int* ptr_ti, const T* ptr_pj, T* ptr_pij, T* ptr_eij, T* ptr_zi2, T* ptr_zj2,
                int* ptr_tij, T* ptr_wij, T* ptr_epsc, int simstep, T kp, T ke, T kzi, T kzj, T kfti,
                T wgain, T eps, T eps2) {
  int row = ptr_ssi[i];
  int col = j;
  int index = row * dim_mcu + col;
  if (j == 0) {
    T zi = ptr_zi[row];
    int ti = ptr_ti[row];
    int pdt = simstep - ti;
    if (pdt <= 0) {
      ptr_zi[row] += kfti;
      ptr_ti[row] = simstep;
    } else {
      T pi = ptr_pi[row];
      T ei = ptr_ei[row];
      pi = (pi - ((ei * kp * kzi - ei * ke * kp + ke * kp * zi) / (ke - kp) + (ke * kp * zi) / (kp - kzi)) /
                     (ke - kzi)) / Fn<T>::exp(mode, kp * pdt) +
           ((Fn<T>::exp(mode, kp * pdt - ke * pdt) * (ei * kp * kzi - ei * ke * kp + ke * kp * zi)) / (ke - kp) +
            (ke * kp * zi * Fn<T>::exp(mode, kp * pdt - kzi * pdt)) / (kp - kzi)) /
               (Fn<T>::exp(mode, kp * pdt) * (ke - kzi));
      ei = (ei - (ke * zi) / (ke - kzi)) / Fn<T>::exp(mode, ke * pdt) +
           (ke * zi * Fn<T>::exp(mode, ke * pdt - kzi * pdt)) / (Fn<T>::exp(mode, ke * pdt) * (ke - kzi));
      zi = zi * Fn<T>::exp(mode, -kzi * pdt) + kfti;
      ti = simstep;
      ptr_pi[row] = pi;
      ptr_ei[row] = ei;
      ptr_zi[row] = zi;
      ptr_ti[row] = ti;
    }
  }
  T pij = ptr_pij[index];
  int tij = ptr_tij[index];
  T zi2 = ptr_zi2[index];
  int pdt = simstep - tij;
  if (pdt <= 0) {
    ptr_zi2[index] += kfti;
    ptr_tij[index] = simstep;
  } else {
    T eij = ptr_eij[index];
    T zj2 = ptr_zj2[index];
    pij = (pij + ((eij * kp * kzi - eij * ke * kp + eij * kp * kzj + ke * kp * zi2 * zj2) / (ke - kp) -
                  (ke * kp * zi2 * zj2) / (kzi - kp + kzj)) / (kzi - ke + kzj)) / Fn<T>::exp(mode, kp * pdt) -
          ((Fn<T>::exp(mode, kp * pdt - ke * pdt) *
            (eij * kp * kzi - eij * ke * kp + eij * kp * kzj + ke * kp * zi2 * zj2)) / (ke - kp) -
           (ke * kp * zi2 * zj2 * Fn<T>::exp(mode, kp * pdt - kzi * pdt - kzj * pdt)) / (kzi - kp + kzj)) /
              (Fn<T>::exp(mode, kp * pdt) * (kzi - ke + kzj));
    eij = (eij + (ke * zi2 * zj2) / (kzi - ke + kzj)) / Fn<T>::exp(mode, ke * pdt) -
          (ke * zi2 * zj2) / (Fn<T>::exp(mode, kzi * pdt) * Fn<T>::exp(mode, kzj * pdt) * (kzi - ke + kzj));
    zi2 = zi2 * Fn<T>::exp(mode, -kzi * pdt) + kfti;
    zj2 = zj2 * Fn<T>::exp(mode, -kzj * pdt);
    tij = simstep;
    ptr_pij[index] = pij;
    ptr_eij[index] = eij;
    ptr_zi2[index] = zi2;
    ptr_zj2[index] = zj2;
    ptr_tij[index] = tij;
    T wij;
    int idx_hcu = row / dim_conn;
    int idx_mcu = idx_hcu * dim_mcu + j;
    if (kp) {
      T pi = ptr_pi[row];
      T pj = ptr_pj[idx_mcu];
      wij = wgain * Fn<T>::log(mode, (pij + eps2) / ((pi + eps) * (pj + eps)));
      ptr_wij[index] = wij;
    } else {
      wij = ptr_wij[index];
    }
    ptr_epsc[idx_mcu] += wij;
  }
}

/* update_col_kernel_cpu, Proj.cpp:481-536. */
template <typename T>
void col_kernel(int mode, int i, int j, int dim_conn, int dim_mcu, const int* ptr_ii, const int* ptr_ssj,
                T* ptr_pij, T* ptr_eij, T* ptr_zi2, T* ptr_zj2, int* ptr_tij, int simstep, T kp, T ke, T kzi,
                T kzj, T kftj) {
  int row = ptr_ssj[j] / dim_mcu * dim_conn + i;
  if (ptr_ii[row] < 0) return;
  int col = ptr_ssj[j] % dim_mcu;
  int index = row * dim_mcu + col;
  int tij = ptr_tij[index];
  T zj2 = ptr_zj2[index];
  int pdt = simstep - tij;
  if (pdt <= 0) {
    zj2 += kftj;
    ptr_zj2[index] = zj2;
    ptr_tij[index] = simstep;
  } else {
    T pij = ptr_pij[index];
    T eij = ptr_eij[index];
    T zi2 = ptr_zi2[index];
    pij = (pij + ((eij * kp * kzi - eij * ke * kp + eij * kp * kzj + ke * kp * zi2 * zj2) / (ke - kp) -
                  (ke * kp * zi2 * zj2) / (kzi - kp + kzj)) / (kzi - ke + kzj)) / Fn<T>::exp(mode, kp * pdt) -
          ((Fn<T>::exp(mode, kp * pdt - ke * pdt) *
            (eij * kp * kzi - eij * ke * kp + eij * kp * kzj + ke * kp * zi2 * zj2)) / (ke - kp) -
           (ke * kp * zi2 * zj2 * Fn<T>::exp(mode, kp * pdt - kzi * pdt - kzj * pdt)) / (kzi - kp + kzj)) /
              (Fn<T>::exp(mode, kp * pdt) * (kzi - ke + kzj));
    eij = (eij + (ke * zi2 * zj2) / (kzi - ke + kzj)) / Fn<T>::exp(mode, ke * pdt) -
          (ke * zi2 * zj2) / (Fn<T>::exp(mode, kzi * pdt) * Fn<T>::exp(mode, kzj * pdt) * (kzi - ke + kzj));
    zi2 = zi2 * Fn<T>::exp(mode, -kzi * pdt);
    zj2 = zj2 * Fn<T>::exp(mode, -kzj * pdt) + kftj;
    tij = simstep;
    ptr_pij[index] = pij;
    ptr_eij[index] = eij;
    ptr_zi2[index] = zi2;
    ptr_zj2[index] = zj2;
    ptr_tij[index] = tij;
  }
}

/* Proj::update_all_cpu, Proj.cpp:538-588. */
template <typename T>
void proj_update_all(Net<T>& net, Proj<T>* j, int simstep, float prn, float old_prn) {
  if (old_prn == prn) return;
  int R = j->dim_hcu * j->dim_conn;
#ifdef BCPNN_ORACLE_REF
  if constexpr (std::is_same<T, float>::value) {
    if (net.math == MATH_REF) {
      for (int i = 0; i < R; i++)
        for (int k = 0; k < j->dim_mcu; k++)
          ref::update_all_kernel_cpu(i, k, j->dim_conn, j->dim_mcu, j->pi.data(), j->ei.data(), j->zi.data(),
                                     j->ti.data(), j->pj.data(), j->pij.data(), j->eij.data(), j->zi2.data(),
                                     j->zj2.data(), j->tij.data(), j->wij.data(), simstep - 1,
                                     j->taupdt * old_prn, j->tauedt, j->tauzidt, j->tauzjdt, j->wgain, j->eps,
                                     j->eps2);
      net.cnt.all_cells += (uint64_t)R * j->dim_mcu;
      return;
    }
  }
#endif
  for (int i = 0; i < R; i++) {
    for (int k = 0; k < j->dim_mcu; k++) {
      all_kernel<T>(net.math, i, k, j->dim_conn, j->dim_mcu, j->pi.data(), j->ei.data(), j->zi.data(),
                    j->ti.data(), j->pj.data(), j->pij.data(), j->eij.data(), j->zi2.data(), j->zj2.data(),
                    j->tij.data(), j->wij.data(), simstep - 1, j->taupdt * (T)old_prn, j->tauedt, j->tauzidt,
                    j->tauzjdt, j->wgain, j->eps, j->eps2);
    }
  }
  net.cnt.all_cells += (uint64_t)R * j->dim_mcu;
}

/* Proj::update_jxx_cpu, Proj.cpp:590-619. */
template <typename T>
void proj_update_jxx(Net<T>& net, Proj<T>* j, float prn) {
  size_t off = (size_t)j->proj_in_pop * j->dim_hcu * j->dim_mcu;
  T* ptr_epsc = j->dest->epsc.data() + off;
  T* ptr_bj = j->dest->bj.data() + off;
  const int8_t* ptr_sj = j->dest->spike.data();
#ifdef BCPNN_ORACLE_REF
  if constexpr (std::is_same<T, float>::value) {
    if (net.math == MATH_REF) {
      for (int i = 0; i < j->dim_hcu * j->dim_mcu; i++)
        ref::update_jxx_kernel_cpu(i, ptr_sj, j->pj.data(), j->ej.data(), j->zj.data(), ptr_bj, ptr_epsc,
                                   j->taupdt * prn, j->tauedt, j->tauzjdt, j->tauzidt, j->tauepscdt, j->kftj,
                                   j->bgain, j->eps);
      return;
    }
  }
#endif
  for (int i = 0; i < j->dim_hcu * j->dim_mcu; i++) {
    jxx_kernel<T>(net.math, i, ptr_sj, j->pj.data(), j->ej.data(), j->zj.data(), ptr_bj, ptr_epsc,
                  j->taupdt * (T)prn, j->tauedt, j->tauzjdt, j->tauepscdt, j->kftj, j->bgain, j->eps);
  }
}

/* Proj::update_ssi_cpu / update_ssj_cpu, Proj.cpp:621-643. */
template <typename T> void proj_update_ssi(Proj<T>* j) {
  j->ssi.clear();
  for (int i = 0; i < j->dim_conn * j->dim_hcu; i++)
    if (j->siq[i] > 0) j->ssi.push_back(i);
}
template <typename T> void proj_update_ssj(Proj<T>* j) {
  j->ssj.clear();
  const int8_t* sj = j->dest->spike.data();
  for (int i = 0; i < j->dim_hcu * j->dim_mcu; i++)
    if (sj[i] > 0) j->ssj.push_back(i);
}

/* Proj::update_que_cpu, Proj.cpp:645-664. */
template <typename T> void proj_update_que(Proj<T>* j) {
  for (int i = 0; i < j->dim_conn * j->dim_hcu; i++) {
    if (j->ii[i] < 0) continue;
    j->siq[i] = j->qi[i] & 0x01;
    j->qi[i] >>= 1;
    int8_t spk = j->si[j->ii[i]];
    if (spk > 0) j->qi[i] |= (0x01 << (j->di[i] - 1));
  }
}

/* Proj::update_row_cpu, Proj.cpp:667-720. */
template <typename T>
void proj_update_row(Net<T>& net, Proj<T>* j, int simstep, float prn) {
  T* ptr_epsc = j->dest->epsc.data() + (size_t)j->proj_in_pop * j->dim_hcu * j->dim_mcu;
  int active_row_num = (int)j->ssi.size();
#ifdef BCPNN_ORACLE_REF
  if constexpr (std::is_same<T, float>::value) {
    if (net.math == MATH_REF) {
      for (int i = 0; i < active_row_num; i++)
        for (int k = 0; k < j->dim_mcu; k++)
          ref::update_row_kernel_cpu(i, k, j->dim_conn, j->dim_mcu, j->ssi.data(), j->pi.data(), j->ei.data(),
                                     j->zi.data(), j->ti.data(), j->pj.data(), j->pij.data(), j->eij.data(),
                                     j->zi2.data(), j->zj2.data(), j->tij.data(), j->wij.data(), ptr_epsc, simstep,
                                     j->taupdt * prn, j->tauedt, j->tauzidt, j->tauzjdt, j->kfti, j->wgain,
                                     j->eps, j->eps2);
      net.cnt.row_cells += (uint64_t)active_row_num * j->dim_mcu;
      return;
    }
  }
#endif
  for (int i = 0; i < active_row_num; i++) {
    for (int k = 0; k < j->dim_mcu; k++) {
      row_kernel<T>(net.math, i, k, j->dim_conn, j->dim_mcu, j->ssi.data(), j->pi.data(), j->ei.data(),
                    j->zi.data(), j->ti.data(), j->pj.data(), j->pij.data(), j->eij.data(), j->zi2.data(),
                    j->zj2.data(), j->tij.data(), j->wij.data(), ptr_epsc, simstep, j->taupdt * (T)prn,
                    j->tauedt, j->tauzidt, j->tauzjdt, j->kfti, j->wgain, j->eps, j->eps2);
    }
  }
  net.cnt.row_cells += (uint64_t)active_row_num * j->dim_mcu;
}

/* Proj::update_col_cpu, Proj.cpp:722-760. */
template <typename T>
void proj_update_col(Net<T>& net, Proj<T>* j, int simstep, float prn) {
  int active_col_num = (int)j->ssj.size();
#ifdef BCPNN_ORACLE_REF
  if constexpr (std::is_same<T, float>::value) {
    if (net.math == MATH_REF) {
      for (int k = 0; k < active_col_num; k++)
        for (int i = 0; i < j->dim_conn; i++)
          ref::update_col_kernel_cpu(i, k, j->dim_conn, j->dim_mcu, j->ii.data(), j->ssj.data(), j->pij.data(),
                                     j->eij.data(), j->zi2.data(), j->zj2.data(), j->tij.data(), simstep,
                                     j->taupdt * prn, j->tauedt, j->tauzidt, j->tauzjdt, j->kftj);
      net.cnt.col_cells += (uint64_t)active_col_num * j->dim_conn;
      return;
    }
  }
#endif
  for (int k = 0; k < active_col_num; k++) {
    for (int i = 0; i < j->dim_conn; i++) {
      col_kernel<T>(net.math, i, k, j->dim_conn, j->dim_mcu, j->ii.data(), j->ssj.data(), j->pij.data(),
                    j->eij.data(), j->zi2.data(), j->zj2.data(), j->tij.data(), simstep, j->taupdt * (T)prn,
                    j->tauedt, j->tauzidt, j->tauzjdt, j->kftj);
    }
  }
  net.cnt.col_cells += (uint64_t)active_col_num * j->dim_conn;
}

/* ProcUpdLazy::update_cpu, ProcUpdLazy.cpp:88-124 (the cycle-flag gate is the
   caller's). */
template <typename T>
void upd_lazy_update(Net<T>& net, int simstep, float prn, float old_prn) {
  for (auto p : net.pops) {
    pop_update_rnd(net, p, simstep);
    pop_update_sup(net, p, simstep);
    pop_fill_spike(p, simstep);
  }
  for (auto j : net.projs) {
    proj_update_all(net, j, simstep, prn, old_prn);
    proj_update_jxx(net, j, prn);
    proj_update_ssi(j);
    proj_update_ssj(j);
    proj_update_row(net, j, simstep, prn);
    proj_update_col(net, j, simstep, prn);
    proj_update_que(j);
  }
}

/* ProcExchangeSpike::update_cpu, ProcExchangeSpike.cpp:94-139, one rank:
   for every projection the DESTINATION population's spikes are copied into
   the shared buffer at that population's offset (:109-119); then every
   projection's si is read from the buffer at its SOURCE population's offset
   (:123-133).  A population that is the destination of no projection is never
   published and its region stays zero. */
template <typename T>
void exchange_spike(Net<T>& net) {
  std::vector<int> offset(net.pops.size());
  int total = 0;
  for (size_t k = 0; k < net.pops.size(); k++) {
    offset[k] = total;
    total += net.pops[k]->dim_hcu * net.pops[k]->dim_mcu;
  }
  if ((int)net.shared_buffer.size() != total) net.shared_buffer.assign(total, 0);
  for (auto j : net.projs) {
    Pop<T>* p = j->dest;
    std::memcpy(&net.shared_buffer[offset[p->id]], p->spike.data(), p->spike.size());
  }
  for (auto j : net.projs) {
    Pop<T>* p = j->src;
    std::memcpy(j->si.data(), &net.shared_buffer[offset[p->id]], j->si.size());
  }
}

}  // namespace oracle

/* ======================================================================== */
/* C API for the Python test harness                                          */
/* ======================================================================== */

using namespace oracle;

struct OracleHandle {
  int real_bits;
  Net<float>* f = nullptr;
  Net<double>* d = nullptr;
};

template <typename T>
static Net<T>* build(int math, float dt, uint32_t seed, float poisson_hz, int n_pops, const int* pop_dims,
                     const float* pop_params, int n_projs, const int* proj_ints, const float* proj_floats) {
  Net<T>* n = new Net<T>();
  n->math = math;
  n->dt = dt;
  n->seed = seed;
  n->poisson_hz = poisson_hz;
  int hcu_cnt = 0, mcu_cnt = 0;
  for (int k = 0; k < n_pops; k++) {
    PopDesc d;
    d.hcu_num = pop_dims[2 * k];
    d.mcu_num = pop_dims[2 * k + 1];
    const float* q = pop_params + 7 * k;
    d.taum = q[0]; d.wtagain = q[1]; d.maxfq = q[2]; d.igain = q[3]; d.wgain = q[4]; d.lgbias = q[5]; d.snoise = q[6];
    pop_init(*n, d, &hcu_cnt, &mcu_cnt);
  }
  for (int k = 0; k < n_projs; k++) {
    ProjDesc d;
    d.src_pop = proj_ints[2 * k];
    d.dest_pop = proj_ints[2 * k + 1];
    const float* q = proj_floats + 9 * k;
    d.tauzi = q[0]; d.tauzj = q[1]; d.taue = q[2]; d.taup = q[3]; d.maxfq = q[4]; d.bgain = q[5];
    d.wgain = q[6]; d.tauepsc = q[7]; d.slot_num = q[8];
    proj_init(*n, d);
  }
  n->lginp.assign(mcu_cnt, 0);
  n->wmask_row.assign(hcu_cnt, 0);
  return n;
}

static char g_empty[8];

template <typename T> static void* find_vec(Net<T>* n, const std::string& name, int* kind, size_t* count) {
  /* kind: 0 = value type T, 1 = int32, 2 = int8; an empty vector resolves to
     a non-null placeholder */
  auto split = name.rfind('_');
  if (split == std::string::npos) return nullptr;
  std::string base = name.substr(0, split);
  int id = std::atoi(name.c_str() + split + 1);
#define RET(vec, k) do { *kind = (k); *count = (vec).size(); return (vec).empty() ? (void*)g_empty : (void*)(vec).data(); } while (0)
  if (id >= 0 && id < (int)n->pops.size()) {
    Pop<T>* p = n->pops[id];
    if (base == "dsup") RET(p->dsup, 0);
    if (base == "act") RET(p->act, 0);
    if (base == "epsc") RET(p->epsc, 0);
    if (base == "bj") RET(p->bj, 0);
    if (base == "spike") RET(p->spike, 2);
    if (base == ".counter") RET(p->counter, 1);
    if (base == ".rnd_uniform01") RET(p->rnd_uniform01, 0);
    if (base == ".rnd_normal") RET(p->rnd_normal, 0);
  }
  if (id >= 0 && id < (int)n->projs.size()) {
    Proj<T>* j = n->projs[id];
    if (base == "ii") RET(j->ii, 1);
    if (base == "qi") RET(j->qi, 1);
    if (base == "di") RET(j->di, 1);
    if (base == "ti") RET(j->ti, 1);
    if (base == "tij") RET(j->tij, 1);
    if (base == ".ssi") RET(j->ssi, 1);
    if (base == ".ssj") RET(j->ssj, 1);
    if (base == ".siq") RET(j->siq, 2);
    if (base == "si") RET(j->si, 2);
    if (base == "pi") RET(j->pi, 0);
    if (base == "ei") RET(j->ei, 0);
    if (base == "zi") RET(j->zi, 0);
    if (base == "pj") RET(j->pj, 0);
    if (base == "ej") RET(j->ej, 0);
    if (base == "zj") RET(j->zj, 0);
    if (base == "pij") RET(j->pij, 0);
    if (base == "eij") RET(j->eij, 0);
    if (base == "zi2") RET(j->zi2, 0);
    if (base == "zj2") RET(j->zj2, 0);
    if (base == "wij") RET(j->wij, 0);
  }
#undef RET
  return nullptr;
}

extern "C" {

void* oracle_create(int real_bits, int math, float dt, uint32_t seed, float poisson_hz, int n_pops,
                    const int* pop_dims, const float* pop_params, int n_projs, const int* proj_ints,
                    const float* proj_floats) {
  /* gsbn's own kernels exist only in the oracle/_ref build, and only in float */
  if (math == MATH_REF && (!kHaveRef || real_bits != 32)) return nullptr;
  OracleHandle* h = new OracleHandle();
  h->real_bits = real_bits;
  if (real_bits == 64)
    h->d = build<double>(math, dt, seed, poisson_hz, n_pops, pop_dims, pop_params, n_projs, proj_ints, proj_floats);
  else
    h->f = build<float>(math, dt, seed, poisson_hz, n_pops, pop_dims, pop_params, n_projs, proj_ints, proj_floats);
  return h;
}

void oracle_destroy(void* hp) {
  OracleHandle* h = (OracleHandle*)hp;
  delete h->f;
  delete h->d;
  delete h;
}

/* lginp: total MCUs, wmask_row: total HCUs, as float (the reference stores
   both as f32, ProcExtGen.cpp:57-59). */
int oracle_set_stimulus(void* hp, const float* lginp, const float* wmask_row) {
  OracleHandle* h = (OracleHandle*)hp;
  if (h->f) {
    for (size_t i = 0; i < h->f->lginp.size(); i++) h->f->lginp[i] = lginp[i];
    for (size_t i = 0; i < h->f->wmask_row.size(); i++) h->f->wmask_row[i] = wmask_row[i];
  } else {
    for (size_t i = 0; i < h->d->lginp.size(); i++) h->d->lginp[i] = lginp[i];
    for (size_t i = 0; i < h->d->wmask_row.size(); i++) h->d->wmask_row[i] = wmask_row[i];
  }
  return 0;
}

/* External spike replay table of one population: n entries of (tick,
   indices[offsets[k]:offsets[k+1]]), Pop.cpp:67-110. */
int oracle_set_ext_spikes(void* hp, int pop, int n, const int* ticks, const int* offsets, const int* idx) {
  OracleHandle* h = (OracleHandle*)hp;
  auto fill = [&](auto* net) {
    auto* p = net->pops[pop];
    p->flag_ext_spike = true;
    p->ext_spikes.clear();
    for (int k = 0; k < n; k++) p->ext_spikes[ticks[k]] = std::vector<int>(idx + offsets[k], idx + offsets[k + 1]);
  };
  if (h->f) fill(h->f); else fill(h->d);
  return 0;
}

int oracle_update(void* hp, int simstep, float prn, float old_prn) {
  OracleHandle* h = (OracleHandle*)hp;
  if (h->f) upd_lazy_update(*h->f, simstep, prn, old_prn);
  else upd_lazy_update(*h->d, simstep, prn, old_prn);
  return 0;
}

int oracle_exchange(void* hp) {
  OracleHandle* h = (OracleHandle*)hp;
  if (h->f) exchange_spike(*h->f); else exchange_spike(*h->d);
  return 0;
}

/* Returns element count (-1 if unknown); *kind: 0 value type, 1 i32, 2 i8. */
long long oracle_state_info(void* hp, const char* name, int* kind) {
  OracleHandle* h = (OracleHandle*)hp;
  size_t count = 0;
  void* p = h->f ? find_vec(h->f, name, kind, &count) : find_vec(h->d, name, kind, &count);
  return p ? (long long)count : -1;
}

int oracle_read_state(void* hp, const char* name, void* out, size_t bytes) {
  OracleHandle* h = (OracleHandle*)hp;
  int kind = 0;
  size_t count = 0;
  void* p = h->f ? find_vec(h->f, name, &kind, &count) : find_vec(h->d, name, &kind, &count);
  if (!p) return -1;
  size_t esz = kind == 0 ? (h->f ? 4 : 8) : (kind == 1 ? 4 : 1);
  if (bytes != count * esz) return -2;
  if (bytes) std::memcpy(out, p, bytes);
  return 0;
}

int oracle_write_state(void* hp, const char* name, const void* in, size_t bytes) {
  OracleHandle* h = (OracleHandle*)hp;
  int kind = 0;
  size_t count = 0;
  void* p = h->f ? find_vec(h->f, name, &kind, &count) : find_vec(h->d, name, &kind, &count);
  if (!p) return -1;
  size_t esz = kind == 0 ? (h->f ? 4 : 8) : (kind == 1 ? 4 : 1);
  if (bytes != count * esz) return -2;
  if (bytes) std::memcpy(p, in, bytes);
  return 0;
}

/* Cells brought to the current tick: row, column and all-cells sweeps. */
void oracle_counters(void* hp, unsigned long long* out3) {
  OracleHandle* h = (OracleHandle*)hp;
  Counters c = h->f ? h->f->cnt : h->d->cnt;
  out3[0] = c.row_cells;
  out3[1] = c.col_cells;
  out3[2] = c.all_cells;
}

float oracle_expf(int math, float x) { return Fn<float>::exp(math, x); }

/* element-wise exp/log of an array (shared or libm definition) */
void oracle_expf_array(int math, long long n, const float* in, float* out) {
  for (long long i = 0; i < n; ++i) out[i] = Fn<float>::exp(math, in[i]);
}
void oracle_logf_array(int math, long long n, const float* in, float* out) {
  for (long long i = 0; i < n; ++i) out[i] = Fn<float>::log(math, in[i]);
}

/* Philox4x32-10 block and the stream map, for the known-answer tests */
void oracle_philox(const uint32_t* ctr, const uint32_t* key, uint32_t* out) {
  bx_u32x4 c;
  for (int i = 0; i < 4; ++i) c.v[i] = ctr[i];
  bx_u32x4 o = bx_philox4x32_10(c, key[0], key[1]);
  for (int i = 0; i < 4; ++i) out[i] = o.v[i];
}
void oracle_uniform_array(uint32_t seed, uint32_t pop, uint32_t tick, int n, float* out) {
  for (int i = 0; i < n; ++i) out[i] = bx_uniform01(seed, pop, tick, (uint32_t)i);
}
void oracle_uniform_poisson_array(uint32_t seed, uint32_t pop, uint32_t tick, int n, float* out) {
  for (int i = 0; i < n; ++i) out[i] = bx_uniform01_poisson(seed, pop, tick, (uint32_t)i);
}
void oracle_normal_array(uint32_t seed, uint32_t pop, uint32_t tick, int n, float* out) {
  for (int i = 0; i < n; ++i) out[i] = bx_normal01(seed, pop, tick, (uint32_t)i);
}
float oracle_logf(int math, float x) { return Fn<float>::log(math, x); }

/* 1 when this build carries gsbn's own kernels (math mode MATH_REF). */
int oracle_has_ref(void) { return kHaveRef ? 1 : 0; }
double oracle_log_double(int math, double x) { return log_double(math, x); }
/* cos(2 pi u) of the Box-Muller draws (the library's bx_cos2pi_d) */
double oracle_cos2pi_double(double u) { return bx_cos2pi_d(u); }

}  // extern "C"
