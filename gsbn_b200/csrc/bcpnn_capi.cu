/*
 * bcpnn_capi.cu -- implementation of include/bcpnn.h for one network on one
 * B200: device allocation with gsbn's initial values, per-run orchestration
 * (decay tables, all-cells catch-up, one fused kernel per tick, captured once
 * per run length into a CUDA graph and replayed), and state import/export in
 * gsbn's Database layouts.
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "bcpnn.h"
#include "bcpnn_device.cuh"
#define BCPNN_TICK_THREADS 512
#define BCPNN_TICK_NS t512
#include "bcpnn_tick.cuh"
#undef BCPNN_TICK_THREADS
#undef BCPNN_TICK_NS
#define BCPNN_TICK_THREADS 256
#define BCPNN_TICK_NS t256
#include "bcpnn_tick.cuh"
#undef BCPNN_TICK_THREADS
#undef BCPNN_TICK_NS
#include "bcpnn_multi.cuh"
#include "bcpnn_numerics.h"

namespace bcpnn {
namespace multi {
/* ProcUpdMulti's persistent launch: the tick loop of bcpnn_multi.cuh with the
   bounded grid barrier of the tick kernel */
__global__ void __launch_bounds__(kProjThreads, 1) tick_kernel(const NetDev* __restrict__ net,
                                                              const RunParams* __restrict__ rp, int it0, int n_ticks,
                                                              unsigned int* bar) {
  __shared__ int s_ok;
  tick_loop(net, rp, it0, n_ticks,
            [&](int k) { return t512::grid_sync(bar, (unsigned int)k * gridDim.x, net->err, &s_ok); });
}
/* the same with each HCU's state resident in shared memory (res_tick_loop) */
__global__ void __launch_bounds__(kProjThreads, 1) res_tick_kernel(const NetDev* __restrict__ net,
                                                                  const RunParams* __restrict__ rp, int it0,
                                                                  int n_ticks, unsigned int* bar) {
  res_tick_loop(net, rp, it0, n_ticks, bar);
}
}  // namespace multi
}  // namespace bcpnn

using namespace bcpnn;

namespace {

struct TableSlot {
  uint32_t kp_bits = 0;
  int len = 0;   /* valid entries */
  int cap = 0;   /* allocated entries */
  float4* ptr = nullptr;    /* cap * 4 float4, then cap * 4 double2 reciprocals (one allocation) */
  double2* rptr = nullptr;
  uint64_t stamp = 0;
};

struct PopHost {
  bcpnn_pop_desc d;
  int H, M, n, hcu_start, mcu_start, dim_proj = 0;
  std::vector<int> in_proj, out_proj;
  int log_words;
  size_t log_offset;  /* words, within the common log buffer */
  int* ext_off = nullptr;
  int* ext_idx = nullptr;
};

struct ProjHost {
  bcpnn_proj_desc d;
  int H, M, C, Ns, proj_in_pop;
  TableSlot slot[2];
};

}  // namespace

struct bcpnn_net {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::vector<void*> allocs;
  std::vector<PopHost> pops;
  std::vector<ProjHost> projs;
  NetDev h;                 /* host image of the device descriptor */
  std::vector<PopDev> hp;   /* host images of the per-population descriptors */
  std::vector<ProjDev> hq;  /* host images of the per-projection descriptors */
  std::vector<TabRef> tabs; /* host image of the run's decay-table references */
  PopDev* d_pops = nullptr;
  ProjDev* d_projs = nullptr;
  TabRef* d_tabs = nullptr;
  NetDev* d_net = nullptr;
  RunParams rp;             /* host image of the run parameters */
  RunParams* d_rp = nullptr;
  int total_hcu = 0, total_mcu = 0, max_m = 1;
  int max_ticks = 0;
  uint32_t* log_buf = nullptr;
  /* bcpnn_get_spike_log_async: the log is copied to one of two device
     staging buffers on the network's stream, and from there to the host on
     copy_stream, so the next run need not wait for the host copy */
  cudaStream_t copy_stream = nullptr;
  uint32_t* log_stage[2] = {nullptr, nullptr};
  cudaEvent_t stage_ready[2] = {nullptr, nullptr}, stage_free[2] = {nullptr, nullptr};
  int stage_next = 0;
  size_t log_words_per_tick = 0;
  int64_t k_total = 0;      /* ticks executed since creation */
  uint32_t tick_serial = 1; /* tags of the softmax seeds (NetDev::seed64); never reset */
  int last_run_ticks = 0;
  bool exchange = false;
  bool direct = false;      /* GSBN_DIRECT_LAUNCH=1: launch kernels one by one (profilers) */
  bool persistent = false;  /* one cooperative launch per run (else one launch per tick) */
  size_t tick_smem = 0;     /* dynamic shared memory of tick_kernel */
  int threads = 512;        /* CTA size of the tick kernel (512 or 256) */
  bool fp64 = false;        /* FP64-built decay tables */
  bool multi = false;       /* ProcUpdMulti variant (bcpnn_multi.cuh) */
  bool multi_persistent = false; /* its one-launch-per-run form */
  bool multi_resident = false;   /* ... with each HCU's state in shared memory */
  size_t multi_smem = 0;
  int ring_len = 1;         /* its spike buffer size */
  const void* tick_fn = nullptr;  /* the tick kernel variant of the persistent launch */
  const void* tick_fn0 = nullptr; /* the same size and decay form with in-CTA columns */
  unsigned int* bar = nullptr; /* persistent kernel: [0] grid barrier arrivals, [1..2] column units by
                                  tick parity, [4 + cta] column units done for each CTA */
  int4* col_ring = nullptr;    /* deferred column units (NetDev::col_ring) */
  std::map<std::pair<int, int>, cudaGraphExec_t> graphs;
  uint64_t launches = 0;
  uint64_t all_cells = 0;   /* cells swept by all-cells catch-ups */
  uint64_t stamp = 0;
  float* stim_lg = nullptr; /* device stimulus tables (bcpnn_upload_stimuli) */
  int32_t* d_lgidx = nullptr; /* one pattern-index row (bcpnn_set_stimulus_idx) */
  std::vector<int32_t*> check_cnt; /* per population: ProcCheck counters [H*M] (bcpnn_check_count) */
  std::vector<int32_t*> check_out; /* per population: [2][H] idx, count of the last check */
  /* per population: check_out written (network's stream) / read by the host
     copies (copy_stream) */
  std::vector<cudaEvent_t> check_ready, check_free;
  float* stim_wm = nullptr;
  int stim_lg_rows = 0, stim_wm_rows = 0;
  int stim_lg_cap = 0, stim_wm_cap = 0; /* rows the stimulus tables have room for */
  int32_t* d_lgidx_tab = nullptr;       /* pattern-index rows (bcpnn_upload_stimuli_idx_async) */
  int lgidx_tab_cap = 0;
  const float* cur_lg = nullptr; /* stimulus of the next run */
  const float* cur_wm = nullptr;
  float* scratch = nullptr; /* staging for strided cell fields */
  size_t scratch_n = 0;
  std::string err;
};

namespace {

constexpr int kMaxDevices = 64; /* device ordinals the per-device kernel attributes track */

int fail(bcpnn_net* net, int code, const std::string& msg) {
  if (net) net->err = msg;
  return code;
}

#define CU(call)                                                                              \
  do {                                                                                        \
    cudaError_t e_ = (call);                                                                  \
    if (e_ != cudaSuccess)                                                                    \
      return fail(net, BCPNN_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));   \
  } while (0)

template <typename T>
int dalloc(bcpnn_net* net, T** p, size_t count) {
  *p = nullptr;
  if (count == 0) count = 1;
  CU(cudaMalloc((void**)p, count * sizeof(T)));
  net->allocs.push_back((void*)*p);
  return BCPNN_OK;
}

int grid_for(size_t n, int block) {
  size_t g = (n + block - 1) / block;
  if (g > 148 * 32) g = 148 * 32;
  if (g < 1) g = 1;
  return (int)g;
}

int check_device_error(bcpnn_net* net) {
  int e = 0;
  CU(cudaMemcpyAsync(&e, net->h.err, sizeof(int), cudaMemcpyDeviceToHost, net->stream));
  CU(cudaStreamSynchronize(net->stream));
  if (e) {
    CU(cudaMemsetAsync(net->h.err, 0, sizeof(int), net->stream));
    std::string why;
    if (e & kErrIndex) why += " a slot's source MCU index is outside the source population;";
    if (e & kErrBarrier) why += " a grid barrier of the persistent tick kernel timed out;";
    if (e & kErrColumns) why += " a wait for the grid's column updates in the persistent tick kernel timed out;";
    if (e & kErrSeed) why += " a softmax seed published for the next tick carried the wrong tick tag;";
    return fail(net, BCPNN_ERR_DEVICE, "kernel reported error word " + std::to_string(e) + ":" + why);
  }
  return BCPNN_OK;
}

/* (re)build the decay table of slot s of projection p for kp = taupdt*prn
   with at least `need` entries */
/* the reciprocals of the constant divisors for kp = taupdt*prn; the divisors
   are the float expressions of make_coef (host float arithmetic without
   contraction gives the same bits), the reciprocals IEEE double divisions */
RCoef rcoef(const ProjDev& D, float prn) {
  const float kp = D.taupdt * prn;
  RCoef r;
  r.Dekp = 1.0 / (double)(D.ke - kp);
  r.D2 = 1.0 / (double)((D.kzi - kp) + D.kzj);
  r.D3 = 1.0 / (double)((D.kzi - D.ke) + D.kzj);
  r.Dpzi = 1.0 / (double)(kp - D.kzi);
  r.Dezi = 1.0 / (double)(D.ke - D.kzi);
  return r;
}

int fill_slot(bcpnn_net* net, int p, int s, float prn, int need) {
  ProjHost& J = net->projs[p];
  const ProjDev& D = net->hq[p];
  float kp = D.taupdt * prn;
  TableSlot& T = J.slot[s];
  if (T.ptr && T.kp_bits == bx_fbits(kp) && T.len >= need) return BCPNN_OK;
  if (T.cap < need) {
    int cap = 1024;
    while (cap < need) cap *= 2;
    if (T.ptr) CU(cudaFree(T.ptr));
    T.ptr = nullptr;
    T.rptr = nullptr;
    CU(cudaMalloc((void**)&T.ptr, (size_t)cap * 4 * (sizeof(float4) + sizeof(double2))));
    T.rptr = (double2*)(T.ptr + (size_t)cap * 4);
    T.cap = cap;
  }
  if (D.fp64)
    build_table_fp64_kernel<<<grid_for(T.cap, 256), 256, 0, net->stream>>>(T.ptr, T.cap, kp, D.ke, D.kzi, D.kzj);
  else
    build_table_kernel<<<grid_for(T.cap, 256), 256, 0, net->stream>>>(T.ptr, T.rptr, T.cap, kp, D.ke, D.kzi, D.kzj);
  CU(cudaGetLastError());
  net->launches++;
  T.kp_bits = bx_fbits(kp);
  T.len = T.cap;
  return BCPNN_OK;
}

/* Tables of projection p for this run: slot *s_cur for prn, and, when the
   all-cells catch-up runs, slot *s_old for old_prn.  Two slots per projection
   cover the usual alternation of training and recall segments. */
int prepare_tables(bcpnn_net* net, int p, float prn, float old_prn, bool with_all, int need_cur, int need_old,
                   int* s_cur, int* s_old) {
  ProjHost& J = net->projs[p];
  const ProjDev& D = net->hq[p];
  uint32_t b_cur = bx_fbits(D.taupdt * prn), b_old = bx_fbits(D.taupdt * old_prn);
  auto lookup = [&](uint32_t b) {
    for (int s = 0; s < 2; ++s)
      if (J.slot[s].ptr && J.slot[s].kp_bits == b) return s;
    return -1;
  };
  int sc = lookup(b_cur);
  int so = with_all ? lookup(b_old) : -1;
  if (with_all && b_old == b_cur) so = sc;
  if (sc < 0) {
    if (so >= 0) sc = so ^ 1;
    else sc = (J.slot[0].stamp <= J.slot[1].stamp) ? 0 : 1;
  }
  if (with_all && so < 0) so = (b_old == b_cur) ? sc : (sc ^ 1);
  int rc = fill_slot(net, p, sc, prn, need_cur);
  if (rc) return rc;
  if (with_all && so != sc && (rc = fill_slot(net, p, so, old_prn, need_old))) return rc;
  if (with_all && so == sc && b_old != b_cur) return fail(net, BCPNN_ERR_STATE, "decay table slot conflict");
  J.slot[sc].stamp = ++net->stamp;
  if (with_all) J.slot[so].stamp = ++net->stamp;
  *s_cur = sc;
  *s_old = so;
  return BCPNN_OK;
}

template <typename T>
int dset(bcpnn_net* net, T* p, size_t n, T v) {
  if (n == 0) return BCPNN_OK;
  fill_kernel<T><<<grid_for(n, 256), 256, 0, net->stream>>>(p, n, v);
  CU(cudaGetLastError());
  net->launches++;
  return BCPNN_OK;
}

int dzero(bcpnn_net* net, void* p, size_t bytes) {
  if (bytes) CU(cudaMemsetAsync(p, 0, bytes, net->stream));
  return BCPNN_OK;
}

/* gsbn's initial values (Pop.cpp:59-65, Proj.cpp:88-105) for every state
   vector; connectivity (ii, di), stimulus and replay tables are kept. */
int reset_state(bcpnn_net* net) {
  int rc;
  for (size_t p = 0; p < net->pops.size(); ++p) {
    const PopHost& P = net->pops[p];
    PopDev& D = net->hp[p];
    size_t n = P.n, ne = n * std::max(1, P.dim_proj);
    for (int b = 0; b < 2; ++b) {
      if ((rc = dset(net, D.dsup[b], n, (float)bx_log_d(1.0 / P.M)))) return rc;   /* log(1.0/M), Pop.cpp:59 */
      if ((rc = dzero(net, D.epsc[b], ne * sizeof(float)))) return rc;
      if ((rc = dzero(net, D.bj[b], ne * sizeof(float)))) return rc;
    }
    if ((rc = dset(net, D.act, n, (float)(1.0 / P.M)))) return rc;                 /* Pop.cpp:60 */
    if ((rc = dzero(net, D.spike, n))) return rc;
    if ((rc = dzero(net, D.counter, n * sizeof(int)))) return rc;
    if (D.ada && (rc = dzero(net, D.ada, n * sizeof(float)))) return rc;
    if (D.ring && (rc = dzero(net, D.ring, n * (size_t)D.ring_len))) return rc;
  }
  for (size_t q = 0; q < net->projs.size(); ++q) {
    const ProjHost& J = net->projs[q];
    ProjDev& D = net->hq[q];
    size_t R = (size_t)J.H * J.C, HM = (size_t)J.H * J.M, cells = R * J.M;
    if ((rc = dzero(net, D.qi, R * sizeof(int)))) return rc;
    if ((rc = dset(net, D.pi, R, (float)(1.0 / J.C)))) return rc;                  /* Proj.cpp:91 */
    if ((rc = dzero(net, D.ei, R * sizeof(float)))) return rc;
    if ((rc = dzero(net, D.zi, R * sizeof(float)))) return rc;
    if ((rc = dzero(net, D.ti, R * sizeof(int)))) return rc;
    if ((rc = dset(net, D.pj, HM, (float)(1.0 / J.M)))) return rc;                 /* Proj.cpp:96 */
    if ((rc = dzero(net, D.ej, HM * sizeof(float)))) return rc;
    if ((rc = dzero(net, D.zj, HM * sizeof(float)))) return rc;
    float pij0 = (float)(1.0 / J.C / J.M);                                         /* Proj.cpp:99 */
    if ((rc = dset(net, D.cell, cells, make_float4(pij0, 0.0f, 0.0f, 0.0f)))) return rc;
    if ((rc = dzero(net, D.tij, cells * sizeof(int)))) return rc;
    if ((rc = dzero(net, D.wij, cells * sizeof(float)))) return rc;
    if ((rc = dzero(net, D.si[0], 4 * (size_t)J.Ns))) return rc;
    if ((rc = dzero(net, D.list_cnt, (size_t)J.H * sizeof(int)))) return rc;
  }
  for (size_t q = 0; q < net->check_cnt.size(); ++q)
    if (net->check_cnt[q] && (rc = dzero(net, net->check_cnt[q], (size_t)net->pops[q].H * net->pops[q].M * sizeof(int32_t))))
      return rc;
  net->k_total = 0;
  return BCPNN_OK;
}

/* the work of one run, queued on the network's stream */
void enqueue_run(bcpnn_net* net, int n_ticks, bool with_all) {
  for (const PopHost& P : net->pops)
    cudaMemsetAsync(net->log_buf + P.log_offset, 0, (size_t)n_ticks * P.log_words * sizeof(uint32_t), net->stream);
  cudaMemsetAsync(net->h.ss_log, 0, (size_t)n_ticks * net->h.n_projs * sizeof(uint32_t), net->stream);
  if (with_all && !net->multi) {
    for (int p = 0; p < net->h.n_projs; ++p) {
      const ProjHost& J = net->projs[p];
      all_rows_kernel<<<grid_for((size_t)J.H * J.C, 256), 256, 0, net->stream>>>(net->d_net, net->d_rp, p);
      all_cells_kernel<<<grid_for((size_t)J.H * J.C * J.M, 256), 256, 0, net->stream>>>(net->d_net, net->d_rp, p);
    }
  }
  size_t smem = net->tick_smem;
  if (net->multi) {
    /* ProcUpdMulti: catch-up at a change of prn, then per tick the
       populations and one launch per projection */
    if (with_all)
      for (int p = 0; p < net->h.n_projs; ++p) {
        const ProjHost& J = net->projs[p];
        multi::all_kernel<<<grid_for((size_t)J.H * J.C * 32, 256), 256, 0, net->stream>>>(net->d_net, net->d_rp, p);
      }
    if (net->multi_persistent) {
      cudaMemsetAsync(net->bar, 0, 4 * sizeof(unsigned int), net->stream);
      int it0 = 0, n = n_ticks;
      void* args[] = {(void*)&net->d_net, (void*)&net->d_rp, (void*)&it0, (void*)&n, (void*)&net->bar};
      cudaLaunchCooperativeKernel(net->multi_resident ? (const void*)multi::res_tick_kernel
                                                      : (const void*)multi::tick_kernel,
                                  dim3(net->total_hcu), dim3(multi::kProjThreads), args, net->multi_smem, net->stream);
      return;
    }
    const size_t pop_smem = (size_t)(2 * net->max_m + net->max_m) * sizeof(float);
    for (int it = 0; it < n_ticks; ++it) {
      multi::pop_kernel<<<net->total_hcu, multi::kPopThreads, pop_smem, net->stream>>>(net->d_net, net->d_rp, it);
      for (int p = 0; p < net->h.n_projs; ++p) {
        const ProjHost& J = net->projs[p];
        multi::proj_kernel<<<J.H, multi::kProjThreads, multi::proj_smem_bytes(J.M, J.C), net->stream>>>(
            net->d_net, net->d_rp, it, p);
      }
    }
    return;
  }
  if (net->persistent) {
    cudaMemsetAsync(net->bar, 0, (4 + (size_t)net->total_hcu) * sizeof(unsigned int), net->stream);
    int it0 = 0, n = n_ticks;
    void* args[] = {(void*)&net->d_net, (void*)&net->d_rp, (void*)&it0, (void*)&n, (void*)&net->bar};
    cudaLaunchCooperativeKernel(net->tick_fn, dim3(net->total_hcu), dim3(net->threads), args, smem, net->stream);
  } else {
    for (int it = 0; it < n_ticks; ++it) {
      if (net->threads == 256 && net->fp64)
        t256::tick_kernel<1, 0><<<net->total_hcu, 256, smem, net->stream>>>(net->d_net, net->d_rp, it, 1, net->bar);
      else if (net->threads == 256)
        t256::tick_kernel<0, 0><<<net->total_hcu, 256, smem, net->stream>>>(net->d_net, net->d_rp, it, 1, net->bar);
      else if (net->fp64)
        t512::tick_kernel<1, 0><<<net->total_hcu, 512, smem, net->stream>>>(net->d_net, net->d_rp, it, 1, net->bar);
      else
        t512::tick_kernel<0, 0><<<net->total_hcu, 512, smem, net->stream>>>(net->d_net, net->d_rp, it, 1, net->bar);
    }
  }
}

int capture_graph(bcpnn_net* net, int n_ticks, bool with_all, cudaGraphExec_t* out) {
  cudaGraph_t g = nullptr;
  CU(cudaStreamBeginCapture(net->stream, cudaStreamCaptureModeThreadLocal));
  enqueue_run(net, n_ticks, with_all);
  cudaError_t le = cudaGetLastError();
  cudaError_t ce = cudaStreamEndCapture(net->stream, &g);
  if (le != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return fail(net, BCPNN_ERR_CUDA, std::string("kernel launch during capture: ") + cudaGetErrorString(le));
  }
  CU(ce);
  cudaError_t ie = cudaGraphInstantiate(out, g, 0);
  cudaGraphDestroy(g);
  CU(ie);
  return BCPNN_OK;
}

/* name -> (kind, pointer, count, element type) resolution */
enum Kind { K_PLAIN, K_PARITY, K_CELL, K_SIQ, K_SI };
struct Resolved {
  Kind kind;
  int type;       /* BCPNN_F32 / I32 / I8 */
  size_t count;
  void* ptr;      /* K_PLAIN */
  void* par[2];   /* K_PARITY, K_SI */
  int field;      /* K_CELL */
  float4* cell;
  int proj;
};

/* the source-spike buffer of the last tick: by tick parity, or, for
   ProcUpdMulti's resident launch, one of four by tick mod 4 (par[0] is the
   block of four) */
static void* si_last(const bcpnn_net* net, const Resolved& r) {
  if (net->multi && net->multi_persistent && net->multi_resident) {
    const long long k = (net->k_total - 1) & 3;
    return (int8_t*)r.par[0] + (size_t)k * r.count;
  }
  return r.par[(int)((net->k_total - 1) & 1)];
}

bool resolve(const bcpnn_net* net, const char* cname, Resolved* r) {
  if (!cname) return false;
  std::string name(cname);
  size_t us = name.rfind('_');
  if (us == std::string::npos || us + 1 >= name.size()) return false;
  std::string base = name.substr(0, us);
  const char* num = name.c_str() + us + 1;
  for (const char* c = num; *c; ++c)
    if (*c < '0' || *c > '9') return false;
  int id = std::atoi(num);
  r->proj = id;
  if (id < (int)net->pops.size()) {
    const PopHost& P = net->pops[id];
    const PopDev& D = net->hp[id];
    size_t n = (size_t)P.n;
    auto plain = [&](void* p, int type, size_t count) { r->kind = K_PLAIN; r->ptr = p; r->type = type; r->count = count; return true; };
    auto parity = [&](float* a, float* b, size_t count) { r->kind = K_PARITY; r->par[0] = a; r->par[1] = b; r->type = BCPNN_F32; r->count = count; return true; };
    if (base == "dsup") return parity(D.dsup[0], D.dsup[1], n);
    if (base == "epsc") return parity(D.epsc[0], D.epsc[1], n * P.dim_proj);
    if (base == "bj") return parity(D.bj[0], D.bj[1], n * P.dim_proj);
    if (base == "act") return plain(D.act, BCPNN_F32, n);
    /* ProcUpdMulti's spike_<pop> is its ring of spike buffer size ticks, slot
       simstep % size (ProcUpdMulti/Pop.cpp:69,329) */
    if (base == "spike") return D.ring ? plain(D.ring, BCPNN_I8, n * (size_t)D.ring_len) : plain(D.spike, BCPNN_I8, n);
    if (base == ".counter") return plain(D.counter, BCPNN_I32, n);
    if (base == "ada" && D.ada) return plain(D.ada, BCPNN_F32, n);
  }
  if (id < (int)net->projs.size()) {
    const ProjHost& J = net->projs[id];
    const ProjDev& D = net->hq[id];
    size_t R = (size_t)J.H * J.C, HM = (size_t)J.H * J.M, cells = R * J.M;
    auto plain = [&](void* p, int type, size_t count) { r->kind = K_PLAIN; r->ptr = p; r->type = type; r->count = count; return true; };
    auto cell = [&](int f) { r->kind = K_CELL; r->field = f; r->cell = D.cell; r->type = BCPNN_F32; r->count = cells; return true; };
    if (base == "ii") return plain(D.ii, BCPNN_I32, R);
    if (base == "di") return plain(D.di, BCPNN_I32, R);
    if (base == "qi") return plain(D.qi, BCPNN_I32, R);
    if (base == "pi") return plain(D.pi, BCPNN_F32, R);
    if (base == "ei") return plain(D.ei, BCPNN_F32, R);
    if (base == "zi") return plain(D.zi, BCPNN_F32, R);
    if (base == "ti") return plain(D.ti, BCPNN_I32, R);
    if (base == "pj") return plain(D.pj, BCPNN_F32, HM);
    if (base == "ej") return plain(D.ej, BCPNN_F32, HM);
    if (base == "zj") return plain(D.zj, BCPNN_F32, HM);
    if (base == "tij") return plain(D.tij, BCPNN_I32, cells);
    if (base == "wij") return plain(D.wij, BCPNN_F32, cells);
    if (base == "pij") return cell(0);
    if (base == "eij") return cell(1);
    if (base == "zi2") return cell(2);
    if (base == "zj2") return cell(3);
    if (base == "si") { r->kind = K_SI; r->par[0] = D.si[0]; r->par[1] = D.si[1]; r->type = BCPNN_I8; r->count = (size_t)J.Ns; return true; }
    if (base == ".siq") { r->kind = K_SIQ; r->type = BCPNN_I8; r->count = R; return true; }
  }
  return false;
}

size_t type_size(int t) { return t == BCPNN_I8 ? 1 : 4; }

int ensure_scratch(bcpnn_net* net, size_t n) {
  if (net->scratch_n >= n) return BCPNN_OK;
  if (net->scratch) CU(cudaFree(net->scratch));
  net->scratch = nullptr;
  CU(cudaMalloc((void**)&net->scratch, n * sizeof(float)));
  net->scratch_n = n;
  return BCPNN_OK;
}

}  // namespace

/* ======================================================================== */

extern "C" {

const char* bcpnn_status_string(int s) {
  switch (s) {
    case BCPNN_OK: return "ok";
    case BCPNN_ERR_INVALID: return "invalid argument";
    case BCPNN_ERR_CUDA: return "CUDA runtime error";
    case BCPNN_ERR_NOT_FOUND: return "unknown state vector";
    case BCPNN_ERR_SIZE: return "size mismatch";
    case BCPNN_ERR_STATE: return "invalid state";
    case BCPNN_ERR_DEVICE: return "device error word set";
  }
  return "unknown status";
}

const char* bcpnn_last_error(const bcpnn_net* net) { return net ? net->err.c_str() : "null handle"; }

int bcpnn_net_create(const bcpnn_net_desc* desc, bcpnn_net** out) {
  if (!out) return BCPNN_ERR_INVALID;
  *out = nullptr;
  if (!desc || desc->n_pops <= 0 || desc->n_pops > kMaxPops || desc->n_projs < 0 || desc->n_projs > kMaxProj ||
      (desc->n_pops && !desc->pops) || (desc->n_projs && !desc->projs) || !(desc->dt > 0.0f) ||
      desc->max_ticks_per_run <= 0 || (desc->tick_threads != 0 && desc->tick_threads != 256 && desc->tick_threads != 512) ||
      desc->update_variant < 0 || desc->update_variant > 1 || desc->spike_buffer_size < 0 ||
      desc->spike_buffer_size > 1024 || (desc->update_variant == 1 && desc->fp64_tables))
    return BCPNN_ERR_INVALID;
  /* a rate dt/tau must be a finite positive number: a zero, negative,
     infinite or NaN time constant (or frequency) makes the closed forms and
     the FP64 propagator meaningless, so it is refused here, before any device
     work */
  auto pos = [](float x) { return x > 0.0f && x <= 3.4028234663852886e38f; };
  if (!pos(desc->dt)) return BCPNN_ERR_INVALID;
  for (int p = 0; p < desc->n_pops; ++p)
    if (!pos(desc->pops[p].taum)) return BCPNN_ERR_INVALID;
  for (int p = 0; p < desc->n_projs; ++p) {
    const bcpnn_proj_desc& d = desc->projs[p];
    if (!pos(d.tauzi) || !pos(d.tauzj) || !pos(d.taue) || !pos(d.taup) || !pos(d.maxfq) ||
        !(d.tauepsc <= 3.4028234663852886e38f))
      return BCPNN_ERR_INVALID;
  }
  for (int p = 0; p < desc->n_pops; ++p)
    if (desc->pops[p].hcu_num <= 0 || desc->pops[p].mcu_num <= 0 ||
        desc->pops[p].mcu_num > (desc->tick_threads == 256 ? 256 : 512) ||
        (desc->update_variant == 1 && !(desc->pops[p].taua > 0.0f)))
      return BCPNN_ERR_INVALID;
  {
    std::vector<int> n_in(desc->n_pops, 0);
    for (int p = 0; p < desc->n_projs; ++p)
      if (desc->projs[p].dest_pop >= 0 && desc->projs[p].dest_pop < desc->n_pops) n_in[desc->projs[p].dest_pop]++;
    for (int c : n_in)
      if (c > kMaxIn) return BCPNN_ERR_INVALID;
  }
  for (int p = 0; p < desc->n_projs; ++p) {
    const bcpnn_proj_desc& d = desc->projs[p];
    /* slot_num is a float in gsbn's schema; (int) of it must be defined and >= 1 */
    if (d.src_pop < 0 || d.src_pop >= desc->n_pops || d.dest_pop < 0 || d.dest_pop >= desc->n_pops ||
        !(d.slot_num >= 1.0f && d.slot_num < 2147483648.0f))
      return BCPNN_ERR_INVALID;
  }
  bcpnn_net* net = new bcpnn_net();
  net->device = desc->device;
  net->max_ticks = desc->max_ticks_per_run;
  net->exchange = desc->exchange_spikes != 0;
  net->threads = desc->tick_threads == 256 ? 256 : 512;
  net->fp64 = desc->fp64_tables != 0;
  net->multi = desc->update_variant == 1;
  net->ring_len = desc->spike_buffer_size > 0 ? desc->spike_buffer_size : 1;
  if (net->threads == 256) {
    net->tick_fn = net->fp64 ? (const void*)t256::tick_kernel<1, 1> : (const void*)t256::tick_kernel<0, 1>;
    net->tick_fn0 = net->fp64 ? (const void*)t256::tick_kernel<1, 0> : (const void*)t256::tick_kernel<0, 0>;
  } else {
    net->tick_fn = net->fp64 ? (const void*)t512::tick_kernel<1, 1> : (const void*)t512::tick_kernel<0, 1>;
    net->tick_fn0 = net->fp64 ? (const void*)t512::tick_kernel<1, 0> : (const void*)t512::tick_kernel<0, 0>;
  }
  {
    const char* e = std::getenv("GSBN_DIRECT_LAUNCH");
    net->direct = e && e[0] == '1';
  }
  std::memset(&net->h, 0, sizeof(NetDev));
  std::memset(&net->rp, 0, sizeof(RunParams));
  int rc = BCPNN_OK;
  auto bail = [&](int code) { *out = net; return code; };
  if (cudaSetDevice(net->device) != cudaSuccess) { net->err = "cudaSetDevice failed"; return bail(BCPNN_ERR_CUDA); }
  if (cudaStreamCreateWithFlags(&net->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&net->copy_stream, cudaStreamNonBlocking) != cudaSuccess) {
    net->err = "cudaStreamCreate failed";
    return bail(BCPNN_ERR_CUDA);
  }
  for (int k = 0; k < 2; ++k)
    if (cudaEventCreateWithFlags(&net->stage_ready[k], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&net->stage_free[k], cudaEventDisableTiming) != cudaSuccess) {
      net->err = "cudaEventCreate failed";
      return bail(BCPNN_ERR_CUDA);
    }

  /* populations: running HCU/MCU offsets (ProcUpdLazy.cpp:19-29) */
  NetDev& H = net->h;
  H.n_pops = desc->n_pops;
  H.n_projs = desc->n_projs;
  H.dt = desc->dt;
  H.poisson_hz = desc->poisson_noise_hz;
  H.seed = desc->seed;
  net->hp.assign(desc->n_pops, PopDev());
  net->hq.assign(desc->n_projs, ProjDev());
  net->tabs.assign(std::max(1, desc->n_projs), TabRef());
  for (int p = 0; p < desc->n_pops; ++p) {
    PopHost P;
    P.d = desc->pops[p];
    P.H = P.d.hcu_num;
    P.M = P.d.mcu_num;
    P.n = P.H * P.M;
    P.hcu_start = net->total_hcu;
    P.mcu_start = net->total_mcu;
    net->total_hcu += P.H;
    net->total_mcu += P.n;
    net->max_m = std::max(net->max_m, P.M);
    net->pops.push_back(P);
  }
  /* projections: dim_conn, proj_in_pop, coefficients (Proj.cpp:16-52) */
  for (int q = 0; q < desc->n_projs; ++q) {
    ProjHost J;
    J.d = desc->projs[q];
    PopHost& src = net->pops[J.d.src_pop];
    PopHost& dst = net->pops[J.d.dest_pop];
    J.H = dst.H;
    J.M = dst.M;
    J.Ns = src.n;
    J.C = src.n;
    int slot = (int)J.d.slot_num;
    if (J.C > slot) J.C = slot;
    J.proj_in_pop = dst.dim_proj++;
    dst.in_proj.push_back(q);
    net->projs.push_back(J);
  }
  /* ProcExchangeSpike publishes the spikes of populations that are the
     destination of a projection (ProcExchangeSpike.cpp:109-119) */
  if (net->exchange) {
    for (int q = 0; q < desc->n_projs; ++q) {
      int s = net->projs[q].d.src_pop;
      if (net->pops[s].in_proj.size() > 0) net->pops[s].out_proj.push_back(q);
    }
  }
  /* spike log: per population a [max_ticks][words] region */
  net->log_words_per_tick = 0;
  for (auto& P : net->pops) {
    P.log_words = (P.n + 31) / 32;
    P.log_offset = net->log_words_per_tick * (size_t)desc->max_ticks_per_run;
    net->log_words_per_tick += P.log_words;
  }

  float dt = desc->dt;
  if ((rc = dalloc(net, &net->log_buf, (size_t)net->max_ticks * net->log_words_per_tick))) return bail(rc);
  for (int k = 0; k < 2; ++k)
    if ((rc = dalloc(net, &net->log_stage[k], (size_t)net->max_ticks * net->log_words_per_tick))) return bail(rc);
  uint32_t* ss = nullptr;
  if ((rc = dalloc(net, &ss, (size_t)net->max_ticks * std::max(1, desc->n_projs)))) return bail(rc);
  H.ss_log = ss;
  unsigned long long* cnt = nullptr;
  if ((rc = dalloc(net, &cnt, 3))) return bail(rc);
  H.counters = cnt;
  int* errw = nullptr;
  if ((rc = dalloc(net, &errw, 1))) return bail(rc);
  H.err = errw;
  unsigned long long* seeds = nullptr;
  if ((rc = dalloc(net, &seeds, 2 * (size_t)desc->n_pops))) return bail(rc);
  if (cudaMemsetAsync(seeds, 0, 2 * (size_t)desc->n_pops * sizeof(unsigned long long), net->stream) != cudaSuccess) {
    net->err = "memset failed";
    return bail(BCPNN_ERR_CUDA);
  }
  H.seed64 = seeds;
  if (cudaMemsetAsync(cnt, 0, 3 * sizeof(unsigned long long), net->stream) != cudaSuccess ||
      cudaMemsetAsync(errw, 0, sizeof(int), net->stream) != cudaSuccess) {
    net->err = "memset failed";
    return bail(BCPNN_ERR_CUDA);
  }
  float* lg = nullptr;
  float* wm = nullptr;
  if ((rc = dalloc(net, &lg, net->total_mcu))) return bail(rc);
  if ((rc = dalloc(net, &wm, net->total_hcu))) return bail(rc);
  H.lginp = lg;
  H.wmask = wm;

  std::vector<int> idx_lists;
  for (int p = 0; p < desc->n_pops; ++p) {
    PopHost& P = net->pops[p];
    PopDev& D = net->hp[p];
    D.H = P.H; D.M = P.M; D.n = P.n; D.hcu_start = P.hcu_start; D.mcu_start = P.mcu_start;
    D.dim_proj = P.dim_proj; D.id = p;
    D.rng_seed = desc->seed; /* Philox key (seed, p*16 + stream); bcpnn_set_pop_rng overrides it */
    D.rng_pop = (uint32_t)p;
    D.taumdt = dt / P.d.taum;                  /* Pop.cpp:34 */
    D.wtagain = P.d.wtagain;
    D.maxfqdt = P.d.maxfq * dt;                /* Pop.cpp:36 */
    D.igain = P.d.igain;
    D.wgain = P.d.wgain;
    D.lgbias = P.d.lgbias;
    D.snoise = P.d.snoise;
    size_t n = P.n, ne = n * std::max(1, P.dim_proj);
    for (int b = 0; b < 2; ++b) {
      if ((rc = dalloc(net, &D.dsup[b], n))) return bail(rc);
      if ((rc = dalloc(net, &D.epsc[b], ne))) return bail(rc);
      if ((rc = dalloc(net, &D.bj[b], ne))) return bail(rc);
      /* dsup = log(1.0/M) in double, stored as float (Pop.cpp:59) */
    }
    if ((rc = dalloc(net, &D.act, n))) return bail(rc);
    if ((rc = dalloc(net, &D.spike, n))) return bail(rc);
    if ((rc = dalloc(net, &D.counter, n))) return bail(rc);
    if (net->multi) {
      if ((rc = dalloc(net, &D.ada, n))) return bail(rc);
      if ((rc = dalloc(net, &D.ring, n * (size_t)net->ring_len))) return bail(rc);
      D.ring_len = net->ring_len;
      D.tauadt = dt / P.d.taua;                /* ProcUpdMulti/Pop.cpp:46 */
      D.adgain = P.d.adgain;
    }
    D.spk_log = net->log_buf + P.log_offset;
    D.log_words = P.log_words;
    D.n_in = (int)P.in_proj.size();
    D.n_out = (int)P.out_proj.size();
    D.ext = 0;
  }
  /* in/out projection index lists */
  {
    std::vector<int> all;
    std::vector<std::pair<size_t, size_t>> off(desc->n_pops);
    for (int p = 0; p < desc->n_pops; ++p) {
      size_t a = all.size();
      for (int q : net->pops[p].in_proj) all.push_back(q);
      size_t b = all.size();
      for (int q : net->pops[p].out_proj) all.push_back(q);
      off[p] = {a, b};
    }
    int* dl = nullptr;
    if ((rc = dalloc(net, &dl, std::max<size_t>(1, all.size())))) return bail(rc);
    if (!all.empty() && cudaMemcpy(dl, all.data(), all.size() * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess) {
      net->err = "copy of projection lists failed";
      return bail(BCPNN_ERR_CUDA);
    }
    for (int p = 0; p < desc->n_pops; ++p) {
      net->hp[p].in_proj = dl + off[p].first;
      net->hp[p].out_proj = dl + off[p].second;
    }
  }
  for (int q = 0; q < desc->n_projs; ++q) {
    ProjHost& J = net->projs[q];
    ProjDev& D = net->hq[q];
    const bcpnn_proj_desc& d = J.d;
    D.src = d.src_pop; D.dest = d.dest_pop; D.H = J.H; D.M = J.M; D.C = J.C; D.Ns = J.Ns;
    D.proj_in_pop = J.proj_in_pop;
    D.kzi = dt / d.tauzi;                       /* Proj.cpp:38-52 */
    D.kzj = dt / d.tauzj;
    D.ke = dt / d.taue;
    D.taupdt = dt / d.taup;
    D.eps = dt / d.taup;
    D.eps2 = (dt / d.taup) * (dt / d.taup);
    D.kfti = 1 / (d.maxfq * d.tauzi);
    D.kftj = 1 / (d.maxfq * d.tauzj);
    D.bgain = d.bgain;
    D.wgain = d.wgain;
    D.kepsc = d.tauepsc > 0.0f ? dt / d.tauepsc : D.kzi;
    D.fp64 = desc->fp64_tables ? 1 : 0;
    size_t R = (size_t)J.H * J.C, HM = (size_t)J.H * J.M, cells = R * J.M;
    if ((rc = dalloc(net, &D.ii, R))) return bail(rc);
    if ((rc = dalloc(net, &D.di, R))) return bail(rc);
    if ((rc = dalloc(net, &D.qi, R))) return bail(rc);
    if ((rc = dalloc(net, &D.pi, R))) return bail(rc);
    if ((rc = dalloc(net, &D.ei, R))) return bail(rc);
    if ((rc = dalloc(net, &D.zi, R))) return bail(rc);
    if ((rc = dalloc(net, &D.ti, R))) return bail(rc);
    if ((rc = dalloc(net, &D.pj, HM))) return bail(rc);
    if ((rc = dalloc(net, &D.ej, HM))) return bail(rc);
    if ((rc = dalloc(net, &D.zj, HM))) return bail(rc);
    if ((rc = dalloc(net, &D.cell, cells))) return bail(rc);
    if ((rc = dalloc(net, &D.tij, cells))) return bail(rc);
    if ((rc = dalloc(net, &D.wij, cells))) return bail(rc);
    /* source spikes: one block of four buffers of Ns; the tick parity
       forms use the first two, ProcUpdMulti's resident launch all four */
    if ((rc = dalloc(net, &D.si[0], 4 * (size_t)J.Ns))) return bail(rc);
    D.si[1] = D.si[0] + J.Ns;
    if ((rc = dalloc(net, &D.list, R))) return bail(rc);
    if ((rc = dalloc(net, &D.list_cnt, J.H))) return bail(rc);
  }
  for (int q = 0; q < desc->n_projs; ++q) {
    const ProjHost& J = net->projs[q];
    size_t R = (size_t)J.H * J.C;
    if ((rc = dset(net, net->hq[q].ii, R, -1))) return bail(rc);                   /* Proj.cpp:88 */
    if ((rc = dzero(net, net->hq[q].di, R * sizeof(int)))) return bail(rc);
  }
  if ((rc = dzero(net, lg, (size_t)net->total_mcu * sizeof(float)))) return bail(rc);
  if ((rc = dzero(net, wm, (size_t)net->total_hcu * sizeof(float)))) return bail(rc);
  net->cur_lg = lg;
  net->cur_wm = wm;
  if ((rc = reset_state(net))) return bail(rc);
  /* CTA -> (population, HCU) */
  {
    std::vector<int> cp, ch;
    for (int p = 0; p < desc->n_pops; ++p)
      for (int hh = 0; hh < net->pops[p].H; ++hh) { cp.push_back(p); ch.push_back(hh); }
    int* dp = nullptr;
    int* dh = nullptr;
    if ((rc = dalloc(net, &dp, cp.size()))) return bail(rc);
    if ((rc = dalloc(net, &dh, ch.size()))) return bail(rc);
    if (cudaMemcpy(dp, cp.data(), cp.size() * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(dh, ch.data(), ch.size() * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess) {
      net->err = "copy of CTA map failed";
      return bail(BCPNN_ERR_CUDA);
    }
    H.cta_pop = dp;
    H.cta_hcu = dh;
  }
  if ((rc = dalloc(net, &net->d_net, 1))) return bail(rc);
  if ((rc = dalloc(net, &net->d_rp, 1))) return bail(rc);
  if ((rc = dalloc(net, &net->d_pops, net->hp.size()))) return bail(rc);
  if ((rc = dalloc(net, &net->d_projs, std::max<size_t>(1, net->hq.size())))) return bail(rc);
  if ((rc = dalloc(net, &net->d_tabs, net->tabs.size()))) return bail(rc);
  H.pops = net->d_pops;
  H.projs = net->d_projs;
  net->rp.tabs = net->d_tabs;
  if (cudaMemcpy(net->d_pops, net->hp.data(), net->hp.size() * sizeof(PopDev), cudaMemcpyHostToDevice) != cudaSuccess ||
      (!net->hq.empty() &&
       cudaMemcpy(net->d_projs, net->hq.data(), net->hq.size() * sizeof(ProjDev), cudaMemcpyHostToDevice) != cudaSuccess) ||
      cudaMemcpy(net->d_net, &net->h, sizeof(NetDev), cudaMemcpyHostToDevice) != cudaSuccess) {
    net->err = "copy of network descriptor failed";
    return bail(BCPNN_ERR_CUDA);
  }
  /* shared memory of the resident tick kernel: the largest population */
  size_t smem = 0;
  for (const PopHost& P : net->pops) {
    int C[kMaxIn] = {0};
    for (size_t q = 0; q < P.in_proj.size(); ++q) C[q] = net->projs[P.in_proj[q]].C;
    smem = std::max(smem, net->threads == 256 ? t256::tick_smem_bytes_for(P.M, (int)P.in_proj.size(), C)
                                              : t512::tick_smem_bytes_for(P.M, (int)P.in_proj.size(), C));
  }
  int smem_max = 0;
  cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, net->device);
  if (smem + 1024 > (size_t)smem_max) {
    net->err = "network too large for the resident tick kernel: " + std::to_string(smem) +
               " bytes of shared memory per HCU";
    return bail(BCPNN_ERR_INVALID);
  }
  net->tick_smem = smem;
  /* the limit is an attribute of the kernel, shared by every network of the
     process: only ever raise it, per device, so that a network created later
     with a smaller need does not lower it under an earlier one */
  {
    static std::mutex mu;
    static size_t raised[4][kMaxDevices] = {{0}};
    std::lock_guard<std::mutex> lock(mu);
    const int dev = net->device, v = (net->threads == 256 ? 1 : 0) + (net->fp64 ? 2 : 0);
    if (dev < 0 || dev >= kMaxDevices) { net->err = "device ordinal out of range"; return bail(BCPNN_ERR_INVALID); }
    if (smem > raised[v][dev]) {
      if (cudaFuncSetAttribute(net->tick_fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
          cudaFuncSetAttribute(net->tick_fn0, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
        net->err = "cannot raise the shared memory limit of tick_kernel";
        return bail(BCPNN_ERR_CUDA);
      }
      raised[v][dev] = smem;
    }
  }
  /* persistent path: every CTA of the grid must be resident at once */
  {
    int coop = 0, sms = 0, per_sm = 0;
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, net->device);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, net->device);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, net->tick_fn, net->threads, smem);
    const char* e = std::getenv("GSBN_PER_TICK");
    bool forced = e && e[0] == '1';
    net->persistent = !forced && coop && (long long)per_sm * sms >= net->total_hcu && !net->multi;
    if ((rc = dalloc(net, &net->bar, 4 + (size_t)net->total_hcu))) return bail(rc);
  }
  /* ProcUpdMulti: shared memory of its projection kernel (largest M, C) */
  if (net->multi) {
    size_t ms = 0;
    for (const ProjHost& J : net->projs) ms = std::max(ms, multi::proj_smem_bytes(J.M, J.C));
    int smem_max = 0;
    cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, net->device);
    if (ms + 1024 > (size_t)smem_max) {
      net->err = "network too large for the ProcUpdMulti projection kernel: " + std::to_string(ms) +
                 " bytes of shared memory per HCU";
      return bail(BCPNN_ERR_INVALID);
    }
    ms = std::max(ms, (size_t)(3 * net->max_m) * sizeof(float)); /* the population update's share */
    /* the resident persistent form: every population's HCU state in shared
       memory, spike ring of at most 32 ticks (its replay masks) */
    size_t rs = 0;
    for (const PopHost& P : net->pops) {
      int C[kMaxIn] = {0};
      for (size_t q = 0; q < P.in_proj.size(); ++q) C[q] = net->projs[P.in_proj[q]].C;
      rs = std::max(rs, multi::res_smem_bytes(P.M, (int)P.in_proj.size(), C));
    }
    const char* er = std::getenv("GSBN_MULTI_RESIDENT");
    net->multi_resident = !(er && er[0] == '0') && net->ring_len <= 32 && rs + 8192 <= (size_t)smem_max;
    if (net->multi_resident) ms = std::max(ms, rs);
    net->multi_smem = ms;
    static std::mutex mu;
    static size_t raised[kMaxDevices] = {0};
    std::lock_guard<std::mutex> lock(mu);
    if (ms > raised[net->device]) {
      if (cudaFuncSetAttribute(multi::proj_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ms) !=
              cudaSuccess ||
          cudaFuncSetAttribute(multi::tick_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ms) !=
              cudaSuccess ||
          cudaFuncSetAttribute(multi::res_tick_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ms) !=
              cudaSuccess) {
        net->err = "cannot raise the shared memory limit of the ProcUpdMulti kernels";
        return bail(BCPNN_ERR_CUDA);
      }
      raised[net->device] = ms;
    }
    int coop = 0, sms = 0, per_sm = 0;
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, net->device);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, net->device);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &per_sm, net->multi_resident ? (const void*)multi::res_tick_kernel : (const void*)multi::tick_kernel,
        multi::kProjThreads, ms);
    const char* e = std::getenv("GSBN_PER_TICK");
    const bool forced = e && e[0] == '1';
    net->multi_persistent = !forced && coop && (long long)per_sm * sms >= net->total_hcu;
  }
  /* deferred columns of the persistent launch: ring halves sized for every
     MCU of every HCU spiking in one tick (units of kColUnit slots) */
  if (net->persistent) {
    long long cap = 0;
    bool fits = true;
    for (const PopHost& P : net->pops) {
      long long parts = 0;
      for (int q : P.in_proj) parts += (net->projs[q].C + kColUnit - 1) / kColUnit;
      cap += (long long)P.H * P.M * parts;
      if (P.M > 0xffff) fits = false;
    }
    /* unit counters are 32-bit within a launch */
    fits = fits && cap > 0 && cap * (long long)net->max_ticks < (1ll << 31);
    if (!fits) net->tick_fn = net->tick_fn0; /* persistent, with in-CTA columns */
    if (fits) {
      if ((rc = dalloc(net, &net->col_ring, 2 * (size_t)cap))) return bail(rc);
      H.col_ring = net->col_ring;
      H.col_cap = (int)cap;
      if (cudaMemcpy(net->d_net, &net->h, sizeof(NetDev), cudaMemcpyHostToDevice) != cudaSuccess) {
        net->err = "copy of network descriptor failed";
        return bail(BCPNN_ERR_CUDA);
      }
    }
  }
  if (cudaStreamSynchronize(net->stream) != cudaSuccess) {
    net->err = "initialisation failed";
    return bail(BCPNN_ERR_CUDA);
  }
  *out = net;
  return BCPNN_OK;
}

int bcpnn_net_destroy(bcpnn_net* net) {
  if (!net) return BCPNN_ERR_INVALID;
  cudaSetDevice(net->device);
  if (net->stream) cudaStreamSynchronize(net->stream);
  if (net->copy_stream) cudaStreamSynchronize(net->copy_stream);
  for (auto& kv : net->graphs) cudaGraphExecDestroy(kv.second);
  for (auto& J : net->projs)
    for (auto& s : J.slot)
      if (s.ptr) cudaFree(s.ptr);
  for (void* p : net->allocs) cudaFree(p);
  if (net->scratch) cudaFree(net->scratch);
  if (net->stim_lg) cudaFree(net->stim_lg);
  if (net->stim_wm) cudaFree(net->stim_wm);
  if (net->d_lgidx_tab) cudaFree(net->d_lgidx_tab);
  if (net->stream) cudaStreamDestroy(net->stream);
  if (net->copy_stream) cudaStreamDestroy(net->copy_stream);
  for (int k = 0; k < 2; ++k) {
    if (net->stage_ready[k]) cudaEventDestroy(net->stage_ready[k]);
    if (net->stage_free[k]) cudaEventDestroy(net->stage_free[k]);
  }
  for (cudaEvent_t e : net->check_ready)
    if (e) cudaEventDestroy(e);
  for (cudaEvent_t e : net->check_free)
    if (e) cudaEventDestroy(e);
  delete net;
  return BCPNN_OK;
}

int bcpnn_set_conn(bcpnn_net* net, int32_t proj, const int32_t* ii, const int32_t* di, size_t n_slots) {
  if (!net) return BCPNN_ERR_INVALID;
  if (proj < 0 || proj >= (int)net->projs.size() || !ii || !di)
    return fail(net, BCPNN_ERR_INVALID, "bcpnn_set_conn: bad projection or null table");
  const ProjHost& J = net->projs[proj];
  if (n_slots != (size_t)J.H * J.C) return fail(net, BCPNN_ERR_SIZE, "bcpnn_set_conn: slot count != H*C");
  for (size_t s = 0; s < n_slots; ++s) {
    if (ii[s] >= J.Ns || ii[s] < -1) return fail(net, BCPNN_ERR_INVALID, "bcpnn_set_conn: ii outside [-1, Hs*Ms)");
    if (ii[s] >= 0 && (di[s] < 1 || di[s] > 31))
      return fail(net, BCPNN_ERR_INVALID, "bcpnn_set_conn: delay outside [1, 31] ticks");
  }
  CU(cudaSetDevice(net->device));
  const ProjDev& D = net->hq[proj];
  CU(cudaMemcpyAsync(D.ii, ii, n_slots * sizeof(int), cudaMemcpyHostToDevice, net->stream));
  CU(cudaMemcpyAsync(D.di, di, n_slots * sizeof(int), cudaMemcpyHostToDevice, net->stream));
  CU(cudaStreamSynchronize(net->stream));
  return BCPNN_OK;
}

int bcpnn_set_stimulus(bcpnn_net* net, const float* lginp, size_t n_mcu, const float* wmask_row, size_t n_hcu) {
  if (!net) return BCPNN_ERR_INVALID;
  if (!lginp || !wmask_row) return fail(net, BCPNN_ERR_INVALID, "bcpnn_set_stimulus: null buffer");
  if (n_mcu != (size_t)net->total_mcu || n_hcu != (size_t)net->total_hcu)
    return fail(net, BCPNN_ERR_SIZE, "bcpnn_set_stimulus: sizes must be total MCUs and total HCUs");
  CU(cudaSetDevice(net->device));
  CU(cudaMemcpyAsync(net->h.lginp, lginp, n_mcu * sizeof(float), cudaMemcpyHostToDevice, net->stream));
  CU(cudaMemcpyAsync(net->h.wmask, wmask_row, n_hcu * sizeof(float), cudaMemcpyHostToDevice, net->stream));
  net->cur_lg = net->h.lginp;
  net->cur_wm = net->h.wmask;
  return BCPNN_OK;
}

int bcpnn_upload_stimuli(bcpnn_net* net, int32_t n_lginp_rows, const float* lginp_rows, int32_t n_wmask_rows,
                         const float* wmask_rows) {
  if (!net) return BCPNN_ERR_INVALID;
  if (n_lginp_rows <= 0 || n_wmask_rows <= 0 || !lginp_rows || !wmask_rows)
    return fail(net, BCPNN_ERR_INVALID, "bcpnn_upload_stimuli: empty tables");
  CU(cudaSetDevice(net->device));
  CU(cudaStreamSynchronize(net->stream));
  if (net->stim_lg) { CU(cudaFree(net->stim_lg)); net->stim_lg = nullptr; }
  if (net->stim_wm) { CU(cudaFree(net->stim_wm)); net->stim_wm = nullptr; }
  size_t nl = (size_t)n_lginp_rows * net->total_mcu, nw = (size_t)n_wmask_rows * net->total_hcu;
  CU(cudaMalloc((void**)&net->stim_lg, nl * sizeof(float)));
  CU(cudaMalloc((void**)&net->stim_wm, nw * sizeof(float)));
  CU(cudaMemcpy(net->stim_lg, lginp_rows, nl * sizeof(float), cudaMemcpyHostToDevice));
  CU(cudaMemcpy(net->stim_wm, wmask_rows, nw * sizeof(float), cudaMemcpyHostToDevice));
  net->stim_lg_rows = net->stim_lg_cap = n_lginp_rows;
  net->stim_wm_rows = net->stim_wm_cap = n_wmask_rows;
  net->cur_lg = net->h.lginp;
  net->cur_wm = net->h.wmask;
  return BCPNN_OK;
}

int bcpnn_use_stimulus(bcpnn_net* net, int32_t lginp_row, int32_t wmask_row) {
  if (!net) return BCPNN_ERR_INVALID;
  if (lginp_row < 0 || lginp_row >= net->stim_lg_rows || wmask_row < 0 || wmask_row >= net->stim_wm_rows)
    return fail(net, BCPNN_ERR_INVALID, "bcpnn_use_stimulus: row outside the uploaded tables");
  net->cur_lg = net->stim_lg + (size_t)lginp_row * net->total_mcu;
  net->cur_wm = net->stim_wm + (size_t)wmask_row * net->total_hcu;
  return BCPNN_OK;
}

/* lginp of every MCU from one row of pattern indices (one MCU index per HCU,
   anything else = no input), ProcExtGen.cpp:130-144: log(1+eps) on the
   indexed MCU, log(0+eps) elsewhere, float logs as the reference computes
   them. */
static void lginp_from_idx(const bcpnn_net* net, const int32_t* lgidx_row, float eps, float* out) {
  float hit = bx_extgen_logf(1 + eps), miss = bx_extgen_logf(0 + eps);
  size_t k = 0;
  int h = 0;
  for (const PopHost& P : net->pops)
    for (int i = 0; i < P.H; ++i, ++h)
      for (int j = 0; j < P.M; ++j) out[k++] = (lgidx_row[h] == j) ? hit : miss;
}

/* lginp of one pattern-index row on the device (the same two float values
   as lginp_from_idx), one CTA per HCU: no host buffer to stage, so with
   page-locked rows the whole upload is queued without a wait */
__global__ void lginp_idx_kernel(const NetDev* __restrict__ net, const int32_t* __restrict__ lgidx, float hit,
                                 float miss, float* __restrict__ out) {
  const PopDev& P = net->pops[net->cta_pop[blockIdx.x]];
  const int h = net->cta_hcu[blockIdx.x];
  const int want = lgidx[P.hcu_start + h];
  for (int j = threadIdx.x; j < P.M; j += blockDim.x) out[P.mcu_start + h * P.M + j] = (want == j) ? hit : miss;
}

int bcpnn_set_stimulus_idx(bcpnn_net* net, const int32_t* lgidx_row, size_t n_hcu, float eps, const float* wmask_row,
                           size_t n_wmask) {
  if (!net) return BCPNN_ERR_INVALID;
  if (!lgidx_row || !wmask_row) return fail(net, BCPNN_ERR_INVALID, "bcpnn_set_stimulus_idx: null buffer");
  if (n_hcu != (size_t)net->total_hcu || n_wmask != (size_t)net->total_hcu)
    return fail(net, BCPNN_ERR_SIZE, "bcpnn_set_stimulus_idx: sizes must be total HCUs");
  CU(cudaSetDevice(net->device));
  if (!net->d_lgidx) {
    int rc = dalloc(net, &net->d_lgidx, (size_t)net->total_hcu);
    if (rc) return rc;
  }
  CU(cudaMemcpyAsync(net->d_lgidx, lgidx_row, n_hcu * sizeof(int32_t), cudaMemcpyHostToDevice, net->stream));
  lginp_idx_kernel<<<net->total_hcu, 128, 0, net->stream>>>(net->d_net, net->d_lgidx, bx_extgen_logf(1 + eps),
                                                            bx_extgen_logf(0 + eps), net->h.lginp);
  CU(cudaGetLastError());
  net->launches += 1;
  CU(cudaMemcpyAsync(net->h.wmask, wmask_row, n_wmask * sizeof(float), cudaMemcpyHostToDevice, net->stream));
  net->cur_lg = net->h.lginp;
  net->cur_wm = net->h.wmask;
  return BCPNN_OK;
}

/* lginp of n pattern-index rows on the device: block (HCU, row), the values
   of lginp_idx_kernel */
__global__ void lginp_idx_rows_kernel(const NetDev* __restrict__ net, const int32_t* __restrict__ lgidx, int n_hcu,
                                      int n_mcu, float hit, float miss, float* __restrict__ out) {
  const PopDev& P = net->pops[net->cta_pop[blockIdx.x]];
  const int h = net->cta_hcu[blockIdx.x];
  const size_t r = blockIdx.y;
  const int want = lgidx[r * n_hcu + P.hcu_start + h];
  float* o = out + r * n_mcu + P.mcu_start + h * P.M;
  for (int j = threadIdx.x; j < P.M; j += blockDim.x) o[j] = (want == j) ? hit : miss;
}

int bcpnn_upload_stimuli_idx_async(bcpnn_net* net, int32_t n_lgidx_rows, const int32_t* lgidx_rows, float eps,
                                   int32_t n_wmask_rows, const float* wmask_rows) {
  if (!net) return BCPNN_ERR_INVALID;
  if (n_lgidx_rows <= 0 || n_wmask_rows <= 0 || !lgidx_rows || !wmask_rows)
    return fail(net, BCPNN_ERR_INVALID, "bcpnn_upload_stimuli_idx_async: empty tables");
  if (n_lgidx_rows > 65535)
    return fail(net, BCPNN_ERR_SIZE, "bcpnn_upload_stimuli_idx_async: at most 65535 pattern-index rows");
  CU(cudaSetDevice(net->device));
  const size_t H = (size_t)net->total_hcu, N = (size_t)net->total_mcu;
  if (n_lgidx_rows > net->stim_lg_cap || n_wmask_rows > net->stim_wm_cap || n_lgidx_rows > net->lgidx_tab_cap) {
    /* larger tables: runs queued earlier may still read the old ones */
    CU(cudaStreamSynchronize(net->stream));
    if (n_lgidx_rows > net->stim_lg_cap) {
      if (net->stim_lg) { CU(cudaFree(net->stim_lg)); net->stim_lg = nullptr; net->stim_lg_cap = 0; }
      CU(cudaMalloc((void**)&net->stim_lg, (size_t)n_lgidx_rows * N * sizeof(float)));
      net->stim_lg_cap = n_lgidx_rows;
    }
    if (n_wmask_rows > net->stim_wm_cap) {
      if (net->stim_wm) { CU(cudaFree(net->stim_wm)); net->stim_wm = nullptr; net->stim_wm_cap = 0; }
      CU(cudaMalloc((void**)&net->stim_wm, (size_t)n_wmask_rows * H * sizeof(float)));
      net->stim_wm_cap = n_wmask_rows;
    }
    if (n_lgidx_rows > net->lgidx_tab_cap) {
      if (net->d_lgidx_tab) { CU(cudaFree(net->d_lgidx_tab)); net->d_lgidx_tab = nullptr; net->lgidx_tab_cap = 0; }
      CU(cudaMalloc((void**)&net->d_lgidx_tab, (size_t)n_lgidx_rows * H * sizeof(int32_t)));
      net->lgidx_tab_cap = n_lgidx_rows;
    }
  }
  CU(cudaMemcpyAsync(net->d_lgidx_tab, lgidx_rows, (size_t)n_lgidx_rows * H * sizeof(int32_t),
                     cudaMemcpyHostToDevice, net->stream));
  lginp_idx_rows_kernel<<<dim3(net->total_hcu, n_lgidx_rows), 128, 0, net->stream>>>(
      net->d_net, net->d_lgidx_tab, net->total_hcu, net->total_mcu, bx_extgen_logf(1 + eps), bx_extgen_logf(0 + eps),
      net->stim_lg);
  CU(cudaGetLastError());
  net->launches += 1;
  CU(cudaMemcpyAsync(net->stim_wm, wmask_rows, (size_t)n_wmask_rows * H * sizeof(float), cudaMemcpyHostToDevice,
                     net->stream));
  net->stim_lg_rows = n_lgidx_rows;
  net->stim_wm_rows = n_wmask_rows;
  net->cur_lg = net->h.lginp;
  net->cur_wm = net->h.wmask;
  return BCPNN_OK;
}

int bcpnn_upload_stimuli_idx(bcpnn_net* net, int32_t n_lgidx_rows, const int32_t* lgidx_rows, float eps,
                             int32_t n_wmask_rows, const float* wmask_rows) {
  if (!net) return BCPNN_ERR_INVALID;
  if (n_lgidx_rows <= 0 || !lgidx_rows) return fail(net, BCPNN_ERR_INVALID, "bcpnn_upload_stimuli_idx: empty table");
  std::vector<float> lg;
  try {
    lg.resize((size_t)n_lgidx_rows * net->total_mcu);
  } catch (const std::bad_alloc&) { /* nothing may be thrown across the C ABI */
    return fail(net, BCPNN_ERR_INVALID, "bcpnn_upload_stimuli_idx: no host memory for the expanded table");
  }
  for (int r = 0; r < n_lgidx_rows; ++r)
    lginp_from_idx(net, lgidx_rows + (size_t)r * net->total_hcu, eps, lg.data() + (size_t)r * net->total_mcu);
  return bcpnn_upload_stimuli(net, n_lgidx_rows, lg.data(), n_wmask_rows, wmask_rows);
}

int bcpnn_reset(bcpnn_net* net) {
  if (!net) return BCPNN_ERR_INVALID;
  CU(cudaSetDevice(net->device));
  int rc = reset_state(net);
  if (rc) return rc;
  return BCPNN_OK;
}

int bcpnn_get_stream(const bcpnn_net* net, void** stream) {
  if (!net || !stream) return BCPNN_ERR_INVALID;
  *stream = (void*)net->stream;
  return BCPNN_OK;
}

int bcpnn_set_ext_spikes(bcpnn_net* net, int32_t pop, int32_t n, const int32_t* ticks, const int32_t* offsets,
                         const int32_t* idx) {
  if (!net) return BCPNN_ERR_INVALID;
  if (pop < 0 || pop >= (int)net->pops.size() || n < 0 || (n > 0 && (!ticks || !offsets || !idx)))
    return fail(net, BCPNN_ERR_INVALID, "bcpnn_set_ext_spikes: bad arguments");
  PopHost& P = net->pops[pop];
  /* later entries for the same tick replace earlier ones (std::map assignment,
     Pop.cpp:97) */
  std::map<int, std::pair<int, int>> by_tick;
  int t0 = 0, t1 = 0;
  for (int k = 0; k < n; ++k) {
    /* ticks a run can never reach (bcpnn_run: simsteps in [1, 2^24)) are dropped */
    if (ticks[k] < 0 || ticks[k] >= (1 << 24)) continue;
    if (offsets[k] < 0 || offsets[k + 1] < offsets[k])
      return fail(net, BCPNN_ERR_INVALID, "bcpnn_set_ext_spikes: bad offsets");
    for (int e = offsets[k]; e < offsets[k + 1]; ++e)
      if (idx[e] < 0 || idx[e] >= P.n)
        return fail(net, BCPNN_ERR_INVALID, "bcpnn_set_ext_spikes: MCU index outside the population");
    by_tick[ticks[k]] = {offsets[k], offsets[k + 1]};
  }
  std::vector<int> off, flat;
  if (!by_tick.empty()) {
    t0 = by_tick.begin()->first;
    t1 = by_tick.rbegin()->first + 1;
    off.assign((size_t)(t1 - t0) + 1, 0);
    for (int t = t0; t < t1; ++t) {
      off[t - t0] = (int)flat.size();
      auto it = by_tick.find(t);
      if (it != by_tick.end())
        for (int e = it->second.first; e < it->second.second; ++e) flat.push_back(idx[e]);
    }
    off[t1 - t0] = (int)flat.size();
  } else {
    off.assign(1, 0);
  }
  CU(cudaSetDevice(net->device));
  CU(cudaStreamSynchronize(net->stream));
  /* an earlier table is freed here and leaves the list bcpnn_net_destroy frees */
  for (int* old : {P.ext_off, P.ext_idx})
    if (old) {
      net->allocs.erase(std::remove(net->allocs.begin(), net->allocs.end(), (void*)old), net->allocs.end());
      CU(cudaFree(old));
    }
  P.ext_off = nullptr;
  P.ext_idx = nullptr;
  CU(cudaMalloc((void**)&P.ext_off, off.size() * sizeof(int)));
  CU(cudaMalloc((void**)&P.ext_idx, std::max<size_t>(1, flat.size()) * sizeof(int)));
  CU(cudaMemcpy(P.ext_off, off.data(), off.size() * sizeof(int), cudaMemcpyHostToDevice));
  if (!flat.empty()) CU(cudaMemcpy(P.ext_idx, flat.data(), flat.size() * sizeof(int), cudaMemcpyHostToDevice));
  net->allocs.push_back(P.ext_off);
  net->allocs.push_back(P.ext_idx);
  PopDev& D = net->hp[pop];
  D.ext = 1;
  D.ext_off = P.ext_off;
  D.ext_idx = P.ext_idx;
  D.ext_t0 = t0;
  D.ext_t1 = t1;
  CU(cudaMemcpy(net->d_pops + pop, &D, sizeof(PopDev), cudaMemcpyHostToDevice));
  return BCPNN_OK;
}

int bcpnn_set_pop_rng(bcpnn_net* net, int32_t pop, uint32_t seed, uint32_t key_pop) {
  if (!net) return BCPNN_ERR_INVALID;
  if (pop < 0 || pop >= (int)net->pops.size()) return fail(net, BCPNN_ERR_INVALID, "bcpnn_set_pop_rng: no such population");
  CU(cudaSetDevice(net->device));
  CU(cudaStreamSynchronize(net->stream));
  PopDev& D = net->hp[pop];
  D.rng_seed = seed;
  D.rng_pop = key_pop;
  CU(cudaMemcpy(net->d_pops + pop, &D, sizeof(PopDev), cudaMemcpyHostToDevice));
  return BCPNN_OK;
}

int bcpnn_run(bcpnn_net* net, int32_t first_simstep, int32_t n_ticks, float prn, float old_prn) {
  if (!net) return BCPNN_ERR_INVALID;
  if (n_ticks <= 0 || n_ticks > net->max_ticks)
    return fail(net, BCPNN_ERR_INVALID, "bcpnn_run: n_ticks outside [1, max_ticks_per_run]");
  if (first_simstep < 1 || (int64_t)first_simstep + n_ticks > (1 << 24))
    return fail(net, BCPNN_ERR_INVALID, "bcpnn_run: simstep outside [1, 2^24)");
  if (!(std::fabs(prn) <= 3.4028234663852886e38f) || !(std::fabs(old_prn) <= 3.4028234663852886e38f))
    return fail(net, BCPNN_ERR_INVALID, "bcpnn_run: prn and old_prn must be finite");
  CU(cudaSetDevice(net->device));
  bool with_all = (old_prn != prn);
  int need = first_simstep + n_ticks + 1;
  for (int p = 0; p < (int)net->projs.size(); ++p) {
    int s = 0, so = -1, rc;
    if ((rc = prepare_tables(net, p, prn, old_prn, with_all, need, first_simstep + 1, &s, &so))) return rc;
    const ProjHost& J = net->projs[p];
    net->tabs[p].tab = J.slot[s].ptr;
    net->tabs[p].rtab = J.slot[s].rptr;
    net->tabs[p].rk = rcoef(net->hq[p], prn);
    net->tabs[p].k = make_coef(net->hq[p].taupdt * prn, net->hq[p].ke, net->hq[p].kzi, net->hq[p].kzj, net->hq[p].fp64);
    net->tabs[p].len = J.slot[s].len;
    if (with_all) {
      net->tabs[p].tab_old = J.slot[so].ptr;
      net->tabs[p].old_len = J.slot[so].len;
    } else {
      net->tabs[p].tab_old = nullptr;
      net->tabs[p].old_len = 0;
    }
  }
  net->rp.simstep0 = first_simstep;
  net->rp.k0 = (int)(net->k_total & 0x7fffffff);
  net->rp.n_ticks = n_ticks;
  net->rp.prn = prn;
  net->rp.old_prn = old_prn;
  net->rp.lginp = net->cur_lg;
  net->rp.wmask = net->cur_wm;
  net->rp.serial0 = net->tick_serial;
  net->tick_serial += (uint32_t)n_ticks;
  if (net->tick_serial == 0) net->tick_serial = 1; /* tag 0 is the slots' initial value */
  CU(cudaMemcpyAsync(net->d_tabs, net->tabs.data(), net->tabs.size() * sizeof(TabRef), cudaMemcpyHostToDevice,
                     net->stream));
  CU(cudaMemcpyAsync(net->d_rp, &net->rp, sizeof(RunParams), cudaMemcpyHostToDevice, net->stream));
  if (net->direct || net->persistent || net->multi_persistent) {
    enqueue_run(net, n_ticks, with_all);
    CU(cudaGetLastError());
  } else {
    auto key = std::make_pair(n_ticks, with_all ? 1 : 0);
    auto it = net->graphs.find(key);
    cudaGraphExec_t ge = nullptr;
    if (it == net->graphs.end()) {
      int rc = capture_graph(net, n_ticks, with_all, &ge);
      if (rc) return rc;
      net->graphs[key] = ge;
    } else {
      ge = it->second;
    }
    CU(cudaGraphLaunch(ge, net->stream));
  }
  if (net->multi)
    net->launches += (net->multi_persistent ? 1u : (uint64_t)n_ticks * (1 + net->projs.size())) +
                     (with_all ? net->projs.size() : 0u);
  else
    net->launches += (uint64_t)(net->persistent ? 1 : n_ticks) + (with_all ? 2u * net->projs.size() : 0u);
  if (with_all)
    for (const ProjHost& J : net->projs) net->all_cells += (uint64_t)J.H * J.C * J.M;
  net->k_total += n_ticks;
  net->last_run_ticks = n_ticks;
  return BCPNN_OK;
}

int bcpnn_sync(bcpnn_net* net) {
  if (!net) return BCPNN_ERR_INVALID;
  CU(cudaSetDevice(net->device));
  CU(cudaStreamSynchronize(net->stream));
  CU(cudaStreamSynchronize(net->copy_stream));
  return check_device_error(net);
}

int bcpnn_spike_log_words(const bcpnn_net* net, int32_t pop, int32_t* words) {
  if (!net || !words || pop < 0 || pop >= (int)net->pops.size()) return BCPNN_ERR_INVALID;
  *words = net->pops[pop].log_words;
  return BCPNN_OK;
}

int bcpnn_get_spike_log(bcpnn_net* net, int32_t pop, uint32_t* out, size_t n_words) {
  if (!net) return BCPNN_ERR_INVALID;
  if (pop < 0 || pop >= (int)net->pops.size() || !out) return fail(net, BCPNN_ERR_INVALID, "bcpnn_get_spike_log: bad arguments");
  const PopHost& P = net->pops[pop];
  size_t need = (size_t)net->last_run_ticks * P.log_words;
  if (n_words != need) return fail(net, BCPNN_ERR_SIZE, "bcpnn_get_spike_log: n_words != last run ticks * words");
  CU(cudaSetDevice(net->device));
  if (need) CU(cudaMemcpyAsync(out, net->log_buf + P.log_offset, need * sizeof(uint32_t), cudaMemcpyDeviceToHost, net->stream));
  CU(cudaStreamSynchronize(net->stream));
  return check_device_error(net);
}

int bcpnn_get_spike_log_async(bcpnn_net* net, int32_t pop, uint32_t* out, size_t n_words) {
  if (!net) return BCPNN_ERR_INVALID;
  if (pop < 0 || pop >= (int)net->pops.size() || !out)
    return fail(net, BCPNN_ERR_INVALID, "bcpnn_get_spike_log_async: bad arguments");
  const PopHost& P = net->pops[pop];
  size_t need = (size_t)net->last_run_ticks * P.log_words;
  if (n_words != need) return fail(net, BCPNN_ERR_SIZE, "bcpnn_get_spike_log_async: n_words != last run ticks * words");
  CU(cudaSetDevice(net->device));
  if (need) {
    /* device copy into a staging slot on the network's stream, once the host
       copy that last read the slot is done; the host copy on copy_stream */
    const int k = net->stage_next;
    net->stage_next ^= 1;
    uint32_t* st = net->log_stage[k] + P.log_offset;
    const size_t bytes = need * sizeof(uint32_t);
    CU(cudaStreamWaitEvent(net->stream, net->stage_free[k], 0));
    CU(cudaMemcpyAsync(st, net->log_buf + P.log_offset, bytes, cudaMemcpyDeviceToDevice, net->stream));
    CU(cudaEventRecord(net->stage_ready[k], net->stream));
    CU(cudaStreamWaitEvent(net->copy_stream, net->stage_ready[k], 0));
    CU(cudaMemcpyAsync(out, st, bytes, cudaMemcpyDeviceToHost, net->copy_stream));
    CU(cudaEventRecord(net->stage_free[k], net->copy_stream));
  }
  return BCPNN_OK;
}

/* ProcCheck/Pop.cpp:36-44: count the spikes of ticks k0..k1-1 of a spike
   log.  Thread (i, s) counts MCU i over the ticks k0 + s, k0 + s + S, ...
   (S = gridDim.y slices, so that a whole window's loads are spread over the
   GPU) and adds its count to counts[i]; integer sums, so the order does not
   matter. */
__global__ void check_count_kernel(const uint32_t* __restrict__ log, int words, int k0, int k1, int n,
                                   int32_t* __restrict__ counts) {
  const int S = gridDim.y, s = blockIdx.y;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int c = 0;
    for (int t = k0 + s; t < k1; t += S) c += (int)((__ldcg(log + (size_t)t * words + (i >> 5)) >> (i & 31)) & 1u);
    if (c) atomicAdd(counts + i, c);
  }
}

/* ProcCheck/Pop.cpp:46-60: per HCU the first MCU with the largest count (-1
   when none counted) and that count; counters cleared.  One warp per HCU:
   each lane keeps the first of its MCUs with its largest positive count,
   then the warp keeps the largest count and, among equal counts, the
   smallest MCU index -- the MCU gsbn's scan in index order with a strict >
   picks. */
__global__ void check_result_kernel(int32_t* __restrict__ counts, int H, int M, int32_t* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int h = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); h < H; h += nw) {
    int best = -1, most = 0;
    for (int j = lane; j < M; j += 32) {
      const int c = counts[(size_t)h * M + j];
      if (c > most) {
        best = j;
        most = c;
      }
      counts[(size_t)h * M + j] = 0;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const int ob = __shfl_xor_sync(0xffffffffu, best, o), om = __shfl_xor_sync(0xffffffffu, most, o);
      if (om > most || (om == most && om > 0 && ob < best)) {
        best = ob;
        most = om;
      }
    }
    if (lane == 0) {
      out[h] = best;
      out[H + h] = most;
    }
  }
}

static int check_buffers(bcpnn_net* net, int pop) {
  if (net->check_cnt.empty()) {
    net->check_cnt.assign(net->pops.size(), nullptr);
    net->check_out.assign(net->pops.size(), nullptr);
    net->check_ready.assign(net->pops.size(), nullptr);
    net->check_free.assign(net->pops.size(), nullptr);
  }
  if (!net->check_cnt[pop]) {
    const PopHost& P = net->pops[pop];
    if (!net->check_ready[pop]) CU(cudaEventCreateWithFlags(&net->check_ready[pop], cudaEventDisableTiming));
    if (!net->check_free[pop]) CU(cudaEventCreateWithFlags(&net->check_free[pop], cudaEventDisableTiming));
    int rc = dalloc(net, &net->check_cnt[pop], (size_t)P.H * P.M);
    if (rc) return rc;
    if ((rc = dalloc(net, &net->check_out[pop], 2 * (size_t)P.H))) return rc;
    CU(cudaMemsetAsync(net->check_cnt[pop], 0, (size_t)P.H * P.M * sizeof(int32_t), net->stream));
  }
  return BCPNN_OK;
}

int bcpnn_check_count(bcpnn_net* net, int32_t pop, int32_t k0, int32_t k1) {
  if (!net) return BCPNN_ERR_INVALID;
  if (pop < 0 || pop >= (int)net->pops.size()) return fail(net, BCPNN_ERR_INVALID, "bcpnn_check_count: bad population");
  if (k0 < 0 || k1 < k0 || k1 > net->last_run_ticks)
    return fail(net, BCPNN_ERR_INVALID, "bcpnn_check_count: ticks outside the last run");
  CU(cudaSetDevice(net->device));
  int rc = check_buffers(net, pop);
  if (rc) return rc;
  if (k1 == k0) return BCPNN_OK;
  const PopHost& P = net->pops[pop];
  const int n = P.H * P.M;
  const int slices = (k1 - k0) < 16 ? (k1 - k0) : 16;
  check_count_kernel<<<dim3((n + 255) / 256, slices), 256, 0, net->stream>>>(net->log_buf + P.log_offset, P.log_words,
                                                                            k0, k1, n, net->check_cnt[pop]);
  CU(cudaGetLastError());
  net->launches += 1;
  return BCPNN_OK;
}

int bcpnn_check_result_async(bcpnn_net* net, int32_t pop, int32_t* idx, int32_t* cnt, size_t n_hcu) {
  if (!net) return BCPNN_ERR_INVALID;
  if (pop < 0 || pop >= (int)net->pops.size() || !idx || !cnt)
    return fail(net, BCPNN_ERR_INVALID, "bcpnn_check_result_async: bad arguments");
  const PopHost& P = net->pops[pop];
  if (n_hcu != (size_t)P.H) return fail(net, BCPNN_ERR_SIZE, "bcpnn_check_result_async: n_hcu != HCUs of the population");
  CU(cudaSetDevice(net->device));
  int rc = check_buffers(net, pop);
  if (rc) return rc;
  /* the result kernel on the network's stream, once the host copies of the
     previous result are done; the host copies on copy_stream, so the next
     run does not wait for them */
  CU(cudaStreamWaitEvent(net->stream, net->check_free[pop], 0));
  check_result_kernel<<<(P.H + 7) / 8, 256, 0, net->stream>>>(net->check_cnt[pop], P.H, P.M, net->check_out[pop]);
  CU(cudaGetLastError());
  net->launches += 1;
  CU(cudaEventRecord(net->check_ready[pop], net->stream));
  CU(cudaStreamWaitEvent(net->copy_stream, net->check_ready[pop], 0));
  CU(cudaMemcpyAsync(idx, net->check_out[pop], n_hcu * sizeof(int32_t), cudaMemcpyDeviceToHost, net->copy_stream));
  CU(cudaMemcpyAsync(cnt, net->check_out[pop] + P.H, n_hcu * sizeof(int32_t), cudaMemcpyDeviceToHost,
                     net->copy_stream));
  CU(cudaEventRecord(net->check_free[pop], net->copy_stream));
  return BCPNN_OK;
}

int bcpnn_get_ss_flags(bcpnn_net* net, uint8_t* out, size_t n_bytes) {
  if (!net) return BCPNN_ERR_INVALID;
  size_t need = (size_t)net->last_run_ticks * net->projs.size();
  if (!out || n_bytes != need) return fail(net, BCPNN_ERR_SIZE, "bcpnn_get_ss_flags: n_bytes != ticks * projections");
  CU(cudaSetDevice(net->device));
  std::vector<uint32_t> w(need);
  if (need) CU(cudaMemcpyAsync(w.data(), net->h.ss_log, need * sizeof(uint32_t), cudaMemcpyDeviceToHost, net->stream));
  CU(cudaStreamSynchronize(net->stream));
  for (size_t i = 0; i < need; ++i) out[i] = (uint8_t)w[i];
  return BCPNN_OK;
}

int bcpnn_state_info(const bcpnn_net* net, const char* name, int32_t* type, size_t* count) {
  if (!net || !type || !count) return BCPNN_ERR_INVALID;
  Resolved r;
  if (!resolve(net, name, &r)) return BCPNN_ERR_NOT_FOUND;
  *type = r.type;
  *count = r.count;
  return BCPNN_OK;
}

int bcpnn_read_state(bcpnn_net* net, const char* name, void* host, size_t bytes) {
  if (!net) return BCPNN_ERR_INVALID;
  Resolved r;
  if (!resolve(net, name, &r)) return fail(net, BCPNN_ERR_NOT_FOUND, std::string("unknown state vector ") + (name ? name : "(null)"));
  if (!host || bytes != r.count * type_size(r.type)) return fail(net, BCPNN_ERR_SIZE, "bcpnn_read_state: size mismatch");
  CU(cudaSetDevice(net->device));
  int last = (int)((net->k_total - 1) & 1);  /* buffer written by the last tick (1 before any tick) */
  switch (r.kind) {
    case K_PLAIN:
      CU(cudaMemcpyAsync(host, r.ptr, bytes, cudaMemcpyDeviceToHost, net->stream));
      break;
    case K_PARITY:
      CU(cudaMemcpyAsync(host, r.par[last], bytes, cudaMemcpyDeviceToHost, net->stream));
      break;
    case K_SI:
      CU(cudaMemcpyAsync(host, si_last(net, r), bytes, cudaMemcpyDeviceToHost, net->stream));
      break;
    case K_CELL: {
      int rc = ensure_scratch(net, r.count);
      if (rc) return rc;
      cell_gather_kernel<<<grid_for(r.count, 256), 256, 0, net->stream>>>(r.cell, r.count, r.field, net->scratch);
      CU(cudaGetLastError());
      net->launches++;
      CU(cudaMemcpyAsync(host, net->scratch, bytes, cudaMemcpyDeviceToHost, net->stream));
      break;
    }
    case K_SIQ: {
      const ProjHost& J = net->projs[r.proj];
      const ProjDev& D = net->hq[r.proj];
      std::vector<int> cnt(J.H), list((size_t)J.H * J.C);
      CU(cudaMemcpyAsync(cnt.data(), D.list_cnt, J.H * sizeof(int), cudaMemcpyDeviceToHost, net->stream));
      CU(cudaMemcpyAsync(list.data(), D.list, list.size() * sizeof(int), cudaMemcpyDeviceToHost, net->stream));
      CU(cudaStreamSynchronize(net->stream));
      int8_t* o = (int8_t*)host;
      std::memset(o, 0, bytes);
      for (int hh = 0; hh < J.H; ++hh)
        for (int e = 0; e < cnt[hh] && e < J.C; ++e) {
          int row = list[(size_t)hh * J.C + e];
          if (row >= 0 && (size_t)row < r.count) o[row] = 1;
        }
      break;
    }
  }
  CU(cudaStreamSynchronize(net->stream));
  return BCPNN_OK;
}

int bcpnn_write_state(bcpnn_net* net, const char* name, const void* host, size_t bytes) {
  if (!net) return BCPNN_ERR_INVALID;
  Resolved r;
  if (!resolve(net, name, &r)) return fail(net, BCPNN_ERR_NOT_FOUND, std::string("unknown state vector ") + (name ? name : "(null)"));
  if (!host || bytes != r.count * type_size(r.type)) return fail(net, BCPNN_ERR_SIZE, "bcpnn_write_state: size mismatch");
  CU(cudaSetDevice(net->device));
  int last = (int)((net->k_total - 1) & 1);
  switch (r.kind) {
    case K_PLAIN:
      CU(cudaMemcpyAsync(r.ptr, host, bytes, cudaMemcpyHostToDevice, net->stream));
      break;
    case K_PARITY:
      CU(cudaMemcpyAsync(r.par[last], host, bytes, cudaMemcpyHostToDevice, net->stream));
      break;
    case K_SI:
      CU(cudaMemcpyAsync(si_last(net, r), host, bytes, cudaMemcpyHostToDevice, net->stream));
      break;
    case K_CELL: {
      int rc = ensure_scratch(net, r.count);
      if (rc) return rc;
      CU(cudaMemcpyAsync(net->scratch, host, bytes, cudaMemcpyHostToDevice, net->stream));
      cell_scatter_kernel<<<grid_for(r.count, 256), 256, 0, net->stream>>>(r.cell, r.count, r.field, net->scratch);
      CU(cudaGetLastError());
      net->launches++;
      break;
    }
    case K_SIQ: {
      const ProjHost& J = net->projs[r.proj];
      const ProjDev& D = net->hq[r.proj];
      const int8_t* in = (const int8_t*)host;
      std::vector<int> cnt(J.H, 0), list((size_t)J.H * J.C, 0);
      for (int hh = 0; hh < J.H; ++hh)
        for (int s = 0; s < J.C; ++s)
          if (in[(size_t)hh * J.C + s] > 0) list[(size_t)hh * J.C + cnt[hh]++] = hh * J.C + s;
      CU(cudaMemcpyAsync(D.list_cnt, cnt.data(), J.H * sizeof(int), cudaMemcpyHostToDevice, net->stream));
      CU(cudaMemcpyAsync(D.list, list.data(), list.size() * sizeof(int), cudaMemcpyHostToDevice, net->stream));
      break;
    }
  }
  CU(cudaStreamSynchronize(net->stream));
  return BCPNN_OK;
}

int bcpnn_prune(bcpnn_net* net, int32_t proj, int32_t threshold_t, float wp, float wn, int32_t* removed_src,
                size_t cap, int32_t* n_removed) {
  if (!net) return BCPNN_ERR_INVALID;
  if (proj < 0 || proj >= (int)net->projs.size() || !removed_src || !n_removed)
    return fail(net, BCPNN_ERR_INVALID, "bcpnn_prune: bad projection or null buffer");
  if (!(wp > wn)) return fail(net, BCPNN_ERR_INVALID, "bcpnn_prune: w+ must be larger than w-");
  const ProjHost& J = net->projs[proj];
  const size_t R = (size_t)J.H * J.C;
  if (cap < R) return fail(net, BCPNN_ERR_SIZE, "bcpnn_prune: removed_src must hold H*C entries");
  CU(cudaSetDevice(net->device));
  int rc = ensure_scratch(net, R);
  if (rc) return rc;
  int* out = reinterpret_cast<int*>(net->scratch);
  prune_rows_kernel<<<grid_for(R * 32, 256), 256, 0, net->stream>>>(net->d_projs, proj, threshold_t, wp, wn, out);
  CU(cudaGetLastError());
  net->launches += 1;
  std::vector<int> all(R);
  CU(cudaMemcpyAsync(all.data(), out, R * sizeof(int), cudaMemcpyDeviceToHost, net->stream));
  CU(cudaStreamSynchronize(net->stream));
  int32_t n = 0;
  for (size_t r = 0; r < R; ++r)
    if (all[r] >= 0) removed_src[n++] = all[r];
  *n_removed = n;
  return BCPNN_OK;
}

int bcpnn_counters(bcpnn_net* net, uint64_t out[3]) {
  if (!net || !out) return BCPNN_ERR_INVALID;
  CU(cudaSetDevice(net->device));
  unsigned long long c[3];
  CU(cudaMemcpyAsync(c, net->h.counters, sizeof(c), cudaMemcpyDeviceToHost, net->stream));
  CU(cudaStreamSynchronize(net->stream));
  /* the all-cells sweep is counted on the host: every cell of every
     projection per sweep (Proj.cpp:558-586 loops over all of them) */
  out[0] = c[0];
  out[1] = c[1];
  out[2] = net->all_cells;
  return BCPNN_OK;
}

int bcpnn_kernel_launches(const bcpnn_net* net, uint64_t* out) {
  if (!net || !out) return BCPNN_ERR_INVALID;
  *out = net->launches;
  return BCPNN_OK;
}

/* pairs for the division self-test: a 64-bit mix of (seed, index), with one
   draw in two forced into a hard class */
__device__ __forceinline__ uint32_t selftest_mix(uint64_t x) {
  x += 0x9e3779b97f4a7c15ull;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
  return (uint32_t)(x ^ (x >> 31));
}

__global__ void division_check_kernel(uint64_t n, uint64_t seed, unsigned long long* tested,
                                      unsigned long long* bad) {
  unsigned long long t = 0, b = 0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t ua = selftest_mix(seed * 0x100000001b3ull + 3 * i), ub = selftest_mix(seed * 0x100000001b3ull + 3 * i + 1);
    switch (selftest_mix(seed + 3 * i + 2) % 20) {
      case 0: ua &= 0x807fffffu; break;                                   /* subnormal numerator  */
      case 1: ub &= 0x807fffffu; break;                                   /* subnormal divisor    */
      case 2: ua &= 0x80000000u; break;                                   /* zero numerator       */
      case 3: ub = (ub & 0x80000000u) | 0x7f800000u; break;               /* infinite divisor     */
      case 4: ua = (ua & 0x80000000u) | 0x7f800000u; break;               /* infinite numerator   */
      case 5: ub &= 0x80000000u; break;                                   /* zero divisor         */
      case 6: ub = (ub & 0x80ffffffu) | 0x7e000000u; break;               /* huge divisor         */
      case 7: ua = (ua & 0x80ffffffu) | 0x7e000000u; ub = (ub & 0x80ffffffu) | 0x01000000u; break; /* overflow */
      case 8: ub = (ub & 0x807fffffu) | (((ua >> 23) & 0xffu) + 100u > 254u ? 0x3f800000u : (((ua >> 23) & 0xffu) + 100u) << 23); break;
      case 9: ua = (ua & 0x807fffffu) | 0x3f800000u; ub = (ub & 0x807fffffu) | 0x3f800000u; break; /* [1, 2) */
      case 10:
      case 11: { /* a / d within an ulp of a float midpoint: a = RN(m d), m = q + ulp(q)/2 */
        const uint32_t uq = (ua & 0x807fffffu) | (((ua >> 23) & 0x3fu) + 96u) << 23;
        ub = (ub & 0x807fffffu) | (((ub >> 23) & 0x3fu) + 96u) << 23;
        const double m = (double)__uint_as_float(uq) + (double)__uint_as_float(uq & 0x7f800000u) * 0x1p-24;
        ua = __float_as_uint(__double2float_rn(m * (double)__uint_as_float(ub))) + (uint32_t)(ua >> 31) -
             (uint32_t)((ua >> 30) & 1u);
        break;
      }
      default: break;
    }
    const float a = __uint_as_float(ua), d = __uint_as_float(ub);
    if (a != a || d != d) continue;
    const float q0 = a / d, q1 = div_rn(a, d);
    ++t;
    if (__float_as_uint(q0) != __float_as_uint(q1) && !(q0 != q0 && q1 != q1)) ++b;
    /* the reciprocal form of the closed forms (qmul), where it claims the
       quotient; a subnormal quotient is left to div_rn by its callers */
    bool slow = false;
    const float q2 = qmul(a, __drcp_rn((double)d), slow);
    if (!slow && __float_as_uint(q0) != __float_as_uint(q2) && !(q0 != q0 && q2 != q2)) ++b;
  }
  atomicAdd(tested, t);
  atomicAdd(bad, b);
}

int bcpnn_phase_probe(bcpnn_net* net, uint64_t* out, int32_t max_ctas, int32_t* n_ctas, int32_t reset) {
  if (!net) return BCPNN_ERR_INVALID;
#ifdef BCPNN_PHASE_PROBE
  if (!n_ctas || (max_ctas > 0 && !out)) return fail(net, BCPNN_ERR_INVALID, "bcpnn_phase_probe: null buffer");
  const int n = std::min(net->total_hcu, kProbeCtas);
  *n_ctas = n;
  CU(cudaSetDevice(net->device));
  CU(cudaStreamSynchronize(net->stream));
  if (max_ctas > 0) {
    const size_t k = (size_t)std::min(n, (int)max_ctas) * kProbeSlots;
    CU(cudaMemcpyFromSymbol(out, g_phase_probe, k * sizeof(uint64_t)));
  }
  if (reset) {
    static const uint64_t zeros[kProbeCtas * kProbeSlots] = {};
    CU(cudaMemcpyToSymbol(g_phase_probe, zeros, sizeof(zeros)));
  }
  return BCPNN_OK;
#else
  (void)out; (void)max_ctas; (void)reset;
  if (n_ctas) *n_ctas = 0;
  return fail(net, BCPNN_ERR_STATE, "bcpnn_phase_probe: this library was built without BCPNN_PHASE_PROBE");
#endif
}

int bcpnn_selftest_division(bcpnn_net* net, uint64_t n_pairs, uint64_t seed, uint64_t* tested, uint64_t* mismatches) {
  if (!net || !tested || !mismatches) return BCPNN_ERR_INVALID;
  cudaSetDevice(net->device);
  unsigned long long* c = nullptr;
  CU(cudaMalloc((void**)&c, 2 * sizeof(unsigned long long)));
  cudaError_t e = cudaMemsetAsync(c, 0, 2 * sizeof(unsigned long long), net->stream);
  if (e == cudaSuccess) {
    division_check_kernel<<<148 * 4, 256, 0, net->stream>>>(n_pairs, seed, c, c + 1);
    e = cudaGetLastError();
  }
  unsigned long long h[2] = {0, 0};
  if (e == cudaSuccess) e = cudaMemcpyAsync(h, c, sizeof(h), cudaMemcpyDeviceToHost, net->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(net->stream);
  cudaFree(c);
  if (e != cudaSuccess) return fail(net, BCPNN_ERR_CUDA, std::string("division self-test: ") + cudaGetErrorString(e));
  *tested = h[0];
  *mismatches = h[1];
  return BCPNN_OK;
}

int bcpnn_selftest_barrier_timeout(bcpnn_net* net, int64_t limit_ns) {
  if (!net) return BCPNN_ERR_INVALID;
  if (limit_ns < 100000 || limit_ns > 2000000000) return fail(net, BCPNN_ERR_INVALID, "bcpnn_selftest_barrier_timeout: limit outside [1e5, 2e9] ns");
  CU(cudaSetDevice(net->device));
  unsigned int* bar = nullptr;
  CU(cudaMalloc((void**)&bar, sizeof(unsigned int)));
  cudaError_t e = cudaMemsetAsync(bar, 0, sizeof(unsigned int), net->stream);
  /* two CTAs, each waiting for a third arrival that never comes */
  if (e == cudaSuccess) {
    t512::barrier_probe_kernel<<<2, 32, 0, net->stream>>>(bar, net->h.err, (unsigned long long)limit_ns);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(net->stream);
  cudaFree(bar);
  if (e != cudaSuccess) return fail(net, BCPNN_ERR_CUDA, std::string("barrier probe: ") + cudaGetErrorString(e));
  net->launches += 1;
  return check_device_error(net);
}

}  // extern "C"

/* ======================================================================== */
/* Allocation-free read of a state vector                                    */
/* ======================================================================== */

/* Scratch of bcpnn_read_state_noalloc: a file-scope device array that every
   GPU loading this library holds until the process exits.  Host code only
   uses its device address from cudaGetSymbolAddress; the name itself is a
   host-side stand-in. */
static constexpr size_t kNoAllocScratchFloats = (size_t)1 << 20; /* 4 MiB */
static __device__ __align__(256) float g_noalloc_scratch[kNoAllocScratchFloats];
static constexpr int kNoAllocMaxDevices = 64;
/* device address per ordinal, set on the first call on that device.  Several
   host threads may set an entry at once (all store the same address), so the
   entries are atomics.  The cached address assumes the device is not reset
   (cudaDeviceReset) while the library is loaded. */
static std::atomic<float*> g_noalloc_scratch_dev[kNoAllocMaxDevices];

namespace {

/* name -> vector, like resolve() but without building any std::string; the
   delay-queue view .siq_<proj> (assembled on the host) is not offered */
bool resolve_noalloc(const bcpnn_net* net, const char* name, Resolved* r) {
  const char* us = std::strrchr(name, '_');
  if (!us || !us[1]) return false;
  char base[16];
  size_t blen = (size_t)(us - name);
  if (blen == 0 || blen >= sizeof(base)) return false;
  std::memcpy(base, name, blen);
  base[blen] = '\0';
  int id = 0;
  for (const char* c = us + 1; *c; ++c) {
    if (*c < '0' || *c > '9' || id > 100000) return false;
    id = id * 10 + (*c - '0');
  }
  auto is = [&](const char* b) { return std::strcmp(base, b) == 0; };
  r->proj = id;
  if (id < (int)net->pops.size()) {
    const PopHost& P = net->pops[id];
    const PopDev& D = net->hp[id];
    size_t n = (size_t)P.n;
    auto plain = [&](void* p, int type, size_t count) { r->kind = K_PLAIN; r->ptr = p; r->type = type; r->count = count; return true; };
    auto parity = [&](float* a, float* b, size_t count) { r->kind = K_PARITY; r->par[0] = a; r->par[1] = b; r->type = BCPNN_F32; r->count = count; return true; };
    if (is("dsup")) return parity(D.dsup[0], D.dsup[1], n);
    if (is("epsc")) return parity(D.epsc[0], D.epsc[1], n * P.dim_proj);
    if (is("bj")) return parity(D.bj[0], D.bj[1], n * P.dim_proj);
    if (is("act")) return plain(D.act, BCPNN_F32, n);
    if (is("spike")) return D.ring ? plain(D.ring, BCPNN_I8, n * (size_t)D.ring_len) : plain(D.spike, BCPNN_I8, n);
    if (is(".counter")) return plain(D.counter, BCPNN_I32, n);
    if (is("ada") && D.ada) return plain(D.ada, BCPNN_F32, n);
  }
  if (id < (int)net->projs.size()) {
    const ProjHost& J = net->projs[id];
    const ProjDev& D = net->hq[id];
    size_t R = (size_t)J.H * J.C, HM = (size_t)J.H * J.M, cells = R * J.M;
    auto plain = [&](void* p, int type, size_t count) { r->kind = K_PLAIN; r->ptr = p; r->type = type; r->count = count; return true; };
    auto cell = [&](int f) { r->kind = K_CELL; r->field = f; r->cell = D.cell; r->type = BCPNN_F32; r->count = cells; return true; };
    if (is("ii")) return plain(D.ii, BCPNN_I32, R);
    if (is("di")) return plain(D.di, BCPNN_I32, R);
    if (is("qi")) return plain(D.qi, BCPNN_I32, R);
    if (is("pi")) return plain(D.pi, BCPNN_F32, R);
    if (is("ei")) return plain(D.ei, BCPNN_F32, R);
    if (is("zi")) return plain(D.zi, BCPNN_F32, R);
    if (is("ti")) return plain(D.ti, BCPNN_I32, R);
    if (is("pj")) return plain(D.pj, BCPNN_F32, HM);
    if (is("ej")) return plain(D.ej, BCPNN_F32, HM);
    if (is("zj")) return plain(D.zj, BCPNN_F32, HM);
    if (is("tij")) return plain(D.tij, BCPNN_I32, cells);
    if (is("wij")) return plain(D.wij, BCPNN_F32, cells);
    if (is("pij")) return cell(0);
    if (is("eij")) return cell(1);
    if (is("zi2")) return cell(2);
    if (is("zj2")) return cell(3);
    if (is("si")) { r->kind = K_SI; r->par[0] = D.si[0]; r->par[1] = D.si[1]; r->type = BCPNN_I8; r->count = (size_t)J.Ns; return true; }
  }
  return false;
}

}  // namespace

extern "C" int bcpnn_read_state_noalloc(bcpnn_net* net, const char* name, void* host, size_t bytes) {
  if (!net) return BCPNN_ERR_INVALID;
  Resolved r;
  if (!name || !resolve_noalloc(net, name, &r))
    return fail(net, BCPNN_ERR_NOT_FOUND, "bcpnn_read_state_noalloc: unknown state vector (or .siq_, not offered)");
  if (!host || bytes != r.count * type_size(r.type))
    return fail(net, BCPNN_ERR_SIZE, "bcpnn_read_state_noalloc: size mismatch");
  if (r.kind == K_CELL && r.count > kNoAllocScratchFloats)
    return fail(net, BCPNN_ERR_SIZE, "bcpnn_read_state_noalloc: the vector has more elements than the static "
                                     "scratch holds (1048576 floats); use bcpnn_read_state");
  if (net->device < 0 || net->device >= kNoAllocMaxDevices)
    return fail(net, BCPNN_ERR_INVALID, "bcpnn_read_state_noalloc: device ordinal beyond 63");
  CU(cudaSetDevice(net->device));
  const int last = (int)((net->k_total - 1) & 1);
  switch (r.kind) {
    case K_PLAIN:
      CU(cudaMemcpyAsync(host, r.ptr, bytes, cudaMemcpyDeviceToHost, net->stream));
      break;
    case K_PARITY:
      CU(cudaMemcpyAsync(host, r.par[last], bytes, cudaMemcpyDeviceToHost, net->stream));
      break;
    case K_SI:
      CU(cudaMemcpyAsync(host, si_last(net, r), bytes, cudaMemcpyDeviceToHost, net->stream));
      break;
    case K_CELL: {
      /* set-up, once per device with that device current: the device address
         of the static scratch */
      float* scratch = g_noalloc_scratch_dev[net->device].load(std::memory_order_relaxed);
      if (!scratch) {
        void* p = nullptr;
        CU(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        scratch = (float*)p;
        g_noalloc_scratch_dev[net->device].store(scratch, std::memory_order_relaxed);
      }
      /* every element read back is written by the gather first, so nothing
         of an earlier call's contents is used */
      cell_gather_kernel<<<grid_for(r.count, 256), 256, 0, net->stream>>>(r.cell, r.count, r.field, scratch);
      CU(cudaGetLastError());
      net->launches++;
      CU(cudaMemcpyAsync(host, scratch, bytes, cudaMemcpyDeviceToHost, net->stream));
      break;
    }
    default:
      return fail(net, BCPNN_ERR_NOT_FOUND, "bcpnn_read_state_noalloc: vector not offered");
  }
  CU(cudaStreamSynchronize(net->stream));
  return BCPNN_OK;
}

/* the batch engine (include/bcpnn_batch.h) shares this unit's device code */
#include "bcpnn_batch.cuh"
