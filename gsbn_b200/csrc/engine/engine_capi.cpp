/* extern "C" layer over the engine (include/gsbn_engine.h). */
#include <cstring>
#include <string>

#include "gsbn_engine.h"
#include "gsbn_engine.hpp"

namespace {
thread_local std::string g_err;

template <class F>
int guarded(F f) {
  try {
    g_err.clear();
    return f();
  } catch (const gsbn::Fatal& e) {
    g_err = e.what();
    return BCPNN_ERR_STATE;
  } catch (const std::bad_alloc&) {
    g_err = "out of host memory";
    return BCPNN_ERR_STATE;
  } catch (const std::exception& e) {
    g_err = e.what();
    return BCPNN_ERR_STATE;
  }
}
}  // namespace

struct gsbn_solver {
  gsbn::Solver* solver;
};

extern "C" {

int gsbn_solver_create(const char* net_path, const char* snapshot_path, int mode, gsbn_solver** out) {
  if (!net_path || !out) return BCPNN_ERR_INVALID;
  *out = nullptr;
  if (mode != GSBN_MODE_CPU && mode != GSBN_MODE_GPU) return BCPNN_ERR_INVALID;
  return guarded([&] {
    bool copy = snapshot_path && *snapshot_path;
    auto* s = new gsbn_solver{nullptr};
    try {
      s->solver = new gsbn::Solver(copy ? gsbn::Solver::COPY_SOLVER : gsbn::Solver::NEW_SOLVER, net_path,
                                   copy ? snapshot_path : "", mode == GSBN_MODE_GPU ? gsbn::GPU : gsbn::CPU);
    } catch (...) {
      delete s;
      throw;
    }
    *out = s;
    return BCPNN_OK;
  });
}

int gsbn_solver_run(gsbn_solver* s, int windows) {
  if (!s || !s->solver) return BCPNN_ERR_INVALID;
  return guarded([&] {
    s->solver->run(windows != 0);
    return BCPNN_OK;
  });
}

int gsbn_solver_stats(const gsbn_solver* s, int64_t* ticks, int64_t* windows, int32_t* correct, int32_t* patterns) {
  if (!s || !s->solver) return BCPNN_ERR_INVALID;
  if (ticks) *ticks = s->solver->ticks_run();
  if (windows) *windows = s->solver->windows_run();
  int c = -1, n = -1;
  auto& pool = s->solver->pool();
  auto ic = pool.find("check-correct"), in = pool.find("check-patterns");
  if (ic != pool.end() && in != pool.end()) {
    c = ic->second.i;
    n = in->second.i;
  }
  if (correct) *correct = c;
  if (patterns) *patterns = n;
  return BCPNN_OK;
}

int gsbn_solver_net(gsbn_solver* s, void** net) {
  if (!s || !s->solver || !net) return BCPNN_ERR_INVALID;
  *net = s->solver->db().net();
  return BCPNN_OK;
}

int gsbn_solver_destroy(gsbn_solver* s) {
  if (!s) return BCPNN_ERR_INVALID;
  delete s->solver;
  delete s;
  return BCPNN_OK;
}

const char* gsbn_engine_last_error(void) { return g_err.c_str(); }

int gsbn_prototxt_dump(const char* path, char* out, size_t cap, size_t* needed) {
  if (!path) return BCPNN_ERR_INVALID;
  return guarded([&] {
    std::string d = gsbn::dump_solver_param(gsbn::read_solver_param(path));
    if (needed) *needed = d.size() + 1;
    if (!out || cap < d.size() + 1) return BCPNN_ERR_SIZE;
    std::memcpy(out, d.c_str(), d.size() + 1);
    return BCPNN_OK;
  });
}

int gsbn_stim_decode(const char* path, uint32_t dims[4], uint32_t* data, size_t data_cap, float* mask, size_t mask_cap) {
  if (!path || !dims) return BCPNN_ERR_INVALID;
  return guarded([&] {
    gsbn::StimRawData s = gsbn::read_stim_raw_data(path);
    dims[0] = s.data_rows;
    dims[1] = s.data_cols;
    dims[2] = s.mask_rows;
    dims[3] = s.mask_cols;
    if (data) {
      if (data_cap < s.data.size()) return BCPNN_ERR_SIZE;
      if (!s.data.empty()) std::memcpy(data, s.data.data(), s.data.size() * 4);
    }
    if (mask) {
      if (mask_cap < s.mask.size()) return BCPNN_ERR_SIZE;
      if (!s.mask.empty()) std::memcpy(mask, s.mask.data(), s.mask.size() * 4);
    }
    return BCPNN_OK;
  });
}

int gsbn_procedure_names(char* out, size_t cap) {
  if (!out) return BCPNN_ERR_INVALID;
  std::string all;
  for (auto& n : gsbn::ProcedureFactory::names()) all += (all.empty() ? "" : ",") + n;
  if (cap < all.size() + 1) return BCPNN_ERR_SIZE;
  std::memcpy(out, all.c_str(), all.size() + 1);
  return BCPNN_OK;
}

}  // extern "C"
