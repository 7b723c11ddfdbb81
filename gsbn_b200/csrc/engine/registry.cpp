/* GlobalVar, Database, ProcedureFactory, Upd and Solver of the host engine.
 *
 * Follows gsbn's Solver (src/gsbn/Solver.cpp:9-92), Upd (src/gsbn/Upd.cpp:12-40),
 * ProcedureFactory (src/gsbn/ProcedureFactory.cpp:9-29) and GlobalVar
 * (src/gsbn/GlobalVar.cpp) in behaviour; the window loop (Upd::update_window)
 * is this library's addition.
 */
#include <sys/stat.h>

#include <algorithm>
#include <chrono>
#include <iomanip>
#include <cerrno>
#include <cstring>
#include <iostream>

#include "gsbn_engine.hpp"

namespace gsbn {

/* ------------------------------------------------------------ GlobalVar */

namespace {
thread_local GlobalVar::Pool* g_bound_pool = nullptr;
GlobalVar::Pool& fallback_pool() {
  static GlobalVar::Pool p;
  return p;
}
}  // namespace

GlobalVar::GlobalVar() : pool_(g_bound_pool ? g_bound_pool : &fallback_pool()) {}

GlobalVar::Pool* GlobalVar::bind(Pool* p) {
  Pool* old = g_bound_pool;
  g_bound_pool = p;
  return old;
}

#define GV_GET(fn, T, member)                                \
  bool GlobalVar::fn(const std::string& key, T& v) const {   \
    auto it = pool_->find(key);                              \
    if (it == pool_->end()) return false;                    \
    v = it->second.member;                                   \
    return true;                                             \
  }
GV_GET(getb, bool, b)
GV_GET(geti, int, i)
GV_GET(getf, float, f)
GV_GET(gets, std::string, s)
#undef GV_GET

/* gsbn's glvar_t is a union: a value put as one type reads back as another
   by reinterpretation.  Procedures never rely on that, so each put writes
   its own member and the rest are left as they were. */
#define GV_PUT(fn, T, member)                                \
  bool GlobalVar::fn(const std::string& key, T v) {          \
    bool existed = pool_->count(key) != 0;                   \
    (*pool_)[key].member = v;                                \
    return existed;                                          \
  }
GV_PUT(putb, bool, b)
GV_PUT(puti, int, i)
GV_PUT(putf, float, f)
#undef GV_PUT

bool GlobalVar::puts(const std::string& key, const std::string& v) {
  bool existed = pool_->count(key) != 0;
  (*pool_)[key].s = v;
  return existed;
}

/* ------------------------------------------------------------- Database */

Database::~Database() {
  if (net_) bcpnn_net_destroy(net_);
}

HostVector<int32_t>* Database::create_vector_i32(const std::string& name) {
  if (i32_.count(name)) return nullptr; /* gsbn: warning + NULL (Database.cpp:124-131) */
  auto& p = i32_[name];
  p.reset(new HostVector<int32_t>());
  return p.get();
}
HostVector<float>* Database::create_vector_f32(const std::string& name) {
  if (f32_.count(name)) return nullptr;
  auto& p = f32_[name];
  p.reset(new HostVector<float>());
  return p.get();
}
HostVector<int32_t>* Database::vector_i32(const std::string& name) {
  auto it = i32_.find(name);
  return it == i32_.end() ? nullptr : it->second.get();
}
HostVector<float>* Database::vector_f32(const std::string& name) {
  auto it = f32_.find(name);
  return it == f32_.end() ? nullptr : it->second.get();
}

bcpnn_net* Database::require_net(const char* who) const {
  if (!net_) fatal(std::string(who) + " needs the network built by ProcUpdLazy: list ProcUpdLazy before it");
  return net_;
}

std::vector<uint8_t> Database::read_state(const std::string& name, int32_t* type) {
  bcpnn_net* n = require_net("Database::read_state");
  int32_t t = 0;
  size_t count = 0;
  int st = bcpnn_state_info(n, name.c_str(), &t, &count);
  if (st != BCPNN_OK) fatal("no state vector " + name);
  size_t bytes = count * (t == BCPNN_I8 ? 1 : 4);
  std::vector<uint8_t> out(bytes);
  st = bcpnn_read_state(n, name.c_str(), out.data(), bytes);
  if (st != BCPNN_OK) fatal("reading " + name + ": " + bcpnn_last_error(n));
  if (type) *type = t;
  return out;
}

void Database::write_state(const std::string& name, const void* data, size_t bytes) {
  bcpnn_net* n = require_net("Database::write_state");
  int st = bcpnn_write_state(n, name.c_str(), data, bytes);
  if (st != BCPNN_OK) fatal("writing " + name + ": " + bcpnn_last_error(n));
}

bool SpikeLog::tick_has_spike(int pop, int k) const {
  const uint32_t* w = bits[pop].data() + (size_t)k * words[pop];
  for (int i = 0; i < words[pop]; i++)
    if (w[i]) return true;
  return false;
}

/* ----------------------------------------------------- ProcedureFactory */

ProcedureCreator::ProcedureCreator(const std::string& classname) { ProcedureFactory::registerit(classname, this); }

std::map<std::string, ProcedureCreator*>& ProcedureFactory::get_table() {
  static std::map<std::string, ProcedureCreator*> table;
  return table;
}

void ProcedureFactory::registerit(const std::string& classname, ProcedureCreator* creator) {
  get_table()[classname] = creator;
}

ProcedureBase* ProcedureFactory::create(const std::string& classname) {
  auto it = get_table().find(classname);
  return it == get_table().end() ? nullptr : it->second->create();
}

std::vector<std::string> ProcedureFactory::names() {
  std::vector<std::string> out;
  for (auto& kv : get_table()) out.push_back(kv.first);
  return out;
}

ProcParam find_proc_param(const SolverParam& sp, const std::string& name) {
  for (const ProcParam& p : sp.proc_param)
    if (p.name == name) return p;
  fatal("No parameters specified for `" + name + "' !");
}

/* ------------------------------------------------------------------ Upd */

Upd::~Upd() {
  for (ProcedureBase* p : procs_) delete p;
}

void Upd::init(const SolverParam& sp, Database& db, bool initialized_db) {
  for (const ProcParam& pp : sp.proc_param) {
    ProcedureBase* p = ProcedureFactory::create(pp.name);
    /* gsbn dereferences the NULL of an unknown name; here it is an error */
    if (!p) {
      std::string known;
      for (auto& n : ProcedureFactory::names()) known += " " + n;
      fatal("unknown procedure `" + pp.name + "' (registered:" + known + ")");
    }
    procs_.push_back(p);
    names_.push_back(pp.name);
    if (!initialized_db)
      p->init_new(sp, db);
    else
      p->init_copy(sp, db);
  }
}

void Upd::update(mode_t mode) {
  for (ProcedureBase* p : procs_) {
    if (mode == GPU)
      p->update_gpu();
    else
      p->update_cpu();
  }
}

bool Upd::all_support_runs() const {
  for (ProcedureBase* p : procs_)
    if (!p->supports_runs()) return false;
  return true;
}

int Upd::update_window(int next_tick) {
  RunWindow w;
  w.first = next_tick;
  w.n = INT_MAX;
  for (ProcedureBase* p : procs_) w.n = std::min(w.n, p->run_horizon(next_tick));
  if (w.n < 1) w.n = 1;
  if (w.n == INT_MAX) fatal("no procedure bounds the run window (is ProcExtGen listed?)");
  for (ProcedureBase* p : procs_) p->update_run(w);
  return w.cycle_flag;
}

/* --------------------------------------------------------------- Solver */

namespace {
struct PoolBinding {
  GlobalVar::Pool* old;
  explicit PoolBinding(GlobalVar::Pool* p) : old(GlobalVar::bind(p)) {}
  ~PoolBinding() { GlobalVar::bind(old); }
};

void make_dirs(const std::string& dir) {
  std::string cur;
  for (size_t i = 0; i < dir.size(); i++) {
    cur.push_back(dir[i]);
    if (dir[i] == '/' || i + 1 == dir.size()) {
      if (cur == "/" || cur == "./" || cur == "../") continue;
      if (mkdir(cur.c_str(), 0755) != 0 && errno != EEXIST) fatal("Cannot create directory " + cur);
    }
  }
}
}  // namespace

Solver::Solver(type_t type, const std::string& n_path, const std::string& s_path, mode_t mode) : mode_(mode) {
  PoolBinding bind(&pool_);
  SolverParam sp = read_solver_param(n_path);
  GlobalVar glv;
  std::string log_dir = sp.rec_param.directory;
  if (log_dir.empty()) log_dir = "./";
  if (log_dir.back() != '/') log_dir += "/";
  struct stat info;
  if (!(stat(log_dir.c_str(), &info) == 0 && (info.st_mode & S_IFDIR))) make_dirs(log_dir);
  glv.puts("log-dir", log_dir);
  glv.puti("rank", 0);
  glv.putf("dt", sp.gen_param.dt);
  if (type == NEW_SOLVER) {
    upd_.init(sp, db_, false);
    glv.puti("simstep", 0);
    glv.puti("cycle-flag", 0);
    glv.putf("prn", 0.f);
    glv.putf("old-prn", 0.f);
  } else {
    read_solver_state(s_path, db_);
    float dt = sp.gen_param.dt;
    glv.puti("simstep", int(db_.snapshot_timestamp / dt));
    glv.putf("prn", db_.snapshot_prn);
    glv.putf("old-prn", db_.snapshot_prn);
    glv.puti("cycle-flag", 0);
    upd_.init(sp, db_, true);
  }
}

Solver::~Solver() {}

void Solver::run(bool windows) {
  PoolBinding bind(&pool_);
  GlobalVar glv;
  float dt = 0.f;
  int simstep = 0;
  glv.getf("dt", dt);
  glv.geti("simstep", simstep);
  float start_time = simstep * dt;
  auto t0 = std::chrono::steady_clock::now();
  int f = 0;
  glv.geti("cycle-flag", f);
  /* windows are the device path; mode CPU goes through update_cpu per tick */
  bool use_windows = windows && mode_ == GPU && upd_.all_support_runs();
  while (f >= 0) {
    if (use_windows) {
      int simstep = 0;
      glv.geti("simstep", simstep);
      f = upd_.update_window(simstep + 1);
      windows_++;
      int now = 0;
      glv.geti("simstep", now);
      ticks_ += now - simstep;
    } else {
      upd_.update(mode_);
      ticks_++;
      if (!glv.geti("cycle-flag", f)) fatal("no procedure sets cycle-flag (is ProcExtGen listed?)");
    }
  }
  glv.geti("simstep", simstep);
  float end_time = simstep * dt;
  double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  /* Solver.cpp:86-91 */
  std::cout << "Total time for [" << end_time - start_time << "]: " << std::setprecision(6) << secs << std::endl;
}

}  // namespace gsbn
