/* Host engine around the B200 tick kernels: gsbn's run-time procedure
 * registry, its prototxt/StimRawData formats and its Solver loop, written for
 * this library.
 *
 * Interface kept from gsbn (so procedure code and network files carry over):
 *   - SolverParam and the messages under it: the fields, types, labels and
 *     defaults of src/gsbn/proto/gsbn.proto, read from protobuf text format
 *     (Solver.cpp:12-15) by a parser written here (no libprotobuf);
 *   - GlobalVar with string keys "simstep", "cycle-flag", "prn", "old-prn",
 *     "dt", "wmask-idx", "lginp-idx", "plasticity", "log-dir", "rank"
 *     (GlobalVar.hpp, ProcExtGen.cpp:113-148, Solver.cpp:35-43);
 *   - ProcedureBase with init_new/init_copy/update_cpu/update_gpu, the
 *     ProcedureFactory table filled at static-initialisation time by
 *     REGISTER/REGISTERIMPL, and get_proc_param looking a procedure's
 *     proc_param up by class name (ProcedureFactory.hpp:17-85);
 *   - Upd running the procedures of proc_param in file order, once per tick
 *     (Upd.cpp:12-40), and Solver looping until "cycle-flag" < 0
 *     (Solver.cpp:67-92);
 *   - Parser argi/argf/args lookups on a ProcParam (Parser.cpp).
 *
 * What is new (the B200 part):
 *   - windows: a procedure may declare supports_runs() and then advance a
 *     whole run of ticks in one update_run() call.  Upd asks every procedure
 *     for its horizon (how many ticks from the next one it can take without a
 *     per-tick look), takes the minimum and hands the same RunWindow to each
 *     procedure in file order.  ProcExtGen's horizon is the rest of the
 *     current stimulus segment, so a segment becomes one bcpnn_run call (one
 *     persistent kernel launch) and the spike log of the whole segment comes
 *     back in one copy.  The per-tick update_gpu() path stays for procedures
 *     that need it;
 *   - Database keeps named host vectors (the ones gsbn's host-side procedures
 *     exchange: .lgidx, .wmask, .lginp) plus the device network handle; the
 *     network state itself stays on the device and is read or written by name
 *     through the C ABI (bcpnn_read_state / bcpnn_write_state);
 *   - errors throw gsbn::Fatal (gsbn aborts through CHECK/LOG(FATAL)); the C
 *     entry points and the command line catch it.
 */
#ifndef GSBN_B200_ENGINE_HPP
#define GSBN_B200_ENGINE_HPP

#include <climits>
#include <cstdint>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "bcpnn.h"

namespace gsbn {

struct Fatal : std::runtime_error {
  explicit Fatal(const std::string& m) : std::runtime_error(m) {}
};

/* ---------------------------------------------------------------- schema */

struct ModeParam {
  float begin_time = 0.f, end_time = 0.f;
  uint32_t begin_lgidx_id = 0, begin_lgexp_id = 0, begin_wmask_id = 0;
  uint32_t time_step = 1, lgidx_step = 1, lgexp_step = 1, wmask_step = 1;
  float prn = 1.0f;
  uint32_t plasticity = 1;
};

struct GenParam {
  std::string stim_file;
  float dt = 0.f;
  float eps = 0.001f;
  std::vector<ModeParam> mode_param;
  std::vector<std::string> procedure;
};

struct PopParam {
  uint32_t pop_num = 0, hcu_num = 0, mcu_num = 0, fanout_num = 0;
  float taum = 0.01f, wtagain = 4.f, maxfq = 100.f, igain = 1.f, wgain = 1.f, lgbias = 0.f, snoise = 0.f;
  float adgain = 1.f, taua = 0.05f;
  std::vector<int32_t> position;
  std::vector<uint32_t> shape;
  uint32_t type = 0, rank = 0;
};

struct ProjParam {
  uint32_t src_pop = 0, dest_pop = 0;
  float tauzi = 0.f, tauzj = 0.f, taue = 0.f, taup = 0.f;
  float maxfq = 100.f, bgain = 0.f, wgain = 0.f;
  bool has_tauepsc = false;
  float tauepsc = 0.f;
  float slot_num = 0.f;
  float distance = 0.f;
};

struct NetParam {
  std::vector<PopParam> pop_param;
  std::vector<ProjParam> proj_param;
};

struct RecParam {
  std::string directory = ".";
};

struct ProcParam {
  std::string name;
  std::vector<std::pair<std::string, int32_t>> argi;
  std::vector<std::pair<std::string, float>> argf;
  std::vector<std::pair<std::string, std::string>> args;
};

struct SolverParam {
  GenParam gen_param;
  NetParam net_param;
  RecParam rec_param;
  std::vector<ProcParam> proc_param;
};

/* Protobuf text format -> SolverParam.  Unknown fields, a repeated optional
   field, a missing required field, a value of the wrong kind or out of range
   are errors (thrown as Fatal with file line numbers). */
SolverParam parse_solver_param_text(const std::string& text);
SolverParam read_solver_param(const std::string& path);
/* Canonical one-field-per-line dump (every field with its value, defaults
   included) used to compare parsers. */
std::string dump_solver_param(const SolverParam& sp);

struct StimRawData {
  uint32_t data_rows = 0, data_cols = 0, mask_rows = 0, mask_cols = 0;
  std::vector<uint32_t> data;
  std::vector<float> mask;
};
/* Protobuf wire format (packed or unpacked repeated fields, unknown fields
   skipped by wire type) -> StimRawData; required fields must be present. */
StimRawData decode_stim_raw_data(const std::string& bytes);
StimRawData read_stim_raw_data(const std::string& path);

/* ProcParam argument lookups, as gsbn's Parser (src/gsbn/Parser.cpp:12-43):
   the first entry with a matching key wins. */
class Parser {
 public:
  explicit Parser(const ProcParam& p) : p_(p) {}
  bool argi(const std::string& key, int& val) const;
  bool argf(const std::string& key, float& val) const;
  bool args(const std::string& key, std::string& val) const;

 private:
  ProcParam p_;
};

/* ------------------------------------------------------------ GlobalVar */

/* A string-keyed variable pool.  gsbn keeps one static pool per process; here
   every Solver owns a pool and binds it while it builds and runs its
   procedures, so GlobalVar objects created inside procedures see that
   solver's pool (several solvers may live in one process, one at a time per
   thread). */
class GlobalVar {
 public:
  struct Value {
    bool b = false;
    int i = 0;
    float f = 0.f;
    std::string s;
  };
  using Pool = std::map<std::string, Value>;

  GlobalVar();
  bool getb(const std::string& key, bool& v) const;
  bool geti(const std::string& key, int& v) const;
  bool getf(const std::string& key, float& v) const;
  bool gets(const std::string& key, std::string& v) const;
  bool putb(const std::string& key, bool v);
  bool puti(const std::string& key, int v);
  bool putf(const std::string& key, float v);
  bool puts(const std::string& key, const std::string& v);

  static Pool* bind(Pool* p); /* returns the previous binding */

 private:
  Pool* pool_;
};

/* ------------------------------------------------------------- Database */

template <class T>
struct HostVector {
  std::vector<T> data;
  size_t ld = 0; /* row length (leading dimension), 0 = not a table */
  const T* row(size_t r) const { return data.data() + r * ld; }
};

/* Spike log of the last window, per population: n ticks of `words` 32-bit
   words, bit (i & 31) of word (i >> 5) = MCU i of the population. */
struct SpikeLog {
  int first = 0, n = 0;
  std::vector<int> words;                   /* per population */
  std::vector<std::vector<uint32_t>> bits;  /* per population, n * words */
  std::vector<uint8_t> ss_flags;            /* n * n_projs, bcpnn_get_ss_flags */
  bool tick_has_spike(int pop, int k) const;
};

class Database {
 public:
  ~Database();
  HostVector<int32_t>* create_vector_i32(const std::string& name);
  HostVector<float>* create_vector_f32(const std::string& name);
  HostVector<int32_t>* vector_i32(const std::string& name);
  HostVector<float>* vector_f32(const std::string& name);

  /* the device network, owned by the Database once set (ProcUpdLazy) */
  void set_net(bcpnn_net* net) { net_ = net; }
  bcpnn_net* net() const { return net_; }
  bcpnn_net* require_net(const char* who) const;

  /* procedures that read spikes ask for the log at init; ProcUpdLazy fills
     it after every window */
  void request_spike_log(bool ss_flags = false) {
    want_spike_log_ = true;
    want_ss_flags_ = want_ss_flags_ || ss_flags;
  }
  bool want_spike_log() const { return want_spike_log_; }
  bool want_ss_flags() const { return want_ss_flags_; }
  SpikeLog& spike_log() { return log_; }

  /* named state of the device network, gsbn layout (bcpnn_read_state) */
  std::vector<uint8_t> read_state(const std::string& name, int32_t* type = nullptr);
  void write_state(const std::string& name, const void* data, size_t bytes);

  /* population / projection shapes as the network was built (ProcUpdLazy) */
  std::vector<bcpnn_pop_desc> pops;
  std::vector<bcpnn_proj_desc> projs;
  /* 0: ProcUpdLazy, 1: ProcUpdMulti (the vectors each creates differ) */
  int update_variant = 0;

  /* vectors of a restored snapshot (SolverState), by gsbn name; consumed by
     init_copy */
  struct StateVec {
    int32_t type;
    std::vector<uint8_t> bytes;
  };
  std::map<std::string, StateVec> snapshot;
  float snapshot_timestamp = 0.f, snapshot_prn = 0.f;

 private:
  std::map<std::string, std::unique_ptr<HostVector<int32_t>>> i32_;
  std::map<std::string, std::unique_ptr<HostVector<float>>> f32_;
  bcpnn_net* net_ = nullptr;
  bool want_spike_log_ = false, want_ss_flags_ = false;
  SpikeLog log_;
};

/* ----------------------------------------------------------- procedures */

/* A run of consecutive ticks first .. first+n-1 with one stimulus and
   plasticity.  Filled by the procedure that owns the tick schedule
   (ProcExtGen) and read by the others. */
struct RunWindow {
  int first = 0;
  int n = 0;
  int cycle_flag = 0; /* 1 active, 0 idle, -1 end (gsbn "cycle-flag") */
  float prn = 0.f;
  float old_prn = 0.f; /* "old-prn" at the first tick */
};

class ProcedureBase {
 public:
  ProcedureBase() {}
  virtual ~ProcedureBase() {}
  virtual void init_new(SolverParam solver_param, Database& db) = 0;
  virtual void init_copy(SolverParam solver_param, Database& db) = 0;
  virtual void update_cpu() = 0;
  virtual void update_gpu() = 0;

  /* window interface (optional) */
  virtual bool supports_runs() const { return false; }
  virtual int run_horizon(int first_tick) { (void)first_tick; return INT_MAX; }
  virtual void update_run(RunWindow& w) { (void)w; }

 protected:
  GlobalVar _glv;
};

class ProcedureCreator {
 public:
  explicit ProcedureCreator(const std::string& classname);
  virtual ~ProcedureCreator() {}
  virtual ProcedureBase* create() = 0;
};

template <class T>
class ProcedureCreatorImpl : public ProcedureCreator {
 public:
  explicit ProcedureCreatorImpl(const std::string& classname) : ProcedureCreator(classname) {}
  ProcedureBase* create() override { return new T; }
};

class ProcedureFactory {
 public:
  /* nullptr for an unknown name */
  static ProcedureBase* create(const std::string& classname);
  static void registerit(const std::string& classname, ProcedureCreator* creator);
  static std::vector<std::string> names();

 private:
  static std::map<std::string, ProcedureCreator*>& get_table();
};

ProcParam find_proc_param(const SolverParam& sp, const std::string& name);

#define REGISTER(classname)                                   \
 private:                                                     \
  static const ProcedureCreatorImpl<classname> creator;       \
  static const std::string proc_name();                       \
  static const ProcParam get_proc_param(const SolverParam& sp);

#define REGISTERIMPL(classname)                                                         \
  const ProcedureCreatorImpl<classname> classname::creator(#classname);                 \
  const std::string classname::proc_name() { return #classname; }                       \
  const ProcParam classname::get_proc_param(const SolverParam& sp) {                    \
    return find_proc_param(sp, #classname);                                             \
  }

/* ------------------------------------------------------------ Upd/Solver */

enum mode_t { CPU = 0, GPU = 1 };

class Upd {
 public:
  ~Upd();
  void init(const SolverParam& sp, Database& db, bool initialized_db);
  /* one tick, every procedure in file order (Upd.cpp:28-40) */
  void update(mode_t mode);
  /* one window of ticks; returns the window's cycle flag */
  int update_window(int next_tick);
  bool all_support_runs() const;
  const std::vector<ProcedureBase*>& procedures() const { return procs_; }

 private:
  std::vector<ProcedureBase*> procs_;
  std::vector<std::string> names_;
};

class Solver {
 public:
  enum type_t { NEW_SOLVER, COPY_SOLVER };
  /* n_path: prototxt network description; s_path: SolverState snapshot for
     COPY_SOLVER (Solver.cpp:9-65) */
  Solver(type_t type, const std::string& n_path, const std::string& s_path, mode_t mode = GPU);
  ~Solver();
  /* runs until cycle-flag < 0 (Solver.cpp:67-92); windows when every
     procedure supports them, otherwise tick by tick */
  void run(bool windows = true);
  Database& db() { return db_; }
  GlobalVar::Pool& pool() { return pool_; }
  int ticks_run() const { return ticks_; }
  int windows_run() const { return windows_; }

 private:
  GlobalVar::Pool pool_;
  Database db_;
  Upd upd_;
  mode_t mode_;
  int ticks_ = 0, windows_ = 0;
};

/* SolverState snapshot (gsbn.proto SolverState: timestamp, prn and one
   VectorState per named vector): decode/encode with the wire codec. */
void read_solver_state(const std::string& path, Database& db);
std::string encode_solver_state(float timestamp, float prn, const std::vector<std::pair<std::string, Database::StateVec>>& vecs);

/* status helper for CHECK-style tests */
[[noreturn]] void fatal(const std::string& msg);

}  // namespace gsbn

#endif
