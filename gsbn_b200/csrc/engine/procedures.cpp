/* The procedures of the ProcUpdLazy path, registered under gsbn's class names:
 * ProcExtGen, ProcUpdLazy, ProcExchangeSpike, ProcInitConn, ProcSpkRec,
 * ProcCheck and ProcSnapshot.  Each reads the same prototxt keys and writes the
 * same files as gsbn's procedure of that name (cited per class); each also
 * takes whole windows of ticks (update_run) so that a stimulus segment runs as
 * one bcpnn_run call on the device.
 */
#include <sys/stat.h>

#include <algorithm>
#include <cmath>
#include <cerrno>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <set>
#include <sstream>

#include "bcpnn_numerics.h"
#include "gsbn_engine.hpp"

namespace gsbn {

namespace {

void check_net(bcpnn_net* net, int st, const std::string& what) {
  if (st != BCPNN_OK)
    fatal(what + ": " + bcpnn_status_string(st) + (net ? std::string(" (") + bcpnn_last_error(net) + ")" : ""));
}

std::string proc_dir(const std::string& name) {
  GlobalVar glv;
  std::string log_dir;
  if (!glv.gets("log-dir", log_dir) || log_dir.empty()) fatal(name + ": GlobalVar log-dir is not set");
  std::string dir = log_dir + name;
  struct stat info;
  if (!(stat(dir.c_str(), &info) == 0 && (info.st_mode & S_IFDIR))) {
    if (mkdir(dir.c_str(), 0755) != 0 && errno != EEXIST) fatal("Cannot create directory " + dir);
  }
  return dir;
}

/* stoi-like: leading whitespace, optional sign, digits; trailing text ignored */
int to_int(const std::string& s, const char* what) {
  const char* p = s.c_str();
  char* end = nullptr;
  errno = 0;
  long v = std::strtol(p, &end, 10);
  if (end == p || errno == ERANGE || v < INT32_MIN || v > INT32_MAX) fatal(std::string(what) + ": bad integer \"" + s + "\"");
  return (int)v;
}

std::vector<std::string> split_commas(const std::string& line) {
  /* gsbn splits with getline(ss, substr, ',') while ss.good() */
  std::vector<std::string> out;
  std::stringstream ss(line);
  while (ss.good()) {
    std::string sub;
    std::getline(ss, sub, ',');
    out.push_back(sub);
  }
  return out;
}

/* expanded segment list of the mode_params (ProcExtGen.cpp:16-55 with
   clamp_end; ProcCheck.cpp:29-66 without, prn != 0 skipped) */
struct Mode {
  int begin_step, end_step, lgidx_id, lgexp_id, wmask_id;
  float prn;
  int plasticity;
};

std::vector<Mode> expand_modes(const GenParam& g, bool clamp_end, bool only_prn0) {
  std::vector<Mode> out;
  float dt = g.dt;
  for (const ModeParam& mp : g.mode_param) {
    int begin_step = int(mp.begin_time / dt);
    int end_step = int(mp.end_time / dt);
    if (end_step < begin_step) fatal("Time range is wrong, abort!");
    if (only_prn0 && mp.prn != 0.0f) continue;
    int lg = (int)mp.begin_lgidx_id, ex = (int)mp.begin_lgexp_id, wm = (int)mp.begin_wmask_id;
    if (mp.time_step == 0 && begin_step < end_step) fatal("mode_param time_step is 0");
    while (begin_step < end_step) {
      Mode m;
      m.begin_step = begin_step;
      m.end_step = begin_step + (int)mp.time_step;
      if (clamp_end && m.end_step >= end_step) m.end_step = end_step;
      m.lgidx_id = lg;
      m.lgexp_id = ex;
      m.wmask_id = wm;
      lg += (int)mp.lgidx_step;
      ex += (int)mp.lgexp_step;
      wm += (int)mp.wmask_step;
      m.prn = mp.prn;
      m.plasticity = (int)mp.plasticity;
      out.push_back(m);
      begin_step = clamp_end ? m.end_step : begin_step + (int)mp.time_step;
    }
  }
  return out;
}

struct PopShape {
  int id, hcu, mcu, hcu_start, mcu_start;
  float maxfq;
};

std::vector<PopShape> pop_shapes(const NetParam& net) {
  std::vector<PopShape> out;
  int h0 = 0, m0 = 0;
  for (const PopParam& pp : net.pop_param)
    for (uint32_t k = 0; k < pp.pop_num; k++) {
      PopShape s{(int)out.size(), (int)pp.hcu_num, (int)pp.mcu_num, h0, m0, pp.maxfq};
      h0 += s.hcu;
      m0 += s.hcu * s.mcu;
      out.push_back(s);
    }
  return out;
}

/* projections whose populations exist, in file order (ProcUpdLazy.cpp:33-45) */
std::vector<const ProjParam*> live_projs(const NetParam& net, int n_pops) {
  std::vector<const ProjParam*> out;
  for (const ProjParam& q : net.proj_param)
    if ((int)q.src_pop < n_pops && (int)q.dest_pop < n_pops) out.push_back(&q);
  return out;
}

bool has_proc(const SolverParam& sp, const char* name) {
  for (const ProcParam& p : sp.proc_param)
    if (p.name == name) return true;
  return false;
}

}  // namespace

/* =================================================================
 * ProcExtGen — stimulus schedule (src/gsbn/procedures/ProcExtGen.cpp:8-153)
 * ================================================================= */
class ProcExtGen : public ProcedureBase {
  REGISTER(ProcExtGen)
 public:
  void init_new(SolverParam sp, Database& db) override {
    _eps = sp.gen_param.eps;
    _glv.putf("dt", sp.gen_param.dt);
    _modes = expand_modes(sp.gen_param, true, false);
    _lgidx = db.create_vector_i32(".lgidx");
    _wmask = db.create_vector_f32(".wmask");
    _lginp = db.create_vector_f32(".lginp");
    if (!_lgidx || !_wmask || !_lginp) fatal("ProcExtGen: stimulus vectors already exist (listed twice?)");
    StimRawData s = read_stim_raw_data(sp.gen_param.stim_file);
    _lgidx->ld = s.data_cols;
    _wmask->ld = s.mask_cols;
    _lgidx->data.assign(s.data.begin(), s.data.end()); /* uint32 -> int32 as gsbn's vector<int> */
    _wmask->data = s.mask;
    /* every population instance (pop_num copies of a PopParam): gsbn counts
       each PopParam once here (ProcExtGen.cpp:91-101), which leaves .lginp
       short when pop_num > 1 and the population update reading past it */
    int mcu_num = 0;
    for (const PopShape& p : pop_shapes(sp.net_param)) {
      mcu_num += p.hcu * p.mcu;
      for (int j = 0; j < p.hcu; j++) _mcu_in_hcu.push_back(p.mcu);
    }
    _lginp->data.assign(mcu_num, 0.f);
    _lginp->ld = mcu_num;
    _lg_hit = bx_extgen_logf(1.0f + _eps);
    _lg_miss = bx_extgen_logf(0.0f + _eps);
    /* every row read later must be wide enough (gsbn reads past the row) */
    for (const Mode& m : _modes) {
      if (m.lgidx_id >= (int)s.data_rows) fatal("ProcExtGen: lgidx row " + std::to_string(m.lgidx_id) + " not in stimulus file");
      if (m.wmask_id >= (int)s.mask_rows) fatal("ProcExtGen: wmask row " + std::to_string(m.wmask_id) + " not in stimulus file");
    }
    if ((int)s.data_cols < (int)_mcu_in_hcu.size()) fatal("ProcExtGen: stimulus rows narrower than the HCU count");
    _cursor = 0;
    _old_lgidx_id = -1;
  }
  void init_copy(SolverParam sp, Database& db) override { init_new(sp, db); }

  void update_cpu() override { tick(); }
  void update_gpu() override { tick(); }

  bool supports_runs() const override { return true; }

  int run_horizon(int t) override {
    for (size_t c = _cursor; c < _modes.size(); c++) {
      const Mode& m = _modes[c];
      if (t > m.begin_step && t <= m.end_step) return m.end_step - t + 1;
      if (t <= m.begin_step) return m.begin_step - t + 1;
    }
    return 1;
  }

  void update_run(RunWindow& w) override {
    float prn_before = 0.f;
    _glv.getf("prn", prn_before);
    tick();
    int cf = 0, simstep = 0;
    _glv.geti("cycle-flag", cf);
    _glv.geti("simstep", simstep);
    if (simstep != w.first) fatal("ProcExtGen: window does not start at the next tick");
    w.cycle_flag = cf;
    _glv.getf("prn", w.prn);
    w.old_prn = cf == 1 ? prn_before : w.prn;
    if (cf < 0) w.n = 1;
    if (w.n > 1) {
      /* the remaining ticks repeat the first one's state; only simstep and
         old-prn move (ProcExtGen.cpp:113-148 applied n-1 more times) */
      _glv.puti("simstep", w.first + w.n - 1);
      if (cf == 1) _glv.putf("old-prn", w.prn);
    }
  }

 private:
  void tick() {
    int t = 0;
    if (!_glv.geti("simstep", t)) fatal("ProcExtGen: simstep not set");
    t++;
    _glv.puti("simstep", t);
    for (; _cursor < _modes.size(); _cursor++) {
      const Mode& m = _modes[_cursor];
      if (t > m.begin_step && t <= m.end_step) {
        float old_prn = 0.f;
        _glv.getf("prn", old_prn);
        _glv.putf("old-prn", old_prn);
        _glv.putf("prn", m.prn);
        _glv.puti("wmask-idx", m.wmask_id);
        _glv.putb("plasticity", m.plasticity != 0);
        _glv.puti("lginp-idx", 0);
        _glv.puti("lgidx-row", m.lgidx_id); /* row of .lgidx that .lginp holds */
        _glv.puti("cycle-flag", 1);
        if (_old_lgidx_id != m.lgidx_id) {
          _old_lgidx_id = m.lgidx_id;
          const int32_t* row = _lgidx->row((size_t)m.lgidx_id);
          float* out = _lginp->data.data();
          for (size_t i = 0; i < _mcu_in_hcu.size(); i++)
            for (int j = 0; j < _mcu_in_hcu[i]; j++) *out++ = (row[i] == j) ? _lg_hit : _lg_miss;
        }
        return;
      } else if (t <= m.begin_step) {
        _glv.puti("cycle-flag", 0);
        return;
      }
    }
    _glv.puti("cycle-flag", -1);
  }

  float _eps = 0.f, _lg_hit = 0.f, _lg_miss = 0.f;
  std::vector<Mode> _modes;
  std::vector<int> _mcu_in_hcu;
  size_t _cursor = 0;
  int _old_lgidx_id = -1;
  HostVector<int32_t>* _lgidx = nullptr;
  HostVector<float>* _wmask = nullptr;
  HostVector<float>* _lginp = nullptr;
};
REGISTERIMPL(ProcExtGen)

/* =================================================================
 * ProcUpdLazy — the B200 network (src/gsbn/procedures/ProcUpdLazy.cpp:8-180,
 * ProcUpdLazy/Pop.cpp, ProcUpdLazy/Proj.cpp)
 * ================================================================= */
class ProcUpdLazy : public ProcedureBase {
  REGISTER(ProcUpdLazy)
 public:
  ~ProcUpdLazy() override {}

  void init_new(SolverParam sp, Database& db) override { build(sp, db, false, get_proc_param(sp), 0); }
  void init_copy(SolverParam sp, Database& db) override { build(sp, db, true, get_proc_param(sp), 0); }

  void update_cpu() override {
    fatal("ProcUpdLazy has no CPU path in this build: run with mode GPU");
  }

  void update_gpu() override {
    RunWindow w;
    _glv.geti("cycle-flag", w.cycle_flag);
    _glv.geti("simstep", w.first);
    _glv.getf("prn", w.prn);
    _glv.getf("old-prn", w.old_prn);
    w.n = 1;
    update_run(w);
  }

  bool supports_runs() const override { return true; }
  int run_horizon(int) override { return INT_MAX; }

  void update_run(RunWindow& w) override {
    if (w.cycle_flag != 1) return;
    set_stimulus();
    SpikeLog& log = _db->spike_log();
    bool want = _db->want_spike_log(), want_ss = _db->want_ss_flags();
    if (want) {
      log.first = w.first;
      log.n = 0;
      log.words = _words;
      log.bits.assign(_words.size(), {});
      for (size_t p = 0; p < _words.size(); p++) log.bits[p].reserve((size_t)w.n * _words[p]);
      log.ss_flags.clear();
    }
    for (int done = 0; done < w.n;) {
      int n = std::min(w.n - done, _max_ticks);
      float old = done == 0 ? w.old_prn : w.prn;
      check_net(_net, bcpnn_run(_net, w.first + done, n, w.prn, old), "bcpnn_run");
      if (want) {
        for (size_t p = 0; p < _words.size(); p++) {
          size_t at = log.bits[p].size();
          log.bits[p].resize(at + (size_t)n * _words[p]);
          check_net(_net, bcpnn_get_spike_log(_net, (int32_t)p, log.bits[p].data() + at, (size_t)n * _words[p]),
                    "bcpnn_get_spike_log");
        }
        if (want_ss && _n_projs) {
          size_t at = log.ss_flags.size();
          log.ss_flags.resize(at + (size_t)n * _n_projs);
          check_net(_net, bcpnn_get_ss_flags(_net, log.ss_flags.data() + at, (size_t)n * _n_projs), "bcpnn_get_ss_flags");
        }
        log.n += n;
      }
      done += n;
    }
  }

 protected:
  /* variant 0: ProcUpdLazy; 1: ProcUpdMulti (its ProcParam, its spike ring) */
  void build(const SolverParam& sp, Database& db, bool copy, const ProcParam& pp, int variant) {
    _db = &db;
    Parser par(pp);
    const NetParam& net = sp.net_param;
    for (const PopParam& p : net.pop_param)
      for (uint32_t k = 0; k < p.pop_num; k++) {
        bcpnn_pop_desc d;
        std::memset(&d, 0, sizeof d);
        d.hcu_num = (int32_t)p.hcu_num;
        d.mcu_num = (int32_t)p.mcu_num;
        d.taum = p.taum;
        d.wtagain = p.wtagain;
        d.maxfq = p.maxfq;
        d.igain = p.igain;
        d.wgain = p.wgain;
        d.lgbias = p.lgbias;
        d.snoise = p.snoise;
        d.taua = p.taua;
        d.adgain = p.adgain;
        db.pops.push_back(d);
      }
    for (const ProjParam* q : live_projs(net, (int)db.pops.size())) {
      bcpnn_proj_desc d;
      std::memset(&d, 0, sizeof d);
      d.src_pop = (int32_t)q->src_pop;
      d.dest_pop = (int32_t)q->dest_pop;
      d.tauzi = q->tauzi;
      d.tauzj = q->tauzj;
      d.taue = q->taue;
      d.taup = q->taup;
      d.maxfq = q->maxfq;
      d.bgain = q->bgain;
      d.wgain = q->wgain;
      d.tauepsc = q->has_tauepsc ? q->tauepsc : 0.f;
      d.slot_num = q->slot_num;
      db.projs.push_back(d);
    }
    int seed = 0, device = 0;
    float noise = 0.f;
    par.argi("seed", seed);
    par.argi("device", device);
    par.argf("poisson-noise-hz", noise);
    _max_ticks = 1024;
    par.argi("max-ticks-per-run", _max_ticks);
    if (_max_ticks < 1) fatal("ProcUpdLazy: max-ticks-per-run must be >= 1");
    bcpnn_net_desc desc;
    std::memset(&desc, 0, sizeof desc);
    desc.n_pops = (int32_t)db.pops.size();
    desc.pops = db.pops.data();
    desc.n_projs = (int32_t)db.projs.size();
    desc.projs = db.projs.data();
    desc.dt = sp.gen_param.dt;
    desc.seed = (uint32_t)seed;
    desc.poisson_noise_hz = noise;
    desc.exchange_spikes = has_proc(sp, "ProcExchangeSpike") ? 1 : 0;
    desc.device = device;
    desc.max_ticks_per_run = _max_ticks;
    desc.update_variant = variant;
    db.update_variant = variant;
    if (variant == 1) {
      int ring = 1; /* ProcUpdMulti/Pop.cpp:31-36 */
      if (par.argi("spike buffer size", ring) && ring <= 0) fatal("ProcUpdMulti: spike buffer size must be > 0");
      desc.spike_buffer_size = ring;
    }
    bcpnn_net* n = nullptr;
    int st = bcpnn_net_create(&desc, &n);
    if (st != BCPNN_OK) fatal(std::string("ProcUpdLazy: bcpnn_net_create: ") + bcpnn_status_string(st));
    _net = n;
    db.set_net(n);
    _n_projs = (int)db.projs.size();
    for (size_t p = 0; p < db.pops.size(); p++) {
      int32_t w = 0;
      check_net(_net, bcpnn_spike_log_words(_net, (int32_t)p, &w), "bcpnn_spike_log_words");
      _words.push_back(w);
    }
    _eps = sp.gen_param.eps;
    _total_hcu = 0;
    for (auto& d : db.pops) _total_hcu += d.hcu_num;

    std::string ext;
    if (par.args("external spike", ext)) load_ext_spikes(ext);
    if (copy) restore(db);
  }

  /* ProcUpdLazy/Pop.cpp:67-110: "tick,pop,idx,idx,..." lines; a later line
     for the same tick replaces an earlier one */
  void load_ext_spikes(const std::string& path) {
    std::ifstream f(path);
    if (!f.is_open()) fatal("Unable to open file to load external spikes: " + path);
    std::vector<std::map<int, std::vector<int>>> table(_db->pops.size());
    std::string line;
    while (std::getline(f, line)) {
      std::vector<std::string> v = split_commas(line);
      if (v.size() <= 2) continue;
      int tick = to_int(v[0], "external spike"), pop = to_int(v[1], "external spike");
      if (tick < 0 || pop < 0 || pop >= (int)table.size()) continue;
      std::vector<int> idx;
      for (size_t i = 2; i < v.size(); i++) idx.push_back(to_int(v[i], "external spike"));
      table[pop][tick] = idx;
    }
    for (size_t p = 0; p < table.size(); p++) {
      std::vector<int32_t> ticks, offsets{0}, idx;
      for (auto& kv : table[p]) {
        ticks.push_back(kv.first);
        idx.insert(idx.end(), kv.second.begin(), kv.second.end());
        offsets.push_back((int32_t)idx.size());
      }
      /* every population of a file-driven run is overridden, listed or not */
      check_net(_net, bcpnn_set_ext_spikes(_net, (int32_t)p, (int32_t)ticks.size(), ticks.data(), offsets.data(),
                                           idx.empty() ? nullptr : idx.data()),
                "bcpnn_set_ext_spikes");
    }
  }

  /* SolverState vectors -> device (ProcUpdLazy/Pop.cpp, Proj.cpp init_copy) */
  void restore(Database& db) {
    int written = 0;
    for (auto& kv : db.snapshot) {
      int32_t type = 0;
      size_t count = 0;
      if (bcpnn_state_info(_net, kv.first.c_str(), &type, &count) != BCPNN_OK) continue;
      if (type != kv.second.type) fatal("snapshot vector " + kv.first + " has the wrong type");
      db.write_state(kv.first, kv.second.bytes.data(), kv.second.bytes.size());
      written++;
    }
    if (!written) fatal("snapshot holds no vector of this network");
  }

  void set_stimulus() {
    int wmask_idx = 0, lgidx_row = -1;
    _glv.geti("wmask-idx", wmask_idx);
    bool by_row = _glv.geti("lgidx-row", lgidx_row) && lgidx_row >= 0;
    HostVector<int32_t>* lgidx = _db->vector_i32(".lgidx");
    HostVector<float>* wmask = _db->vector_f32(".wmask");
    if (!wmask) fatal("ProcUpdLazy: no .wmask vector (list ProcExtGen first)");
    if (wmask_idx < 0 || (size_t)(wmask_idx + 1) * wmask->ld > wmask->data.size()) fatal("ProcUpdLazy: wmask-idx out of range");
    if (by_row && lgidx) {
      if (!_uploaded) {
        int32_t rows = (int32_t)(lgidx->data.size() / std::max<size_t>(1, lgidx->ld));
        int32_t wrows = (int32_t)(wmask->data.size() / std::max<size_t>(1, wmask->ld));
        if ((int)lgidx->ld < _total_hcu || (int)wmask->ld < _total_hcu)
          fatal("ProcUpdLazy: stimulus rows narrower than the HCU count");
        /* tables keep total-HCU columns: re-pack if the file rows are wider */
        std::vector<int32_t> lg((size_t)rows * _total_hcu);
        std::vector<float> wm((size_t)wrows * _total_hcu);
        for (int32_t r = 0; r < rows; r++)
          std::copy(lgidx->row(r), lgidx->row(r) + _total_hcu, lg.begin() + (size_t)r * _total_hcu);
        for (int32_t r = 0; r < wrows; r++)
          std::copy(wmask->row(r), wmask->row(r) + _total_hcu, wm.begin() + (size_t)r * _total_hcu);
        check_net(_net, bcpnn_upload_stimuli_idx(_net, rows, lg.data(), _eps, wrows, wm.data()), "bcpnn_upload_stimuli_idx");
        _uploaded = true;
      }
      if (lgidx_row != _cur_lg || wmask_idx != _cur_wm) {
        check_net(_net, bcpnn_use_stimulus(_net, lgidx_row, wmask_idx), "bcpnn_use_stimulus");
        _cur_lg = lgidx_row;
        _cur_wm = wmask_idx;
      }
      return;
    }
    HostVector<float>* lginp = _db->vector_f32(".lginp");
    if (!lginp) fatal("ProcUpdLazy: no .lginp vector (list ProcExtGen first)");
    check_net(_net, bcpnn_set_stimulus(_net, lginp->data.data(), lginp->data.size(), wmask->row(wmask_idx), (size_t)_total_hcu),
              "bcpnn_set_stimulus");
    _cur_lg = _cur_wm = -1;
  }

  Database* _db = nullptr;
  bcpnn_net* _net = nullptr; /* owned by the Database */
  std::vector<int32_t> _words;
  int _n_projs = 0, _max_ticks = 1024, _total_hcu = 0;
  float _eps = 0.f;
  bool _uploaded = false;
  int _cur_lg = -1, _cur_wm = -1;
};
REGISTERIMPL(ProcUpdLazy)

/* =================================================================
 * ProcUpdMulti (src/gsbn/procedures/ProcUpdMulti.cpp:8-180): the row-only
 * update with a ring of postsynaptic spikes and an adaptation current, on
 * the same device network (bcpnn_net_desc.update_variant = 1, per-tick
 * launches).  Keys: argi "spike buffer size" (default 1) and ProcUpdLazy's
 * "seed", "device", "max-ticks-per-run", "external spike".
 * ================================================================= */
class ProcUpdMulti : public ProcUpdLazy {
  REGISTER(ProcUpdMulti)
 public:
  void init_new(SolverParam sp, Database& db) override { build(sp, db, false, get_proc_param(sp), 1); }
  void init_copy(SolverParam sp, Database& db) override { build(sp, db, true, get_proc_param(sp), 1); }
  void update_cpu() override { fatal("ProcUpdMulti has no CPU path in this build: run with mode GPU"); }
};
REGISTERIMPL(ProcUpdMulti)

/* =================================================================
 * ProcExchangeSpike (src/gsbn/procedures/ProcExchangeSpike.cpp:94-139):
 * si_<proj> <- spike_<src_pop> after every tick.  Fused into the tick kernel
 * (the network is built with exchange_spikes when this procedure is listed),
 * so the procedure itself only checks the set-up.
 * ================================================================= */
class ProcExchangeSpike : public ProcedureBase {
  REGISTER(ProcExchangeSpike)
 public:
  void init_new(SolverParam sp, Database&) override {
    get_proc_param(sp);
    if (!has_proc(sp, "ProcUpdLazy") && !has_proc(sp, "ProcUpdMulti"))
      fatal("ProcExchangeSpike needs ProcUpdLazy or ProcUpdMulti");
  }
  void init_copy(SolverParam sp, Database& db) override { init_new(sp, db); }
  void update_cpu() override {}
  void update_gpu() override {}
  bool supports_runs() const override { return true; }
};
REGISTERIMPL(ProcExchangeSpike)

/* =================================================================
 * ProcInitConn (src/gsbn/procedures/ProcInitConn.cpp:8-103): connection map
 * "proj,dest_hcu,src_mcu,delay,src_mcu,delay,...", each pair into the first
 * empty slot (ii < 0) of the destination HCU, dropped when none is left.
 * ================================================================= */
class ProcInitConn : public ProcedureBase {
  REGISTER(ProcInitConn)
 public:
  void init_new(SolverParam sp, Database& db) override { load(sp, db, false); }
  void init_copy(SolverParam sp, Database& db) override { load(sp, db, true); }
  void update_cpu() override {}
  void update_gpu() override {}
  bool supports_runs() const override { return true; }

 private:
  void load(const SolverParam& sp, Database& db, bool keep_existing) {
    Parser par(get_proc_param(sp));
    std::string path;
    if (!par.args("conn-map-file", path)) fatal("Connection map is not specified! Abort");
    bcpnn_net* net = db.require_net("ProcInitConn");
    size_t n_projs = db.projs.size();
    std::vector<std::vector<int32_t>> ii(n_projs), di(n_projs);
    std::vector<std::vector<int32_t>> fill(n_projs);
    std::vector<int> C(n_projs), H(n_projs);
    for (size_t k = 0; k < n_projs; k++) {
      const bcpnn_proj_desc& q = db.projs[k];
      const bcpnn_pop_desc& s = db.pops[q.src_pop];
      H[k] = db.pops[q.dest_pop].hcu_num;
      C[k] = (int)std::min<long long>((long long)s.hcu_num * s.mcu_num, (long long)q.slot_num); /* Proj.cpp:22-26 */
      if (keep_existing) {
        auto a = db.read_state("ii_" + std::to_string(k));
        auto b = db.read_state("di_" + std::to_string(k));
        ii[k].resize(a.size() / 4);
        di[k].resize(b.size() / 4);
        std::memcpy(ii[k].data(), a.data(), a.size());
        std::memcpy(di[k].data(), b.data(), b.size());
      } else {
        ii[k].assign((size_t)H[k] * C[k], -1);
        di[k].assign((size_t)H[k] * C[k], 0);
      }
      fill[k].assign(H[k], 0);
    }
    std::ifstream f(path);
    if (f.is_open()) { /* gsbn silently skips a missing file */
      std::string line;
      while (std::getline(f, line)) {
        std::vector<std::string> v = split_commas(line);
        if (v.size() <= 2) continue;
        int prj = to_int(v[0], "conn-map"), hcu = to_int(v[1], "conn-map");
        if (prj < 0 || prj >= (int)n_projs) fatal("conn-map: projection " + std::to_string(prj) + " does not exist");
        if (hcu < 0 || hcu >= H[prj]) fatal("conn-map: HCU " + std::to_string(hcu) + " out of range");
        if ((v.size() - 2) % 2) fatal("conn-map: odd number of values after proj,hcu: " + line);
        int32_t* rii = ii[prj].data() + (size_t)hcu * C[prj];
        int32_t* rdi = di[prj].data() + (size_t)hcu * C[prj];
        int32_t& ptr = fill[prj][hcu];
        for (size_t i = 2; i + 1 < v.size(); i += 2) {
          int src = to_int(v[i], "conn-map"), delay = to_int(v[i + 1], "conn-map");
          /* first slot with ii < 0: slots only turn non-negative, so a running
             pointer finds it */
          while (ptr < C[prj] && rii[ptr] >= 0) ptr++;
          if (ptr < C[prj]) {
            rii[ptr] = src < 0 ? -1 : src; /* any negative source is an empty slot */
            rdi[ptr] = delay;
          }
        }
      }
    }
    for (size_t k = 0; k < n_projs; k++)
      check_net(net, bcpnn_set_conn(net, (int32_t)k, ii[k].data(), di[k].data(), ii[k].size()), "bcpnn_set_conn");
  }
};
REGISTERIMPL(ProcInitConn)

/* =================================================================
 * ProcSpkRec (src/gsbn/procedures/ProcSpkRec.cpp:10-206, ProcSpkRec/Pop.cpp:30-52,
 * ProcSpkRec/Prj.cpp:95-138): spk_pop_<pop>.csv ("H,M,dt,maxfq" header, then
 * "t,idx,idx,..." for ticks with spikes), ssi_pop_/ssj_pop_<proj>.csv
 * ("t,flag" per recorded tick).
 * ================================================================= */
class ProcSpkRec : public ProcedureBase {
  REGISTER(ProcSpkRec)
 public:
  void init_new(SolverParam sp, Database& db) override {
    _db = &db;
    _dir = proc_dir("ProcSpkRec");
    Parser par(get_proc_param(sp));
    if (!par.argi("offset", _offset))
      _offset = 0;
    else if (_offset < 0)
      fatal("ProcSpkRec: offset must be >= 0");
    if (!par.argi("period", _period))
      _period = 1;
    else if (_period <= 0)
      fatal("ProcSpkRec: period must be > 0");
    float dt = sp.gen_param.dt;
    _pops = pop_shapes(sp.net_param);
    _n_projs = (int)live_projs(sp.net_param, (int)_pops.size()).size();
    /* gsbn lists every proj_param here, live or not (ProcSpkRec.cpp:79-89) */
    int n_files = (int)sp.net_param.proj_param.size();
    for (const PopShape& p : _pops) {
      std::ofstream o(_dir + "/spk_pop_" + std::to_string(p.id) + ".csv", std::ios::out | std::ios::trunc);
      o << p.hcu << "," << p.mcu << "," << dt << "," << p.maxfq << std::endl;
    }
    for (int k = 0; k < n_files; k++) {
      std::ofstream(_dir + "/ssi_pop_" + std::to_string(k) + ".csv", std::ios::out | std::ios::trunc);
      std::ofstream(_dir + "/ssj_pop_" + std::to_string(k) + ".csv", std::ios::out | std::ios::trunc);
    }
    _n_files = n_files;
    db.request_spike_log(true);
  }
  void init_copy(SolverParam sp, Database& db) override { init_new(sp, db); }
  void update_cpu() override { update_gpu(); }
  void update_gpu() override {
    RunWindow w;
    _glv.geti("cycle-flag", w.cycle_flag);
    _glv.geti("simstep", w.first);
    w.n = 1;
    update_run(w);
  }
  bool supports_runs() const override { return true; }

  void update_run(RunWindow& w) override {
    if (w.cycle_flag != 1) return;
    const SpikeLog& log = _db->spike_log();
    if (log.first != w.first || log.n != w.n) fatal("ProcSpkRec: spike log does not cover this window (list ProcUpdLazy first)");
    std::vector<std::string> spk(_pops.size()), ssi(_n_files), ssj(_n_files);
    for (int k = 0; k < w.n; k++) {
      int t = w.first + k;
      if (t < 0) fatal("ProcSpkRec: negative simstep");
      if (t < _offset || t % _period != 0) continue;
      for (size_t p = 0; p < _pops.size(); p++) {
        const uint32_t* row = log.bits[p].data() + (size_t)k * log.words[p];
        bool first = true;
        int n = _pops[p].hcu * _pops[p].mcu;
        for (int wd = 0; wd < log.words[p]; wd++) {
          uint32_t b = row[wd];
          while (b) {
            int i = wd * 32 + __builtin_ctz(b);
            b &= b - 1;
            if (i >= n) break;
            if (first) {
              spk[p] += std::to_string(t);
              first = false;
            }
            spk[p] += "," + std::to_string(i);
          }
        }
        if (!first) spk[p] += "\n";
      }
      for (int q = 0; q < _n_files; q++) {
        uint8_t fl = (q < _n_projs && !log.ss_flags.empty()) ? log.ss_flags[(size_t)k * _n_projs + q] : 0;
        ssj[q] += std::to_string(t) + "," + ((fl & 2) ? "1" : "0") + "\n";
        ssi[q] += std::to_string(t) + "," + ((fl & 1) ? "1" : "0") + "\n";
      }
    }
    for (size_t p = 0; p < _pops.size(); p++)
      if (!spk[p].empty()) append(_dir + "/spk_pop_" + std::to_string(_pops[p].id) + ".csv", spk[p]);
    for (int q = 0; q < _n_files; q++) {
      if (!ssj[q].empty()) append(_dir + "/ssj_pop_" + std::to_string(q) + ".csv", ssj[q]);
      if (!ssi[q].empty()) append(_dir + "/ssi_pop_" + std::to_string(q) + ".csv", ssi[q]);
    }
  }

 private:
  static void append(const std::string& path, const std::string& text) {
    std::ofstream o(path, std::ios::out | std::ios::app);
    o << text;
    if (!o) fatal("cannot write " + path);
  }
  Database* _db = nullptr;
  std::string _dir;
  int _offset = 0, _period = 1, _n_projs = 0, _n_files = 0;
  std::vector<PopShape> _pops;
};
REGISTERIMPL(ProcSpkRec)

/* =================================================================
 * ProcCheck (src/gsbn/procedures/ProcCheck.cpp:8-237, ProcCheck/Pop.cpp:6-60):
 * per recall segment (prn 0) count the spikes of every MCU, take the
 * most-spiking MCU of each HCU and compare with the segment's expected row of
 * .lgidx; write check_result.txt and the final "correct pattern" line.
 * ================================================================= */
class ProcCheck : public ProcedureBase {
  REGISTER(ProcCheck)
 public:
  void init_new(SolverParam sp, Database& db) override {
    _db = &db;
    _logfile = proc_dir("ProcCheck") + "/check_result.txt";
    _modes = expand_modes(sp.gen_param, false, true);
    _lgidx = db.vector_i32(".lgidx");
    if (!_lgidx || !db.vector_f32(".lginp") || !db.vector_f32(".wmask"))
      fatal("ProcCheck needs the stimulus vectors of ProcExtGen: list ProcExtGen first");
    _pops = pop_shapes(sp.net_param);
    _total_hcu = 0;
    for (const PopShape& p : _pops) {
      _counter.emplace_back((size_t)p.hcu * p.mcu, 0);
      _total_hcu += p.hcu;
    }
    for (const Mode& m : _modes)
      if (m.lgexp_id >= (int)(_lgidx->data.size() / std::max<size_t>(1, _lgidx->ld)))
        fatal("ProcCheck: lgexp row " + std::to_string(m.lgexp_id) + " not in stimulus file");
    if ((int)_lgidx->ld < _total_hcu) fatal("ProcCheck: stimulus rows narrower than the HCU count");
    _shared_idx.assign(_total_hcu, 0);
    _shared_cnt.assign(_total_hcu, 0);
    Parser par(get_proc_param(sp));
    if (!par.argi("threashold", _threshold)) _threshold = 0;
    std::ofstream o(_logfile, std::ios::out | std::ios::trunc);
    o << "result | reference pattern | recorded pattern | recorded pattern spike count" << std::endl;
    db.request_spike_log();
    _glv.puti("check-correct", 0);
    _glv.puti("check-patterns", 0);
  }
  void init_copy(SolverParam sp, Database& db) override { init_new(sp, db); }
  void update_cpu() override { update_gpu(); }
  void update_gpu() override {
    RunWindow w;
    _glv.geti("cycle-flag", w.cycle_flag);
    _glv.geti("simstep", w.first);
    w.n = 1;
    update_run(w);
  }
  bool supports_runs() const override { return true; }

  void update_run(RunWindow& w) override {
    if (w.cycle_flag == 0) return;
    if (w.cycle_flag < 0) {
      double pct = _correct * 100.0 / float(_patterns);
      std::cout << "correct pattern: " << _correct << "/" << _patterns << "(" << pct << "%)" << std::endl;
      std::ofstream o(_logfile, std::ios::out | std::ios::app);
      o << "correct pattern: " << _correct << "/" << _patterns << "(" << pct << "%)" << std::endl;
      return;
    }
    const SpikeLog& log = _db->spike_log();
    if (log.first != w.first || log.n != w.n) fatal("ProcCheck: spike log does not cover this window (list ProcUpdLazy first)");
    for (int k = 0; k < w.n; k++) tick(w.first + k, log, k);
  }

  int correct() const { return _correct; }
  int patterns() const { return _patterns; }

 private:
  void tick(int t, const SpikeLog& log, int k) {
    if (_cursor >= _modes.size()) return; /* gsbn reads past the list here */
    const Mode& m = _modes[_cursor];
    if (t <= m.begin_step) return;
    if (t < m.end_step) {
      for (size_t p = 0; p < _pops.size(); p++) {
        const uint32_t* row = log.bits[p].data() + (size_t)k * log.words[p];
        int n = _pops[p].hcu * _pops[p].mcu;
        for (int wd = 0; wd < log.words[p]; wd++) {
          uint32_t b = row[wd];
          while (b) {
            int i = wd * 32 + __builtin_ctz(b);
            b &= b - 1;
            if (i < n) _counter[p][i]++;
          }
        }
      }
      _updated = true;
      return;
    }
    if (!_updated) {
      while (_cursor < _modes.size() && t >= _modes[_cursor].end_step) _cursor++;
      return;
    }
    int h = 0;
    for (size_t p = 0; p < _pops.size(); p++) {
      for (int i = 0; i < _pops[p].hcu; i++) {
        int max_idx = -1, max_cnt = 0;
        for (int j = 0; j < _pops[p].mcu; j++) {
          int& c = _counter[p][(size_t)i * _pops[p].mcu + j];
          if (c > max_cnt) {
            max_idx = j;
            max_cnt = c;
          }
          c = 0;
        }
        _shared_idx[h + i] = max_idx;
        _shared_cnt[h + i] = max_cnt;
      }
      h += _pops[p].hcu;
    }
    const int32_t* exp = _lgidx->row((size_t)m.lgexp_id);
    bool flag = true;
    for (int i = 0; i < _total_hcu; i++) {
      if (((_shared_cnt[i] < _threshold || _shared_idx[i] != exp[i]) && exp[i] >= 0) ||
          (_shared_cnt[i] > _threshold && exp[i] < 0)) {
        flag = false;
        break;
      }
    }
    std::ofstream o(_logfile, std::ios::out | std::ios::app);
    o << flag << "|[";
    for (int i = 0; i < _total_hcu; i++) o << exp[i] << ",";
    o << "]|[";
    for (int v : _shared_idx) o << v << ",";
    o << "]|[";
    for (int v : _shared_cnt) o << v << ",";
    o << "]" << std::endl;
    _patterns++;
    if (flag) _correct++;
    _cursor++;
    /* counts for the C entry point (gsbn_solver_stats) */
    _glv.puti("check-correct", _correct);
    _glv.puti("check-patterns", _patterns);
  }

  Database* _db = nullptr;
  std::string _logfile;
  std::vector<Mode> _modes;
  HostVector<int32_t>* _lgidx = nullptr;
  std::vector<PopShape> _pops;
  std::vector<std::vector<int>> _counter;
  std::vector<int> _shared_idx, _shared_cnt;
  int _total_hcu = 0, _threshold = 0, _patterns = 0, _correct = 0;
  size_t _cursor = 0;
  bool _updated = false;
};
REGISTERIMPL(ProcCheck)

/* =================================================================
 * ProcSnapshot (src/gsbn/procedures/ProcSnapshot.cpp:8-80,
 * src/gsbn/Database.cpp:257-295): every `period` ticks from `offset`, write
 * ProcSnapshot/Snapshot_<simstep*dt>.bin, a SolverState with every named
 * (non-'.') vector of the network.
 * ================================================================= */
class ProcSnapshot : public ProcedureBase {
  REGISTER(ProcSnapshot)
 public:
  void init_new(SolverParam sp, Database& db) override {
    _db = &db;
    _dir = proc_dir("ProcSnapshot");
    Parser par(get_proc_param(sp));
    if (!par.argi("offset", _offset))
      _offset = 0;
    else if (_offset < 0)
      fatal("ProcSnapshot: offset must be >= 0");
    if (!par.argi("period", _period))
      _period = 1;
    else if (_period <= 0)
      fatal("ProcSnapshot: period must be > 0");
  }
  void init_copy(SolverParam sp, Database& db) override { init_new(sp, db); }
  void update_cpu() override { update_gpu(); }
  void update_gpu() override {
    int cf = 0, t = 0;
    _glv.geti("cycle-flag", cf);
    _glv.geti("simstep", t);
    if (cf == 1 && t >= _offset && t % _period == 0) write(t);
  }
  bool supports_runs() const override { return true; }
  /* a snapshot needs the state right after its tick: end windows there */
  int run_horizon(int t) override {
    int next = std::max(t, _offset);
    int r = next % _period;
    if (r) next += _period - r;
    return next - t + 1;
  }
  void update_run(RunWindow& w) override {
    if (w.cycle_flag != 1) return;
    int last = w.first + w.n - 1;
    if (last >= _offset && last % _period == 0) write(last);
  }

 private:
  void write(int simstep) {
    float dt = 0.f, prn = 0.f;
    _glv.getf("dt", dt);
    _glv.getf("prn", prn);
    std::vector<std::pair<std::string, Database::StateVec>> vecs;
    /* the non-'.' vectors each variant's Pop/Proj create: ProcUpdLazy/Pop.cpp:
       47-52, Proj.cpp:64-83; ProcUpdMulti/Pop.cpp:54-59, Proj.cpp:63-80 (no
       per-cell zi2 or tij) */
    static const char* pop_names[] = {"dsup", "act", "ada", "spike", "epsc", "bj"};
    static const char* lazy_proj[] = {"ii", "di", "qi", "pi", "ei", "zi", "ti", "pj", "ej", "zj",
                                      "pij", "eij", "zi2", "zj2", "tij", "wij", "si"};
    static const char* multi_proj[] = {"ii", "di", "qi", "pi", "ei", "zi", "ti", "pj", "ej", "zj",
                                       "pij", "eij", "zj2", "wij", "si"};
    const bool multi = _db->update_variant == 1;
    auto add = [&](const std::string& name) {
      Database::StateVec v;
      v.bytes = _db->read_state(name, &v.type);
      vecs.emplace_back(name, std::move(v));
    };
    for (size_t p = 0; p < _db->pops.size(); p++)
      for (const char* n : pop_names) {
        std::string name = std::string(n) + "_" + std::to_string(p);
        if (!multi && std::strcmp(n, "ada") == 0) {
          /* ProcUpdLazy creates ada_<pop> and never updates it (its lines
             are commented out, Pop.cpp:258,322): H*M zeros */
          Database::StateVec v;
          v.type = BCPNN_F32;
          v.bytes.assign((size_t)_db->pops[p].hcu_num * _db->pops[p].mcu_num * sizeof(float), 0);
          vecs.emplace_back(name, std::move(v));
        } else {
          add(name);
        }
      }
    for (size_t q = 0; q < _db->projs.size(); q++) {
      if (multi)
        for (const char* n : multi_proj) add(std::string(n) + "_" + std::to_string(q));
      else
        for (const char* n : lazy_proj) add(std::string(n) + "_" + std::to_string(q));
    }
    /* gsbn iterates its vector map, keyed "<name>_<type>" (Database.cpp:
       260-290): sort by that key, so "pi_10" comes before "pi_1" as there */
    auto key = [](const std::pair<std::string, Database::StateVec>& a) {
      return a.first + (a.second.type == BCPNN_I8 ? "_i08" : a.second.type == BCPNN_I32 ? "_i32" : "_f32");
    };
    std::sort(vecs.begin(), vecs.end(), [&](const std::pair<std::string, Database::StateVec>& a,
                                            const std::pair<std::string, Database::StateVec>& b) { return key(a) < key(b); });
    std::string bytes = encode_solver_state(simstep * dt, prn, vecs);
    std::string path = _dir + "/Snapshot_" + std::to_string(simstep * dt) + ".bin";
    std::ofstream o(path, std::ios::out | std::ios::trunc | std::ios::binary);
    o.write(bytes.data(), (std::streamsize)bytes.size());
    if (!o) fatal("Failed to write states.");
  }
  Database* _db = nullptr;
  std::string _dir;
  int _offset = 0, _period = 1;
};
REGISTERIMPL(ProcSnapshot)

/* =================================================================
 * ProcStructuralPlasticity (src/gsbn/procedures/ProcStructuralPlasitcity.cpp:8-631,
 * ProcStructuralPlasticity/Prj.cpp, Pop.cpp): every `pruning-period` ticks,
 * disconnect slot rows that are stale (row tick older than `t-th` ticks) or
 * weak (no weight reaches `wp` or `wn`), on the device (bcpnn_prune), and
 * give each removed row's source MCU its fanout back; every `period` ticks,
 * connect active source MCUs to active destination HCUs through free slots.
 * Only during plastic segments (mode_param plasticity != 0).
 *
 * Kept from gsbn: the loop order and every selection rule, including two
 * quirks: a destination HCU counts as having a free slot when HCU 0 has one
 * (Prj.cpp:111-117 scans the first dim_conn slots for every HCU), and the
 * HCU-activity threshold 0.5 is passed as an int, i.e. 0 (:426).  Reading a
 * source MCU's activity clears the population's spike counters (Pop.cpp:60-70).
 * Changed: gsbn draws from std::random_device (unreplayable); here every
 * draw comes from a Philox4x32-10 stream keyed (argi "seed", 0x5350), draw i
 * at counter (i, i >> 32, 0x53505241, 0), uniform (x >> 8) * 2^-24, and
 * shuffles are Fisher-Yates from the back with j = floor(u * (i + 1)).
 * Geometric delays (enable-geometry) must land in 1..31 ticks.
 * ================================================================= */
class ProcStructuralPlasticity : public ProcedureBase {
  REGISTER(ProcStructuralPlasticity)
 public:
  void init_new(SolverParam sp, Database& db) override {
    _db = &db;
    _net = db.require_net("ProcStructuralPlasticity");
    Parser par(get_proc_param(sp));
    _glv.getf("dt", _dt);
    if (par.argf("d-norm", _d_norm) && _d_norm < 0) _d_norm = 0;
    if (par.argf("v-cond", _v_cond) && _v_cond <= 0) _v_cond = 1;
    if (par.argi("t-th", _t_th) && _t_th <= 0) _t_th = 100;
    if (par.argi("period", _period) && _period <= 0) _period = 100;
    if (par.argi("pruning-period", _pruning_period) && _pruning_period <= 0) _pruning_period = 1000;
    if (par.argi("enable-geometry", _geometry) && _geometry != 0) _geometry = 1;
    if (par.argi("enable-init-conn", _init_conn) && _init_conn != 0) _init_conn = 1;
    par.argf("wp", _wp);
    par.argf("wn", _wn);
    int seed = 0;
    par.argi("seed", seed);
    _seed = (uint32_t)seed;
    if (!(_wp > _wn)) fatal("ProcStructuralPlasticity: w+ should be larger than w- !!");
    for (const PopParam& pp : sp.net_param.pop_param)
      for (uint32_t k = 0; k < pp.pop_num; k++) {
        PopInfo P;
        P.H = (int)pp.hcu_num;
        P.M = (int)pp.mcu_num;
        P.fanout.assign((size_t)P.H * P.M, (int)pp.fanout_num);
        P.shape.assign(pp.shape.begin(), pp.shape.end());
        P.position.assign(pp.position.begin(), pp.position.end());
        _pops.push_back(P);
      }
    for (size_t k = 0; k < db.projs.size(); k++) {
      const bcpnn_proj_desc& q = db.projs[k];
      PrjInfo J;
      J.src = q.src_pop;
      J.dest = q.dest_pop;
      J.H = _pops[J.dest].H;
      J.M = _pops[J.dest].M;
      J.C = (int)std::min<long long>((long long)_pops[J.src].H * _pops[J.src].M, (long long)q.slot_num);
      _prjs.push_back(J);
      _pops[J.src].out.push_back((int)k);
    }
    if (_init_conn) grow(-1, -1);
  }
  void init_copy(SolverParam sp, Database& db) override { init_new(sp, db); }
  void update_cpu() override { update_gpu(); }
  void update_gpu() override {
    int cf = 0, t = 0;
    _glv.geti("cycle-flag", cf);
    _glv.geti("simstep", t);
    if (cf == 1) at_tick(t);
  }
  bool supports_runs() const override { return true; }
  /* the work happens right after ticks that are multiples of the periods */
  int run_horizon(int t) override {
    auto next = [&](int period) { int r = t % period; return r ? t + period - r : t; };
    return std::min(next(_period), next(_pruning_period)) - t + 1;
  }
  void update_run(RunWindow& w) override {
    if (w.cycle_flag != 1) return;
    at_tick(w.first + w.n - 1);
  }

 private:
  struct PopInfo {
    int H = 0, M = 0;
    std::vector<int> fanout;
    std::vector<int> shape, position;
    std::vector<int> out; /* projections with this population as source, in id order */
  };
  struct PrjInfo {
    int src = 0, dest = 0, H = 0, M = 0, C = 0;
  };

  void at_tick(int t) {
    bool plastic = false;
    _glv.getb("plasticity", plastic);
    if (!plastic) return;
    if (t % _pruning_period == 0) prune(t);
    if (t % _period == 0) grow(0, (int)(0.2 * _period * 100 * _dt)); /* ProcStructuralPlasitcity.cpp:426-458 */
  }

  /* stages 1-2 (ProcStructuralPlasitcity.cpp:275-350) */
  void prune(int t) {
    for (size_t k = 0; k < _prjs.size(); k++) {
      const PrjInfo& J = _prjs[k];
      std::vector<int32_t> removed((size_t)J.H * J.C + 1);
      int32_t n = 0;
      int st = bcpnn_prune(_net, (int32_t)k, t - _t_th, _wp, _wn, removed.data(), removed.size(), &n);
      if (st != BCPNN_OK) fatal(std::string("bcpnn_prune: ") + bcpnn_last_error(_net));
      std::vector<int>& fan = _pops[J.src].fanout;
      for (int32_t i = 0; i < n; i++) fan[removed[i]] += 1;
    }
  }

  std::vector<int32_t> read_i32(const std::string& name) {
    std::vector<uint8_t> b = _db->read_state(name);
    std::vector<int32_t> v(b.size() / 4);
    if (!v.empty()) std::memcpy(v.data(), b.data(), b.size());
    return v;
  }
  std::vector<float> read_f32(const std::string& name) {
    std::vector<uint8_t> b = _db->read_state(name);
    std::vector<float> v(b.size() / 4);
    if (!v.empty()) std::memcpy(v.data(), b.data(), b.size());
    return v;
  }

  float uniform() {
    bx_u32x4 c;
    c.v[0] = (uint32_t)_draws;
    c.v[1] = (uint32_t)(_draws >> 32);
    c.v[2] = 0x53505241u;
    c.v[3] = 0u;
    _draws++;
    return bx_u01(bx_philox4x32_10(c, _seed, 0x5350u).v[0]);
  }
  void shuffle(std::vector<int>& a) {
    for (size_t i = a.size(); i-- > 1;) {
      size_t j = (size_t)((double)uniform() * (double)(i + 1));
      if (j > i) j = i;
      std::swap(a[i], a[j]);
    }
  }

  /* stages 3-5 (ProcStructuralPlasitcity.cpp:352-560; init_conn :113-258 with
     thresholds -1) */
  void grow(int hcu_threshold, int mcu_threshold) {
    const size_t np = _prjs.size();
    std::vector<std::vector<int32_t>> local(np), avail_hcu(np);
    for (size_t k = 0; k < np; k++) {
      const PrjInfo& J = _prjs[k];
      local[k] = read_i32("ii_" + std::to_string(k));
      std::vector<float> ej = read_f32("ej_" + std::to_string(k));
      bool free_slot = false; /* gsbn scans HCU 0's slots for every HCU (Prj.cpp:111-117) */
      for (int j = 0; j < J.C; j++)
        if (local[k][j] < 0) {
          free_slot = true;
          break;
        }
      for (int i = 0; i < J.H; i++) {
        float acc = 0;
        for (int j = 0; j < J.M; j++) acc += ej[(size_t)i * J.M + j];
        if (acc > (float)hcu_threshold && free_slot) avail_hcu[k].push_back(i);
      }
    }
    for (size_t pi = 0; pi < _pops.size(); pi++) {
      PopInfo& P = _pops[pi];
      /* active source MCUs; the counters are cleared as they are read (Pop.cpp:60-70) */
      const std::string cname = ".counter_" + std::to_string(pi);
      std::vector<int32_t> cnt = read_i32(cname);
      std::vector<int> active;
      for (size_t i = 0; i < cnt.size(); i++)
        if (cnt[i] > mcu_threshold) active.push_back((int)i);
      std::vector<int32_t> zero(cnt.size(), 0);
      _db->write_state(cname, zero.data(), zero.size() * 4);
      std::vector<int> prjs = P.out;
      while (!prjs.empty() && !active.empty()) {
        float u = uniform();
        size_t idx = (size_t)(int)(u * (float)prjs.size());
        if (idx >= prjs.size()) idx = prjs.size() - 1;
        const int k = prjs[idx];
        const PrjInfo& J = _prjs[k];
        std::vector<int> hcus(avail_hcu[k].begin(), avail_hcu[k].end());
        if (hcus.empty()) break;
        shuffle(hcus);
        for (int h : hcus) {
          std::vector<int> cand = active;
          for (int s = 0; s < J.C; s++) {
            int c = local[k][(size_t)h * J.C + s];
            if (c >= 0) cand.erase(std::remove(cand.begin(), cand.end(), c), cand.end());
          }
          if (cand.empty()) continue;
          shuffle(cand);
          size_t l = 0;
          for (int s = 0; s < J.C && l < cand.size(); s++) {
            int32_t& slot = local[k][(size_t)h * J.C + s];
            if (slot < 0) slot = cand[l++];
          }
          for (size_t i = 0; i < l; i++) {
            int mcu = cand[i];
            if (--P.fanout[mcu] <= 0) active.erase(std::remove(active.begin(), active.end(), mcu), active.end());
          }
        }
        prjs.erase(prjs.begin() + idx);
      }
    }
    /* stage 5: new rows into the first free slot of their HCU (add_row, :576-588) */
    for (size_t k = 0; k < np; k++) {
      const PrjInfo& J = _prjs[k];
      std::vector<int32_t> ii = read_i32("ii_" + std::to_string(k));
      std::vector<int32_t> di = read_i32("di_" + std::to_string(k));
      const std::vector<int32_t> cur = ii;
      bool changed = false;
      for (int h = 0; h < J.H; h++)
        for (int s = 0; s < J.C; s++) {
          const size_t index = (size_t)h * J.C + s;
          if (cur[index] >= 0 || ii[index] >= 0 || local[k][index] < 0) continue;
          const int src = local[k][index];
          const int delay = _geometry ? delay_cycle(J, src, h) : 1;
          for (int f = 0; f < J.C; f++) {
            if (ii[(size_t)h * J.C + f] < 0) {
              ii[(size_t)h * J.C + f] = src;
              di[(size_t)h * J.C + f] = delay;
              changed = true;
              break;
            }
          }
        }
      if (changed) {
        int st = bcpnn_set_conn(_net, (int32_t)k, ii.data(), di.data(), ii.size());
        if (st != BCPNN_OK) fatal(std::string("ProcStructuralPlasticity: ") + bcpnn_last_error(_net));
      }
    }
  }

  std::vector<int> hcu_coor(const PopInfo& P, int hcu) const { /* Pop.cpp:72-91 */
    std::vector<int> coor(P.shape.size());
    int index = hcu;
    for (size_t i = 0; i < P.shape.size(); i++) {
      if (P.shape[i] <= 0) fatal("ProcStructuralPlasticity: population shape entries must be > 0");
      coor[i] = index % P.shape[i];
      index /= P.shape[i];
    }
    for (size_t i = 0; i < P.position.size(); i++) {
      if (i < coor.size())
        coor[i] += P.position[i];
      else
        coor.push_back(P.position[i]);
    }
    return coor;
  }

  int delay_cycle(const PrjInfo& J, int src_mcu, int dest_hcu) { /* :590-625 */
    const PopInfo& P0 = _pops[J.src];
    const PopInfo& P1 = _pops[J.dest];
    std::vector<int> a = hcu_coor(P0, src_mcu / P0.M), b = hcu_coor(P1, dest_hcu);
    while (a.size() < b.size()) a.push_back(0);
    while (b.size() < a.size()) b.push_back(0);
    float d2 = 0;
    for (size_t i = 0; i < a.size(); i++) d2 += (float)((a[i] - b[i]) * (a[i] - b[i]));
    const float distance = (float)std::sqrt((double)d2);
    const float mean = _d_norm * distance / _v_cond + 1;
    /* normal(mean, 0.1 mean) by Box-Muller from two draws of the stream */
    const double u1 = 1.0 - (double)uniform(), u2 = (double)uniform();
    const double z = std::sqrt(-2.0 * bx_log_d(u1)) * bx_cos2pi_d(u2);
    const float tij = (float)(mean + 0.1 * mean * z);
    return (int)std::ceil(tij * 0.001 / _dt);
  }

  Database* _db = nullptr;
  bcpnn_net* _net = nullptr;
  float _dt = 0.001f, _d_norm = 0.75f, _v_cond = 0.2f, _wp = 0.5f, _wn = -0.5f;
  int _t_th = 100, _period = 100, _pruning_period = 1000, _geometry = 0, _init_conn = 0;
  uint32_t _seed = 0;
  uint64_t _draws = 0;
  std::vector<PopInfo> _pops;
  std::vector<PrjInfo> _prjs;
};
REGISTERIMPL(ProcStructuralPlasticity)

}  // namespace gsbn
