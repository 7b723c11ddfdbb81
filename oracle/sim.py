"""TEST INFRASTRUCTURE, NOT PART OF THE PRODUCT.

Python half of the CPU oracle: a ctypes wrapper over the C++ restatement of
ProcUpdLazy (oracle/bcpnn_oracle.cpp) and restatements of the host-side
procedures around the hot path, each citing the reference code it follows
(paths relative to the gsbn source tree):

  ProcExtGen        src/gsbn/procedures/ProcExtGen.cpp:8-153
  ProcInitConn      src/gsbn/procedures/ProcInitConn.cpp:8-103
  external spikes   src/gsbn/procedures/ProcUpdLazy/Pop.cpp:67-110
  ProcCheck         src/gsbn/procedures/ProcCheck.cpp:8-237, ProcCheck/Pop.cpp:6-60
  ProcSpkRec        src/gsbn/procedures/ProcSpkRec.cpp:10-206, ProcSpkRec/Pop.cpp:30-52,
                    ProcSpkRec/Prj.cpp:95-138
  Solver loop       src/gsbn/Solver.cpp:67-92, src/gsbn/Upd.cpp:28-40

Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline use it.

Math modes of the C++ oracle:
  MATH_SHARED  the restatement with the shared exp/log (bit-exact with the GPU);
  MATH_LIBM    the restatement with glibc expf/logf, as gsbn's float calls;
  MATH_REF     gsbn's own update_*_kernel_cpu functions, compiled from the gsbn
               sources into oracle/_ref/libbcpnn_oracle_ref.so (oracle/Makefile
               target `ref`), driven by the same loops.  The whole gsbn program
               cannot be built (protobuf, MPI), but these free functions can.
The restatement is pinned against MATH_REF, on the reference's fixtures and on
the published Philox known-answer vectors.
"""
import ctypes
import math
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libbcpnn_oracle.so")
LIB_REF = os.path.join(HERE, "_ref", "libbcpnn_oracle_ref.so")
MATH_LIBM, MATH_SHARED, MATH_REF = 0, 1, 2
f32 = np.float32

_lib = None
_lib_ref = None


def build():
    """The oracle, and oracle/_ref when the gsbn sources are present."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    subprocess.run(["make", "-s", "-C", HERE, "ref-if-present"], check=True)


def reference_root():
    """The gsbn source tree ($GSBN_REFERENCE_ROOT, else oracle/Makefile's
    REF_ROOT), or None when it is not present."""
    r = os.environ.get("GSBN_REFERENCE_ROOT")
    if not r:
        r = subprocess.run(["make", "-s", "-C", HERE, "ref-root"], capture_output=True, text=True).stdout.strip()
    return r if r and os.path.isdir(r) else None


def ref_available():
    """True when oracle/_ref (gsbn's own kernels) is built."""
    return os.path.exists(LIB_REF)


def load(ref=False):
    """The oracle library; ref=True: the build that carries gsbn's kernels."""
    global _lib, _lib_ref
    if ref:
        if _lib_ref is not None:
            return _lib_ref
        if not os.path.exists(LIB_REF):
            raise RuntimeError("oracle/_ref is not built (make -C oracle ref, with the gsbn sources present)")
        _lib_ref = _bind(ctypes.CDLL(LIB_REF))
        return _lib_ref
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB):
        build()
    _lib = _bind(ctypes.CDLL(LIB))
    return _lib


def _bind(lib):
    vp, i32, u32, fl, sz = ctypes.c_void_p, ctypes.c_int, ctypes.c_uint32, ctypes.c_float, ctypes.c_size_t
    lib.oracle_create.restype = vp
    lib.oracle_create.argtypes = [i32, i32, fl, u32, fl, i32, vp, vp, i32, vp, vp]
    lib.oracle_destroy.argtypes = [vp]
    lib.oracle_set_stimulus.argtypes = [vp, vp, vp]
    lib.oracle_set_ext_spikes.argtypes = [vp, i32, i32, vp, vp, vp]
    lib.oracle_update.argtypes = [vp, i32, fl, fl]
    lib.oracle_exchange.argtypes = [vp]
    lib.oracle_state_info.restype = ctypes.c_longlong
    lib.oracle_state_info.argtypes = [vp, ctypes.c_char_p, ctypes.POINTER(i32)]
    lib.oracle_read_state.argtypes = [vp, ctypes.c_char_p, vp, sz]
    lib.oracle_write_state.argtypes = [vp, ctypes.c_char_p, vp, sz]
    lib.oracle_counters.argtypes = [vp, ctypes.POINTER(ctypes.c_ulonglong)]
    lib.oracle_expf.restype = fl
    lib.oracle_expf.argtypes = [i32, fl]
    lib.oracle_logf.restype = fl
    lib.oracle_logf.argtypes = [i32, fl]
    lib.oracle_log_double.restype = ctypes.c_double
    lib.oracle_log_double.argtypes = [i32, ctypes.c_double]
    lib.oracle_cos2pi_double.restype = ctypes.c_double
    lib.oracle_cos2pi_double.argtypes = [ctypes.c_double]
    lib.oracle_expf_array.argtypes = [i32, ctypes.c_longlong, vp, vp]
    lib.oracle_logf_array.argtypes = [i32, ctypes.c_longlong, vp, vp]
    lib.oracle_philox.argtypes = [vp, vp, vp]
    lib.oracle_uniform_array.argtypes = [u32, u32, u32, i32, vp]
    lib.oracle_uniform_poisson_array.argtypes = [u32, u32, u32, i32, vp]
    lib.oracle_normal_array.argtypes = [u32, u32, u32, i32, vp]
    lib.oracle_has_ref.restype = i32
    return lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def expf(x, math=MATH_SHARED):
    x = np.ascontiguousarray(x, dtype=np.float32)
    out = np.empty_like(x)
    load().oracle_expf_array(math, x.size, _p(x), _p(out))
    return out


def logf(x, math=MATH_SHARED):
    x = np.ascontiguousarray(x, dtype=np.float32)
    out = np.empty_like(x)
    load().oracle_logf_array(math, x.size, _p(x), _p(out))
    return out


def extgen_logf(x):
    """ProcExtGen's lginp values log(1+eps), log(0+eps) (ProcExtGen.cpp:130-144):
    gsbn computes them on the host with glibc's float log in every mode, and
    so does the product's host code; the stimulus rows are gsbn's bit for bit."""
    return np.float32(load().oracle_logf(MATH_LIBM, float(np.float32(x))))


def philox(ctr, key):
    c = np.ascontiguousarray(ctr, dtype=np.uint32)
    k = np.ascontiguousarray(key, dtype=np.uint32)
    out = np.zeros(4, np.uint32)
    load().oracle_philox(_p(c), _p(k), _p(out))
    return out


def uniforms(seed, pop, tick, n):
    out = np.zeros(n, np.float32)
    load().oracle_uniform_array(seed, pop, tick, n, _p(out))
    return out


def uniforms_poisson(seed, pop, tick, n):
    out = np.zeros(n, np.float32)
    load().oracle_uniform_poisson_array(seed, pop, tick, n, _p(out))
    return out


def normals(seed, pop, tick, n):
    out = np.zeros(n, np.float32)
    load().oracle_normal_array(seed, pop, tick, n, _p(out))
    return out


POP_KEYS = ("taum", "wtagain", "maxfq", "igain", "wgain", "lgbias", "snoise")
PROJ_KEYS = ("tauzi", "tauzj", "taue", "taup", "maxfq", "bgain", "wgain", "tauepsc", "slot_num")


class OracleNet:
    """CPU restatement of one network (same call shape as gsbn_b200.capi.Net)."""

    def __init__(self, pops, projs, dt, seed=0, poisson_hz=0.0, real_bits=32, math=MATH_SHARED):
        self.lib = load(ref=(math == MATH_REF))
        self.real_bits = real_bits
        self.math = math
        dims = np.array([[p["hcu_num"], p["mcu_num"]] for p in pops], dtype=np.int32).reshape(-1)
        pp = np.array([[p[k] for k in POP_KEYS] for p in pops], dtype=np.float32).reshape(-1)
        pi = np.array([[q["src_pop"], q["dest_pop"]] for q in projs], dtype=np.int32).reshape(-1)
        pf = np.array([[q[k] for k in PROJ_KEYS] for q in projs], dtype=np.float32).reshape(-1)
        if pi.size == 0:
            pi = np.zeros(2, np.int32)
            pf = np.zeros(9, np.float32)
        self.h = self.lib.oracle_create(real_bits, math, dt, seed, poisson_hz, len(pops), _p(dims), _p(pp),
                                        len(projs), _p(pi), _p(pf))
        if not self.h:
            raise RuntimeError("MATH_REF needs the float oracle built with gsbn's kernels (oracle/_ref)")
        self.n_pops, self.n_projs = len(pops), len(projs)

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.oracle_destroy(self.h)
            self.h = None

    def _vec(self, name):
        kind = ctypes.c_int()
        n = self.lib.oracle_state_info(self.h, name.encode(), ctypes.byref(kind))
        if n < 0:
            raise KeyError(name)
        dt = {0: (np.float32 if self.real_bits == 32 else np.float64), 1: np.int32, 2: np.int8}[kind.value]
        return n, dt

    def read(self, name):
        n, dt = self._vec(name)
        out = np.zeros(n, dtype=dt)
        rc = self.lib.oracle_read_state(self.h, name.encode(), _p(out), out.nbytes)
        assert rc == 0, rc
        return out

    def write(self, name, arr):
        n, dt = self._vec(name)
        a = np.ascontiguousarray(arr, dtype=dt)
        assert a.size == n
        assert self.lib.oracle_write_state(self.h, name.encode(), _p(a), a.nbytes) == 0

    def set_conn(self, proj, ii, di):
        self.write(f"ii_{proj}", ii)
        self.write(f"di_{proj}", di)

    def set_stimulus(self, lginp, wmask_row):
        lg = np.ascontiguousarray(lginp, dtype=np.float32)
        wm = np.ascontiguousarray(wmask_row, dtype=np.float32)
        self.lib.oracle_set_stimulus(self.h, _p(lg), _p(wm))

    def set_ext_spikes(self, pop, table):
        ticks = np.array(sorted(table), dtype=np.int32)
        offs, flat = [0], []
        for t in ticks:
            flat.extend(table[int(t)])
            offs.append(len(flat))
        offs = np.array(offs, dtype=np.int32)
        flat = np.array(flat if flat else [0], dtype=np.int32)
        self.lib.oracle_set_ext_spikes(self.h, pop, len(ticks), _p(ticks), _p(offs), _p(flat))

    def update(self, simstep, prn, old_prn):
        """ProcUpdLazy::update_cpu for one tick."""
        self.lib.oracle_update(self.h, simstep, prn, old_prn)

    def exchange(self):
        """ProcExchangeSpike::update_cpu for one tick."""
        self.lib.oracle_exchange(self.h)

    def run(self, first_simstep, n_ticks, prn, old_prn, exchange=True, spikes=True):
        """n ticks of ProcUpdLazy (+ ProcExchangeSpike); returns per tick and per
        population the ascending spike indices."""
        out = []
        for k in range(n_ticks):
            self.update(first_simstep + k, prn, old_prn if k == 0 else prn)
            if exchange:
                self.exchange()
            if spikes:
                out.append([np.nonzero(self.read(f"spike_{p}"))[0] for p in range(self.n_pops)])
        return out

    def counters(self):
        c = (ctypes.c_ulonglong * 3)()
        self.lib.oracle_counters(self.h, c)
        return [int(c[0]), int(c[1]), int(c[2])]

    def logf(self, x):
        """ProcExtGen's float log (host code in gsbn, glibc logf in every math
        mode): the stimulus values log(1+eps) and log(eps)."""
        return extgen_logf(x)


# ---------------------------------------------------------------------------
# network description from a SolverParam (ProcUpdLazy.cpp:19-45)
# ---------------------------------------------------------------------------

def net_from_solver_param(sp):
    """Populations (pop_num copies of each PopParam) and the projections whose
    src and dest populations exist, as plain dicts."""
    pops = []
    for pp in sp.net_param.pop_param:
        for _ in range(pp.pop_num):
            pops.append(dict(hcu_num=pp.hcu_num, mcu_num=pp.mcu_num, taum=pp.taum, wtagain=pp.wtagain,
                             maxfq=pp.maxfq, igain=pp.igain, wgain=pp.wgain, lgbias=pp.lgbias, snoise=pp.snoise))
    projs = []
    for q in sp.net_param.proj_param:
        if q.src_pop < len(pops) and q.dest_pop < len(pops):
            projs.append(dict(src_pop=q.src_pop, dest_pop=q.dest_pop, tauzi=q.tauzi, tauzj=q.tauzj, taue=q.taue,
                              taup=q.taup, maxfq=q.maxfq, bgain=q.bgain, wgain=q.wgain,
                              tauepsc=q.tauepsc if q.HasField("tauepsc") else 0.0, slot_num=q.slot_num))
    return pops, projs


def dim_conn(pops, q):
    """Proj.cpp:22-26."""
    c = pops[q["src_pop"]]["hcu_num"] * pops[q["src_pop"]]["mcu_num"]
    return min(c, int(q["slot_num"]))


def log_double(x):
    """the library's double log (bx_log_d), as the oracle computes it"""
    return load().oracle_log_double(MATH_SHARED, x)


def proc_args(sp, name):
    """argi/argf/args of the proc_param named `name` (Parser.cpp:12-43)."""
    for pp in sp.proc_param:
        if pp.name == name:
            return ({a.key: a.val for a in pp.argi}, {a.key: a.val for a in pp.argf},
                    {a.key: a.val for a in pp.args})
    return None


# ---------------------------------------------------------------------------
# ProcInitConn (ProcInitConn.cpp:48-103)
# ---------------------------------------------------------------------------

def parse_conn_map(text, pops, projs):
    """Slot tables (ii, di) per projection from a connection map: lines
    `proj,dest_hcu,src_mcu,delay,src_mcu,delay,...`; each pair fills the first
    empty slot of the destination HCU and is dropped when none is left.  Slots
    only ever fill in order here, so the first empty slot is a running count."""
    tables, fill = [], []
    for q in projs:
        C = dim_conn(pops, q)
        H = pops[q["dest_pop"]]["hcu_num"]
        tables.append((np.full(H * C, -1, np.int32), np.zeros(H * C, np.int32), C))
        fill.append(np.zeros(H, np.int64))
    for line in text.splitlines():
        v = line.split(",")
        if len(v) > 2:
            prj = int(v[0])
            hcu = int(v[1])
            ii, di, C = tables[prj]
            for i in range(2, len(v) - 1, 2):
                s = fill[prj][hcu]
                if s < C:
                    ii[hcu * C + s] = int(v[i])
                    di[hcu * C + s] = int(v[i + 1])
                    if int(v[i]) >= 0:  # a negative source leaves the slot empty
                        fill[prj][hcu] = s + 1
    return [(t[0], t[1]) for t in tables]


# ---------------------------------------------------------------------------
# external spike file (Pop.cpp:67-110)
# ---------------------------------------------------------------------------

def parse_ext_spikes(text, pop_id):
    table = {}
    for line in text.splitlines():
        v = line.split(",")
        if len(v) > 2 and int(v[1]) == pop_id and int(v[0]) >= 0:
            table[int(v[0])] = [int(x) for x in v[2:]]
    return table


# ---------------------------------------------------------------------------
# ProcExtGen (ProcExtGen.cpp:8-153)
# ---------------------------------------------------------------------------

def extgen_modes(gen_param):
    """Expand mode_param into per-pattern segments (ProcExtGen.cpp:16-55)."""
    dt = f32(gen_param.dt)
    modes = []
    for mp in gen_param.mode_param:
        begin_step = int(f32(mp.begin_time) / dt)
        end_step = int(f32(mp.end_time) / dt)
        if end_step < begin_step:
            raise ValueError("Time range is wrong")
        lgidx, lgexp, wmask = mp.begin_lgidx_id, mp.begin_lgexp_id, mp.begin_wmask_id
        while begin_step < end_step:
            e = begin_step + mp.time_step
            if e >= end_step:
                e = end_step
            modes.append(dict(begin_step=begin_step, end_step=e, lgidx_id=lgidx, lgexp_id=lgexp, wmask_id=wmask,
                              prn=float(f32(mp.prn)), plasticity=mp.plasticity))
            lgidx += mp.lgidx_step
            lgexp += mp.lgexp_step
            wmask += mp.wmask_step
            begin_step = e
    return modes


def as_int32(v):
    v = int(v) & 0xFFFFFFFF
    return v - (1 << 32) if v >= (1 << 31) else v


class ExtGen:
    """Per-tick stimulus and phase state (ProcExtGen.cpp:113-153)."""

    def __init__(self, sp, stim, mcu_in_hcu, logf):
        self.modes = extgen_modes(sp.gen_param)
        self.eps = f32(sp.gen_param.eps)
        self.lgidx = np.array([as_int32(x) for x in stim.data], dtype=np.int64).reshape(stim.data_rows,
                                                                                       stim.data_cols)
        self.wmask = np.array(stim.mask, dtype=np.float32).reshape(stim.mask_rows, stim.mask_cols)
        self.mcu_in_hcu = mcu_in_hcu
        self.lg_hit = f32(logf(f32(1) + self.eps))
        self.lg_miss = f32(logf(f32(0) + self.eps))
        self.lginp = np.zeros(sum(mcu_in_hcu), dtype=np.float32)
        self.cursor = 0
        self.old_lgidx_id = -1
        self.simstep = 0
        self.prn = 0.0
        self.old_prn = 0.0
        self.cycle_flag = 0
        self.wmask_idx = 0
        self.lginp_changed = False
        self.plasticity = False

    def tick(self):
        self.simstep += 1
        t = self.simstep
        self.lginp_changed = False
        while self.cursor < len(self.modes):
            m = self.modes[self.cursor]
            if m["begin_step"] < t <= m["end_step"]:
                self.old_prn = self.prn
                self.prn = m["prn"]
                self.wmask_idx = m["wmask_id"]
                self.plasticity = bool(m["plasticity"])
                self.cycle_flag = 1
                if self.old_lgidx_id != m["lgidx_id"]:
                    self.old_lgidx_id = m["lgidx_id"]
                    row = self.lgidx[m["lgidx_id"]]
                    k = 0
                    for i, nm in enumerate(self.mcu_in_hcu):
                        for j in range(nm):
                            self.lginp[k] = self.lg_hit if row[i] == j else self.lg_miss
                            k += 1
                    self.lginp_changed = True
                return
            elif t <= m["begin_step"]:
                self.cycle_flag = 0
                return
            self.cursor += 1
        self.cycle_flag = -1

    def wmask_row(self):
        return self.wmask[self.wmask_idx]


# ---------------------------------------------------------------------------
# ProcCheck (ProcCheck.cpp:8-237, ProcCheck/Pop.cpp:6-60)
# ---------------------------------------------------------------------------

class Check:
    def __init__(self, sp, lgidx, pops, threshold=0):
        dt = f32(sp.gen_param.dt)
        self.modes = []
        for mp in sp.gen_param.mode_param:
            begin_step = int(f32(mp.begin_time) / dt)
            end_step = int(f32(mp.end_time) / dt)
            if f32(mp.prn) != 0.0:
                continue
            lgidx_, lgexp, wmask = mp.begin_lgidx_id, mp.begin_lgexp_id, mp.begin_wmask_id
            while begin_step < end_step:
                self.modes.append(dict(begin_step=begin_step, end_step=begin_step + mp.time_step, lgexp_id=lgexp))
                lgidx_ += mp.lgidx_step
                lgexp += mp.lgexp_step
                wmask += mp.wmask_step
                begin_step += mp.time_step
        self.lgidx = lgidx
        self.pops = pops
        self.counter = [np.zeros((p["hcu_num"], p["mcu_num"]), np.int64) for p in pops]
        self.total_hcu = sum(p["hcu_num"] for p in pops)
        self.shared_idx = np.zeros(self.total_hcu, np.int64)
        self.shared_cnt = np.zeros(self.total_hcu, np.int64)
        self.threshold = threshold
        self.cursor = 0
        self.pattern_num = 0
        self.correct = 0
        self.updated = False
        self.lines = ["result | reference pattern | recorded pattern | recorded pattern spike count"]
        self.summary = None

    def update(self, cycle_flag, simstep, spikes):
        """spikes: per population the int8 spike vector of this tick."""
        if cycle_flag == 0:
            return
        if cycle_flag > 0:
            if self.cursor >= len(self.modes):
                return
            m = self.modes[self.cursor]
            if simstep <= m["begin_step"]:
                return
            if simstep < m["end_step"]:
                for c, s, p in zip(self.counter, spikes, self.pops):
                    c += (np.asarray(s).reshape(p["hcu_num"], p["mcu_num"]) > 0)
                self.updated = True
                return
            if not self.updated:
                while self.cursor < len(self.modes) and simstep >= self.modes[self.cursor]["end_step"]:
                    self.cursor += 1
                return
            hcu = 0
            for c in self.counter:
                for i in range(c.shape[0]):
                    max_idx, max_cnt = -1, 0
                    for j in range(c.shape[1]):
                        if c[i, j] > max_cnt:
                            max_idx, max_cnt = j, int(c[i, j])
                    self.shared_idx[hcu + i] = max_idx
                    self.shared_cnt[hcu + i] = max_cnt
                c[:] = 0
                hcu += c.shape[0]
            exp = self.lgidx[m["lgexp_id"]]
            flag = True
            for i in range(self.total_hcu):
                e = exp[i]
                if ((self.shared_cnt[i] < self.threshold or self.shared_idx[i] != e) and e >= 0) or \
                        (self.shared_cnt[i] > self.threshold and e < 0):
                    flag = False
                    break
            self.lines.append(f"{int(flag)}|[" + "".join(f"{int(v)}," for v in exp[:self.total_hcu]) + "]|[" +
                              "".join(f"{int(v)}," for v in self.shared_idx) + "]|[" +
                              "".join(f"{int(v)}," for v in self.shared_cnt) + "]")
            self.pattern_num += 1
            self.correct += int(flag)
            self.cursor += 1
        else:
            pct = self.correct * 100.0 / self.pattern_num if self.pattern_num else float("nan")
            self.summary = f"correct pattern: {self.correct}/{self.pattern_num}({cpp_g(pct)}%)"
            self.lines.append(self.summary)


def cpp_g(x):
    """std::ostream << double with the default precision 6 (%g)."""
    if x != x:
        return "nan"
    if x == float("inf"):
        return "inf"
    return format(x, "g")


# ---------------------------------------------------------------------------
# ProcSpkRec (ProcSpkRec.cpp:10-206)
# ---------------------------------------------------------------------------

class SpkRec:
    def __init__(self, sp, pops, n_projs, offset=0, period=1):
        dt = f32(sp.gen_param.dt)
        self.offset, self.period = offset, period
        self.spk = [[f"{p['hcu_num']},{p['mcu_num']},{cpp_g(float(dt))},{cpp_g(float(f32(p['maxfq'])))}"]
                    for p in pops]
        self.ssi = [[] for _ in range(n_projs)]
        self.ssj = [[] for _ in range(n_projs)]

    def update(self, cycle_flag, simstep, spikes, ss_flags):
        """spikes: per population ascending spike indices; ss_flags: per
        projection (row 9 in .ssi, MCU 9 in .ssj)."""
        if cycle_flag != 1 or simstep < self.offset or simstep % self.period != 0:
            return
        for k, s in enumerate(spikes):
            if len(s):
                self.spk[k].append(str(simstep) + "".join(f",{int(i)}" for i in s))
        for k, (fi, fj) in enumerate(ss_flags):
            self.ssj[k].append(f"{simstep},{1 if fj else 0}")
            self.ssi[k].append(f"{simstep},{1 if fi else 0}")

    def files(self):
        out = {}
        for k, lines in enumerate(self.spk):
            out[f"spk_pop_{k}.csv"] = "\n".join(lines) + "\n"
        for k in range(len(self.ssi)):
            out[f"ssi_pop_{k}.csv"] = "".join(l + "\n" for l in self.ssi[k])
            out[f"ssj_pop_{k}.csv"] = "".join(l + "\n" for l in self.ssj[k])
        return out


# ---------------------------------------------------------------------------
# ProcStructuralPlasticity (ProcStructuralPlasitcity.cpp:8-631,
# ProcStructuralPlasticity/Prj.cpp:69-165, Pop.cpp:6-91), with gsbn's
# random_device draws replaced by the seeded Philox stream the product uses:
# draw i = philox((i, i >> 32, 0x53505241, 0), (seed, 0x5350))[0], uniform
# (x >> 8) * 2^-24; Fisher-Yates from the back with j = floor(u * (i + 1)).
# enable-geometry: a grown row's delay is ceil(tij * 0.001 / dt) ticks with
# tij ~ normal(mean, 0.1 mean), mean = d_norm * distance / v_cond + 1 in float
# over the HCUs' grid coordinates (delay_cycle, ProcStructuralPlasitcity.cpp:
# 597-627; Pop::hcu_coor, ProcStructuralPlasticity/Pop.cpp:64-88); gsbn's
# normal draw is restated as Box-Muller in double from two uniforms of the
# stream, z = sqrt(-2 log(1 - u1)) cos(2 pi u2).
# ---------------------------------------------------------------------------

class StructuralPlasticity:
    def __init__(self, sp, net, pops, projs, dt):
        argi, argf, _ = proc_args(sp, "ProcStructuralPlasticity")
        self.net, self.pops, self.projs, self.dt = net, pops, projs, f32(dt)
        self.t_th = argi.get("t-th", 100) if argi.get("t-th", 100) > 0 else 100
        self.period = argi.get("period", 100) if argi.get("period", 100) > 0 else 100
        pp = argi.get("pruning-period", 1000)
        self.pruning_period = pp if pp > 0 else 1000
        self.geometry = argi.get("enable-geometry", 0) != 0
        self.d_norm = f32(argf.get("d-norm", 0.75))
        if "d-norm" in argf and self.d_norm < 0:
            self.d_norm = f32(0)
        self.v_cond = f32(argf.get("v-cond", 0.2))
        if "v-cond" in argf and self.v_cond <= 0:
            self.v_cond = f32(1)
        self.geo = [(list(pp.shape), list(pp.position)) for pp in sp.net_param.pop_param for _ in range(pp.pop_num)]
        self.wp, self.wn = f32(argf.get("wp", 0.5)), f32(argf.get("wn", -0.5))
        self.seed = argi.get("seed", 0) & 0xFFFFFFFF
        self.draws = 0
        fan = [pp.fanout_num for pp in sp.net_param.pop_param for _ in range(pp.pop_num)]
        self.fanout = [np.full(p["hcu_num"] * p["mcu_num"], fan[i], np.int64) for i, p in enumerate(pops)]
        self.out = [[k for k, q in enumerate(projs) if q["src_pop"] == i] for i in range(len(pops))]
        if argi.get("enable-init-conn", 0):
            self.grow(-1, -1)

    def uniform(self):
        i = self.draws
        self.draws += 1
        x = philox([i & 0xFFFFFFFF, (i >> 32) & 0xFFFFFFFF, 0x53505241, 0], [self.seed, 0x5350])[0]
        return f32(int(x) >> 8) * f32(2.0 ** -24)

    def hcu_coor(self, pop, hcu):
        """Pop::hcu_coor (ProcStructuralPlasticity/Pop.cpp:64-88)"""
        shape, position = self.geo[pop]
        coor, index = [], hcu
        for d in shape:
            if d <= 0:
                raise ValueError("population shape entries must be > 0")
            coor.append(index % d)
            index //= d
        for i, p in enumerate(position):
            if i < len(coor):
                coor[i] += p
            else:
                coor.append(p)
        return coor

    def delay_cycle(self, k, src_mcu, dest_hcu):
        """ProcStructuralPlasticity::delay_cycle (ProcStructuralPlasitcity.cpp:597-627)"""
        q = self.projs[k]
        a = self.hcu_coor(q["src_pop"], src_mcu // self.pops[q["src_pop"]]["mcu_num"])
        b = self.hcu_coor(q["dest_pop"], dest_hcu)
        n = max(len(a), len(b))
        a, b = a + [0] * (n - len(a)), b + [0] * (n - len(b))
        d2 = f32(0)
        for x, y in zip(a, b):
            d2 = f32(d2 + f32((x - y) * (x - y)))
        distance = f32(math.sqrt(float(d2)))
        mean = f32(f32(f32(self.d_norm * distance) / self.v_cond) + f32(1))
        u1 = 1.0 - float(self.uniform())
        u2 = float(self.uniform())
        z = math.sqrt(-2.0 * log_double(u1)) * load().oracle_cos2pi_double(u2)
        m = float(mean)
        tij = f32(m + 0.1 * m * z)
        return int(math.ceil(float(tij) * 0.001 / float(self.dt)))

    def shuffle(self, a):
        for i in range(len(a) - 1, 0, -1):
            j = min(i, int(float(self.uniform()) * (i + 1)))
            a[i], a[j] = a[j], a[i]

    def update(self, cycle_flag, simstep, plasticity):
        if cycle_flag != 1 or not plasticity:
            return
        if simstep % self.pruning_period == 0:
            self.prune(simstep)
        if simstep % self.period == 0:
            self.grow(0, int(0.2 * self.period * 100 * float(self.dt)))

    def prune(self, t):
        """Prj::prune + remove_conn for every projection, fanout given back"""
        for k, q in enumerate(self.projs):
            ii, ti, wij = self.net.read(f"ii_{k}"), self.net.read(f"ti_{k}"), self.net.read(f"wij_{k}")
            M = self.pops[q["dest_pop"]]["mcu_num"]
            w = wij.reshape(-1, M)
            strong = np.any((w >= self.wp) | (w <= self.wn), axis=1)
            removed = (ii >= 0) & ((ti < t - self.t_th) | ~strong)
            src = ii[removed].copy()
            if removed.any():
                for name, val in (("ii", -1), ("di", 0), ("ti", 0), ("pi", 0), ("ei", 0)):
                    a = self.net.read(f"{name}_{k}")
                    a[removed] = val
                    self.net.write(f"{name}_{k}", a)
                cells = np.repeat(removed, M)
                for name in ("pij", "eij", "zj2"):
                    a = self.net.read(f"{name}_{k}")
                    a[cells] = 0
                    self.net.write(f"{name}_{k}", a)
            for c in src:
                self.fanout[q["src_pop"]][c] += 1

    def grow(self, hcu_threshold, mcu_threshold):
        local, avail_hcu = [], []
        for k, q in enumerate(self.projs):
            dest, srcp = self.pops[q["dest_pop"]], self.pops[q["src_pop"]]
            H, M = dest["hcu_num"], dest["mcu_num"]
            C = min(srcp["hcu_num"] * srcp["mcu_num"], int(q["slot_num"]))
            ii = self.net.read(f"ii_{k}").copy()
            ej = self.net.read(f"ej_{k}").astype(np.float32)
            free_slot = bool(np.any(ii[:C] < 0))  # gsbn looks at HCU 0's slots for every HCU
            hcus = []
            for i in range(H):
                acc = f32(0)
                for j in range(M):
                    acc = f32(acc + ej[i * M + j])
                if acc > f32(hcu_threshold) and free_slot:
                    hcus.append(i)
            local.append(ii)
            avail_hcu.append((hcus, C))
        for pi, p in enumerate(self.pops):
            cnt = self.net.read(f".counter_{pi}")
            active = [int(i) for i in np.nonzero(cnt > mcu_threshold)[0]]
            self.net.write(f".counter_{pi}", np.zeros_like(cnt))
            prjs = list(self.out[pi])
            fan = self.fanout[pi]
            while prjs and active:
                u = self.uniform()
                idx = min(int(f32(u) * f32(len(prjs))), len(prjs) - 1)
                k = prjs[idx]
                hcus, C = avail_hcu[k]
                hcus = list(hcus)
                if not hcus:
                    break
                self.shuffle(hcus)
                for h in hcus:
                    row = local[k][h * C:(h + 1) * C]
                    taken = set(int(c) for c in row if c >= 0)
                    cand = [m for m in active if m not in taken]
                    if not cand:
                        continue
                    self.shuffle(cand)
                    l = 0
                    for s in range(C):
                        if l >= len(cand):
                            break
                        if row[s] < 0:
                            row[s] = cand[l]
                            l += 1
                    for m in cand[:l]:
                        fan[m] -= 1
                        if fan[m] <= 0:
                            active = [x for x in active if x != m]
                del prjs[idx]
        for k, q in enumerate(self.projs):
            hcus, C = avail_hcu[k]
            ii = self.net.read(f"ii_{k}").copy()
            di = self.net.read(f"di_{k}").copy()
            H = self.pops[q["dest_pop"]]["hcu_num"]
            for h in range(H):
                for s in range(C):
                    idx = h * C + s
                    if ii[idx] >= 0 or local[k][idx] < 0:
                        continue
                    free = np.nonzero(ii[h * C:(h + 1) * C] < 0)[0]
                    f = h * C + int(free[0])
                    ii[f] = local[k][idx]
                    di[f] = self.delay_cycle(k, int(local[k][idx]), h) if self.geometry else 1
            self.net.write(f"ii_{k}", ii)
            self.net.write(f"di_{k}", di)


# ---------------------------------------------------------------------------
# Solver loop (Solver.cpp:67-92, Upd.cpp:28-40)
# ---------------------------------------------------------------------------

def simulate(sp, base_dir, real_bits=32, math=MATH_SHARED, max_ticks=None, stim=None, conn_text=None,
             ext_text=None):
    """Run the procedures named in sp.proc_param (ProcExtGen, ProcUpdLazy,
    ProcExchangeSpike, ProcInitConn, ProcSpkRec, ProcCheck) in file order on
    the CPU oracle.  Returns a dict with the recorder files, the check lines
    and the oracle network."""
    from gsbn_b200 import schema  # protobuf schema only
    names = [p.name for p in sp.proc_param]
    pops, projs = net_from_solver_param(sp)
    upd = proc_args(sp, "ProcUpdLazy")
    argi, argf, args = upd if upd else ({}, {}, {})
    seed = int(argi.get("seed", 0))
    poisson_hz = float(argf.get("poisson-noise-hz", 0.0))
    net = OracleNet(pops, projs, float(f32(sp.gen_param.dt)), seed=seed, poisson_hz=poisson_hz,
                    real_bits=real_bits, math=math)
    if stim is None:
        stim = schema.read_stim(os.path.join(base_dir, sp.gen_param.stim_file))
    mcu_in_hcu = [p["mcu_num"] for p in pops for _ in range(p["hcu_num"])]
    gen = ExtGen(sp, stim, mcu_in_hcu, net.logf)
    if "ProcInitConn" in names:
        a = proc_args(sp, "ProcInitConn")
        if conn_text is None:
            with open(os.path.join(base_dir, a[2]["conn-map-file"])) as f:
                conn_text = f.read()
        for k, (ii, di) in enumerate(parse_conn_map(conn_text, pops, projs)):
            net.set_conn(k, ii, di)
    if "external spike" in args:
        if ext_text is None:
            with open(os.path.join(base_dir, args["external spike"])) as f:
                ext_text = f.read()
        for k in range(len(pops)):
            net.set_ext_spikes(k, parse_ext_spikes(ext_text, k))
    rec = None
    if "ProcSpkRec" in names:
        a = proc_args(sp, "ProcSpkRec")[0]
        rec = SpkRec(sp, pops, len(projs), a.get("offset", 0), a.get("period", 1))
    spl = None
    if "ProcStructuralPlasticity" in names:
        spl = StructuralPlasticity(sp, net, pops, projs, float(f32(sp.gen_param.dt)))
    chk = None
    if "ProcCheck" in names:
        chk = Check(sp, gen.lgidx, pops, proc_args(sp, "ProcCheck")[0].get("threashold", 0))
    ticks = 0
    while True:
        spikes_i8 = None
        for name in names:
            if name == "ProcExtGen":
                gen.tick()
                if gen.lginp_changed or gen.cycle_flag == 1:
                    net.set_stimulus(gen.lginp, gen.wmask_row())
            elif name == "ProcUpdLazy":
                if gen.cycle_flag == 1:
                    net.update(gen.simstep, gen.prn, gen.old_prn)
            elif name == "ProcExchangeSpike":
                if gen.cycle_flag == 1:
                    net.exchange()
            elif name == "ProcSpkRec" and rec is not None:
                if gen.cycle_flag == 1:
                    sp_idx = [np.nonzero(net.read(f"spike_{k}"))[0] for k in range(len(pops))]
                    flags = []
                    for k in range(len(projs)):
                        ssi = net.read(f".ssi_{k}")
                        ssj = net.read(f".ssj_{k}")
                        flags.append((bool(np.any(ssi == 9)), bool(np.any(ssj == 9))))
                    rec.update(gen.cycle_flag, gen.simstep, sp_idx, flags)
            elif name == "ProcStructuralPlasticity" and spl is not None:
                spl.update(gen.cycle_flag, gen.simstep, gen.plasticity)
            elif name == "ProcCheck" and chk is not None:
                spikes_i8 = [net.read(f"spike_{k}") for k in range(len(pops))] if gen.cycle_flag > 0 else None
                chk.update(gen.cycle_flag, gen.simstep, spikes_i8)
        ticks += 1
        if gen.cycle_flag < 0 or (max_ticks is not None and ticks >= max_ticks):
            break
    return dict(net=net, rec=rec.files() if rec else {}, check=chk.lines if chk else [],
                correct=(chk.correct, chk.pattern_num) if chk else None, simstep=gen.simstep, pops=pops,
                projs=projs)
