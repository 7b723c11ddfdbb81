"""Batches of independent networks on one GPU: ctypes binding of the batch
engine (include/bcpnn_batch.h) and the batch workload.

A batch member is a complete network of its own (one population with a full
recurrent projection, its own patterns, connectivity and Philox seed, keyed as
population 0 of a network of its own), so it draws exactly the numbers, and
computes exactly the state, it would alone.  The engine advances every member
over the same ticks in one persistent kernel per run; its launch shape (CTA
size, the cost model of the warp schedule) is chosen by its own tuner
(bcpnn_batch_tune, C++), which times the candidates on training and recall
ticks.
"""
import ctypes

import numpy as np

from . import capi, extgen, schema, workloads

BATCH_EXPORTS = (
    "bcpnn_batch_create", "bcpnn_batch_destroy", "bcpnn_batch_set_conn", "bcpnn_batch_upload_stimuli_idx",
    "bcpnn_batch_use_stimulus", "bcpnn_batch_run", "bcpnn_batch_reset", "bcpnn_batch_sync", "bcpnn_batch_get_stream",
    "bcpnn_batch_state_info", "bcpnn_batch_read_state", "bcpnn_batch_get_spike_log", "bcpnn_batch_counters",
    "bcpnn_batch_kernel_launches", "bcpnn_batch_tune", "bcpnn_batch_last_error", "bcpnn_batch_phase_probe",
)

F32 = np.float32


class Member:
    """One network of the batch: H x M, full recurrent, P patterns."""

    def __init__(self, index, hcu, mcu, seed, n_patterns=20, cue_frac=0.3):
        self.index, self.H, self.M, self.seed = index, hcu, mcu, seed
        rng = np.random.default_rng(seed)
        self.patterns = workloads.draw_patterns(rng, n_patterns, hcu, mcu)
        self.n_cued = int(np.ceil(hcu * cue_frac - 1e-9))
        stim = schema.StimRawData()
        stim.ParseFromString(workloads.stim_bytes(self.patterns, self.n_cued, hcu))
        self.lgidx, self.wmask = extgen.stim_tables(stim)
        self.C = hcu * mcu
        conn = "\n".join(workloads._hcu_conn(rng, hcu, hcu, mcu, hcu)) + "\n"
        self.pop = dict(hcu_num=hcu, mcu_num=mcu, taum=F32(0.005), wtagain=1.0, maxfq=100.0, igain=1.0, wgain=1.0,
                        lgbias=F32(workloads.LGBIAS), snoise=0.0)
        self.proj = dict(src_pop=0, dest_pop=0, tauzi=F32(0.01), tauzj=F32(0.01), taue=F32(0.02), taup=1.0,
                         maxfq=100.0, bgain=1.0, wgain=1.0, tauepsc=0.0, slot_num=float(self.C))
        self.ii, self.di = workloads.read_conn_map(conn, [self.pop], [self.proj])[0]
        self.cells = hcu * self.C * mcu


def make_members(n=256, seed=0, hcu=(8, 64), mcu=(5, 50), n_patterns=20):
    """B networks with HCU and MCU counts drawn uniformly (inclusive) and
    per-network seeds."""
    rng = np.random.default_rng(seed)
    hs = rng.integers(hcu[0], hcu[1] + 1, n)
    ms = rng.integers(mcu[0], mcu[1] + 1, n)
    return [Member(i, int(hs[i]), int(ms[i]), seed * 100003 + i + 1, n_patterns) for i in range(n)]


def schedule(n_patterns, train_ticks=100, recall_ticks=50):
    """(first, n, prn, old_prn, lgidx_row, wmask_row) runs: every pattern
    trained, then every pattern recalled from its cue (rows as stim_bytes lays
    them out)."""
    runs, t, prn = [], 1, 0.0
    for k in range(n_patterns):
        runs.append((t, train_ticks, 1.0, prn, k, 0))
        prn = 1.0
        t += train_ticks
    for k in range(n_patterns):
        runs.append((t, recall_ticks, 0.0, prn, n_patterns + k, 1))
        prn = 0.0
        t += recall_ticks
    return runs


class MemberDesc(ctypes.Structure):
    _fields_ = [("pop", capi.PopDesc), ("proj", capi.ProjDesc), ("seed", ctypes.c_uint32)]


class BatchDesc(ctypes.Structure):
    _fields_ = [("n_members", ctypes.c_int32), ("members", ctypes.POINTER(MemberDesc)), ("dt", ctypes.c_float),
                ("poisson_noise_hz", ctypes.c_float), ("device", ctypes.c_int32),
                ("max_ticks_per_run", ctypes.c_int32), ("threads", ctypes.c_int32),
                ("lpt_weights", ctypes.c_int32 * 3)]


_lib = None


def load():
    global _lib
    if _lib is not None:
        return _lib
    lib = capi.load()
    vp, i32, sz = ctypes.c_void_p, ctypes.c_int32, ctypes.c_size_t
    P = ctypes.POINTER
    sig = {
        "bcpnn_batch_create": (ctypes.c_int, [P(BatchDesc), P(vp)]),
        "bcpnn_batch_destroy": (ctypes.c_int, [vp]),
        "bcpnn_batch_set_conn": (ctypes.c_int, [vp, i32, vp, vp, sz]),
        "bcpnn_batch_upload_stimuli_idx": (ctypes.c_int, [vp, i32, i32, vp, ctypes.c_float, i32, vp]),
        "bcpnn_batch_use_stimulus": (ctypes.c_int, [vp, i32, i32]),
        "bcpnn_batch_run": (ctypes.c_int, [vp, i32, i32, ctypes.c_float, ctypes.c_float]),
        "bcpnn_batch_reset": (ctypes.c_int, [vp]),
        "bcpnn_batch_sync": (ctypes.c_int, [vp]),
        "bcpnn_batch_get_stream": (ctypes.c_int, [vp, P(vp)]),
        "bcpnn_batch_state_info": (ctypes.c_int, [vp, i32, ctypes.c_char_p, P(i32), P(sz)]),
        "bcpnn_batch_read_state": (ctypes.c_int, [vp, i32, ctypes.c_char_p, vp, sz]),
        "bcpnn_batch_get_spike_log": (ctypes.c_int, [vp, i32, vp, sz]),
        "bcpnn_batch_counters": (ctypes.c_int, [vp, P(ctypes.c_uint64)]),
        "bcpnn_batch_kernel_launches": (ctypes.c_int, [vp, P(ctypes.c_uint64)]),
        "bcpnn_batch_tune": (ctypes.c_int, [vp, i32, i32, i32, i32, i32, P(i32), P(ctypes.c_float)]),
        "bcpnn_batch_last_error": (ctypes.c_char_p, [vp]),
        "bcpnn_batch_phase_probe": (ctypes.c_int, [vp, vp, i32, P(i32), i32]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class BatchEngine:
    """The members on one GPU, driven through the batch C ABI."""

    def __init__(self, members, dt=0.001, eps=1e-4, device=0, max_ticks=128, threads=512, lpt=(0, 0, 0),
                 poisson_hz=0.0):
        self._lib = load()
        self._h = ctypes.c_void_p()
        self.members = members
        arr = (MemberDesc * len(members))(*[MemberDesc(capi.PopDesc(**m.pop), capi.ProjDesc(**m.proj), m.seed)
                                            for m in members])
        self._arr = arr
        d = BatchDesc(len(members), arr, dt, poisson_hz, device, max_ticks, threads, (ctypes.c_int32 * 3)(*lpt))
        rc = self._lib.bcpnn_batch_create(ctypes.byref(d), ctypes.byref(self._h))
        if rc != 0:
            msg = self._lib.bcpnn_batch_last_error(self._h).decode() if self._h else ""
            if self._h:
                self._lib.bcpnn_batch_destroy(self._h)
                self._h = ctypes.c_void_p()
            raise capi.BcpnnError(rc, msg or self._lib.bcpnn_status_string(rc).decode())
        for i, m in enumerate(members):
            ii = np.ascontiguousarray(m.ii, np.int32)
            di = np.ascontiguousarray(m.di, np.int32)
            self._check(self._lib.bcpnn_batch_set_conn(self._h, i, _p(ii), _p(di), ii.size))
            lg = np.ascontiguousarray(m.lgidx, np.int32)
            wm = np.ascontiguousarray(m.wmask, np.float32)
            self._check(self._lib.bcpnn_batch_upload_stimuli_idx(self._h, i, lg.shape[0], _p(lg), eps, wm.shape[0],
                                                                 _p(wm)))
        self.last_ticks = 0

    def _check(self, rc):
        if rc != 0:
            raise capi.BcpnnError(rc, self._lib.bcpnn_batch_last_error(self._h).decode())

    def run_segment(self, first, n, prn, old_prn, lg_row, wm_row):
        self._check(self._lib.bcpnn_batch_use_stimulus(self._h, lg_row, wm_row))
        self._check(self._lib.bcpnn_batch_run(self._h, first, n, prn, old_prn))
        self.last_ticks = n

    def reset(self):
        self._check(self._lib.bcpnn_batch_reset(self._h))

    def sync(self):
        self._check(self._lib.bcpnn_batch_sync(self._h))

    def stream(self):
        s = ctypes.c_void_p()
        self._check(self._lib.bcpnn_batch_get_stream(self._h, ctypes.byref(s)))
        return s.value

    def read(self, member, name):
        t, n = ctypes.c_int32(), ctypes.c_size_t()
        self._check(self._lib.bcpnn_batch_state_info(self._h, member, name.encode(), ctypes.byref(t), ctypes.byref(n)))
        out = np.zeros(n.value, dtype={0: np.float32, 1: np.int32, 2: np.int8}[t.value])
        self._check(self._lib.bcpnn_batch_read_state(self._h, member, name.encode(), _p(out), out.nbytes))
        return out

    def spike_log(self, member):
        m = self.members[member]
        words = (m.H * m.M + 31) // 32
        out = np.zeros((self.last_ticks, words), np.uint32)
        self._check(self._lib.bcpnn_batch_get_spike_log(self._h, member, _p(out), out.size))
        return out

    def counters(self):
        c = (ctypes.c_uint64 * 3)()
        self._check(self._lib.bcpnn_batch_counters(self._h, c))
        return [int(c[0]), int(c[1]), int(c[2])]

    def launches(self):
        c = ctypes.c_uint64()
        self._check(self._lib.bcpnn_batch_kernel_launches(self._h, ctypes.byref(c)))
        return int(c.value)

    def tune(self, probe_ticks, train_rows=(0, 0), recall_rows=(1, 1)):
        """the engine's tuner: ((threads, w0, w1, w2), us per tick); leaves the
        batch reset under the chosen shape"""
        out = (ctypes.c_int32 * 4)()
        us = ctypes.c_float()
        self._check(self._lib.bcpnn_batch_tune(self._h, probe_ticks, train_rows[0], train_rows[1], recall_rows[0],
                                               recall_rows[1], out, ctypes.byref(us)))
        return tuple(int(v) for v in out), float(us.value)

    def phase_probe(self, reset=True):
        """uint64 [CTAs, 32] batch-kernel phase counters (library built with
        BCPNN_PHASE_PROBE; see bcpnn_batch_phase_probe)"""
        n = ctypes.c_int32()
        self._check(self._lib.bcpnn_batch_phase_probe(self._h, None, 0, ctypes.byref(n), 0))
        out = np.zeros((n.value, 32), np.uint64)
        self._check(self._lib.bcpnn_batch_phase_probe(self._h, _p(out), n.value, ctypes.byref(n), 1 if reset else 0))
        return out

    def close(self):
        if self._h:
            self._lib.bcpnn_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Plain:
    """The same members as networks of their own through the single-network C
    ABI, one after the other (one network per launch): the comparison path."""

    def __init__(self, members, dt=0.001, eps=1e-4, device=0, max_ticks=128):
        self.members = members
        self.nets = []
        for m in members:
            net = capi.Net([m.pop], [m.proj], dt, seed=m.seed, device=device, max_ticks=max_ticks)
            net.set_conn(0, m.ii, m.di)
            net.upload_stimuli_idx(m.lgidx, eps, m.wmask)
            self.nets.append(net)

    def run_segment(self, first, n, prn, old_prn, lg_row, wm_row):
        for net in self.nets:
            net.use_stimulus(lg_row, wm_row)
            net.run(first, n, prn, old_prn)

    def sync(self):
        for net in self.nets:
            net.sync()

    def reset(self):
        for net in self.nets:
            net.reset()

    def counters(self):
        return sum(sum(net.counters()) for net in self.nets)

    def close(self):
        for net in self.nets:
            net.close()
