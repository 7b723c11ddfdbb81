"""ctypes binding of the replicate recall engine (include/bcpnn_recall.h) and
the host steps around it: take a trained network from the plain path, build
W (w_ij by source MCU x destination MCU, after the prn-change catch-up), b_j
and the end-of-training state, and hand them to the engine.
"""
import ctypes

import numpy as np

from . import capi

RECALL_EXPORTS = (
    "bcpnn_recall_create", "bcpnn_recall_destroy", "bcpnn_recall_load", "bcpnn_recall_set_cues", "bcpnn_recall_run",
    "bcpnn_recall_clear_counts", "bcpnn_recall_read", "bcpnn_recall_write", "bcpnn_recall_get_stream",
    "bcpnn_recall_launches", "bcpnn_recall_last_error", "bcpnn_recall_timing", "bcpnn_recall_contraction_time",
)


class RecallDesc(ctypes.Structure):
    _fields_ = [("hcu_num", ctypes.c_int32), ("mcu_num", ctypes.c_int32), ("replicates", ctypes.c_int32),
                ("pop", capi.PopDesc), ("dt", ctypes.c_float), ("kepsc", ctypes.c_float),
                ("seed_base", ctypes.c_uint32), ("poisson_noise_hz", ctypes.c_float), ("device", ctypes.c_int32),
                ("contraction", ctypes.c_int32)]


CONTRACTIONS = {"bf16": 0, "fp32": 1}


_lib = None


def load():
    global _lib
    if _lib is not None:
        return _lib
    lib = capi.load()
    vp, i32, sz = ctypes.c_void_p, ctypes.c_int32, ctypes.c_size_t
    P = ctypes.POINTER
    sig = {
        "bcpnn_recall_create": (ctypes.c_int, [P(RecallDesc), P(vp)]),
        "bcpnn_recall_destroy": (ctypes.c_int, [vp]),
        "bcpnn_recall_load": (ctypes.c_int, [vp, vp, vp, vp, vp, vp, vp, vp]),
        "bcpnn_recall_set_cues": (ctypes.c_int, [vp, vp, ctypes.c_float, vp]),
        "bcpnn_recall_run": (ctypes.c_int, [vp, i32, i32, i32, i32]),
        "bcpnn_recall_clear_counts": (ctypes.c_int, [vp]),
        "bcpnn_recall_read": (ctypes.c_int, [vp, ctypes.c_char_p, i32, i32, vp, sz]),
        "bcpnn_recall_write": (ctypes.c_int, [vp, ctypes.c_char_p, i32, i32, vp, sz]),
        "bcpnn_recall_get_stream": (ctypes.c_int, [vp, P(vp)]),
        "bcpnn_recall_launches": (ctypes.c_int, [vp, P(ctypes.c_uint64)]),
        "bcpnn_recall_last_error": (ctypes.c_char_p, [vp]),
        "bcpnn_recall_timing": (ctypes.c_int, [vp, i32]),
        "bcpnn_recall_contraction_time": (ctypes.c_int, [vp, P(ctypes.c_double), P(ctypes.c_uint64)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class Recall:
    """R replicates of one trained population on one GPU; `contraction` is
    "bf16" (tensor cores, W rounded to BF16) or "fp32" (SIMT, W in FP32)."""

    def __init__(self, hcu, mcu, replicates, pop, dt, kepsc, seed_base=0, poisson_hz=0.0, device=0,
                 contraction="bf16"):
        self._lib = load()
        self._h = ctypes.c_void_p()
        self.H, self.M, self.R, self.N = hcu, mcu, replicates, hcu * mcu
        self.contraction = contraction
        d = RecallDesc(hcu, mcu, replicates, capi.PopDesc(**pop), dt, kepsc, seed_base, poisson_hz, device,
                       CONTRACTIONS[contraction])
        rc = self._lib.bcpnn_recall_create(ctypes.byref(d), ctypes.byref(self._h))
        if rc != 0:
            raise capi.BcpnnError(rc, self._lib.bcpnn_status_string(rc).decode())

    def _check(self, rc):
        if rc != 0:
            raise capi.BcpnnError(rc, self._lib.bcpnn_recall_last_error(self._h).decode())

    def load_state(self, w, bj, epsc, dsup, s_tm3, s_tm2, s_tm1):
        N = self.N
        arrs = [np.ascontiguousarray(w, np.float32).reshape(N * N)] + \
            [np.ascontiguousarray(a, np.float32).reshape(N) for a in (bj, epsc, dsup)] + \
            [np.ascontiguousarray(a, np.int8).reshape(N) for a in (s_tm3, s_tm2, s_tm1)]
        self._check(self._lib.bcpnn_recall_load(self._h, *[_p(a) for a in arrs]))

    def set_cues(self, lgidx, eps, wmask):
        lg = np.ascontiguousarray(lgidx, np.int32).reshape(self.R * self.H)
        wm = np.ascontiguousarray(wmask, np.float32).reshape(self.R * self.H)
        self._check(self._lib.bcpnn_recall_set_cues(self._h, _p(lg), eps, _p(wm)))

    def run(self, first, n, count_first=0, count_last=-1):
        self._check(self._lib.bcpnn_recall_run(self._h, first, n, count_first, count_last))

    def clear_counts(self):
        self._check(self._lib.bcpnn_recall_clear_counts(self._h))

    def read(self, name, row0=0, n_rows=None):
        n_rows = self.R - row0 if n_rows is None else n_rows
        dt = {"dsup": np.float32, "epsc": np.float32, "counts": np.uint8}.get(name, np.int8)
        out = np.zeros((n_rows, self.N), dt)
        self._check(self._lib.bcpnn_recall_read(self._h, name.encode(), row0, n_rows, _p(out), out.nbytes))
        return out

    def write(self, name, arr, row0=0):
        dt = np.float32 if name in ("dsup", "epsc") else np.int8
        a = np.ascontiguousarray(arr, dt).reshape(-1, self.N)
        self._check(self._lib.bcpnn_recall_write(self._h, name.encode(), row0, a.shape[0], _p(a), a.nbytes))

    def stream(self):
        s = ctypes.c_void_p()
        self._check(self._lib.bcpnn_recall_get_stream(self._h, ctypes.byref(s)))
        return s.value

    def launches(self):
        v = ctypes.c_uint64()
        self._check(self._lib.bcpnn_recall_launches(self._h, ctypes.byref(v)))
        return v.value

    def timing(self, on=True):
        """switch the in-place timing of the contraction launches (clears the sums)"""
        self._check(self._lib.bcpnn_recall_timing(self._h, 1 if on else 0))

    def contraction_time(self):
        """(summed milliseconds, launches) of the timed contraction launches"""
        ms, n = ctypes.c_double(), ctypes.c_uint64()
        self._check(self._lib.bcpnn_recall_contraction_time(self._h, ctypes.byref(ms), ctypes.byref(n)))
        return ms.value, n.value

    def close(self):
        if self._h:
            self._lib.bcpnn_recall_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def kepsc_of(proj, dt):
    """the projection's epsc decay rate as the library computes it"""
    dt = np.float32(dt)
    if proj.get("tauepsc", 0.0) and proj["tauepsc"] > 0:
        return float(dt / np.float32(proj["tauepsc"]))
    return float(dt / np.float32(proj["tauzi"]))


def slot_sources(net, H, C):
    """ii of the slots of every destination HCU; each must be a permutation of
    the source MCUs (full connectivity) with delay 1."""
    ii = net.read("ii_0").reshape(H, C)
    di = net.read("di_0").reshape(H, C)
    N = C
    for h in range(H):
        if not np.array_equal(np.sort(ii[h]), np.arange(N)):
            raise ValueError("replicate recall needs one slot per source MCU in every destination HCU")
    if np.any(di != 1):
        raise ValueError("replicate recall needs delay 1 on every slot")
    return ii


def end_of_training_state(net, H, M):
    """State at the end of the last training tick, by source MCU: epsc, dsup,
    bj and the spikes of the last three ticks (.siq, qi bit 0, si)."""
    N = H * M
    ii = slot_sources(net, H, N)[0]
    qi = net.read("qi_0")[:N]
    siq = net.read(".siq_0")[:N]
    s_tm3 = np.zeros(N, np.int8)
    s_tm2 = np.zeros(N, np.int8)
    s_tm3[ii] = (siq != 0).astype(np.int8)
    s_tm2[ii] = (qi & 1).astype(np.int8)
    s_tm1 = (net.read("si_0") != 0).astype(np.int8)
    return dict(epsc=net.read("epsc_0"), dsup=net.read("dsup_0"), bj=net.read("bj_0"), s_tm3=s_tm3, s_tm2=s_tm2,
                s_tm1=s_tm1)


def weights_by_source(net, H, M):
    """W[i, j] = w_ij of the slot of destination HCU j // M holding source MCU
    i (row-major [source][destination])."""
    N = H * M
    ii = slot_sources(net, H, N)
    wij = net.read("wij_0").reshape(H, N, M)  # [dest HCU][slot][dest MCU]
    W = np.empty((N, N), np.float32)
    for h in range(H):
        W[ii[h], h * M:(h + 1) * M] = wij[h]
    return W


class Trained:
    """A network trained on the plain FP32 path, stopped before its first
    recall segment (tick t0)."""

    def __init__(self, work, directory, device=0, max_ticks=1024):
        import os
        from . import extgen, schema, workloads
        path = work.write(directory)
        with open(path) as f:
            sp = schema.parse_prototxt(f.read())
        self.sp = sp
        self.pops, self.projs = workloads.net_from_solver_param(sp)
        if len(self.pops) != 1 or len(self.projs) != 1:
            raise ValueError("replicate recall takes one population with one projection")
        upd = [p for p in sp.proc_param if p.name == "ProcUpdLazy"][0]
        seed = {a.key: a.val for a in upd.argi}.get("seed", 0)
        self.poisson_hz = float({a.key: a.val for a in upd.argf}.get("poisson-noise-hz", 0.0))
        self.dt = float(np.float32(sp.gen_param.dt))
        self.eps = float(np.float32(sp.gen_param.eps))
        self.H, self.M = self.pops[0]["hcu_num"], self.pops[0]["mcu_num"]
        self.net = capi.Net(self.pops, self.projs, self.dt, seed=seed, poisson_hz=self.poisson_hz, device=device,
                            max_ticks=max_ticks)
        conn = [p for p in sp.proc_param if p.name == "ProcInitConn"][0]
        with open({a.key: a.val for a in conn.args}["conn-map-file"]) as f:
            for k, (ii, di) in enumerate(workloads.read_conn_map(f.read(), self.pops, self.projs)):
                self.net.set_conn(k, ii, di)
        self.lgidx, self.wmask = extgen.stim_tables(schema.read_stim(sp.gen_param.stim_file))
        self.net.upload_stimuli_idx(self.lgidx, self.eps, self.wmask)
        runs = extgen.segments(sp)
        k = next(i for i, r in enumerate(runs) if r.prn == 0.0)
        self.train_runs, self.recall_runs = runs[:k], runs[k:]
        for r in self.train_runs:
            self.net.use_stimulus(r.lgidx, r.wmask)
            self.net.run(r.first, r.n, r.prn, r.old_prn)
        self.t0 = self.recall_runs[0].first
        self.old_prn = self.recall_runs[0].old_prn
        self.n_patterns = work.meta["patterns"]
        self.n_cued = work.meta["n_cued"]

    def snapshot(self, names):
        """named state vectors at the end of training"""
        return {n: self.net.read(n) for n in names}

    def recall_inputs(self):
        """(W, end-of-training state): the state is read first, then the
        first recall tick runs on the plain network, whose prn-change catch-up
        leaves w_ij as every recall tick uses it."""
        st = end_of_training_state(self.net, self.H, self.M)
        r = self.recall_runs[0]
        self.net.use_stimulus(r.lgidx, r.wmask)
        self.net.run(self.t0, 1, 0.0, self.old_prn)
        return weights_by_source(self.net, self.H, self.M), st

    def cues(self, replicates):
        """replicate r recalls pattern r % P from its cue row (first n_cued
        HCUs) with the recall mask"""
        P = self.n_patterns
        lg = np.stack([self.lgidx[P + (r % P)] for r in range(replicates)]).astype(np.int32)
        wm = np.stack([self.wmask[1]] * replicates).astype(np.float32)
        expected = np.stack([self.lgidx[r % P] for r in range(replicates)]).astype(np.int32)
        return lg, wm, expected


def hcu_accuracy(counts, H, M, expected):
    """per replicate row: the fraction of cued-pattern HCUs (expected >= 0)
    whose most-spiking MCU (first on ties, none if silent) is the expected
    one -- a graded view of the decision ProcCheck takes over all HCUs"""
    c = counts.reshape(counts.shape[0], H, M).astype(np.int64)
    mx = c.max(axis=2)
    idx = np.where(mx > 0, c.argmax(axis=2), -1)
    exp = expected.astype(np.int64)
    valid = exp >= 0
    return ((idx == exp) & valid).sum(axis=1) / np.maximum(valid.sum(axis=1), 1)


def recall_decisions(counts, H, M, expected, threshold=0):
    """ProcCheck's per-segment decision (ProcCheck.cpp:185-199, Pop.cpp:35-52)
    for each replicate row: most-spiking MCU per HCU (first on ties, -1 if
    none) against the expected pattern."""
    c = counts.reshape(counts.shape[0], H, M).astype(np.int64)
    mx = c.max(axis=2)
    idx = np.where(mx > 0, c.argmax(axis=2), -1)
    exp = expected.astype(np.int64)
    bad = (((mx < threshold) | (idx != exp)) & (exp >= 0)) | ((mx > threshold) & (exp < 0))
    return ~bad.any(axis=1)
