"""ctypes binding of libgsbn_b200.so (include/bcpnn.h).

Thin and loud: every non-zero status raises BcpnnError with the library's own
message.  There is no CPU fallback: if the shared library is missing or no
CUDA device can be opened, the calls fail.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# the library; GSBN_B200_LIB selects another build of it (the phase-probe
# build, gsbn_b200/libgsbn_b200_probe.so)
LIB_PATH = os.environ.get("GSBN_B200_LIB") or os.path.join(_HERE, "libgsbn_b200.so")

F32, I32, I8 = 0, 1, 2
_NP = {F32: np.float32, I32: np.int32, I8: np.int8}

# every entry point declared in include/bcpnn.h
EXPORTS = (
    "bcpnn_net_create", "bcpnn_net_destroy", "bcpnn_set_conn", "bcpnn_set_stimulus", "bcpnn_upload_stimuli",
    "bcpnn_use_stimulus", "bcpnn_set_stimulus_idx", "bcpnn_upload_stimuli_idx", "bcpnn_upload_stimuli_idx_async", "bcpnn_set_ext_spikes", "bcpnn_reset", "bcpnn_get_stream",
    "bcpnn_run", "bcpnn_sync", "bcpnn_spike_log_words", "bcpnn_get_spike_log", "bcpnn_get_spike_log_async", "bcpnn_check_count",
    "bcpnn_check_result_async", "bcpnn_get_ss_flags",
    "bcpnn_state_info", "bcpnn_read_state", "bcpnn_write_state", "bcpnn_read_state_noalloc", "bcpnn_counters", "bcpnn_kernel_launches",
    "bcpnn_selftest_barrier_timeout", "bcpnn_selftest_division", "bcpnn_phase_probe", "bcpnn_set_pop_rng", "bcpnn_prune",
    "bcpnn_last_error",
    "bcpnn_status_string",
)


class BcpnnError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"bcpnn status {status}: {message}")
        self.status = status


class PopDesc(ctypes.Structure):
    _fields_ = [("hcu_num", ctypes.c_int32), ("mcu_num", ctypes.c_int32), ("taum", ctypes.c_float),
                ("wtagain", ctypes.c_float), ("maxfq", ctypes.c_float), ("igain", ctypes.c_float),
                ("wgain", ctypes.c_float), ("lgbias", ctypes.c_float), ("snoise", ctypes.c_float),
                ("taua", ctypes.c_float), ("adgain", ctypes.c_float)]


class ProjDesc(ctypes.Structure):
    _fields_ = [("src_pop", ctypes.c_int32), ("dest_pop", ctypes.c_int32), ("tauzi", ctypes.c_float),
                ("tauzj", ctypes.c_float), ("taue", ctypes.c_float), ("taup", ctypes.c_float),
                ("maxfq", ctypes.c_float), ("bgain", ctypes.c_float), ("wgain", ctypes.c_float),
                ("tauepsc", ctypes.c_float), ("slot_num", ctypes.c_float)]


class NetDesc(ctypes.Structure):
    _fields_ = [("n_pops", ctypes.c_int32), ("pops", ctypes.POINTER(PopDesc)), ("n_projs", ctypes.c_int32),
                ("projs", ctypes.POINTER(ProjDesc)), ("dt", ctypes.c_float), ("seed", ctypes.c_uint32),
                ("poisson_noise_hz", ctypes.c_float), ("exchange_spikes", ctypes.c_int32),
                ("device", ctypes.c_int32), ("max_ticks_per_run", ctypes.c_int32), ("tick_threads", ctypes.c_int32),
                ("fp64_tables", ctypes.c_int32), ("update_variant", ctypes.c_int32),
                ("spike_buffer_size", ctypes.c_int32)]


_lib = None


def load():
    """Load the shared library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise OSError(f"{LIB_PATH} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'`")
    lib = ctypes.CDLL(LIB_PATH)
    vp, i32, sz = ctypes.c_void_p, ctypes.c_int32, ctypes.c_size_t
    P = ctypes.POINTER
    sig = {
        "bcpnn_net_create": (ctypes.c_int, [P(NetDesc), P(vp)]),
        "bcpnn_net_destroy": (ctypes.c_int, [vp]),
        "bcpnn_set_conn": (ctypes.c_int, [vp, i32, vp, vp, sz]),
        "bcpnn_set_stimulus": (ctypes.c_int, [vp, vp, sz, vp, sz]),
        "bcpnn_upload_stimuli": (ctypes.c_int, [vp, i32, vp, i32, vp]),
        "bcpnn_use_stimulus": (ctypes.c_int, [vp, i32, i32]),
        "bcpnn_set_stimulus_idx": (ctypes.c_int, [vp, vp, sz, ctypes.c_float, vp, sz]),
        "bcpnn_upload_stimuli_idx": (ctypes.c_int, [vp, i32, vp, ctypes.c_float, i32, vp]),
        "bcpnn_upload_stimuli_idx_async": (ctypes.c_int, [vp, i32, vp, ctypes.c_float, i32, vp]),
        "bcpnn_set_ext_spikes": (ctypes.c_int, [vp, i32, i32, vp, vp, vp]),
        "bcpnn_reset": (ctypes.c_int, [vp]),
        "bcpnn_get_stream": (ctypes.c_int, [vp, P(vp)]),
        "bcpnn_run": (ctypes.c_int, [vp, i32, i32, ctypes.c_float, ctypes.c_float]),
        "bcpnn_phase_probe": (ctypes.c_int, [vp, vp, i32, P(i32), i32]),
        "bcpnn_sync": (ctypes.c_int, [vp]),
        "bcpnn_spike_log_words": (ctypes.c_int, [vp, i32, P(i32)]),
        "bcpnn_get_spike_log": (ctypes.c_int, [vp, i32, vp, sz]),
        "bcpnn_get_spike_log_async": (ctypes.c_int, [vp, i32, vp, sz]),
        "bcpnn_check_count": (ctypes.c_int, [vp, i32, i32, i32]),
        "bcpnn_check_result_async": (ctypes.c_int, [vp, i32, vp, vp, sz]),
        "bcpnn_get_ss_flags": (ctypes.c_int, [vp, vp, sz]),
        "bcpnn_state_info": (ctypes.c_int, [vp, ctypes.c_char_p, P(i32), P(sz)]),
        "bcpnn_read_state": (ctypes.c_int, [vp, ctypes.c_char_p, vp, sz]),
        "bcpnn_write_state": (ctypes.c_int, [vp, ctypes.c_char_p, vp, sz]),
        "bcpnn_read_state_noalloc": (ctypes.c_int, [vp, ctypes.c_char_p, vp, sz]),
        "bcpnn_counters": (ctypes.c_int, [vp, P(ctypes.c_uint64)]),
        "bcpnn_kernel_launches": (ctypes.c_int, [vp, P(ctypes.c_uint64)]),
        "bcpnn_selftest_barrier_timeout": (ctypes.c_int, [vp, ctypes.c_int64]),
        "bcpnn_selftest_division": (ctypes.c_int, [vp, ctypes.c_uint64, ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64),
                                                   ctypes.POINTER(ctypes.c_uint64)]),
        "bcpnn_set_pop_rng": (ctypes.c_int, [vp, i32, ctypes.c_uint32, ctypes.c_uint32]),
        "bcpnn_prune": (ctypes.c_int, [vp, i32, i32, ctypes.c_float, ctypes.c_float, vp, sz, P(i32)]),
        "bcpnn_last_error": (ctypes.c_char_p, [vp]),
        "bcpnn_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _out_buffer(a, dtype):
    """A caller's array that the library writes into by element count: it
    must be a writable C-contiguous array of exactly that element type, or
    the copy would write past its end."""
    if not isinstance(a, np.ndarray) or a.dtype != dtype or not a.flags.c_contiguous or not a.flags.writeable:
        raise ValueError(f"expected a writable C-contiguous {np.dtype(dtype).name} array")


class Net:
    """One network on one GPU, driven through the C ABI."""

    def __init__(self, pops, projs, dt, seed=0, poisson_hz=0.0, exchange=True, device=0, max_ticks=1024,
                 tick_threads=0, fp64_tables=0, variant=0, spike_buffer=1):
        """variant 0: ProcUpdLazy; 1: ProcUpdMulti with a ring of `spike_buffer`
        ticks (populations then need taua and adgain)"""
        self._lib = load()
        self._h = ctypes.c_void_p()
        self.n_pops, self.n_projs = len(pops), len(projs)
        self._pops = (PopDesc * max(1, len(pops)))(*[PopDesc(**p) for p in pops])
        self._projs = (ProjDesc * max(1, len(projs)))(*[ProjDesc(**p) for p in projs])
        desc = NetDesc(len(pops), self._pops, len(projs), self._projs, dt, seed, poisson_hz, 1 if exchange else 0,
                       device, max_ticks, tick_threads, fp64_tables, variant, spike_buffer)
        rc = self._lib.bcpnn_net_create(ctypes.byref(desc), ctypes.byref(self._h))
        if rc != 0:
            msg = self._lib.bcpnn_last_error(self._h).decode() if self._h else ""
            if self._h:
                self._lib.bcpnn_net_destroy(self._h)
                self._h = ctypes.c_void_p()
            raise BcpnnError(rc, msg or self._lib.bcpnn_status_string(rc).decode())
        self.last_ticks = 0

    def _check(self, rc):
        if rc != 0:
            raise BcpnnError(rc, self._lib.bcpnn_last_error(self._h).decode())

    def close(self):
        if self._h:
            self._lib.bcpnn_net_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_conn(self, proj, ii, di):
        ii = np.ascontiguousarray(ii, dtype=np.int32)
        di = np.ascontiguousarray(di, dtype=np.int32)
        self._check(self._lib.bcpnn_set_conn(self._h, proj, _ptr(ii), _ptr(di), ii.size))

    def set_stimulus(self, lginp, wmask_row):
        lg = np.ascontiguousarray(lginp, dtype=np.float32)
        wm = np.ascontiguousarray(wmask_row, dtype=np.float32)
        self._check(self._lib.bcpnn_set_stimulus(self._h, _ptr(lg), lg.size, _ptr(wm), wm.size))

    def upload_stimuli(self, lginp_rows, wmask_rows):
        lg = np.ascontiguousarray(lginp_rows, dtype=np.float32)
        wm = np.ascontiguousarray(wmask_rows, dtype=np.float32)
        self._check(self._lib.bcpnn_upload_stimuli(self._h, lg.shape[0], _ptr(lg), wm.shape[0], _ptr(wm)))

    def set_stimulus_idx(self, lgidx_row, eps, wmask_row):
        lg = np.ascontiguousarray(lgidx_row, dtype=np.int32)
        wm = np.ascontiguousarray(wmask_row, dtype=np.float32)
        self._check(self._lib.bcpnn_set_stimulus_idx(self._h, _ptr(lg), lg.size, eps, _ptr(wm), wm.size))

    def upload_stimuli_idx(self, lgidx_rows, eps, wmask_rows):
        lg = np.ascontiguousarray(lgidx_rows, dtype=np.int32)
        wm = np.ascontiguousarray(wmask_rows, dtype=np.float32)
        self._check(self._lib.bcpnn_upload_stimuli_idx(self._h, lg.shape[0], _ptr(lg), eps, wm.shape[0], _ptr(wm)))

    def upload_stimuli_idx_async(self, lgidx_rows, eps, wmask_rows):
        """the tables of upload_stimuli_idx, queued on the network's stream;
        page-locked arrays are read when the stream reaches the copies, so
        the caller keeps them unchanged until sync()"""
        lg = np.ascontiguousarray(lgidx_rows, dtype=np.int32)
        wm = np.ascontiguousarray(wmask_rows, dtype=np.float32)
        if lg.ndim != 2 or wm.ndim != 2:
            raise ValueError("tables of rows expected")
        self._check(self._lib.bcpnn_upload_stimuli_idx_async(self._h, lg.shape[0], _ptr(lg), eps, wm.shape[0],
                                                             _ptr(wm)))

    def use_stimulus(self, lginp_row, wmask_row):
        self._check(self._lib.bcpnn_use_stimulus(self._h, lginp_row, wmask_row))

    def reset(self):
        self._check(self._lib.bcpnn_reset(self._h))

    def stream(self):
        s = ctypes.c_void_p()
        self._check(self._lib.bcpnn_get_stream(self._h, ctypes.byref(s)))
        return s.value

    def set_ext_spikes(self, pop, table):
        """table: dict tick -> list of MCU indices."""
        ticks = np.array(sorted(table), dtype=np.int32)
        offs, flat = [0], []
        for t in ticks:
            flat.extend(table[int(t)])
            offs.append(len(flat))
        offs = np.array(offs, dtype=np.int32)
        flat = np.array(flat if flat else [0], dtype=np.int32)
        self._check(self._lib.bcpnn_set_ext_spikes(self._h, pop, len(ticks), _ptr(ticks), _ptr(offs), _ptr(flat)))

    def run(self, first_simstep, n_ticks, prn, old_prn):
        self._check(self._lib.bcpnn_run(self._h, first_simstep, n_ticks, prn, old_prn))
        self.last_ticks = n_ticks

    def phase_probe(self, reset=True):
        """uint64 [CTAs, 32] tick-kernel phase counters (library built with
        BCPNN_PHASE_PROBE; see bcpnn_phase_probe)"""
        n = ctypes.c_int32()
        self._check(self._lib.bcpnn_phase_probe(self._h, None, 0, ctypes.byref(n), 0))
        out = np.zeros((n.value, 32), np.uint64)
        self._check(self._lib.bcpnn_phase_probe(self._h, _ptr(out), n.value, ctypes.byref(n), 1 if reset else 0))
        return out

    def sync(self):
        self._check(self._lib.bcpnn_sync(self._h))

    def spike_log(self, pop):
        """uint32 [ticks of the last run, words] spike bitmask."""
        w = ctypes.c_int32()
        self._check(self._lib.bcpnn_spike_log_words(self._h, pop, ctypes.byref(w)))
        out = np.zeros((self.last_ticks, w.value), dtype=np.uint32)
        self._check(self._lib.bcpnn_get_spike_log(self._h, pop, _ptr(out), out.size))
        return out

    def spike_log_async(self, pop, out):
        """Queue the copy of the last run's spike log of `pop` into `out`
        (uint32 [ticks, words], page-locked for an asynchronous copy); `out`
        is complete after the next sync()."""
        _out_buffer(out, np.uint32)
        self._check(self._lib.bcpnn_get_spike_log_async(self._h, pop, _ptr(out), out.size))

    def check_count(self, pop, k0, k1):
        """add the spikes of ticks k0..k1-1 of the last run to `pop`'s recall counters"""
        self._check(self._lib.bcpnn_check_count(self._h, pop, int(k0), int(k1)))

    def check_result_async(self, pop, idx, cnt):
        """queue per-HCU (first most-spiking MCU or -1, its count) of `pop`
        into int32 idx/cnt and clear the counters; complete after sync()"""
        _out_buffer(idx, np.int32)
        _out_buffer(cnt, np.int32)
        if cnt.size != idx.size:
            raise ValueError("idx and cnt must have the same size")
        self._check(self._lib.bcpnn_check_result_async(self._h, pop, _ptr(idx), _ptr(cnt), idx.size))

    def ss_flags(self):
        out = np.zeros((self.last_ticks, self.n_projs), dtype=np.uint8)
        self._check(self._lib.bcpnn_get_ss_flags(self._h, _ptr(out), out.size))
        return out

    def info(self, name):
        t, n = ctypes.c_int32(), ctypes.c_size_t()
        self._check(self._lib.bcpnn_state_info(self._h, name.encode(), ctypes.byref(t), ctypes.byref(n)))
        return t.value, n.value

    def read(self, name):
        t, n = self.info(name)
        out = np.zeros(n, dtype=_NP[t])
        self._check(self._lib.bcpnn_read_state(self._h, name.encode(), _ptr(out), out.nbytes))
        return out

    def read_noalloc(self, name):
        """bcpnn_read_state_noalloc: the same read without any device allocation."""
        t, n = self.info(name)
        out = np.zeros(n, dtype=_NP[t])
        self._check(self._lib.bcpnn_read_state_noalloc(self._h, name.encode(), _ptr(out), out.nbytes))
        return out

    def write(self, name, arr):
        t, n = self.info(name)
        a = np.ascontiguousarray(arr, dtype=_NP[t])
        self._check(self._lib.bcpnn_write_state(self._h, name.encode(), _ptr(a), a.nbytes))

    def counters(self):
        out = (ctypes.c_uint64 * 3)()
        self._check(self._lib.bcpnn_counters(self._h, out))
        return [int(out[0]), int(out[1]), int(out[2])]

    def prune(self, proj, threshold_t, wp, wn):
        """disconnect weak or stale rows; returns their source MCUs in row order"""
        n_slots = self.info(f"ii_{proj}")[1]
        out = np.zeros(max(1, n_slots), np.int32)
        n = ctypes.c_int32()
        self._check(self._lib.bcpnn_prune(self._h, proj, threshold_t, wp, wn, _ptr(out), out.size, ctypes.byref(n)))
        return out[:n.value].copy()

    def set_pop_rng(self, pop, seed, key_pop):
        self._check(self._lib.bcpnn_set_pop_rng(self._h, pop, seed, key_pop))

    def selftest_division(self, n_pairs, seed=1):
        """(pairs compared, quotients that differ) of the exact warp-uniform
        division against `/` on this network's device"""
        t, b = ctypes.c_uint64(0), ctypes.c_uint64(0)
        self._check(self._lib.bcpnn_selftest_division(self._h, int(n_pairs), int(seed), ctypes.byref(t), ctypes.byref(b)))
        return t.value, b.value

    def selftest_barrier_timeout(self, limit_ns):
        """status of the barrier self-test (BCPNN_ERR_DEVICE = -6 expected)"""
        return self._lib.bcpnn_selftest_barrier_timeout(self._h, int(limit_ns)), \
            self._lib.bcpnn_last_error(self._h).decode()

    def kernel_launches(self):
        out = ctypes.c_uint64()
        self._check(self._lib.bcpnn_kernel_launches(self._h, ctypes.byref(out)))
        return int(out.value)


def spikes_from_log(log_row, n):
    """Ascending MCU indices set in one row of a spike log."""
    bits = np.unpackbits(log_row.view(np.uint8), bitorder="little")[:n]
    return np.nonzero(bits)[0]
