"""ctypes binding of the host engine (include/gsbn_engine.h): gsbn's Solver
with its procedure registry, and the prototxt / StimRawData readers.

Solver(net_path) builds the procedures listed in the network description and
runs them on the GPU; the record files (ProcSpkRec, ProcCheck, ProcSnapshot)
land under rec_param.directory exactly as gsbn writes them.
"""
import ctypes

import numpy as np

from . import capi

ENGINE_EXPORTS = (
    "gsbn_solver_create", "gsbn_solver_run", "gsbn_solver_stats", "gsbn_solver_net", "gsbn_solver_destroy",
    "gsbn_engine_last_error", "gsbn_prototxt_dump", "gsbn_stim_decode", "gsbn_procedure_names",
)
MODE_CPU, MODE_GPU = 0, 1

_lib = None


class EngineError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"gsbn engine status {status}: {message}")
        self.status = status


def load():
    global _lib
    if _lib is not None:
        return _lib
    lib = capi.load()
    vp, sz, i32, i64 = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int32, ctypes.c_int64
    P = ctypes.POINTER
    sig = {
        "gsbn_solver_create": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int, P(vp)]),
        "gsbn_solver_run": (ctypes.c_int, [vp, ctypes.c_int]),
        "gsbn_solver_stats": (ctypes.c_int, [vp, P(i64), P(i64), P(i32), P(i32)]),
        "gsbn_solver_net": (ctypes.c_int, [vp, P(vp)]),
        "gsbn_solver_destroy": (ctypes.c_int, [vp]),
        "gsbn_engine_last_error": (ctypes.c_char_p, []),
        "gsbn_prototxt_dump": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p, sz, P(sz)]),
        "gsbn_stim_decode": (ctypes.c_int, [ctypes.c_char_p, P(ctypes.c_uint32), vp, sz, vp, sz]),
        "gsbn_procedure_names": (ctypes.c_int, [ctypes.c_char_p, sz]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _check(rc):
    if rc != 0:
        raise EngineError(rc, load().gsbn_engine_last_error().decode())


def prototxt_dump(path):
    """Canonical dump of a parsed network description (one field per line)."""
    lib = load()
    need = ctypes.c_size_t(0)
    rc = lib.gsbn_prototxt_dump(path.encode(), None, 0, ctypes.byref(need))
    if rc not in (0, -4):  # BCPNN_ERR_SIZE: only the size was asked for
        _check(rc)
    buf = ctypes.create_string_buffer(need.value)
    _check(lib.gsbn_prototxt_dump(path.encode(), buf, need.value, ctypes.byref(need)))
    return buf.value.decode()


def stim_decode(path):
    """(lgidx rows as uint32 [rows, cols], wmask rows as float32 [rows, cols])."""
    lib = load()
    dims = (ctypes.c_uint32 * 4)()
    _check(lib.gsbn_stim_decode(path.encode(), dims, None, 0, None, 0))
    data = np.zeros(dims[0] * dims[1], np.uint32)
    mask = np.zeros(dims[2] * dims[3], np.float32)
    _check(lib.gsbn_stim_decode(path.encode(), dims, data.ctypes.data_as(ctypes.c_void_p), data.size,
                                mask.ctypes.data_as(ctypes.c_void_p), mask.size))
    return data.reshape(dims[0], dims[1]), mask.reshape(dims[2], dims[3])


def procedure_names():
    buf = ctypes.create_string_buffer(4096)
    _check(load().gsbn_procedure_names(buf, 4096))
    return buf.value.decode().split(",")


class _BorrowedNet(capi.Net):
    """capi.Net view of the network owned by a Solver (not destroyed here)."""

    def __init__(self, handle, n_pops, n_projs):
        self._lib = capi.load()
        self._h = ctypes.c_void_p(handle)
        self.n_pops, self.n_projs = n_pops, n_projs
        self.last_ticks = 0

    def close(self):
        self._h = ctypes.c_void_p()


class Solver:
    """gsbn Solver: Solver(net_path) or Solver(net_path, snapshot_path)."""

    def __init__(self, net_path, snapshot_path=None, mode=MODE_GPU):
        self._lib = load()
        self._h = ctypes.c_void_p()
        _check(self._lib.gsbn_solver_create(net_path.encode(), snapshot_path.encode() if snapshot_path else None, mode,
                                            ctypes.byref(self._h)))

    def run(self, windows=True):
        _check(self._lib.gsbn_solver_run(self._h, 1 if windows else 0))

    def stats(self):
        t, w = ctypes.c_int64(), ctypes.c_int64()
        c, n = ctypes.c_int32(), ctypes.c_int32()
        _check(self._lib.gsbn_solver_stats(self._h, ctypes.byref(t), ctypes.byref(w), ctypes.byref(c), ctypes.byref(n)))
        return dict(ticks=t.value, windows=w.value, correct=c.value, patterns=n.value)

    def net(self, n_pops, n_projs):
        h = ctypes.c_void_p()
        _check(self._lib.gsbn_solver_net(self._h, ctypes.byref(h)))
        if not h.value:
            raise EngineError(-5, "no network (ProcUpdLazy not listed)")
        return _BorrowedNet(h.value, n_pops, n_projs)

    def close(self):
        if self._h:
            self._lib.gsbn_solver_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
