"""The C ABI library without a GPU: it loads, exports every entry point that
include/bcpnn.h declares, and rejects invalid network descriptions before it
touches a device."""
import ctypes
import os
import re

import numpy as np
import pytest

from gsbn_b200 import capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared(prefix="bcpnn_"):
    names = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        if h.endswith(".h"):
            text = open(os.path.join(ROOT, "include", h)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            names |= set(re.findall(r"\b(" + prefix + r"[a-z_0-9]+)\s*\(", text))
    return names


def test_every_declared_entry_point_is_exported():
    from gsbn_b200 import batch, engine, recall
    lib = capi.load()
    names = declared("bcpnn_") | declared("gsbn_")
    assert len(names) >= 40
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing
    bound = set(capi.EXPORTS) | set(recall.RECALL_EXPORTS) | set(engine.ENGINE_EXPORTS) | set(batch.BATCH_EXPORTS)
    assert names <= bound, sorted(names - bound)


def test_recall_rejects_bad_shapes_before_the_device():
    from gsbn_b200 import recall
    pop = dict(hcu_num=8, mcu_num=32, taum=0.005, wtagain=1.0, maxfq=100.0, igain=1.0, wgain=1.0, lgbias=0.0,
               snoise=0.0)
    for H, M, R in [(8, 32, 100), (3, 32, 128), (8, 48, 128), (5, 64, 128), (8, 32, 0)]:
        with pytest.raises(capi.BcpnnError) as e:
            recall.Recall(H, M, R, dict(pop, hcu_num=H, mcu_num=M), 0.001, 0.1)
        assert e.value.status == -1
    # a contraction form other than BF16 (0) or FP32 (1)
    recall.CONTRACTIONS["unknown"] = 7
    try:
        with pytest.raises(capi.BcpnnError) as e:
            recall.Recall(8, 32, 128, pop, 0.001, 0.1, contraction="unknown")
        assert e.value.status == -1
    finally:
        del recall.CONTRACTIONS["unknown"]


def test_status_strings():
    lib = capi.load()
    assert lib.bcpnn_status_string(0) == b"ok"
    assert lib.bcpnn_status_string(-3) == b"unknown state vector"
    assert lib.bcpnn_status_string(-99) == b"unknown status"


POP = dict(hcu_num=2, mcu_num=3, taum=0.01, wtagain=1.0, maxfq=100.0, igain=1.0, wgain=1.0, lgbias=0.0, snoise=0.0)
PROJ = dict(src_pop=0, dest_pop=0, tauzi=0.01, tauzj=0.01, taue=0.02, taup=1.0, maxfq=100.0, bgain=1.0, wgain=1.0,
            tauepsc=0.0, slot_num=6.0)


@pytest.mark.parametrize("pops,projs,kw", [
    ([], [], {}),
    ([dict(POP, mcu_num=0)], [], {}),
    ([dict(POP, mcu_num=513)], [], {}),
    ([POP], [dict(PROJ, dest_pop=1)], {}),
    ([POP], [dict(PROJ, slot_num=0.0)], {}),
    ([POP], [dict(PROJ, slot_num=float("nan"))], {}),
    ([POP], [dict(PROJ, slot_num=1e30)], {}),
    ([POP], [PROJ] * 9, {}),
    ([POP], [PROJ], dict(dt=0.0)),
    ([POP], [PROJ], dict(dt=float("inf"))),
    ([POP], [PROJ], dict(max_ticks=0)),
    # time constants and frequencies whose rate dt/tau is not a finite
    # positive number (the FP64 propagator and the closed forms need one)
    ([dict(POP, taum=0.0)], [PROJ], {}),
    ([POP], [dict(PROJ, tauzi=0.0)], {}),
    ([POP], [dict(PROJ, tauzj=-0.01)], {}),
    ([POP], [dict(PROJ, taue=0.0)], {}),
    ([POP], [dict(PROJ, taup=float("inf"))], {}),
    ([POP], [dict(PROJ, taup=float("nan"))], {}),
    ([POP], [dict(PROJ, maxfq=0.0)], {}),
    ([POP], [dict(PROJ, tauepsc=float("inf"))], {}),
    ([POP], [dict(PROJ, taue=0.0)], dict(fp64_tables=1)),
])
def test_invalid_descriptions_are_rejected(pops, projs, kw):
    args = dict(dt=0.001, max_ticks=16)
    args.update(kw)
    dt = args.pop("dt")
    with pytest.raises(capi.BcpnnError) as e:
        capi.Net(pops, projs, dt, **args)
    assert e.value.status == -1


def test_null_handle_calls_fail_cleanly():
    lib = capi.load()
    assert lib.bcpnn_run(None, 1, 1, 1.0, 0.0) == -1
    assert lib.bcpnn_sync(None) == -1
    assert lib.bcpnn_net_destroy(None) == -1
    assert lib.bcpnn_last_error(None) == b"null handle"
    out = ctypes.c_void_p()
    assert lib.bcpnn_net_create(None, ctypes.byref(out)) == -1
    lg = np.zeros(4, np.int32)
    wm = np.zeros(4, np.float32)
    assert lib.bcpnn_upload_stimuli_idx_async(None, 1, lg.ctypes.data, 1e-4, 1, wm.ctypes.data) == -1
    assert lib.bcpnn_get_spike_log_async(None, 0, lg.ctypes.data, 4) == -1


def test_output_buffers_are_checked_before_the_library_writes():
    """The asynchronous copies write by element count into the caller's
    array: a wrong element type, a strided view or a read-only array is
    refused in Python, before any pointer reaches the library."""
    import numpy as np
    good = np.zeros((4, 3), np.uint32)
    capi._out_buffer(good, np.uint32)
    for bad in (np.zeros((4, 3), np.uint8), np.zeros((4, 6), np.uint32)[:, ::2], [0, 1, 2]):
        with pytest.raises(ValueError):
            capi._out_buffer(bad, np.uint32)
    ro = np.zeros(3, np.int32)
    ro.flags.writeable = False
    with pytest.raises(ValueError):
        capi._out_buffer(ro, np.int32)


@pytest.mark.parametrize("prn,old_prn", [(float("inf"), 1.0), (1.0, float("-inf")), (float("nan"), 0.0)])
def test_non_finite_prn_is_rejected_before_any_launch(prn, old_prn):
    """bcpnn_run refuses a prn that is not finite before it touches the device
    (kp = prn dt/taup would be infinite).  Without a GPU the network's creation
    stops at cudaSetDevice but still hands back a handle; with one it
    succeeds.  Either way the run returns BCPNN_ERR_INVALID."""
    lib = capi.load()
    pops = (capi.PopDesc * 1)(capi.PopDesc(**POP))
    projs = (capi.ProjDesc * 1)(capi.ProjDesc(**PROJ))
    desc = capi.NetDesc(1, pops, 1, projs, 0.001, 0, 0.0, 1, 0, 16, 0, 0, 0, 1)
    h = ctypes.c_void_p()
    lib.bcpnn_net_create(ctypes.byref(desc), ctypes.byref(h))
    assert h
    try:
        assert lib.bcpnn_run(h, 1, 1, prn, old_prn) == -1
        assert b"finite" in lib.bcpnn_last_error(h)
    finally:
        lib.bcpnn_net_destroy(h)


def test_batch_rejects_bad_members_before_the_device():
    """bcpnn_batch_create refuses members beyond the engine's limits (64 MCUs
    per HCU, one recurrent projection) and non-positive rates, before any
    device work."""
    from gsbn_b200 import batch
    good = batch.make_members(n=1, seed=1, hcu=(8, 8), mcu=(5, 5), n_patterns=2)[0]
    for edit in (dict(pop=dict(good.pop, mcu_num=65)), dict(proj=dict(good.proj, src_pop=1)),
                 dict(proj=dict(good.proj, taue=0.0)), dict(pop=dict(good.pop, taum=float("nan")))):
        m = batch.Member.__new__(batch.Member)
        m.__dict__.update(good.__dict__)
        m.__dict__.update(edit)
        with pytest.raises(capi.BcpnnError) as e:
            batch.BatchEngine([m], max_ticks=8)
        assert e.value.status == -1
    # CTA sizes other than 256, 384 and 512 threads
    for threads in (128, 300, 448, 1024):
        with pytest.raises(capi.BcpnnError) as e:
            batch.BatchEngine([good], max_ticks=8, threads=threads)
        assert e.value.status == -1
