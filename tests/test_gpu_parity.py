"""Parity of the sm_100a path (through the C ABI) with the CPU oracle.

Bar: bit-identical spikes and state vectors (every float compared by its bit
pattern) on the same seeded inputs and Philox stream, tick by tick and run by
run, for the 10x10 workload, the two-population workload with Poisson input
noise, a reduced copy of the 100x100 workload, external spike replay, and the
all-cells catch-up at every change of prn.
"""
import os

import numpy as np
import pytest

from gsbn_b200 import capi, workloads
from oracle import sim
from tests.harness import first_mismatch, load_workload, schedule, state

pytestmark = pytest.mark.gpu


def gpu_net(*args, per_tick=False, **kw):
    """a capi.Net on the persistent cooperative path (default) or on the
    one-launch-per-tick path; per_tick="t256" is the persistent path with
    256-thread CTAs, per_tick="global" (ProcUpdMulti) the persistent launch
    that keeps the HCU state in global memory instead of shared memory"""
    saved = {k: os.environ.get(k) for k in ("GSBN_PER_TICK", "GSBN_MULTI_RESIDENT")}
    if per_tick == "t256":
        kw["tick_threads"] = 256
        per_tick = False
    os.environ["GSBN_MULTI_RESIDENT"] = "0" if per_tick == "global" else "1"
    if per_tick == "global":
        per_tick = False
    os.environ["GSBN_PER_TICK"] = "1" if per_tick else "0"
    try:
        return capi.Net(*args, **kw)
    finally:
        for k, v in saved.items():
            if v is None:
                del os.environ[k]
            else:
                os.environ[k] = v


@pytest.fixture(params=["persistent", "per_tick", "t256"])
def mode(request):
    return {"persistent": False, "per_tick": True, "t256": "t256"}[request.param]


def make_pair(w, directory, max_ticks=256, exchange=True, per_tick=False):
    sp, pops, projs, stim, conn, seed, phz = load_workload(w, str(directory))
    dt = float(np.float32(sp.gen_param.dt))
    orc = sim.OracleNet(pops, projs, dt, seed=seed, poisson_hz=phz)
    gpu = gpu_net(pops, projs, dt, seed=seed, poisson_hz=phz, exchange=exchange, max_ticks=max_ticks,
                  per_tick=per_tick)
    for k, (ii, di) in enumerate(conn):
        orc.set_conn(k, ii, di)
        gpu.set_conn(k, ii, di)
    runs = schedule(sp, stim, pops, orc.logf)
    return sp, pops, projs, orc, gpu, runs


def spikes_of(gpu, pops, n):
    logs = [gpu.spike_log(p) for p in range(len(pops))]
    out = []
    for t in range(n):
        out.append([capi.spikes_from_log(logs[p][t], pops[p]["hcu_num"] * pops[p]["mcu_num"])
                    for p in range(len(pops))])
    return out


def compare_runs(pops, projs, orc, gpu, runs, full_every_run=True, limit=None):
    n_spikes = 0
    for ri, r in enumerate(runs if limit is None else runs[:limit]):
        orc.set_stimulus(r.lginp, r.wmask)
        gpu.set_stimulus(r.lginp, r.wmask)
        ref = orc.run(r.first, r.n, r.prn, r.old_prn)
        gpu.run(r.first, r.n, r.prn, r.old_prn)
        got = spikes_of(gpu, pops, r.n)
        for t in range(r.n):
            for p in range(len(pops)):
                assert np.array_equal(ref[t][p], got[t][p]), f"spikes differ at simstep {r.first + t} pop {p}"
                n_spikes += len(ref[t][p])
        if full_every_run or ri == len(runs) - 1:
            msg = first_mismatch(state(orc, len(pops), len(projs)), state(gpu, len(pops), len(projs)))
            assert msg is None, f"after run {ri} (simstep {r.first}..{r.first + r.n - 1}): {msg}"
    return n_spikes


def test_config0_tick_by_tick(tmp_path, mode):
    sp, pops, projs, orc, gpu, runs = make_pair(workloads.config0(), tmp_path, per_tick=mode)
    ticks = 0
    for r in runs:
        orc.set_stimulus(r.lginp, r.wmask)
        gpu.set_stimulus(r.lginp, r.wmask)
        for k in range(r.n):
            old = r.old_prn if k == 0 else r.prn
            orc.update(r.first + k, r.prn, old)
            orc.exchange()
            gpu.run(r.first + k, 1, r.prn, old)
            ticks += 1
            if ticks <= 400 or k == 0 or k == r.n - 1:
                msg = first_mismatch(state(orc, 1, 1), state(gpu, 1, 1))
                assert msg is None, f"simstep {r.first + k}: {msg}"
    assert ticks == 2200
    assert orc.counters() == gpu.counters()


def test_config0_runs(tmp_path, mode):
    sp, pops, projs, orc, gpu, runs = make_pair(workloads.config0(), tmp_path, per_tick=mode)
    n = compare_runs(pops, projs, orc, gpu, runs)
    assert n > 100
    assert orc.counters() == gpu.counters()


def test_config2_two_projections_poisson(tmp_path, mode):
    w = workloads.config2(n_patterns=12, train_ticks=80, recall_ticks=20)
    sp, pops, projs, orc, gpu, runs = make_pair(w, tmp_path, per_tick=mode)
    n = compare_runs(pops, projs, orc, gpu, runs)
    assert n > 100
    assert orc.counters() == gpu.counters()


def test_config2_full_size(tmp_path, mode):
    """The two-population workload at its real size: 50 patterns, 5,000
    ticks, in every launch mode."""
    sp, pops, projs, orc, gpu, runs = make_pair(workloads.config2(), tmp_path, per_tick=mode)
    try:
        assert sum(r.n for r in runs) == 5000
        n = compare_runs(pops, projs, orc, gpu, runs, full_every_run=False)
        assert n > 1000
        assert orc.counters() == gpu.counters()
    finally:
        gpu.close()


def test_reduced_100x100(tmp_path, mode):
    w = workloads.small_scale(hcu=24, mcu=20, src=6, n_patterns=8, train_ticks=50, recall_ticks=30)
    sp, pops, projs, orc, gpu, runs = make_pair(w, tmp_path, per_tick=mode)
    compare_runs(pops, projs, orc, gpu, runs, full_every_run=False)
    assert orc.counters() == gpu.counters()


def test_external_spike_replay(tmp_path, mode):
    w = workloads.config0()
    sp, pops, projs, orc, gpu, runs = make_pair(w, tmp_path, per_tick=mode)
    rng = np.random.default_rng(7)
    table = {}
    for t in range(1, 2201):
        k = int(rng.integers(0, 4))
        table[t] = sorted(rng.choice(100, size=k, replace=False).tolist())
    orc.set_ext_spikes(0, table)
    gpu.set_ext_spikes(0, table)
    compare_runs(pops, projs, orc, gpu, runs, limit=12)


def test_no_exchange_keeps_si_zero(tmp_path):
    w = workloads.config0()
    sp, pops, projs, stim, conn, seed, phz = load_workload(w, str(tmp_path))
    gpu = gpu_net(pops, projs, 0.001, seed=seed, exchange=False, max_ticks=256)
    for k, (ii, di) in enumerate(conn):
        gpu.set_conn(k, ii, di)
    r = schedule(sp, stim, pops, lambda x: np.float32(np.log(x)))[0]
    gpu.set_stimulus(r.lginp, r.wmask)
    gpu.run(r.first, r.n, r.prn, r.old_prn)
    assert not gpu.read("si_0").any()
    assert gpu.counters()[0] == 0


def test_determinism_and_paths(tmp_path):
    """a run on the persistent path and the same run cut into one-tick calls on
    the per-tick path (CUDA-graph replay of cached run lengths) give the same
    bits."""
    w = workloads.config0()
    sp, pops, projs, orc, a, runs = make_pair(w, tmp_path / "a")
    _, _, _, _, b, _ = make_pair(w, tmp_path / "b", per_tick=True)
    for r in runs[:6]:
        for net in (a, b):
            net.set_stimulus(r.lginp, r.wmask)
        a.run(r.first, r.n, r.prn, r.old_prn)
        for k in range(r.n):
            b.run(r.first + k, 1, r.prn, r.old_prn if k == 0 else r.prn)
    assert first_mismatch(state(a, 1, 1), state(b, 1, 1)) is None


def test_state_roundtrip(tmp_path):
    w = workloads.config0()
    sp, pops, projs, orc, gpu, runs = make_pair(w, tmp_path)
    rng = np.random.default_rng(3)
    for name in ("pij_0", "eij_0", "zi2_0", "zj2_0", "wij_0", "tij_0", "pi_0", "dsup_0", "epsc_0", "qi_0"):
        t, n = gpu.info(name)
        a = rng.standard_normal(n).astype(np.float32) if t == capi.F32 else rng.integers(0, 50, n).astype(np.int32)
        gpu.write(name, a)
        assert np.array_equal(gpu.read(name), a), name
    with pytest.raises(capi.BcpnnError):
        gpu.read("nonexistent_0")
    with pytest.raises(capi.BcpnnError):
        gpu.run(1, 100000, 1.0, 0.0)


def test_bad_connection_rejected(tmp_path):
    w = workloads.config0()
    sp, pops, projs, orc, gpu, runs = make_pair(w, tmp_path)
    ii = np.full(1000, -1, np.int32)
    di = np.ones(1000, np.int32)
    ii[5] = 100  # outside the 100 source MCUs
    with pytest.raises(capi.BcpnnError):
        gpu.set_conn(0, ii, di)
    ii[5] = 3
    di[5] = 0  # delay must be >= 1
    with pytest.raises(capi.BcpnnError):
        gpu.set_conn(0, ii, di)
