"""The sm_100a path against gsbn's own kernels.

The CPU side here is the oracle in math mode MATH_REF: its population and
projection loops call gsbn's update_*_kernel_cpu functions
(ProcUpdLazy/Proj.cpp:209-536, ProcUpdLazy/Pop.cpp:229-323) compiled from the
gsbn sources (oracle/_ref), with glibc expf/logf as gsbn calls them.  Both
sides get the same stimulus rows (ProcExtGen's lginp computed with glibc logf),
connectivity and Philox stream.  The bar, per the plain FP32 contract:
identical spike trains over the run, the same cell-update counts, and traces
and weights within 1e-5 of each array's largest magnitude (w_ij = log(ratio)
is near zero for many cells, so the bound is not taken element by element).
"""
import numpy as np
import pytest

from gsbn_b200 import workloads
from oracle import sim
from tests.harness import load_workload, schedule, state
from tests.test_gpu_parity import gpu_net, spikes_of

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not sim.ref_available(), reason="oracle/_ref not built (gsbn sources absent)")]

TRACE_TOL = 1e-5


def ref_pair(w, directory, per_tick=False):
    sp, pops, projs, stim, conn, seed, phz = load_workload(w, str(directory))
    dt = float(np.float32(sp.gen_param.dt))
    ref = sim.OracleNet(pops, projs, dt, seed=seed, poisson_hz=phz, math=sim.MATH_REF)
    gpu = gpu_net(pops, projs, dt, seed=seed, poisson_hz=phz, max_ticks=256, per_tick=per_tick)
    for k, (ii, di) in enumerate(conn):
        ref.set_conn(k, ii, di)
        gpu.set_conn(k, ii, di)
    return pops, projs, ref, gpu, schedule(sp, stim, pops, ref.logf)


def run_against_ref(pops, projs, ref, gpu, runs, max_ticks=None):
    ticks = spikes = 0
    for r in runs:
        n = r.n if max_ticks is None else min(r.n, max_ticks - ticks)
        if n <= 0:
            break
        ref.set_stimulus(r.lginp, r.wmask)
        gpu.set_stimulus(r.lginp, r.wmask)
        want = ref.run(r.first, n, r.prn, r.old_prn)
        gpu.run(r.first, n, r.prn, r.old_prn)
        got = spikes_of(gpu, pops, n)
        for t in range(n):
            for p in range(len(pops)):
                assert np.array_equal(want[t][p], got[t][p]), f"spikes differ at simstep {r.first + t} pop {p}"
                spikes += len(want[t][p])
        ticks += n
    a, b = state(gpu, len(pops), len(projs)), state(ref, len(pops), len(projs))
    for k, y in b.items():
        x = a[k]
        if y.dtype.kind != "f":
            assert np.array_equal(x, y), k
            continue
        if y.size == 0:
            continue
        scale = max(float(np.abs(y).max()), np.finfo(np.float32).tiny)
        err = float(np.abs(x.astype(np.float64) - y).max())
        assert err <= TRACE_TOL * scale, f"{k}: {err / scale:.3g} of scale"
    assert gpu.counters() == ref.counters()
    return ticks, spikes


@pytest.mark.parametrize("per_tick", [False, True])
def test_config0_whole_schedule(tmp_path, per_tick):
    """10x10, all 2,200 ticks (training, rests, recall)."""
    pops, projs, ref, gpu, runs = ref_pair(workloads.config0(), tmp_path, per_tick)
    try:
        ticks, spikes = run_against_ref(pops, projs, ref, gpu, runs)
        assert ticks == 2200 and spikes > 1000
    finally:
        gpu.close()


def test_config1_first_3000_ticks(tmp_path):
    """The 100x100 network at density 0.1 (C = 1000, 1e7 cells): the first
    3,000 ticks of its training schedule."""
    pops, projs, ref, gpu, runs = ref_pair(workloads.config1(), tmp_path)
    try:
        ticks, spikes = run_against_ref(pops, projs, ref, gpu, runs, max_ticks=3000)
        assert ticks == 3000 and spikes > 10000
    finally:
        gpu.close()


def test_config1_training_to_recall(tmp_path):
    """The same network with 20 patterns: 2,000 training ticks, the all-cells
    catch-up at the change of prn, and 1,000 recall ticks."""
    w = workloads.config1(n_patterns=20, train_ticks=100, recall_ticks=50)
    pops, projs, ref, gpu, runs = ref_pair(w, tmp_path)
    try:
        assert any(r.prn != r.old_prn for r in runs[1:])
        ticks, spikes = run_against_ref(pops, projs, ref, gpu, runs)
        assert ticks == 3000 and spikes > 10000
    finally:
        gpu.close()


def test_config2_whole_schedule(tmp_path):
    """Two populations, two projections with their own tau_z, 10 Hz Poisson
    input noise: all 50 patterns, 5,000 ticks."""
    pops, projs, ref, gpu, runs = ref_pair(workloads.config2(), tmp_path)
    try:
        ticks, spikes = run_against_ref(pops, projs, ref, gpu, runs)
        assert ticks == 5000 and spikes > 1000
    finally:
        gpu.close()
