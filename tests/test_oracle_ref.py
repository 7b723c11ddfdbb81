"""The oracle's restatement against gsbn's own kernels.

oracle/_ref/libbcpnn_oracle_ref.so carries gsbn's update_*_kernel_cpu
functions (ProcUpdLazy/Proj.cpp:209-536, ProcUpdLazy/Pop.cpp:229-323),
compiled from the gsbn sources by oracle/Makefile's `ref` target.  Math mode
MATH_REF drives them with the oracle's loops, so these tests pin:

  - MATH_LIBM (the restatement with glibc expf/logf, gsbn's math) equals gsbn's
    kernels bit for bit: free runs of the 10x10 and the two-population
    workloads, and an external-spike replay;
  - MATH_SHARED (the restatement with the shared exp/log, which the GPU
    kernels match bit for bit) gives the same spike trains as gsbn's kernels
    over the whole 10x10 schedule, with traces and weights within 1e-5 of each
    array's largest magnitude.
"""
import numpy as np
import pytest

from gsbn_b200 import workloads
from oracle import sim
from tests.harness import first_mismatch, load_workload, schedule, state

pytestmark = pytest.mark.skipif(not sim.ref_available(), reason="oracle/_ref not built (gsbn sources absent)")

TRACE_TOL = 1e-5


def make_net(w, directory, math):
    sp, pops, projs, stim, conn, seed, phz = load_workload(w, str(directory))
    dt = float(np.float32(sp.gen_param.dt))
    net = sim.OracleNet(pops, projs, dt, seed=seed, poisson_hz=phz, math=math)
    for k, (ii, di) in enumerate(conn):
        net.set_conn(k, ii, di)
    return sp, pops, projs, stim, net


def free_run(w, directory, math, max_ticks=None, ext=None):
    """Spike trains (one list of per-population index arrays per tick) and the
    final state of a run of the workload's ProcExtGen schedule."""
    sp, pops, projs, stim, net = make_net(w, directory, math)
    if ext is not None:
        net.set_ext_spikes(0, ext)
    spikes, done = [], 0
    for r in schedule(sp, stim, pops, net.logf):
        n = r.n if max_ticks is None else min(r.n, max_ticks - done)
        if n <= 0:
            break
        net.set_stimulus(r.lginp, r.wmask)
        spikes += net.run(r.first, n, r.prn, r.old_prn)
        done += n
    return spikes, state(net, len(pops), len(projs)), net.counters()


def first_spike_difference(a, b):
    for t, (x, y) in enumerate(zip(a, b)):
        for p, (u, v) in enumerate(zip(x, y)):
            if not np.array_equal(u, v):
                return f"tick {t} population {p}: {u.tolist()} vs {v.tolist()}"
    return None if len(a) == len(b) else f"{len(a)} vs {len(b)} ticks"


@pytest.mark.parametrize("cfg", ["config0", "config2"])
def test_libm_restatement_is_gsbn_kernels_bit_for_bit(tmp_path, cfg):
    """Free runs from the same Philox stream: every spike, every state vector
    (compared by bit pattern) and the cell counters agree."""
    w = workloads.config0() if cfg == "config0" else workloads.config2(n_patterns=8, train_ticks=60, recall_ticks=20)
    ticks = None if cfg == "config0" else 700
    sa, xa, ca = free_run(w, tmp_path / "a", sim.MATH_LIBM, ticks)
    sb, xb, cb = free_run(w, tmp_path / "b", sim.MATH_REF, ticks)
    assert first_spike_difference(sa, sb) is None
    assert sum(len(p) for t in sb for p in t) > 100
    assert first_mismatch(xa, xb) is None
    assert ca == cb


def test_libm_restatement_is_gsbn_kernels_on_replay(tmp_path):
    """External-spike replay (Pop.cpp:389-409), gsbn's own mechanism for
    pinning the trace arithmetic: 600 ticks of a seeded spike file."""
    w = workloads.config0()
    rng = np.random.default_rng(11)
    table = {t: sorted(rng.choice(100, size=int(rng.integers(0, 6)), replace=False).tolist())
             for t in range(1, 601)}
    _, xa, _ = free_run(w, tmp_path / "a", sim.MATH_LIBM, 600, ext=table)
    _, xb, _ = free_run(w, tmp_path / "b", sim.MATH_REF, 600, ext=table)
    assert first_mismatch(xa, xb) is None


def test_shared_math_spike_trains_equal_gsbn_kernels(tmp_path):
    """The arithmetic the GPU reproduces bit for bit (shared exp/log) against
    gsbn's kernels with glibc: identical spike trains over the 2,200-tick 10x10
    schedule, traces and weights within 1e-5 of each array's scale."""
    w = workloads.config0()
    sa, xa, ca = free_run(w, tmp_path / "a", sim.MATH_SHARED)
    sb, xb, cb = free_run(w, tmp_path / "b", sim.MATH_REF)
    assert len(sb) == 2200
    assert first_spike_difference(sa, sb) is None
    assert ca == cb
    for k, b in xb.items():
        a = xa[k]
        if b.dtype.kind != "f":
            assert np.array_equal(a, b), k
            continue
        scale = max(float(np.abs(b).max()), np.finfo(np.float32).tiny)
        assert float(np.abs(a.astype(np.float64) - b).max()) <= TRACE_TOL * scale, k


def test_ref_mode_needs_the_ref_build():
    """MATH_REF exists only in float and only in the oracle/_ref build."""
    pops = [dict(hcu_num=1, mcu_num=2, taum=0.01, wtagain=1.0, maxfq=100.0, igain=1.0, wgain=1.0, lgbias=0.0,
                 snoise=0.0)]
    with pytest.raises(RuntimeError):
        sim.OracleNet(pops, [], 0.001, real_bits=64, math=sim.MATH_REF)
    assert sim.load().oracle_has_ref() == 0
    assert sim.load(ref=True).oracle_has_ref() == 1
