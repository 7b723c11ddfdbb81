"""bench.py's CPU baselines on the CPU, on small samples: the headline's
oracle sample, the batched workload over spawned workers, one recall
replicate from a trained state, and the compiled ProcUpdMulti oracle.  These
run on the B200 host's cores beside the GPU measurements; here they are
checked to run and to report positive rates."""
import tempfile

import numpy as np

import bench
from gsbn_b200 import batch, extgen, workloads
from oracle import sim
from tests.harness import load_workload, schedule


def test_lginp_row_follows_extgen():
    """ProcExtGen's lginp (ProcExtGen.cpp:130-144): log(1+eps) on the
    indexed MCU, log(eps) elsewhere, and on every MCU of an HCU whose index
    is out of range (no input)."""
    H, M = 6, 5
    eps = np.float32(1e-4)
    hit, miss = np.float32(np.log(1 + eps)), np.float32(np.log(eps))
    row = np.array([0, 4, 2, -1, 5, 0x7FFFFFFF], np.int64)
    got = bench._lginp_row(row, H, M, hit, miss).reshape(H, M)
    want = np.array([[hit if row[h] == m else miss for m in range(M)] for h in range(H)], np.float32)
    assert np.array_equal(got, want)
    assert (got == hit).sum() == 3


def test_reference_windows_cover_the_schedule_once():
    """The reference arm's windows: contiguous, equal tick counts, every tick
    of the schedule exactly once, old_prn of a split run set to its prn."""
    w = workloads.config0()
    sp, pops, projs, stim, conn, seed, phz = load_workload(w, tempfile.mkdtemp())
    runs = extgen.segments(sp)
    hr = bench.host_runs(sp, pops, runs)
    windows, bounds = bench.cut_windows(hr, 7)
    ticks = [first + k for win in windows for first, n, *_ in win for k in range(n)]
    assert ticks == [r.first + k for r in runs for k in range(r.n)]
    assert [sum(p[1] for p in win) for win in windows] == [b - a for a, b in zip(bounds, bounds[1:])]
    for win in windows:
        for first, n, prn, old_prn, lg, wm in win:
            src = next(r for r in runs if r.first <= first < r.first + r.n)
            assert prn == src.prn and old_prn == (src.old_prn if first == src.first else src.prn)


def test_cpu_spread_sample_from_oracle_states():
    """The in-line CPU sample, fed states that the shared-math oracle
    produced at the picked segments (the device's states in the bench)."""
    w = workloads.config0()
    sp, pops, projs, stim, conn, seed, phz = load_workload(w, tempfile.mkdtemp())
    runs = extgen.segments(sp)
    hr = bench.host_runs(sp, pops, runs)
    orc = sim.OracleNet(pops, projs, 0.001, seed=seed)
    for k, (ii, di) in enumerate(conn):
        orc.set_conn(k, ii, di)
    first_recall = next(i for i, r in enumerate(runs) if r.prn == 0.0)
    picks = {0, 3, first_recall, len(runs) - 1}
    states = {}
    for i, (first, n, prn, old_prn, lg, wm) in enumerate(hr):
        if i in picks:
            states[i] = {f"{k}_0": orc.read(f"{k}_0") for k in bench.ORACLE_POP + bench.ORACLE_PROJ}
        orc.set_stimulus(lg, wm)
        orc.run(first, n, prn, old_prn, spikes=False)
    v, kind, sample, spent = bench.cpu_spread_sample(sp, pops, projs, seed, runs, states, sum(orc.counters()))
    assert v > 0 and spent > 0
    assert kind == ("reference" if sim.ref_available() else "port")
    assert "4 segments" in sample


def test_spike_digests_are_reproducible():
    """The committed digests of gsbn's kernels on the 100x100 step are what
    the generator gives (first three segments), and spike_parity accepts the
    matching logs and names the first differing segment otherwise."""
    import json
    import os
    from tests.golden import make_spike_digests as mk
    if not sim.ref_available():
        import pytest
        pytest.skip("oracle/_ref not built")
    with open(bench.GOLDEN_DIGESTS) as f:
        gold = json.load(f)
    got = mk.digests(sim.MATH_REF, max_segments=3)
    assert [(s["first"], s["ticks"], s["spikes"], s["sha256"]) for s in gold["segments"][:3]] == got
    assert gold["ticks"] == 20000 and len(gold["segments"]) == 200
    # spike_parity on a two-segment golden file
    logs = [np.zeros((3, 2), np.uint32), np.zeros((2, 2), np.uint32)]
    logs[1][1, 0] = 5
    import hashlib
    doc = {"ticks": 5, "spikes": 2, "math": "test", "segments": [
        {"first": 1, "ticks": 3, "spikes": 0, "sha256": hashlib.sha256(logs[0].tobytes()).hexdigest()},
        {"first": 4, "ticks": 2, "spikes": 2, "sha256": hashlib.sha256(logs[1].tobytes()).hexdigest()}]}
    path = os.path.join(tempfile.mkdtemp(), "d.json")
    with open(path, "w") as f:
        json.dump(doc, f)
    assert bench.spike_parity(logs, path)["status"] == "identical"
    logs[1][0, 1] = 1
    bad = bench.spike_parity(logs, path)
    assert bad["status"] == "differs" and bad["first_difference"]["segment"] == 1


def test_cpu_batch_sample_spawned_workers():
    members = batch.make_members(n=4, seed=3, hcu=(8, 10), mcu=(5, 6), n_patterns=2)
    runs = batch.schedule(2, train_ticks=10, recall_ticks=6)
    v, cores, sample = bench.cpu_batch_sample(members, runs, k_tr=3, k_rc=2)
    assert v > 0 and 1 <= cores <= 4 and "all 4 networks" in sample


def test_cpu_recall_sample_from_trained_state():
    w = workloads.config0()
    sp, pops, projs, stim, conn, seed, phz = load_workload(w, tempfile.mkdtemp())
    dt, eps = float(np.float32(sp.gen_param.dt)), float(np.float32(sp.gen_param.eps))
    orc = sim.OracleNet(pops, projs, dt, seed=seed)
    for k, (ii, di) in enumerate(conn):
        orc.set_conn(k, ii, di)
    runs = schedule(sp, stim, pops, orc.logf)
    first_recall = next(i for i, r in enumerate(runs) if r.prn == 0.0)
    for r in runs[:3]:
        orc.set_stimulus(r.lginp, r.wmask)
        orc.run(r.first, r.n, r.prn, r.old_prn, spikes=False)
    state = {n: orc.read(n) for n in bench.RECALL_STATE}
    lgidx, wmask = extgen.stim_tables(stim)
    r = runs[first_recall]
    v, sample = bench.cpu_recall_sample(pops, projs, dt, 20.0, state, lgidx[w.meta["patterns"]], wmask[1], eps,
                                        r.first, 1.0, 200, 1, k=10)
    assert v > 0 and "1+10 recall ticks" in sample


def test_cpu_multi_sample_reports_a_rate():
    v, sample = bench.cpu_multi_sample(25, sample_ticks=60)
    assert v > 0 and "60 training ticks + 30 recall ticks" in sample
