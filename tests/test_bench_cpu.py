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


def test_cpu_sample_reports_a_rate():
    v, sample, secs = bench.cpu_sample(40)
    assert v > 0 and secs > 0 and "40 training ticks + 20 recall ticks" in sample


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
