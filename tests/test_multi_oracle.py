"""The ProcUpdMulti oracle restatements on the CPU: the Python one
(oracle/multi.py) with gsbn's initial values (ProcUpdMulti/Pop.cpp:66-73,
Proj.cpp:92-108), a ring of postsynaptic spikes that replays into active
cells, the adaptation current following act, and spikes in recall; and the
compiled one (oracle/bcpnn_oracle_multi.cpp) held to the Python one bit for
bit."""
import warnings

import numpy as np
import pytest

from gsbn_b200 import extgen, schema, workloads
from oracle import multi, sim


def test_multi_oracle_runs_config0(tmp_path):
    w = workloads.config0()
    sp, _ = w.solver_param(str(tmp_path))
    pops, projs = workloads.net_from_solver_param(sp)
    for p in pops:
        p.update(taua=0.05, adgain=1.0)
    conn = workloads.read_conn_map(w.conn, pops, projs)
    lgidx, wmask = extgen.stim_tables(schema.read_stim(sp.gen_param.stim_file))
    eps = np.float32(sp.gen_param.eps)
    hit = np.float32(sim.extgen_logf(np.float32(1) + eps))
    miss = np.float32(sim.extgen_logf(np.float32(0) + eps))
    net = multi.MultiNet(pops, projs, float(np.float32(sp.gen_param.dt)), seed=w.meta["seed"], spike_buffer=25)
    assert np.all(net.read("pij_0") == np.float32(1.0 / 100 / 10))
    assert np.all(net.read("dsup_0") == np.float32(np.log(0.1)))
    for k, (ii, di) in enumerate(conn):
        net.set_conn(k, ii, di)
    spikes = 0
    for r in extgen.segments(sp)[:4]:
        row = lgidx[r.lgidx]
        net.set_stimulus(np.array([hit if row[h] == m else miss for h in range(10) for m in range(10)], np.float32),
                         wmask[r.wmask])
        logs = net.run(r.first, r.n, r.prn, r.old_prn)
        spikes += int(np.unpackbits(logs[0].view(np.uint8)).sum())
    assert spikes > 50
    ada, act = net.read("ada_0"), net.read("act_0")
    assert np.all(ada > 0) and np.all(np.isfinite(ada)) and np.corrcoef(ada, act)[0, 1] > 0.5
    wij = net.read("wij_0")
    assert np.count_nonzero(wij) > 100 and np.all(np.isfinite(wij))


def _lginp(row, pops, eps):
    hit = np.float32(sim.extgen_logf(np.float32(1) + eps))
    miss = np.float32(sim.extgen_logf(np.float32(0) + eps))
    out, hoff = [], 0
    for p in pops:
        H, M = p["hcu_num"], p["mcu_num"]
        out += [hit if row[hoff + h] == m else miss for h in range(H) for m in range(M)]
        hoff += H
    return np.array(out, np.float32)


@pytest.mark.parametrize("make,ring,snoise", [("config0", 25, 0.0), ("config0", 3, 0.0), ("config0", 1, 0.0),
                                              ("config2", 5, 0.2)])
def test_compiled_multi_matches_python(tmp_path, make, ring, snoise):
    """The compiled restatement (oracle/bcpnn_oracle_multi.cpp, the one fast
    enough for 100x100 networks) computes the same bits as the Python one:
    spike trains and every state vector after each run of a training ->
    recall -> training schedule (both directions of the catch-up at a change
    of prn), for rings of 25, 3 and 1 ticks, and for two populations with
    two projections and normal input noise."""
    w = workloads.config0() if make == "config0" else workloads.config2(n_patterns=4, train_ticks=30, recall_ticks=20)
    sp, _ = w.solver_param(str(tmp_path))
    pops, projs = workloads.net_from_solver_param(sp)
    for p in pops:
        p.update(taua=0.05, adgain=1.0, snoise=snoise)
    conn = workloads.read_conn_map(w.conn, pops, projs)
    lgidx, wmask = extgen.stim_tables(schema.read_stim(sp.gen_param.stim_file))
    eps = np.float32(sp.gen_param.eps)
    dt = float(np.float32(sp.gen_param.dt))
    py = multi.MultiNet(pops, projs, dt, seed=7, spike_buffer=ring)
    cc = multi.MultiNetC(pops, projs, dt, seed=7, spike_buffer=ring)
    for k, (ii, di) in enumerate(conn):
        py.set_conn(k, ii, di)
        cc.set_conn(k, ii, di)
    P = lgidx.shape[0] // 2
    names = [f"{k}_{q}" for q in range(len(pops)) for k in ("dsup", "act", "ada", ".counter", "epsc", "bj", "spike")]
    names += [f"{k}_{q}" for q in range(len(projs))
              for k in ("pi", "ei", "zi", "ti", "pj", "ej", "zj", "pij", "eij", "zj2", "wij", "qi", "siq", "si")]
    spikes = 0
    for first, n, prn, old, lr, wr in ((1, 40, 1.0, 0.0, 0, 0), (41, 20, 0.0, 1.0, P, 1), (61, 15, 1.0, 0.0, 1, 0)):
        lg = _lginp(lgidx[lr], pops, eps)
        py.set_stimulus(lg, wmask[wr])
        cc.set_stimulus(lg, wmask[wr])
        with warnings.catch_warnings():
            warnings.simplefilter("ignore")
            want = py.run(first, n, prn, old)
        got = cc.run(first, n, prn, old)
        for a, b in zip(got, want):
            assert np.array_equal(a, b), f"spikes of the run at {first}"
            spikes += int(np.unpackbits(a.view(np.uint8)).sum())
        for name in names:
            a, b = cc.read(name), py.read(name)
            assert a.dtype == b.dtype and np.array_equal(a.view(np.uint8), b.view(np.uint8)), f"{name} at {first}"
    assert spikes > 50
    row, _, sweeps = cc.counters()
    # each of the three runs starts with a change of prn: three all-cells sweeps
    cells = 0
    for q in projs:
        src, dst = pops[q["src_pop"]], pops[q["dest_pop"]]
        cells += dst["hcu_num"] * min(src["hcu_num"] * src["mcu_num"], int(np.float32(q["slot_num"]))) * dst["mcu_num"]
    assert row > 0 and sweeps == 3 * cells
