"""The ProcUpdMulti oracle restatement (oracle/multi.py) on the CPU: gsbn's
initial values (ProcUpdMulti/Pop.cpp:66-73, Proj.cpp:92-108), a ring of
postsynaptic spikes that replays into active cells, the adaptation current
following act, and spikes in recall."""
import warnings

import numpy as np

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
    hit = np.float32(sim.logf(np.array([np.float32(1) + eps], np.float32))[0])
    miss = np.float32(sim.logf(np.array([np.float32(0) + eps], np.float32))[0])
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
