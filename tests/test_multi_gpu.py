"""ProcUpdMulti (the row-only update with a postsynaptic spike ring,
ProcUpdMulti.cpp:94-125) on the GPU through the C ABI (update_variant 1)
against the oracle's restatement (oracle/multi.py): spike trains and every
state vector bit-identical, run by run over the 10x10 workload's training
and recall segments (so the catch-up at each change of prn is covered), for
a ring of 25 ticks (the reference prototxts' value) and of 1 tick."""
import numpy as np
import pytest

from gsbn_b200 import capi, extgen, schema, workloads
from oracle import multi, sim

pytestmark = pytest.mark.gpu

ARRAYS = ("dsup_0", "act_0", "ada_0", ".counter_0", "epsc_0", "bj_0", "pi_0", "ei_0", "zi_0", "ti_0", "pj_0", "ej_0",
          "zj_0", "pij_0", "eij_0", "zj2_0", "wij_0", "qi_0")


def lginp_row(row, pops, eps):
    hit = np.float32(sim.logf(np.array([np.float32(1) + eps], np.float32))[0])
    miss = np.float32(sim.logf(np.array([np.float32(0) + eps], np.float32))[0])
    H, M = pops[0]["hcu_num"], pops[0]["mcu_num"]
    return np.array([hit if row[h] == m else miss for h in range(H) for m in range(M)], np.float32)


@pytest.mark.parametrize("ring", [25, 1])
def test_multi_matches_oracle(tmp_path, ring):
    w = workloads.config0()
    sp, _ = w.solver_param(str(tmp_path))
    pops, projs = workloads.net_from_solver_param(sp)
    for p in pops:
        p.update(taua=0.05, adgain=1.0)
    conn = workloads.read_conn_map(w.conn, pops, projs)
    lgidx, wmask = extgen.stim_tables(schema.read_stim(sp.gen_param.stim_file))
    eps = np.float32(sp.gen_param.eps)
    runs = extgen.segments(sp)[:22]
    assert any(r.prn != r.old_prn for r in runs[1:])
    dt = float(np.float32(sp.gen_param.dt))
    orc = multi.MultiNet(pops, projs, dt, seed=w.meta["seed"], spike_buffer=ring)
    gpu = capi.Net(pops, projs, dt, seed=w.meta["seed"], max_ticks=256, variant=1, spike_buffer=ring)
    try:
        for k, (ii, di) in enumerate(conn):
            orc.set_conn(k, ii, di)
            gpu.set_conn(k, ii, di)
        spikes = 0
        for r in runs:
            lg, wm = lginp_row(lgidx[r.lgidx], pops, eps), wmask[r.wmask]
            orc.set_stimulus(lg, wm)
            gpu.set_stimulus(lg, wm)
            want = orc.run(r.first, r.n, r.prn, r.old_prn)
            gpu.run(r.first, r.n, r.prn, r.old_prn)
            got = gpu.spike_log(0)
            assert np.array_equal(got, want[0]), f"spikes differ in the run at {r.first}"
            spikes += int(np.unpackbits(got.view(np.uint8)).sum())
            for name in ARRAYS:
                a, b = gpu.read(name), orc.read(name)
                b = np.asarray(b).astype(a.dtype)
                assert np.array_equal(a.view(np.uint8), b.view(np.uint8)), f"{name} after the run at {r.first}"
        assert spikes > 20
    finally:
        gpu.close()
