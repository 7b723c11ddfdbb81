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
    hit = np.float32(sim.extgen_logf(np.float32(1) + eps))
    miss = np.float32(sim.extgen_logf(np.float32(0) + eps))
    H, M = pops[0]["hcu_num"], pops[0]["mcu_num"]
    return np.array([hit if row[h] == m else miss for h in range(H) for m in range(M)], np.float32)


@pytest.mark.parametrize("ring,per_tick", [(25, False), (25, True), (25, "global"), (1, False), (40, False)])
def test_multi_matches_oracle(tmp_path, ring, per_tick):
    """persistent launch (one per run; with the HCU state in shared memory,
    or in global memory with "global" and for rings longer than 32 ticks)
    and one launch per tick"""
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
    from tests.test_gpu_parity import gpu_net
    gpu = gpu_net(pops, projs, dt, seed=w.meta["seed"], max_ticks=256, variant=1, spike_buffer=ring, per_tick=per_tick)
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


def test_engine_runs_procupdmulti(tmp_path):
    """A prototxt naming ProcUpdMulti (with gsbn's "spike buffer size" 25)
    through the host engine's registry records the same spike trains as the
    same network driven directly through the C ABI."""
    from gsbn_b200 import engine
    w = workloads.config0()
    path = w.write(str(tmp_path))
    with open(path) as f:
        text = f.read()
    assert 'name: "ProcUpdLazy"' in text
    text = text.replace('name: "ProcUpdLazy"', 'name: "ProcUpdMulti"\n  argi { key: "spike buffer size" val: 25 }')
    with open(path, "w") as f:
        f.write(text)
    with open(path) as f:
        sp = schema.parse_prototxt(f.read())
    s = engine.Solver(path)
    s.run(True)
    s.close()
    import os
    rec = {}
    with open(os.path.join(sp.rec_param.directory, "ProcSpkRec", "spk_pop_0.csv")) as f:
        for line in f.read().splitlines()[1:]:
            v = [int(x) for x in line.split(",")]
            rec[v[0]] = v[1:]
    pops, projs = workloads.net_from_solver_param(sp)
    for p in pops:
        p.update(taua=0.05, adgain=1.0)
    conn = workloads.read_conn_map(w.conn, pops, projs)
    lgidx, wmask = extgen.stim_tables(schema.read_stim(sp.gen_param.stim_file))
    eps = float(np.float32(sp.gen_param.eps))
    net = capi.Net(pops, projs, float(np.float32(sp.gen_param.dt)), seed=w.meta["seed"], max_ticks=256, variant=1,
                   spike_buffer=25)
    try:
        for k, (ii, di) in enumerate(conn):
            net.set_conn(k, ii, di)
        net.upload_stimuli_idx(lgidx, eps, wmask)
        want = {}
        for r in extgen.segments(sp):
            net.use_stimulus(r.lgidx, r.wmask)
            net.run(r.first, r.n, r.prn, r.old_prn)
            bits = np.unpackbits(net.spike_log(0).view(np.uint8), axis=1, bitorder="little")
            for k in range(r.n):
                idx = np.nonzero(bits[k])[0].tolist()
                if idx:
                    want[r.first + k] = idx
    finally:
        net.close()
    assert rec == want
    assert len(want) > 100
