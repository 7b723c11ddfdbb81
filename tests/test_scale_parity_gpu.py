"""Parity at the 100x100 network's full size: 100 HCUs x 100 MCUs, recurrent
density 0.1, so C = 1000 slots per HCU and 1e7 synaptic cells.  The sm_100a
path through the C ABI is held to the oracle on a short schedule of that
network: 3 patterns trained 100 ticks each, then 3 recalls of 50 ticks, so
the all-cells catch-up at the change of prn is included.  At this size one
spiking MCU's column is four 256-slot units that the whole grid shares in
the persistent launch; the smaller parity workloads (C <= 120) never split
a column.  Spikes are compared every tick, every state vector by bit
pattern at the end, and the cell-update counters.  ProcUpdMulti is held to
its compiled oracle (oracle/bcpnn_oracle_multi.cpp) the same way."""
import numpy as np
import pytest

from gsbn_b200 import extgen, schema, workloads
from oracle import multi
from tests.test_gpu_parity import compare_runs, gpu_net, make_pair
from tests.test_multi_gpu import ARRAYS, lginp_row

pytestmark = pytest.mark.gpu


def workload():
    return workloads.small_scale(hcu=100, mcu=100, src=10, n_patterns=3, train_ticks=100, recall_ticks=50)


@pytest.fixture(params=["persistent", "per_tick", "t256"])
def mode(request):
    return {"persistent": False, "per_tick": True, "t256": "t256"}[request.param]


def test_full_size_100x100(tmp_path, mode):
    sp, pops, projs, orc, gpu, runs = make_pair(workload(), tmp_path, per_tick=mode)
    try:
        assert min(pops[0]["hcu_num"] * pops[0]["mcu_num"], int(np.float32(projs[0]["slot_num"]))) == 1000
        assert any(r.prn != r.old_prn for r in runs[1:])
        n = compare_runs(pops, projs, orc, gpu, runs, full_every_run=False)
        assert n > 1000
        assert orc.counters() == gpu.counters()
    finally:
        gpu.close()


@pytest.mark.parametrize("per_tick", [False, True])
def test_full_size_100x100_procupdmulti(tmp_path, per_tick):
    w = workload()
    sp, _ = w.solver_param(str(tmp_path))
    pops, projs = workloads.net_from_solver_param(sp)
    for p in pops:
        p.update(taua=0.05, adgain=1.0)
    conn = workloads.read_conn_map(w.conn, pops, projs)
    lgidx, wmask = extgen.stim_tables(schema.read_stim(sp.gen_param.stim_file))
    eps = np.float32(sp.gen_param.eps)
    dt = float(np.float32(sp.gen_param.dt))
    runs = extgen.segments(sp)
    assert any(r.prn != r.old_prn for r in runs[1:])
    orc = multi.MultiNetC(pops, projs, dt, seed=w.meta["seed"], spike_buffer=25)
    gpu = gpu_net(pops, projs, dt, seed=w.meta["seed"], max_ticks=256, variant=1, spike_buffer=25, per_tick=per_tick)
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
            assert np.array_equal(a.view(np.uint8), b.view(np.uint8)), f"{name} at the end"
        assert spikes > 1000
        assert orc.counters() == gpu.counters()
    finally:
        gpu.close()
