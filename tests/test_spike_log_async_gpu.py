"""bcpnn_get_spike_log_async: each run's spike log queued into its own
page-locked buffer with no wait, one bcpnn_sync at the end, must equal the
logs read synchronously after every run by a second network on the same
inputs (config 0, 10x10, every segment)."""
import numpy as np
import pytest
import torch

from tests.harness import load_workload, schedule
from tests.test_gpu_parity import gpu_net
from oracle import sim
from gsbn_b200 import workloads

pytestmark = pytest.mark.gpu


def test_async_logs_equal_sync_logs(tmp_path):
    sp, pops, projs, stim, conn, seed, phz = load_workload(workloads.config0(), str(tmp_path))
    dt = float(np.float32(sp.gen_param.dt))
    orc = sim.OracleNet(pops, projs, dt, seed=seed, poisson_hz=phz)
    runs = schedule(sp, stim, pops, orc.logf)
    nets = [gpu_net(pops, projs, dt, seed=seed, poisson_hz=phz, max_ticks=256) for _ in range(2)]
    try:
        for net in nets:
            for k, (ii, di) in enumerate(conn):
                net.set_conn(k, ii, di)
        words = (pops[0]["hcu_num"] * pops[0]["mcu_num"] + 31) // 32
        pinned = [torch.zeros((r.n, words), dtype=torch.int32, pin_memory=True).numpy().view(np.uint32) for r in runs]
        want = []
        for r, buf in zip(runs, pinned):
            for net in nets:
                net.set_stimulus(r.lginp, r.wmask)
                net.run(r.first, r.n, r.prn, r.old_prn)
            nets[0].spike_log_async(0, buf)
            want.append(nets[1].spike_log(0))
        nets[0].sync()
        assert len(runs) > 10
        for k, (a, b) in enumerate(zip(pinned, want)):
            assert np.array_equal(a, b), k
        assert sum(int(np.unpackbits(a.view(np.uint8)).sum()) for a in pinned) > 100
    finally:
        for net in nets:
            net.close()


def test_stimulus_rows_from_indices_on_device(tmp_path):
    """bcpnn_set_stimulus_idx builds the lginp row on the device; a network fed
    that way must spike exactly like one fed from device stimulus tables built
    on the host (bcpnn_upload_stimuli_idx + bcpnn_use_stimulus)."""
    from gsbn_b200 import extgen, schema
    w = workloads.config0()
    sp, path = w.solver_param(str(tmp_path))
    pops, projs = workloads.net_from_solver_param(sp)
    conn = workloads.read_conn_map(w.conn, pops, projs)
    lgidx, wmask = extgen.stim_tables(schema.read_stim(sp.gen_param.stim_file))
    eps = float(np.float32(sp.gen_param.eps))
    runs = extgen.segments(sp)
    dt = float(np.float32(sp.gen_param.dt))
    nets = [gpu_net(pops, projs, dt, seed=w.meta["seed"], max_ticks=256) for _ in range(2)]
    try:
        for net in nets:
            for k, (ii, di) in enumerate(conn):
                net.set_conn(k, ii, di)
        nets[1].upload_stimuli_idx(lgidx, eps, wmask)
        for r in runs:
            nets[0].set_stimulus_idx(lgidx[r.lgidx], eps, wmask[r.wmask])
            nets[1].use_stimulus(r.lgidx, r.wmask)
            for net in nets:
                net.run(r.first, r.n, r.prn, r.old_prn)
            assert np.array_equal(nets[0].spike_log(0), nets[1].spike_log(0)), r.first
        assert len(runs) > 10
    finally:
        for net in nets:
            net.close()


@pytest.mark.parametrize("make", ["config0", "config2"])
def test_stimulus_tables_uploaded_async(tmp_path, make):
    """bcpnn_upload_stimuli_idx_async, once per pass from page-locked tables,
    then bcpnn_use_stimulus per segment, with no wait between: the same
    spikes and end state as tables uploaded synchronously; a second pass
    re-uploads into the tables (no growth), a third with an extra row grows
    them."""
    from gsbn_b200 import extgen
    sp, pops, projs, stim, conn, seed, phz = load_workload(getattr(workloads, make)(), str(tmp_path))
    lgidx, wmask = extgen.stim_tables(stim)
    eps = float(np.float32(sp.gen_param.eps))
    runs = extgen.segments(sp)[:30]
    dt = float(np.float32(sp.gen_param.dt))
    nets = [gpu_net(pops, projs, dt, seed=seed, poisson_hz=phz, max_ticks=256) for _ in range(2)]
    words = (pops[0]["hcu_num"] * pops[0]["mcu_num"] + 31) // 32
    try:
        for net in nets:
            for k, (ii, di) in enumerate(conn):
                net.set_conn(k, ii, di)
        nets[0].upload_stimuli_idx(lgidx, eps, wmask)
        lg_pin = torch.zeros(lgidx.shape, dtype=torch.int32, pin_memory=True).numpy()
        wm_pin = torch.zeros(wmask.shape, dtype=torch.float32, pin_memory=True).numpy()
        lg_pin[:], wm_pin[:] = lgidx, wmask
        logs = [torch.zeros((r.n, words), dtype=torch.int32, pin_memory=True).numpy().view(np.uint32) for r in runs]
        for extra in (0, 0, 1):
            lg_t, wm_t = lg_pin, wm_pin
            if extra:
                lg_t = torch.zeros((lgidx.shape[0] + 1, lgidx.shape[1]), dtype=torch.int32, pin_memory=True).numpy()
                wm_t = torch.zeros((wmask.shape[0] + 1, wmask.shape[1]), dtype=torch.float32, pin_memory=True).numpy()
                lg_t[:-1], wm_t[:-1] = lgidx, wmask
                lg_t[-1], wm_t[-1] = -1, 1.0
            for net in nets:
                net.reset()
            nets[1].upload_stimuli_idx_async(lg_t, eps, wm_t)
            want = []
            for r, buf in zip(runs, logs):
                for net in nets:
                    net.use_stimulus(r.lgidx, r.wmask)
                    net.run(r.first, r.n, r.prn, r.old_prn)
                nets[1].spike_log_async(0, buf)
                want.append(nets[0].spike_log(0))
            nets[1].sync()
            for k, (a, b) in enumerate(zip(logs, want)):
                assert np.array_equal(a, b), (extra, k)
            for name in ("dsup_0", "pij_0", "wij_0", "epsc_0"):
                assert np.array_equal(nets[0].read(name).view(np.uint32), nets[1].read(name).view(np.uint32)), name
        assert sum(int(np.unpackbits(a.view(np.uint8)).sum()) for a in logs) > 100
    finally:
        for net in nets:
            net.close()


@pytest.mark.parametrize("make", ["config0", "config2"])
def test_recall_counters_on_device(tmp_path, make):
    """ProcCheck's counters on the device (extgen.DeviceCheck) must give the
    same (correct, evaluated) as the host evaluation of the spike logs, and
    per evaluated segment the same per-HCU winner and count."""
    from gsbn_b200 import extgen, schema
    w = workloads.config2(n_patterns=8, train_ticks=60, recall_ticks=30) if make == "config2" else workloads.config0()
    sp, path = w.solver_param(str(tmp_path))
    pops, projs = workloads.net_from_solver_param(sp)
    conn = workloads.read_conn_map(w.conn, pops, projs)
    lgidx, wmask = extgen.stim_tables(schema.read_stim(sp.gen_param.stim_file))
    eps = float(np.float32(sp.gen_param.eps))
    runs = extgen.segments(sp)
    dt = float(np.float32(sp.gen_param.dt))
    shapes = [(p["hcu_num"], p["mcu_num"]) for p in pops]
    _, _, _, _, _, seed, phz = load_workload(w, str(tmp_path / "w"))
    net = gpu_net(pops, projs, dt, seed=seed, poisson_hz=phz, max_ticks=256)
    try:
        for k, (ii, di) in enumerate(conn):
            net.set_conn(k, ii, di)
        net.upload_stimuli_idx(lgidx, eps, wmask)
        dc = extgen.DeviceCheck(sp, lgidx, net, shapes)
        logs = []
        for r in runs:
            net.use_stimulus(r.lgidx, r.wmask)
            net.run(r.first, r.n, r.prn, r.old_prn)
            dc.after_run(r)
            logs.append([net.spike_log(p) for p in range(len(pops))])
        net.sync()
        want = extgen.recall(sp, lgidx, shapes, runs, logs)
        assert dc.result() == want
        assert want[1] > 0
        # winners and counts of each evaluated segment from the logs on the host
        checks = dc.checks
        for c, idx, cnt in dc.details():
            b, e = checks[c]["begin"], checks[c]["end"]
            tot = []
            for (h, m), p in zip(shapes, range(len(shapes))):
                acc = np.zeros(h * m, np.int64)
                for r, lg in zip(runs, logs):
                    bits = np.unpackbits(lg[p].view(np.uint8), axis=1, bitorder="little")[:, :h * m]
                    ks = [k for k in range(r.n) if b < r.first + k < e]
                    if ks:
                        acc += bits[ks].sum(axis=0, dtype=np.int64)
                tot.append(acc.reshape(h, m))
            exp_idx = np.concatenate([np.where(a.max(1) > 0, a.argmax(1), -1) for a in tot])
            exp_cnt = np.concatenate([a.max(1) for a in tot])
            assert np.array_equal(idx, exp_idx) and np.array_equal(cnt, exp_cnt), c
    finally:
        net.close()
