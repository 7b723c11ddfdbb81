"""Failure detection on the GPU without a fault: the bounded grid-barrier wait
of the persistent tick kernel runs out on an arrival nothing provides, the
kernel returns, the host reads the error word as BCPNN_ERR_DEVICE, and the
context keeps working (a parity run right after is still bit-exact)."""
import time

import numpy as np
import pytest

from gsbn_b200 import capi, workloads
from oracle import sim
from tests.harness import first_mismatch, load_workload, schedule, state

pytestmark = pytest.mark.gpu


def test_barrier_timeout_reported_and_context_survives(tmp_path):
    sp, pops, projs, stim, conn, seed, phz = load_workload(workloads.config0(), str(tmp_path))
    dt = float(np.float32(sp.gen_param.dt))
    gpu = capi.Net(pops, projs, dt, seed=seed)
    orc = sim.OracleNet(pops, projs, dt, seed=seed)
    for k, (ii, di) in enumerate(conn):
        gpu.set_conn(k, ii, di)
        orc.set_conn(k, ii, di)
    t0 = time.perf_counter()
    rc, msg = gpu.selftest_barrier_timeout(20_000_000)  # 20 ms
    elapsed = time.perf_counter() - t0
    assert rc == -6, msg
    assert "grid barrier" in msg and "timed out" in msg
    assert 0.015 < elapsed < 5.0
    # the error word was cleared and the context is usable
    runs = schedule(sp, stim, pops, orc.logf)
    for r in runs[:3]:
        orc.set_stimulus(r.lginp, r.wmask)
        gpu.set_stimulus(r.lginp, r.wmask)
        orc.run(r.first, r.n, r.prn, r.old_prn)
        gpu.run(r.first, r.n, r.prn, r.old_prn)
    assert first_mismatch(state(orc, 1, 1), state(gpu, 1, 1)) is None
    with pytest.raises(capi.BcpnnError):
        gpu._check(gpu._lib.bcpnn_selftest_barrier_timeout(gpu._h, 10))  # limit out of range
