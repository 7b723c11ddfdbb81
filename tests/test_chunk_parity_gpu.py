"""Parity where a tick's active rows overflow one row chunk.

The tick kernel stages the active rows of a destination HCU in chunks of as
many cells as the CTA has threads (512, or 256 for 256-thread CTAs), i.e. 25
or 12 rows of 20 MCUs; ProcUpdMulti stages 1024 cells (51 rows).  Only a
network whose HCUs see more active rows per tick than that exercises the
chunk loop, and the benchmark-shaped workloads rarely do.  A small network
firing fast does: 40 HCUs x 20 MCUs with maxfq = 1000 Hz (maxfq dt = 1, so
about one spike per HCU per tick), each HCU fed by 30 source HCUs (C = 600,
4.8e5 cells).  The ProcUpdMulti variant uses 64 HCUs fed by 60 sources
(C = 1200) to cross its 51-row chunk.  Patterns change every 40 ticks and
prn switches from training to recall, so the catch-up sweep is included.
Spikes are compared every run and every state vector by bit pattern at the
end, against the oracle with the shared exp/log (MATH_SHARED for ProcUpdLazy,
the compiled ProcUpdMulti restatement for the variant)."""
import numpy as np
import pytest

from oracle import multi, sim
from tests.harness import first_mismatch, state
from tests.test_gpu_parity import gpu_net, spikes_of
from tests.test_multi_gpu import ARRAYS

pytestmark = pytest.mark.gpu

M = 20
EPS = np.float32(1e-4)


def network(H, S, seed):
    pops = [dict(hcu_num=H, mcu_num=M, taum=0.005, wtagain=1.0, maxfq=1000.0, igain=1.0, wgain=1.0, lgbias=0.0,
                 snoise=0.0)]
    projs = [dict(src_pop=0, dest_pop=0, tauzi=0.01, tauzj=0.01, taue=0.02, taup=1.0, maxfq=1000.0, bgain=1.0,
                  wgain=1.0, tauepsc=0.0, slot_num=float(S * M))]
    rng = np.random.default_rng(seed)
    C = S * M
    ii = np.full(H * C, -1, np.int32)
    di = np.zeros(H * C, np.int32)
    for h in range(H):
        src = np.sort(rng.choice(H, S, replace=False))
        ii[h * C:(h + 1) * C] = np.concatenate([np.arange(s * M, (s + 1) * M) for s in src])
        di[h * C:(h + 1) * C] = 1 + (np.arange(C) % 3)   # delays 1..3 ticks
    return pops, projs, ii, di, rng


def runs_of(H, rng, n_train=4, n_recall=2, train=40, recall=30):
    """(first, n, prn, old_prn, lginp, wmask) per run: training patterns
    without recurrent support, then recalls with a third of the HCUs cued."""
    hit, miss = sim.extgen_logf(1 + EPS), sim.extgen_logf(EPS)
    pats = rng.integers(0, M, (n_train, H))
    out, t, prn = [], 1, 0.0
    for k in range(n_train):
        lg = np.full(H * M, miss, np.float32)
        lg[np.arange(H) * M + pats[k]] = hit
        out.append((t, train, 1.0, prn, lg, np.zeros(H, np.float32)))
        t, prn = t + train, 1.0
    for k in range(n_recall):
        lg = np.full(H * M, miss, np.float32)
        cued = np.arange(H // 3)
        lg[cued * M + pats[k][cued]] = hit
        wm = np.ones(H, np.float32)
        wm[cued] = 0.0
        out.append((t, recall, 0.0, prn, lg, wm))
        t, prn = t + recall, 0.0
    return out


@pytest.mark.parametrize("mode", ["t512", "t256", "per_tick"])
def test_row_chunks_overflow_procupdlazy(mode):
    H, S = 40, 30
    pops, projs, ii, di, rng = network(H, S, seed=3)
    orc = sim.OracleNet(pops, projs, 0.001, seed=5)
    kw = dict(tick_threads=256) if mode == "t256" else {}
    gpu = gpu_net(pops, projs, 0.001, seed=5, max_ticks=64, per_tick=(mode == "per_tick"), **kw)
    rows_per_chunk = (256 if mode == "t256" else 512) // M
    try:
        orc.set_conn(0, ii, di)
        gpu.set_conn(0, ii, di)
        most_rows, ticks_over = 0, 0
        for first, n, prn, old_prn, lg, wm in runs_of(H, rng):
            orc.set_stimulus(lg, wm)
            gpu.set_stimulus(lg, wm)
            want = []
            for k in range(n):
                orc.update(first + k, prn, old_prn if k == 0 else prn)
                orc.exchange()
                want.append(np.nonzero(orc.read("spike_0"))[0])
                rows = orc.read(".siq_0").reshape(H, S * M).sum(axis=1)
                most_rows = max(most_rows, int(rows.max()))
                ticks_over += int(rows.max() > rows_per_chunk)
            gpu.run(first, n, prn, old_prn)
            got = spikes_of(gpu, pops, n)
            for t in range(n):
                assert np.array_equal(want[t], got[t][0]), f"spikes differ at simstep {first + t}"
        # the case is only meaningful if the chunk loop ran
        assert ticks_over > 100 and most_rows > rows_per_chunk + 5, (ticks_over, most_rows)
        msg = first_mismatch(state(orc, 1, 1), state(gpu, 1, 1))
        assert msg is None, msg
        assert orc.counters() == gpu.counters()
    finally:
        gpu.close()


@pytest.mark.parametrize("per_tick", [False, True, "global"])
def test_row_chunks_overflow_procupdmulti(per_tick):
    H, S = 64, 60
    pops, projs, ii, di, rng = network(H, S, seed=4)
    for p in pops:
        p.update(taua=0.05, adgain=1.0)
    orc = multi.MultiNetC(pops, projs, 0.001, seed=6, spike_buffer=25)
    gpu = gpu_net(pops, projs, 0.001, seed=6, max_ticks=64, variant=1, spike_buffer=25, per_tick=per_tick)
    try:
        orc.set_conn(0, ii, di)
        gpu.set_conn(0, ii, di)
        spikes = 0
        for first, n, prn, old_prn, lg, wm in runs_of(H, rng, n_train=3, n_recall=2, train=30, recall=20):
            orc.set_stimulus(lg, wm)
            gpu.set_stimulus(lg, wm)
            want = orc.run(first, n, prn, old_prn)
            gpu.run(first, n, prn, old_prn)
            got = gpu.spike_log(0)
            assert np.array_equal(got, want[0]), f"spikes differ in the run at {first}"
            spikes += int(np.unpackbits(got.view(np.uint8)).sum())
        # about one spike per HCU per tick: a destination HCU sees up to ~60
        # active 20-cell rows per tick (71 of the 130 ticks beyond 51 in the
        # ProcUpdLazy oracle of the same network)
        assert spikes > 64 * 130 * 0.5
        for name in ARRAYS:
            a, b = gpu.read(name), orc.read(name)
            b = np.asarray(b).astype(a.dtype)
            assert np.array_equal(a.view(np.uint8), b.view(np.uint8)), name
        assert orc.counters() == gpu.counters()
    finally:
        gpu.close()
