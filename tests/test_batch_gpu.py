"""The batch engine (include/bcpnn_batch.h) against the oracle, member by
member.

Eight members span the batch workload's shapes (HCUs 8 to 64, MCUs 5 to 50,
full recurrent connectivity, up to C = 3200 slots per HCU, 1e7 cells), each
with its own seed, patterns and connectivity.  They run one schedule together
-- two patterns trained 40 ticks each, then two recalls of 25 ticks, so the
all-cells catch-up at the change of prn is included -- under several launch
shapes of the engine (CTA size, cost model of the warp schedule).  Every
member's spike train is compared with its own CPU oracle (the shared-math
restatement, one network alone) tick by tick, and every state vector bit for
bit at the end, including the delay queue (qi, .siq) that the engine keeps
as an arrival ring.
"""
import numpy as np
import pytest

from gsbn_b200 import batch, capi
from oracle import sim
from tests.harness import first_mismatch

pytestmark = pytest.mark.gpu

SHAPES = [(8, 5), (8, 50), (64, 5), (64, 50), (20, 12), (33, 27), (12, 40), (50, 9)]
NAMES = ("pij_0", "eij_0", "zi2_0", "zj2_0", "wij_0", "tij_0", "pi_0", "ei_0", "zi_0", "ti_0", "qi_0", ".siq_0",
         "pj_0", "ej_0", "zj_0", "dsup_0", "act_0", "epsc_0", "bj_0", "spike_0", "si_0", ".counter_0")


def members():
    out = []
    for k, (H, M) in enumerate(SHAPES):
        m = batch.make_members(n=1, seed=100 + k, hcu=(H, H), mcu=(M, M), n_patterns=2)[0]
        out.append(m)
    return out


def oracle_of(m):
    orc = sim.OracleNet([m.pop], [m.proj], 0.001, seed=m.seed)
    orc.set_conn(0, m.ii, m.di)
    return orc


def lginp(m, row):
    hit, miss = sim.extgen_logf(np.float32(1) + np.float32(1e-4)), sim.extgen_logf(np.float32(1e-4))
    out = np.full(m.H * m.M, miss, np.float32)
    for h in range(m.H):
        if 0 <= m.lgidx[row][h] < m.M:
            out[h * m.M + m.lgidx[row][h]] = hit
    return out


@pytest.mark.parametrize("threads,lpt", [(512, (0, 0, 0)), (384, (0, 0, 0)), (256, (0, 0, 0)), (512, (1, 0, 0))])
def test_batch_members_match_their_oracles(threads, lpt):
    ms = members()
    eng = batch.BatchEngine(ms, max_ticks=64, threads=threads, lpt=lpt)
    orcs = [oracle_of(m) for m in ms]
    runs = batch.schedule(2, train_ticks=40, recall_ticks=25)
    assert any(r[2] != r[3] for r in runs[1:])
    try:
        spikes = 0
        for first, n, prn, old_prn, lg_row, wm_row in runs:
            eng.run_segment(first, n, prn, old_prn, lg_row, wm_row)
            for k, (m, orc) in enumerate(zip(ms, orcs)):
                orc.set_stimulus(lginp(m, lg_row), m.wmask[wm_row][:m.H])
                want = orc.run(first, n, prn, old_prn)
                bits = np.unpackbits(eng.spike_log(k).view(np.uint8), axis=1, bitorder="little")[:, :m.H * m.M]
                for t in range(n):
                    got = np.nonzero(bits[t])[0]
                    assert np.array_equal(got, want[t][0]), f"member {k} {m.H}x{m.M}: spikes differ at {first + t}"
                    spikes += len(got)
        for k, (m, orc) in enumerate(zip(ms, orcs)):
            msg = first_mismatch({n: orc.read(n) for n in NAMES}, {n: eng.read(k, n) for n in NAMES})
            assert msg is None, f"member {k} {m.H}x{m.M}: {msg}"
        assert spikes > 1000
        rows = sum(o.counters()[0] for o in orcs)
        cols = sum(o.counters()[1] for o in orcs)
        alls = sum(o.counters()[2] for o in orcs)
        assert eng.counters() == [rows, cols, alls]
    finally:
        eng.close()


def test_batch_tuner_picks_a_shape_and_resets():
    ms = members()[:4]
    eng = batch.BatchEngine(ms, max_ticks=64)
    try:
        shape, us = eng.tune(8, train_rows=(0, 0), recall_rows=(2, 1))
        assert shape[0] in (256, 384, 512) and us > 0
        # the batch is back at the initial state: a run matches the oracle
        orc = oracle_of(ms[0])
        eng.run_segment(1, 20, 1.0, 0.0, 0, 0)
        orc.set_stimulus(lginp(ms[0], 0), ms[0].wmask[0][:ms[0].H])
        orc.run(1, 20, 1.0, 0.0)
        assert first_mismatch({n: orc.read(n) for n in NAMES}, {n: eng.read(0, n) for n in NAMES}) is None
    finally:
        eng.close()
