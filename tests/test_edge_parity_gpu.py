"""Parity at the edges of what the slot tables and populations allow.

gsbn starts every slot of a projection empty (ii = -1, Proj.cpp:88) and
ProcInitConn fills slots from a map file (ProcInitConn.cpp:92-103), so an
HCU may have any number of its C slots filled, in any position, and a source
MCU may appear in more than one slot.  Delays run from 1 to 31 ticks: the
delay queue is a 32-bit shift register that a spike enters at bit di - 1
(Proj.cpp:645-664).  A population may have one HCU or one MCU per HCU.
The cases:

  - sparse: 12x8 recurrent with C = 48; HCU 0 has no slot filled, HCU 1
    every slot, the others a random half at random positions (sources
    drawn with repetition); delays 1..31;
  - tiny: a 3x1 population (one MCU per HCU) and a 1x7 population (one
    HCU) with 30 Hz Poisson input noise; 3x1 -> 1x7 filled, 1x7 -> 3x1
    with every slot empty, 1x7 -> 1x7 with 31-tick delays;
  - widest: 2x512, the most MCUs a 512-thread CTA takes, full recurrent
    (C = 1024, 10^6 cells).

The time constants of a projection stay distinct (tauzi, tauzj != taue):
gsbn's closed-form decays divide by their differences.

Each case runs training segments and then recall segments (prn changes, so
the all-cells catch-up runs), compares the spikes of every tick and, at the
end, every state vector by bit pattern and the cell-update counters with the
oracle using the shared exp/log; every case also runs through the
ProcUpdMulti variant against its compiled restatement.
"""
import numpy as np
import pytest

from oracle import multi, sim
from tests.harness import first_mismatch, state
from tests.test_gpu_parity import gpu_net, spikes_of
from tests.test_multi_gpu import ARRAYS

pytestmark = pytest.mark.gpu

EPS = np.float32(1e-4)
DT = 0.001


def pop(H, M, maxfq=1000.0):
    return dict(hcu_num=H, mcu_num=M, taum=0.005, wtagain=1.0, maxfq=maxfq, igain=1.0, wgain=1.0, lgbias=0.0,
                snoise=0.0)


def proj(src, dest, C, tau=0.01):
    return dict(src_pop=src, dest_pop=dest, tauzi=tau, tauzj=tau, taue=0.02, taup=1.0, maxfq=1000.0, bgain=1.0,
                wgain=1.0, tauepsc=0.0, slot_num=float(C))


def sparse_case(rng):
    H, M, C = 12, 8, 48
    ii = np.full(H * C, -1, np.int32)
    di = np.zeros(H * C, np.int32)
    for h in range(H):
        filled = np.arange(C) if h == 1 else (np.array([], int) if h == 0 else
                                             np.sort(rng.choice(C, C // 2, replace=False)))
        ii[h * C + filled] = rng.integers(0, H * M, filled.size)
        di[h * C + filled] = rng.integers(1, 32, filled.size)
    di[1 * C:2 * C] = np.arange(C) % 31 + 1   # HCU 1 holds every delay
    return [pop(H, M)], [proj(0, 0, C)], [(ii, di)], 0.0


def tiny_case(rng):
    pops = [pop(3, 1), pop(1, 7)]
    projs = [proj(0, 1, 3), proj(1, 0, 7, tau=0.005), proj(1, 1, 7, tau=0.03)]
    conn = [(np.arange(3, dtype=np.int32), np.array([1, 2, 3], np.int32)),
            (np.full(3 * 7, -1, np.int32), np.zeros(3 * 7, np.int32)),
            (np.arange(7, dtype=np.int32), np.full(7, 31, np.int32))]
    return pops, projs, conn, 30.0


def widest_case(rng):
    H, M = 2, 512
    C = H * M
    ii = np.tile(np.arange(C, dtype=np.int32), H)
    di = rng.integers(1, 4, H * C).astype(np.int32)
    return [pop(H, M)], [proj(0, 0, C)], [(ii, di)], 0.0


CASES = {"sparse": sparse_case, "tiny": tiny_case, "widest": widest_case}


def runs_of(pops, rng, n_train=4, n_recall=2, train=40, recall=30):
    """(first, n, prn, old_prn, lginp, wmask) per run: training patterns
    (one MCU per HCU) without recurrent support, then recalls with the first
    third of every population's HCUs cued (at least one)."""
    hit, miss = sim.extgen_logf(1 + EPS), sim.extgen_logf(EPS)
    n_mcu = sum(p["hcu_num"] * p["mcu_num"] for p in pops)
    n_hcu = sum(p["hcu_num"] for p in pops)
    pats = []
    for _ in range(n_train):
        pat, off = np.full(n_mcu, miss, np.float32), 0
        for p in pops:
            H, M = p["hcu_num"], p["mcu_num"]
            pat[off + np.arange(H) * M + rng.integers(0, M, H)] = hit
            off += H * M
        pats.append(pat)
    out, t, prn = [], 1, 0.0
    for k in range(n_train):
        out.append((t, train, 1.0, prn, pats[k], np.zeros(n_hcu, np.float32)))
        t, prn = t + train, 1.0
    for k in range(n_recall):
        lg, wm = np.full(n_mcu, miss, np.float32), np.ones(n_hcu, np.float32)
        off, hoff = 0, 0
        for p in pops:
            H, M = p["hcu_num"], p["mcu_num"]
            cued = np.arange(max(1, H // 3))
            sel = off + (cued[:, None] * M + np.arange(M)).reshape(-1)
            lg[sel] = pats[k][sel]
            wm[hoff + cued] = 0.0
            off, hoff = off + H * M, hoff + H
        out.append((t, recall, 0.0, prn, lg, wm))
        t, prn = t + recall, 0.0
    return out


@pytest.mark.parametrize("mode", ["t512", "t256", "per_tick"])
@pytest.mark.parametrize("case", sorted(CASES))
def test_edge_parity_procupdlazy(case, mode):
    rng = np.random.default_rng(7)
    pops, projs, conn, phz = CASES[case](rng)
    if mode == "t256" and max(p["mcu_num"] for p in pops) > 256:
        pytest.skip("256-thread CTAs take at most 256 MCUs per HCU")
    orc = sim.OracleNet(pops, projs, DT, seed=9, poisson_hz=phz)
    kw = dict(tick_threads=256) if mode == "t256" else {}
    gpu = gpu_net(pops, projs, DT, seed=9, poisson_hz=phz, max_ticks=64, per_tick=(mode == "per_tick"), **kw)
    try:
        for q, (ii, di) in enumerate(conn):
            orc.set_conn(q, ii, di)
            gpu.set_conn(q, ii, di)
        spikes = 0
        for first, n, prn, old_prn, lg, wm in runs_of(pops, rng):
            orc.set_stimulus(lg, wm)
            gpu.set_stimulus(lg, wm)
            want = orc.run(first, n, prn, old_prn)
            gpu.run(first, n, prn, old_prn)
            got = spikes_of(gpu, pops, n)
            for t in range(n):
                for p in range(len(pops)):
                    assert np.array_equal(want[t][p], got[t][p]), f"spikes differ at simstep {first + t} pop {p}"
                    spikes += len(want[t][p])
        assert spikes > 100, spikes
        msg = first_mismatch(state(orc, len(pops), len(projs)), state(gpu, len(pops), len(projs)))
        assert msg is None, msg
        assert orc.counters() == gpu.counters()
    finally:
        gpu.close()


@pytest.mark.parametrize("per_tick", [False, True, "global"])
@pytest.mark.parametrize("case", sorted(CASES))
def test_edge_parity_procupdmulti(case, per_tick):
    """the same cases through the ProcUpdMulti variant (spike ring of 32
    ticks, adaptation on; without Poisson input noise, which the variant's
    restatement does not draw): the resident persistent launch (False), the
    persistent launch with the state in global memory, one launch per tick"""
    rng = np.random.default_rng(7)
    pops, projs, conn, _ = CASES[case](rng)
    for p in pops:
        p.update(taua=0.05, adgain=1.0)
    orc = multi.MultiNetC(pops, projs, DT, seed=9, spike_buffer=32)
    gpu = gpu_net(pops, projs, DT, seed=9, max_ticks=64, variant=1, spike_buffer=32, per_tick=per_tick)
    try:
        for q, (ii, di) in enumerate(conn):
            orc.set_conn(q, ii, di)
            gpu.set_conn(q, ii, di)
        spikes = 0
        for first, n, prn, old_prn, lg, wm in runs_of(pops, rng):
            orc.set_stimulus(lg, wm)
            gpu.set_stimulus(lg, wm)
            want = orc.run(first, n, prn, old_prn)
            gpu.run(first, n, prn, old_prn)
            for p in range(len(pops)):
                got = gpu.spike_log(p)
                assert np.array_equal(got, want[p]), f"pop {p}: spikes differ in the run at {first}"
                spikes += int(np.unpackbits(got.view(np.uint8)).sum())
        assert spikes > 100, spikes
        names = [f"{k}_{p}" for p in range(len(pops)) for k in ("dsup", "act", "ada", ".counter", "epsc", "bj")]
        names += [f"{k}_{q}" for q in range(len(projs))
                  for k in ("pi", "ei", "zi", "ti", "pj", "ej", "zj", "pij", "eij", "zj2", "wij", "qi")]
        for name in names:
            a, b = gpu.read(name), orc.read(name)
            b = np.asarray(b).astype(a.dtype)
            assert np.array_equal(a.view(np.uint8), b.view(np.uint8)), name
        assert orc.counters() == gpu.counters()
    finally:
        gpu.close()
