"""Checks of the CPU oracle itself: its transcription of the closed-form
trace decay against an independent solution of the trace ODEs, its
exp/log definition against the reference's libm calls, and its host-side
restatements against the reference's own fixture files."""
import json
import os

import numpy as np
import pytest
import scipy.linalg

from gsbn_b200 import schema, workloads
from oracle import sim
from tests.harness import load_workload, schedule

# the gsbn source tree ($GSBN_REFERENCE_ROOT, else oracle/Makefile's REF_ROOT), or None
REF = sim.reference_root()
GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "reference_fixtures.json")


def tiny_net(real_bits=64, taus=(0.004, 0.007, 0.02, 0.5)):
    pops = [dict(hcu_num=1, mcu_num=3, taum=0.01, wtagain=1.0, maxfq=100.0, igain=1.0, wgain=1.0, lgbias=0.0,
                 snoise=0.0)]
    tauzi, tauzj, taue, taup = taus
    projs = [dict(src_pop=0, dest_pop=0, tauzi=tauzi, tauzj=tauzj, taue=taue, taup=taup, maxfq=100.0, bgain=1.0,
                  wgain=1.0, tauepsc=0.0, slot_num=2.0)]
    return sim.OracleNet(pops, projs, 0.001, real_bits=real_bits), pops, projs


def test_closed_form_solves_the_trace_odes():
    """update_all (Proj.cpp:209-308) brings every cell from tij to simstep-1 in
    closed form; compare with expm of the linear system
    z' = -(kzi+kzj) z, e' = ke (z - e), p' = kp (e - p) (z = zi2*zj2) and
    zi' = -kzi zi, ei' = ke (zi - ei), pi' = kp (ei - pi) for the row."""
    net, pops, projs = tiny_net()
    rng = np.random.default_rng(5)
    n = 2 * 3
    pij, eij = rng.uniform(0.01, 0.2, n), rng.uniform(0.0, 0.3, n)
    zi2, zj2 = rng.uniform(0.0, 1.0, n), rng.uniform(0.0, 1.0, n)
    pi, ei, zi = rng.uniform(0.05, 0.5, 2), rng.uniform(0.0, 0.4, 2), rng.uniform(0.0, 1.0, 2)
    for k, v in dict(pij_0=pij, eij_0=eij, zi2_0=zi2, zj2_0=zj2, pi_0=pi, ei_0=ei, zi_0=zi).items():
        net.write(k, v)
    T = 37
    net.update(T + 1, 0.0, 1.0)   # prn 1 -> 0: all cells to simstep-1 = T with kp = dt/taup
    # gsbn holds dt and the time constants as float (gsbn.proto:13, 64-67)
    dt, tauzi, tauzj, taue, taup = (float(np.float32(v)) for v in (0.001, 0.004, 0.007, 0.02, 0.5))
    kzi, kzj, ke, kp = dt / tauzi, dt / tauzj, dt / taue, dt / taup
    A = np.array([[-(kzi + kzj), 0, 0], [ke, -ke, 0], [0, kp, -kp]])
    E = scipy.linalg.expm(A * T)
    x = E @ np.stack([zi2 * zj2, eij, pij])
    np.testing.assert_allclose(net.read("eij_0"), x[1], rtol=1e-9, atol=1e-14)
    np.testing.assert_allclose(net.read("pij_0"), x[2], rtol=1e-9, atol=1e-14)
    np.testing.assert_allclose(net.read("zi2_0"), zi2 * np.exp(-kzi * T), rtol=1e-12)
    np.testing.assert_allclose(net.read("zj2_0"), zj2 * np.exp(-kzj * T), rtol=1e-12)
    Ar = np.array([[-kzi, 0, 0], [ke, -ke, 0], [0, kp, -kp]])
    xr = scipy.linalg.expm(Ar * T) @ np.stack([zi, ei, pi])
    np.testing.assert_allclose(net.read("ei_0"), xr[1], rtol=1e-9)
    np.testing.assert_allclose(net.read("pi_0"), xr[2], rtol=1e-9)
    assert np.all(net.read("tij_0") == T) and np.all(net.read("ti_0") == T)


def replay_run(w, directory, ticks, **kw):
    sp, pops, projs, stim, conn, seed, phz = load_workload(w, directory)
    net = sim.OracleNet(pops, projs, 0.001, seed=seed, **kw)
    for k, (ii, di) in enumerate(conn):
        net.set_conn(k, ii, di)
    rng = np.random.default_rng(11)
    table = {t: sorted(rng.choice(pops[0]["hcu_num"] * pops[0]["mcu_num"], size=int(rng.integers(0, 5)),
                                  replace=False).tolist()) for t in range(1, ticks + 1)}
    net.set_ext_spikes(0, table)
    done = 0
    for r in schedule(sp, stim, pops, lambda x: np.float32(np.log(np.float64(x)))):
        n = min(r.n, ticks - done)
        if n <= 0:
            break
        net.set_stimulus(r.lginp, r.wmask)
        net.run(r.first, n, r.prn, r.old_prn, spikes=False)
        done += n
    return net


@pytest.mark.parametrize("name", ["pij_0", "eij_0", "wij_0", "pi_0", "pj_0", "epsc_0", "bj_0", "dsup_0"])
def test_shared_math_tracks_libm(tmp_path, name):
    """Same replayed spikes for 600 ticks: the oracle with the shared exp/log
    and with the reference's glibc calls agree to 1e-5 of each array's scale
    (its largest magnitude) on traces and weights; w_ij = log(ratio) is near
    zero for many cells, so the bound is not taken element by element."""
    w = workloads.config0()
    a = replay_run(w, str(tmp_path / "a"), 600).read(name).astype(np.float64)
    b = replay_run(w, str(tmp_path / "b"), 600, math=sim.MATH_LIBM).read(name).astype(np.float64)
    assert np.max(np.abs(a - b)) <= 1e-5 * np.abs(b).max()


def test_fp32_tracks_fp64(tmp_path):
    w = workloads.config0()
    a = replay_run(w, str(tmp_path / "a"), 400)
    b = replay_run(w, str(tmp_path / "b"), 400, real_bits=64)
    for name in ("pij_0", "eij_0", "wij_0"):
        x, y = a.read(name).astype(np.float64), b.read(name)
        assert np.max(np.abs(x - y)) <= 1e-4 * np.abs(y).max(), name


def test_exchange_spike_publishes_only_destination_populations():
    """ProcExchangeSpike copies the spikes of populations that receive a
    projection (ProcExchangeSpike.cpp:109-119); a pure source population's
    region of the shared buffer stays zero."""
    pops = [dict(hcu_num=2, mcu_num=2, taum=0.01, wtagain=1.0, maxfq=100.0, igain=1.0, wgain=1.0, lgbias=0.0,
                 snoise=0.0)] * 2
    q = dict(tauzi=0.01, tauzj=0.01, taue=0.02, taup=1.0, maxfq=100.0, bgain=1.0, wgain=1.0, tauepsc=0.0,
             slot_num=4.0)
    net = sim.OracleNet(pops, [dict(src_pop=0, dest_pop=1, **q), dict(src_pop=1, dest_pop=1, **q)], 0.001)
    net.set_ext_spikes(0, {1: [0, 3]})
    net.set_ext_spikes(1, {1: [1, 2]})
    net.set_stimulus(np.zeros(8, np.float32), np.zeros(4, np.float32))
    net.update(1, 1.0, 0.0)
    net.exchange()
    assert list(net.read("si_0")) == [0, 0, 0, 0]
    assert list(net.read("si_1")) == [0, 1, 1, 0]


def test_external_spike_file_format():
    text = "5,0,1,2\n5,1,7\n6,0\n-1,0,3,4\n7,0,9\n7,0,8\n"
    assert sim.parse_ext_spikes(text, 0) == {5: [1, 2], 7: [8]}
    assert sim.parse_ext_spikes(text, 1) == {5: [7]}


def test_recorder_and_check_formats(tmp_path):
    w = workloads.config0()
    sp, path = w.solver_param(str(tmp_path))
    r = sim.simulate(sp, str(tmp_path))
    assert r["rec"]["spk_pop_0.csv"].startswith("10,10,0.001,100\n")
    for line in r["rec"]["spk_pop_0.csv"].splitlines()[1:]:
        v = [int(x) for x in line.split(",")]
        assert v[1:] == sorted(v[1:]) and all(0 <= i < 100 for i in v[1:])
    assert r["check"][0].startswith("result | reference pattern")
    assert r["check"][-1].startswith("correct pattern: ")
    assert len(r["check"]) == 1 + 10 + 1
    assert r["correct"][1] == 10


@pytest.fixture(scope="module")
def golden():
    with open(GOLDEN) as f:
        return json.load(f)


@pytest.mark.skipif(REF is None, reason="reference tree not present")
def test_extgen_expansion_of_reference_prototxts(golden):
    for name, g in golden["prototxt"].items():
        with open(os.path.join(REF, "data", name)) as f:
            sp = schema.parse_prototxt(f.read())
        got = [[m["begin_step"], m["end_step"], m["lgidx_id"], m["lgexp_id"], m["wmask_id"], m["prn"]]
               for m in sim.extgen_modes(sp.gen_param)]
        assert got == g["modes"], name


@pytest.mark.skipif(REF is None, reason="reference tree not present")
def test_conn_map_of_reference_fixtures(golden):
    pops = [dict(hcu_num=400, mcu_num=10)]
    for name, g in golden["conn_map"].items():
        with open(os.path.join(REF, "data", name)) as f:
            text = f.read()
        projs = [dict(src_pop=0, dest_pop=0, slot_num=4000.0)]
        ii, di = sim.parse_conn_map(text, pops, projs)[0]
        C = 4000
        for prj, hcu, npairs, ssum, dsum in g["rows"]:
            row_ii, row_di = ii[hcu * C:(hcu + 1) * C], di[hcu * C:(hcu + 1) * C]
            assert int((row_ii >= 0).sum()) == npairs and int(row_ii[row_ii >= 0].sum()) == ssum
            assert int(row_di[row_ii >= 0].sum()) == dsum


def test_stimulus_fixture_decode(golden):
    g = golden["stim"]["stimuli_10x10_100_-1_rnd.bin"]
    assert (g["data_rows"], g["data_cols"], g["mask_rows"], g["mask_cols"]) == (200, 10, 2, 10)
    assert g["mask_head"][:20] == [0.0] * 19 + [1.0]
