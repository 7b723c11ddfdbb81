"""Schema declaration, synthetic workloads and the product-side schedule /
connectivity helpers, cross-checked against the oracle's restatements."""
import numpy as np
import pytest

from gsbn_b200 import extgen, schema, workloads
from oracle import sim
from tests.harness import load_workload, schedule


def test_tick_time_truncation():
    for t in (0, 1, 99, 100, 119, 120, 1200, 2200, 9999, 10000, 20000):
        x = workloads.tick_time(t, 0.001)
        assert int(np.float32(x) / np.float32(0.001)) == t


@pytest.mark.parametrize("make", [workloads.config0, workloads.config1, workloads.config2,
                                  lambda: workloads.small_scale(hcu=12, mcu=7, src=3)])
def test_product_schedule_and_connectivity_match_oracle(tmp_path, make):
    w = make()
    sp, pops, projs, stim, conn, seed, phz = load_workload(w, str(tmp_path))
    ref = schedule(sp, stim, pops, lambda x: np.float32(np.log(np.float64(x))))
    got = extgen.segments(sp)
    assert [(r.first, r.n, r.prn, r.old_prn) for r in got] == [(r.first, r.n, r.prn, r.old_prn) for r in ref]
    lgidx, wmask = extgen.stim_tables(stim)
    for a, b in zip(got, ref):
        assert np.array_equal(wmask[a.wmask], b.wmask)
    p2, q2 = workloads.net_from_solver_param(sp)
    assert (p2, q2) == sim.net_from_solver_param(sp)
    for (ii, di), (jj, dj) in zip(workloads.read_conn_map(w.conn, pops, projs), conn):
        assert np.array_equal(ii, jj) and np.array_equal(di, dj)


def test_config_shapes():
    w = workloads.config1()
    assert w.meta["cells"] == 10 ** 7 and w.meta["C"] == 1000 and w.meta["ticks"] == 20000
    w0 = workloads.config0()
    assert w0.meta["ticks"] == 2200 and w0.meta["C"] == 100


def test_stim_roundtrip(tmp_path):
    w = workloads.config0()
    path = w.write(str(tmp_path))
    sp = schema.parse_prototxt(open(path).read())
    st = schema.read_stim(sp.gen_param.stim_file)
    lg, wm = extgen.stim_tables(st)
    assert lg.shape == (21, 10) and wm.shape == (2, 10)
    assert np.all(lg[20] == 0x7FFFFFFF)
    assert list(wm[1]) == [0, 0, 0, 1, 1, 1, 1, 1, 1, 1]


def test_conn_map_first_empty_slot_semantics():
    pops = [dict(hcu_num=2, mcu_num=2)]
    projs = [dict(src_pop=0, dest_pop=0, slot_num=3.0)]
    text = "0,1,3,2,-1,1,2,1,0,1\n0,0\n0,0,1,1\n"
    (ii, di), = workloads.read_conn_map(text, pops, projs)
    (jj, dj), = sim.parse_conn_map(text, pops, projs)
    assert list(ii) == [1, -1, -1, 3, 2, 0] and list(di) == [1, 0, 0, 2, 1, 1]
    assert np.array_equal(ii, jj) and np.array_equal(di, dj)
