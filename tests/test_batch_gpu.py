"""Batches of independent networks: a member inside a group (one
multi-population network, per-population Philox keys) computes the same bits
as the same network alone, whether its group runs alone or beside other
groups on other streams; the schedule tuner picks a candidate and caches it."""
import json

import numpy as np
import pytest

from gsbn_b200 import batch, capi

pytestmark = pytest.mark.gpu

NAMES = ("pij_0", "eij_0", "zi2_0", "zj2_0", "wij_0", "tij_0", "pi_0", "qi_0", "pj_0", "dsup_0", "epsc_0", "bj_0",
         "spike_0", ".counter_0")


def standalone(m):
    net = capi.Net([m.pop], [m.proj], 0.001, seed=m.seed, max_ticks=128)
    net.set_conn(0, m.ii, m.di)
    net.upload_stimuli_idx(m.lgidx, 1e-4, m.wmask)
    return net


@pytest.mark.parametrize("groups,concurrent,threads", [([[0, 1, 2, 3, 4]], False, 512),
                                                        ([[0, 3], [1, 2, 4]], True, 512),
                                                        ([[0, 1, 2, 3, 4]], False, 256),
                                                        ([[0, 3], [1, 2, 4]], True, 256)])
def test_members_match_standalone(groups, concurrent, threads):
    ms = batch.make_members(n=5, seed=3, hcu=(8, 14), mcu=(5, 12), n_patterns=3)
    runs = batch.schedule(3, train_ticks=30, recall_ticks=20)
    b = batch.Batch(ms, groups, concurrent=concurrent, threads=threads)
    singles = [standalone(m) for m in ms]
    for first, n, prn, old, lg, wm in runs:
        b.run_segment(first, n, prn, old, lg, wm)
        for net in singles:
            net.use_stimulus(lg, wm)
            net.run(first, n, prn, old)
    b.sync()
    for i in range(len(ms)):
        for name in NAMES:
            got, want = b.member_state(i, name), singles[i].read(name)
            assert np.array_equal(got.view(np.uint8), want.view(np.uint8)), f"member {i} {name}"
    assert b.counters() == sum(sum(n.counters()) for n in singles)
    b.close()


def test_tuner_picks_and_caches(tmp_path):
    ms = batch.make_members(n=6, seed=5, hcu=(8, 12), mcu=(5, 8), n_patterns=2)
    cache = str(tmp_path / "tune.json")
    cands = [("one", 1, 512), ("buckets", 2, 256), ("plain", 1, 512)]
    best, times = batch.tune(ms, probe_ticks=5, cache=cache, candidates=cands)
    assert best in cands and set(times) == {"one1/t512", "buckets2/t256", "plain1/t512"}
    with open(cache) as f:
        assert batch.shape_key(ms) in json.load(f)
    again, times2 = batch.tune(ms, probe_ticks=5, cache=cache, candidates=cands)
    assert tuple(again) == tuple(best) and times2 == times
