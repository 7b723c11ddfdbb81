"""Host recall evaluation (gsbn_b200.extgen.recall, ProcCheck.cpp:149-237,
ProcCheck/Pop.cpp:35-60) sums the ticks inside a check window as spans; it
must give the same (correct, evaluated) as a tick-by-tick cursor walk, on the
workloads' schedules and on random spike logs dense enough that recall both
passes and fails."""
import numpy as np
import pytest

from gsbn_b200 import extgen, workloads


def tick_by_tick(sp, lgidx, pop_shapes, runs, logs, threshold=0):
    checks = extgen._modes(sp.gen_param, only_prn0=True, clamp=False)
    counters = [np.zeros((h, m), np.int64) for h, m in pop_shapes]
    total_hcu = sum(h for h, _ in pop_shapes)
    cursor, correct, evaluated, updated = 0, 0, 0, False
    for r, plog in zip(runs, logs):
        bits = [np.unpackbits(l.view(np.uint8), axis=1, bitorder="little")[:, :h * m]
                for l, (h, m) in zip(plog, pop_shapes)]
        for k in range(r.n):
            t = r.first + k
            if cursor >= len(checks):
                break
            c = checks[cursor]
            if t <= c["begin"]:
                continue
            if t < c["end"]:
                for cnt, b, (h, m) in zip(counters, bits, pop_shapes):
                    cnt += b[k].reshape(h, m)
                updated = True
                continue
            if not updated:
                while cursor < len(checks) and t >= checks[cursor]["end"]:
                    cursor += 1
                continue
            idx, num = [], []
            for cnt in counters:
                idx.extend(np.where(cnt.max(axis=1) > 0, cnt.argmax(axis=1), -1).tolist())
                num.extend(cnt.max(axis=1).tolist())
                cnt[:] = 0
            exp = lgidx[c["lgexp"]][:total_hcu]
            ok = all(not (((num[i] < threshold or idx[i] != exp[i]) and exp[i] >= 0) or (num[i] > threshold and exp[i] < 0))
                     for i in range(total_hcu))
            correct += int(ok)
            evaluated += 1
            cursor += 1
    return correct, evaluated


@pytest.mark.parametrize("make,seed,density", [("config0", 1, 0.02), ("config0", 2, 0.3), ("config2", 3, 0.05)])
def test_span_sums_equal_tick_walk(tmp_path, make, seed, density):
    kw = dict(n_patterns=6, train_ticks=40, recall_ticks=30) if make == "config2" else {}
    w = getattr(workloads, make)(**kw)
    sp, _ = w.solver_param(str(tmp_path))
    pops, _ = workloads.net_from_solver_param(sp)
    shapes = [(p["hcu_num"], p["mcu_num"]) for p in pops]
    from gsbn_b200 import schema
    lgidx, _ = extgen.stim_tables(schema.read_stim(sp.gen_param.stim_file))
    runs = extgen.segments(sp)
    rng = np.random.default_rng(seed)
    logs = []
    for r in runs:
        per = []
        for h, m in shapes:
            words = (h * m + 31) // 32
            b = (rng.random((r.n, words * 32)) < density).astype(np.uint8)
            # make the expected MCU of each HCU fire often in half the runs, so some recalls pass
            per.append(np.packbits(b, axis=1, bitorder="little").view(np.uint32).reshape(r.n, words))
        logs.append(per)
    checks = extgen._modes(sp.gen_param, only_prn0=True, clamp=False)
    total = sum(h for h, _ in shapes)
    for r, per in zip(runs, logs):
        cs = [c for c in checks if c["begin"] < r.first < c["end"]]
        if r.prn == 0.0 and cs and rng.random() < 0.5:
            # this run's ticks spike exactly the expected MCU of every HCU: its recall passes
            exp = lgidx[cs[0]["lgexp"]][:total]
            off = 0
            for (h, m), lg in zip(shapes, per):
                bits = np.zeros((r.n, lg.shape[1] * 32), np.uint8)
                for hh in range(h):
                    if 0 <= exp[off + hh] < m:
                        bits[:, hh * m + exp[off + hh]] = 1
                lg[:] = np.packbits(bits, axis=1, bitorder="little").view(np.uint32).reshape(lg.shape)
                off += h
    got = extgen.recall(sp, lgidx, shapes, runs, logs)
    want = tick_by_tick(sp, lgidx, shapes, runs, logs)
    assert got == want
    assert want[1] > 0 and 0 < want[0] < want[1]
