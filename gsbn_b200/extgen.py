"""Stimulus schedule and recall evaluation for driving the C ABI from Python.

segments() expands a SolverParam's mode_param list the way ProcExtGen does
(src/gsbn/procedures/ProcExtGen.cpp:16-55 for the segment list, :113-153 for
the per-tick phase state) into runs of ticks with constant stimulus rows and
plasticity, ready for bcpnn_use_stimulus/bcpnn_set_stimulus_idx + bcpnn_run.
recall() applies ProcCheck's per-segment decision (ProcCheck.cpp:149-237,
ProcCheck/Pop.cpp:35-60) to spike logs.
"""
import numpy as np

f32 = np.float32


def _modes(gen_param, only_prn0=False, clamp=True):
    dt = f32(gen_param.dt)
    out = []
    for mp in gen_param.mode_param:
        b = int(f32(mp.begin_time) / dt)
        e = int(f32(mp.end_time) / dt)
        if e < b:
            raise ValueError("mode_param: end_time before begin_time")
        if only_prn0 and f32(mp.prn) != 0.0:
            continue
        lg, ex, wm = mp.begin_lgidx_id, mp.begin_lgexp_id, mp.begin_wmask_id
        while b < e:
            end = b + mp.time_step
            if clamp and end >= e:
                end = e
            out.append(dict(begin=b, end=end, lgidx=lg, lgexp=ex, wmask=wm, prn=float(f32(mp.prn))))
            lg += mp.lgidx_step
            ex += mp.lgexp_step
            wm += mp.wmask_step
            b = b + mp.time_step if not clamp else end
    return out


class Run:
    __slots__ = ("first", "n", "prn", "old_prn", "lgidx", "wmask")

    def __init__(self, first, n, prn, old_prn, lgidx, wmask):
        self.first, self.n, self.prn, self.old_prn, self.lgidx, self.wmask = first, n, prn, old_prn, lgidx, wmask


def segments(sp):
    """Runs of consecutive active ticks (cycle-flag 1) within one segment.
    old_prn is GlobalVar "old-prn" at a run's first tick: the previous active
    tick's prn (0 before the first, Solver.cpp:204-207)."""
    runs = []
    prn = 0.0
    last = 0  # last active tick; a segment overlapping its predecessor starts after it
    for m in _modes(sp.gen_param):
        first = max(m["begin"] + 1, last + 1)
        n = m["end"] - first + 1
        if n <= 0:
            continue
        runs.append(Run(first, n, m["prn"], prn, m["lgidx"], m["wmask"]))
        prn = m["prn"]
        last = m["end"]
    return runs


def stim_tables(stim):
    """(lgidx rows as int32, wmask rows as float32) of a StimRawData."""
    lg = np.array(stim.data, dtype=np.uint32).astype(np.int64)
    lg = np.where(lg >= 2 ** 31, lg - 2 ** 32, lg).astype(np.int32).reshape(stim.data_rows, stim.data_cols)
    wm = np.array(stim.mask, dtype=np.float32).reshape(stim.mask_rows, stim.mask_cols)
    return lg, wm


def recall(sp, lgidx, pop_shapes, runs, logs, threshold=0):
    """Correct / evaluated recall patterns from per-run spike logs of every
    population (logs[run][pop] = uint32 [ticks, words])."""
    checks = _modes(sp.gen_param, only_prn0=True, clamp=False)
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
                best = np.where(cnt.max(axis=1) > 0, cnt.argmax(axis=1), -1)
                idx.extend(best.tolist())
                num.extend(cnt.max(axis=1).tolist())
                cnt[:] = 0
            exp = lgidx[c["lgexp"]][:total_hcu]
            ok = True
            for i in range(total_hcu):
                if ((num[i] < threshold or idx[i] != exp[i]) and exp[i] >= 0) or (num[i] > threshold and exp[i] < 0):
                    ok = False
                    break
            correct += int(ok)
            evaluated += 1
            cursor += 1
    return correct, evaluated
