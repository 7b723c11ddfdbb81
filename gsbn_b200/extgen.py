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
    population (logs[run][pop] = uint32 [ticks, words]).  Tick by tick this is
    ProcCheck's cursor walk; the ticks strictly inside a check window are
    summed as one span per run."""
    checks = _modes(sp.gen_param, only_prn0=True, clamp=False)
    counters = [np.zeros((h, m), np.int64) for h, m in pop_shapes]
    total_hcu = sum(h for h, _ in pop_shapes)
    cursor, correct, evaluated, updated = 0, 0, 0, False
    for r, plog in zip(runs, logs):
        bits = None
        k = 0
        while k < r.n and cursor < len(checks):
            t = r.first + k
            c = checks[cursor]
            if t <= c["begin"]:
                k += min(c["begin"] + 1 - t, r.n - k)  # ticks up to begin are skipped
                continue
            if t < c["end"]:
                k1 = min(c["end"] - r.first, r.n)  # ticks t .. end-1 of this run
                if bits is None:
                    bits = [np.unpackbits(l.view(np.uint8), axis=1, bitorder="little")[:, :h * m]
                            for l, (h, m) in zip(plog, pop_shapes)]
                for cnt, b, (h, m) in zip(counters, bits, pop_shapes):
                    cnt += b[k:k1].sum(axis=0, dtype=np.int64).reshape(h, m)
                updated = True
                k = k1
                continue
            if not updated:
                while cursor < len(checks) and t >= checks[cursor]["end"]:
                    cursor += 1
                k += 1
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
            k += 1
    return correct, evaluated


class DeviceCheck:
    """ProcCheck's evaluation (ProcCheck.cpp:149-237) with its counters on the
    device (bcpnn_check_count / bcpnn_check_result_async): call after_run(r)
    right after each net.run(r), then result() after net.sync().  The tick
    cursor is walked here exactly as recall() walks it; no spike log has to
    reach the host.  `alloc(n)` gives an int32 host buffer of n elements
    (page-locked, for copies that do not wait)."""

    def __init__(self, sp, lgidx, net, pop_shapes, threshold=0, alloc=None):
        self.checks = _modes(sp.gen_param, only_prn0=True, clamp=False)
        self.lgidx, self.net, self.shapes, self.threshold = lgidx, net, pop_shapes, threshold
        self.total_hcu = sum(h for h, _ in pop_shapes)
        alloc = alloc or (lambda n: np.zeros(n, np.int32))
        self.bufs = [[(alloc(h), alloc(h)) for h, _ in pop_shapes] for _ in self.checks]
        self.reset()

    def reset(self):
        self.cursor, self.updated, self.pending = 0, False, []

    def after_run(self, r):
        k = 0
        while k < r.n and self.cursor < len(self.checks):
            t = r.first + k
            c = self.checks[self.cursor]
            if t <= c["begin"]:
                k += min(c["begin"] + 1 - t, r.n - k)
                continue
            if t < c["end"]:
                k1 = min(c["end"] - r.first, r.n)
                for p in range(len(self.shapes)):
                    self.net.check_count(p, k, k1)
                self.updated = True
                k = k1
                continue
            if not self.updated:
                while self.cursor < len(self.checks) and t >= self.checks[self.cursor]["end"]:
                    self.cursor += 1
                k += 1
                continue
            for p, (idx, cnt) in enumerate(self.bufs[self.cursor]):
                self.net.check_result_async(p, idx, cnt)
            self.pending.append(self.cursor)
            self.cursor += 1
            k += 1

    def details(self):
        """[(check index, idx over all HCUs, count over all HCUs)] of the evaluated checks (after sync)"""
        return [(c, np.concatenate([b[0] for b in self.bufs[c]]), np.concatenate([b[1] for b in self.bufs[c]]))
                for c in self.pending]

    def result(self):
        """(correct, evaluated) after net.sync()"""
        correct = 0
        th = self.threshold
        for c, idx, num in self.details():
            exp = self.lgidx[self.checks[c]["lgexp"]][:self.total_hcu]
            ok = True
            for i in range(self.total_hcu):
                if ((num[i] < th or idx[i] != exp[i]) and exp[i] >= 0) or (num[i] > th and exp[i] < 0):
                    ok = False
                    break
            correct += int(ok)
        return correct, len(self.pending)
