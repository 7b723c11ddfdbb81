"""Batches of independent networks on one GPU.

A batch member is a complete network of its own (one population with a full
recurrent projection, its own patterns, connectivity and Philox seed).  Members
are packed into groups; a group is built as one multi-population network
through the C ABI, one population and one projection per member, each
population keyed with its member's seed as population 0
(bcpnn_set_pop_rng), so a member draws exactly the numbers, and computes
exactly the state, it would as a network of its own.  Several groups run side
by side on their own CUDA streams (one CUDA-graph-captured launch per tick
each); a lone group whose HCUs all fit on the GPU at once runs one persistent
launch per segment.

The schedule (which members go together, and the CTA size of the tick
kernel) is chosen by `tune`: it times each candidate on the first training
ticks and keeps the fastest, cached by the member shapes.  Candidates:
everything in one group; k groups of similar size (sorted by slots per HCU,
so that a group's shared memory is sized for members like it); one group per
member run one after the other (one network per launch, the plain path);
each with 512-thread CTAs (one per SM) or 256-thread CTAs (two per SM, for
small HCUs).
"""
import hashlib
import json
import os
import time

import numpy as np

from . import capi, extgen, schema, workloads

F32 = np.float32


class Member:
    """One network of the batch: H x M, full recurrent, P patterns."""

    def __init__(self, index, hcu, mcu, seed, n_patterns=20, cue_frac=0.3):
        self.index, self.H, self.M, self.seed = index, hcu, mcu, seed
        rng = np.random.default_rng(seed)
        self.patterns = workloads.draw_patterns(rng, n_patterns, hcu, mcu)
        self.n_cued = int(np.ceil(hcu * cue_frac - 1e-9))
        stim = schema.StimRawData()
        stim.ParseFromString(workloads.stim_bytes(self.patterns, self.n_cued, hcu))
        self.lgidx, self.wmask = extgen.stim_tables(stim)
        self.C = hcu * mcu
        conn = "\n".join(workloads._hcu_conn(rng, hcu, hcu, mcu, hcu)) + "\n"
        self.pop = dict(hcu_num=hcu, mcu_num=mcu, taum=F32(0.005), wtagain=1.0, maxfq=100.0, igain=1.0, wgain=1.0,
                        lgbias=F32(workloads.LGBIAS), snoise=0.0)
        self.proj = dict(src_pop=0, dest_pop=0, tauzi=F32(0.01), tauzj=F32(0.01), taue=F32(0.02), taup=1.0,
                         maxfq=100.0, bgain=1.0, wgain=1.0, tauepsc=0.0, slot_num=float(self.C))
        self.ii, self.di = workloads.read_conn_map(conn, [self.pop], [self.proj])[0]
        self.cells = hcu * self.C * mcu


def make_members(n=256, seed=0, hcu=(8, 64), mcu=(5, 50), n_patterns=20):
    """B networks with HCU and MCU counts drawn uniformly (inclusive) and
    per-network seeds."""
    rng = np.random.default_rng(seed)
    hs = rng.integers(hcu[0], hcu[1] + 1, n)
    ms = rng.integers(mcu[0], mcu[1] + 1, n)
    return [Member(i, int(hs[i]), int(ms[i]), seed * 100003 + i + 1, n_patterns) for i in range(n)]


def schedule(n_patterns, train_ticks=100, recall_ticks=50):
    """(first, n, prn, old_prn, lgidx_row, wmask_row) runs: every pattern
    trained, then every pattern recalled from its cue (rows as stim_bytes lays
    them out)."""
    runs, t, prn = [], 1, 0.0
    for k in range(n_patterns):
        runs.append((t, train_ticks, 1.0, prn, k, 0))
        prn = 1.0
        t += train_ticks
    for k in range(n_patterns):
        runs.append((t, recall_ticks, 0.0, prn, n_patterns + k, 1))
        prn = 0.0
        t += recall_ticks
    return runs


class Group:
    """Members built as one multi-population network.  per_tick forces one
    launch per tick (no cooperative persistent launch), which is what groups
    that run side by side on several streams use: a persistent launch relies
    on every CTA of its grid being resident at once."""

    def __init__(self, members, dt=0.001, eps=1e-4, device=0, max_ticks=128, per_tick=False, threads=512):
        self.members = members
        pops = [m.pop for m in members]
        projs = [dict(m.proj, src_pop=i, dest_pop=i) for i, m in enumerate(members)]
        old = os.environ.get("GSBN_PER_TICK")
        os.environ["GSBN_PER_TICK"] = "1" if per_tick else "0"
        try:
            self.net = capi.Net(pops, projs, dt, seed=0, device=device, max_ticks=max_ticks, tick_threads=threads)
        finally:
            if old is None:
                del os.environ["GSBN_PER_TICK"]
            else:
                os.environ["GSBN_PER_TICK"] = old
        for i, m in enumerate(members):
            self.net.set_pop_rng(i, m.seed, 0)
            self.net.set_conn(i, m.ii, m.di)
        lg = np.concatenate([m.lgidx for m in members], axis=1)
        wm = np.concatenate([m.wmask for m in members], axis=1)
        self.net.upload_stimuli_idx(lg, eps, wm)

    def run(self, first, n, prn, old_prn, lg_row, wm_row):
        self.net.use_stimulus(lg_row, wm_row)
        self.net.run(first, n, prn, old_prn)

    def close(self):
        self.net.close()


def partition(members, kind, k=1):
    """member index groups of one candidate schedule"""
    if kind == "one":
        return [list(range(len(members)))]
    if kind == "plain":
        return [[i] for i in range(len(members))]
    order = sorted(range(len(members)), key=lambda i: (members[i].C, members[i].H))
    total = sum(members[i].cells for i in order)
    groups, cur, acc = [], [], 0
    for i in order:  # k groups of about equal cell count, similar shapes together
        cur.append(i)
        acc += members[i].cells
        if acc >= total * (len(groups) + 1) / k and len(groups) < k - 1:
            groups.append(cur)
            cur = []
    if cur:
        groups.append(cur)
    return groups


# (partition kind, groups, tick-kernel CTA size)
CANDIDATES = [("one", 1, 512), ("one", 1, 256), ("buckets", 4, 512), ("buckets", 4, 256), ("buckets", 8, 256),
              ("buckets", 16, 256), ("buckets", 16, 512), ("plain", 1, 512)]


def cand_name(c):
    return f"{c[0]}{c[1]}/t{c[2]}"


class Batch:
    """The batch on the GPU under one schedule.  concurrent: groups run side by
    side on their own streams (one launch per tick each); otherwise one group
    after the other (a group may then use the persistent launch)."""

    def __init__(self, members, groups, device=0, concurrent=None, threads=512):
        self.members = members
        self.groups_idx = groups
        self.concurrent = (1 < len(groups) <= 64) if concurrent is None else concurrent
        self.threads = threads
        self.groups = [Group([members[i] for i in g], device=device, per_tick=self.concurrent, threads=threads)
                       for g in groups]

    def run_segment(self, first, n, prn, old_prn, lg_row, wm_row):
        for g in self.groups:
            g.run(first, n, prn, old_prn, lg_row, wm_row)
            if not self.concurrent:
                g.net.sync()

    def sync(self):
        for g in self.groups:
            g.net.sync()

    def reset(self):
        for g in self.groups:
            g.net.reset()

    def counters(self):
        return sum(sum(g.net.counters()) for g in self.groups)

    def launches(self):
        return sum(g.net.kernel_launches() for g in self.groups)

    def member_state(self, index, name):
        """state vector `name` (gsbn name with the member's own index 0) of one member"""
        for gi, g in enumerate(self.groups_idx):
            if index in g:
                local = g.index(index)
                base = name.rsplit("_", 1)[0]
                return self.groups[gi].net.read(f"{base}_{local}")
        raise KeyError(index)

    def close(self):
        for g in self.groups:
            g.close()


def shape_key(members):
    """cache key: the sorted (H, M) list"""
    return hashlib.sha1(json.dumps(sorted((m.H, m.M) for m in members)).encode()).hexdigest()[:16]


def tune(members, device=0, probe_ticks=20, cache=None, candidates=CANDIDATES):
    """Time every candidate schedule on the first `probe_ticks` training ticks
    from the initial state; return (best (kind, k, threads), {name: seconds}).  With
    `cache` (a JSON path), a result for the same member shapes is reused."""
    key = shape_key(members)
    if cache and os.path.exists(cache):
        with open(cache) as f:
            known = json.load(f)
        if key in known:
            return tuple(known[key]["best"]), known[key]["times"]
    times = {}
    for c in candidates:
        kind, k, threads = c
        b = Batch(members, partition(members, kind, k), device, threads=threads)
        b.run_segment(1, 2, 1.0, 0.0, 0, 0)  # warm-up: graphs, tables, the first catch-up
        b.sync()
        t0 = time.perf_counter()
        b.run_segment(3, probe_ticks, 1.0, 1.0, 0, 0)
        b.sync()
        times[cand_name(c)] = time.perf_counter() - t0
        b.close()
    best = min(candidates, key=lambda c: times[cand_name(c)])
    if cache:
        known = {}
        if os.path.exists(cache):
            with open(cache) as f:
                known = json.load(f)
        known[key] = {"best": list(best), "times": times}
        with open(cache, "w") as f:
            json.dump(known, f)
    return tuple(best), times
