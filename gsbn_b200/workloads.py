"""Seeded synthetic workloads in gsbn's own input formats.

Each workload is a network description (prototxt text using the reference's
schema and Procedure names), a StimRawData stimulus file and a ProcInitConn
connection map.  Conventions follow the reference's stimulus generator
(tools/stimgen/gen_rnd.py:39-75):
  - a pattern is one uniformly drawn MCU per HCU, duplicates rejected;
  - cue rows keep the pattern on the first HCUs and write 0x7fffffff (no
    input) on the silenced ones;
  - mask row 0 is all 0 (training, no recurrent support); mask row 1 is 0 on
    cued HCUs and 1 on the others.
A rest row (all 0x7fffffff) is appended for rest segments.  All randomness
(patterns, connectivity) comes from one numpy seed; spike sampling uses the
Philox stream seeded through ProcUpdLazy's `argi "seed"`.
"""
import os

import numpy as np

from . import schema

NO_INPUT = 0x7FFFFFFF
# lgbias cancels the log(eps) input of silenced HCUs (ProcExtGen.cpp:139,
# eps = 1e-4), so recall is driven by recurrent support rather than silenced.
LGBIAS = 9.21


def tick_time(ticks, dt):
    """A float time t with int(float32(t)/float32(dt)) == ticks, the
    truncation ProcExtGen applies to mode boundaries (ProcExtGen.cpp:22-23)."""
    dt32 = np.float32(dt)
    t = np.float32(ticks * float(dt32))
    for _ in range(64):
        q = int(np.float32(t) / dt32)
        if q == ticks:
            return float(t)
        t = np.nextafter(t, np.float32(np.inf if q < ticks else -np.inf), dtype=np.float32)
    raise ValueError(f"no float time maps to tick {ticks}")


def fmt(x):
    return repr(float(np.float32(x)))


def draw_patterns(rng, n_patterns, hcus, mcus):
    pats, seen = [], set()
    while len(pats) < n_patterns:
        p = tuple(int(rng.integers(0, mcus)) for _ in range(hcus))
        if p not in seen:
            seen.add(p)
            pats.append(p)
    return pats


def stim_bytes(patterns, n_cued, total_hcu):
    """rows [0,P) patterns, [P,2P) cues, 2P rest; masks 0 (train), 1 (recall)."""
    rd = schema.StimRawData()
    P = len(patterns)
    rd.data_rows = 2 * P + 1
    rd.data_cols = total_hcu
    rd.mask_rows = 2
    rd.mask_cols = total_hcu
    for p in patterns:
        rd.data.extend(p)
    for p in patterns:
        rd.data.extend(v if i < n_cued else NO_INPUT for i, v in enumerate(p))
    rd.data.extend([NO_INPUT] * total_hcu)
    rd.mask.extend([0.0] * total_hcu)
    rd.mask.extend([0.0 if i < n_cued else 1.0 for i in range(total_hcu)])
    return rd.SerializeToString()


def mode(begin, end, step, lgidx, lgidx_step, wmask, prn, dt, lgexp=None, lgexp_step=None):
    s = ["  mode_param {", f"    begin_time: {fmt(tick_time(begin, dt))}", f"    end_time: {fmt(tick_time(end, dt))}",
         f"    time_step: {step}", f"    begin_lgidx_id: {lgidx}", f"    lgidx_step: {lgidx_step}",
         f"    begin_wmask_id: {wmask}", "    wmask_step: 0", f"    prn: {fmt(prn)}", "    plasticity: 0"]
    if lgexp is not None:
        s += [f"    begin_lgexp_id: {lgexp}", f"    lgexp_step: {lgexp_step}"]
    return "\n".join(s + ["  }"])


def pop_block(hcu, mcu, taum, maxfq=100.0, wtagain=1.0, lgbias=LGBIAS):
    return "\n".join(["  pop_param {", "    pop_num: 1", f"    hcu_num: {hcu}", f"    mcu_num: {mcu}",
                      f"    fanout_num: {mcu}", f"    taum: {fmt(taum)}", f"    wtagain: {fmt(wtagain)}",
                      f"    maxfq: {fmt(maxfq)}", "    igain: 1", "    wgain: 1", f"    lgbias: {fmt(lgbias)}", "    snoise: 0",
                      "  }"])


def proj_block(src, dest, tauzi, tauzj, taue, taup, slot_num, maxfq=100.0, tauepsc=None):
    s = ["  proj_param {", f"    src_pop: {src}", f"    dest_pop: {dest}", f"    tauzi: {fmt(tauzi)}",
         f"    tauzj: {fmt(tauzj)}", f"    taue: {fmt(taue)}", f"    taup: {fmt(taup)}", f"    maxfq: {fmt(maxfq)}",
         "    wgain: 1", "    bgain: 1", f"    slot_num: {slot_num}"]
    if tauepsc is not None:
        s.append(f"    tauepsc: {fmt(tauepsc)}")
    return "\n".join(s + ["  }"])


def procs(conn_path, seed, poisson_hz=0.0, record=True, check=True):
    s = ['proc_param { name: "ProcExtGen" }',
         'proc_param {\n  name: "ProcUpdLazy"\n  argi { key: "seed" val: %d }\n  argf { key: "poisson-noise-hz" '
         'val: %s }\n}' % (seed, fmt(poisson_hz)),
         'proc_param { name: "ProcExchangeSpike" }',
         'proc_param {\n  name: "ProcInitConn"\n  args { key: "conn-map-file" val: "%s" }\n}' % conn_path]
    if record:
        s.append('proc_param {\n  name: "ProcSpkRec"\n  argi { key: "period" val: 1 }\n  argi { key: "offset" '
                 'val: 0 }\n}')
    if check:
        s.append('proc_param { name: "ProcCheck" }')
    return "\n".join(s)


class Workload:
    """A generated network: prototxt text plus the files it names."""

    def __init__(self, name, prototxt, stim, conn, meta):
        self.name, self.prototxt, self.stim, self.conn, self.meta = name, prototxt, stim, conn, meta

    def write(self, directory):
        """Write the three files; returns the prototxt path."""
        os.makedirs(directory, exist_ok=True)
        stim_path = os.path.join(directory, "stim.bin")
        conn_path = os.path.join(directory, "conn.map")
        with open(stim_path, "wb") as f:
            f.write(self.stim)
        with open(conn_path, "w") as f:
            f.write(self.conn)
        text = self.prototxt.replace("@STIM@", stim_path).replace("@CONN@", conn_path).replace(
            "@REC@", os.path.join(directory, "rec"))
        path = os.path.join(directory, "net.prototxt")
        with open(path, "w") as f:
            f.write(text)
        return path

    def solver_param(self, directory):
        path = self.write(directory)
        with open(path) as f:
            return schema.parse_prototxt(f.read()), path


def _hcu_conn(rng, dest_hcus, src_hcus, src_mcus, n_src_hcus, proj=0, delay=1):
    """each destination HCU receives every MCU of n_src_hcus distinct source
    HCUs drawn at random (HCU-level density n_src_hcus / src_hcus)."""
    lines = []
    for h in range(dest_hcus):
        srcs = sorted(rng.choice(src_hcus, size=n_src_hcus, replace=False).tolist())
        pairs = []
        for s in srcs:
            for m in range(src_mcus):
                pairs += [s * src_mcus + m, delay]
        lines.append(",".join(str(v) for v in [proj, h] + pairs))
    return lines


def _mcu_conn(rng, dest_hcus, n_src, n_slots, proj, delay=1):
    """each destination HCU receives n_slots distinct source MCUs."""
    lines = []
    for h in range(dest_hcus):
        srcs = sorted(rng.choice(n_src, size=n_slots, replace=False).tolist())
        pairs = []
        for s in srcs:
            pairs += [s, delay]
        lines.append(",".join(str(v) for v in [proj, h] + pairs))
    return lines


def single_pop(name, hcu, mcu, n_patterns, train_ticks, rest_ticks, recall_ticks, cue_frac, src_hcus_per_dest,
               seed=0, dt=0.001, eps=1e-4, tauz=0.01, taue=0.02, taup=1.0, taum=0.005, record=True, check=True,
               poisson_hz=0.0):
    """One population with a recurrent projection: the 10x10 and 100x100
    workloads.  Training segments (prn 1, mask 0) of train_ticks, optional
    rest segments (prn 1, rest row) and recall segments (prn 0, cue rows,
    recall mask)."""
    rng = np.random.default_rng(seed)
    pats = draw_patterns(rng, n_patterns, hcu, mcu)
    n_cued = int(np.ceil(hcu * cue_frac - 1e-9))
    stim = stim_bytes(pats, n_cued, hcu)
    C = src_hcus_per_dest * mcu
    conn = "\n".join(_hcu_conn(rng, hcu, hcu, mcu, src_hcus_per_dest)) + "\n"
    modes = []
    t = 0
    rest_row = 2 * n_patterns
    if rest_ticks:
        for k in range(n_patterns):
            modes.append(mode(t, t + train_ticks, train_ticks, k, 1, 0, 1.0, dt))
            t += train_ticks
            modes.append(mode(t, t + rest_ticks, rest_ticks, rest_row, 0, 0, 1.0, dt))
            t += rest_ticks
    else:
        modes.append(mode(t, t + n_patterns * train_ticks, train_ticks, 0, 1, 0, 1.0, dt))
        t += n_patterns * train_ticks
    modes.append(mode(t, t + n_patterns * recall_ticks, recall_ticks, n_patterns, 1, 1, 0.0, dt, lgexp=0,
                      lgexp_step=1))
    t += n_patterns * recall_ticks
    text = "\n".join([
        "gen_param {", '  stim_file: "@STIM@"', f"  dt: {fmt(dt)}", f"  eps: {fmt(eps)}"] + modes + ["}",
        "net_param {", pop_block(hcu, mcu, taum), proj_block(0, 0, tauz, tauz, taue, taup, C), "}",
        'rec_param { directory: "@REC@" }', procs("@CONN@", seed, poisson_hz, record=record, check=check)]) + "\n"
    meta = dict(H=hcu, M=mcu, C=C, patterns=n_patterns, ticks=t, n_cued=n_cued, seed=seed,
                cells=hcu * C * mcu, poisson_hz=poisson_hz)
    return Workload(name, text, stim, conn, meta)


def config0(seed=0, record=True, check=True):
    """10x10, full recurrent (C=100); 10 patterns x (100 train + 20 rest), 10
    recalls of 100 ticks with 3 of 10 HCUs cued; 2200 ticks."""
    return single_pop("10x10 full recurrent", 10, 10, 10, 100, 20, 100, 0.3, 10, seed=seed, record=record,
                      check=check)


def config1(seed=0, record=True, check=True, n_patterns=100, train_ticks=100, recall_ticks=100):
    """100x100, each destination HCU fed by 10 random source HCUs (density 0.1,
    C=1000, 1e7 cells); 100 patterns trained 100 ticks each (1e4 ticks), then
    100 recalls of 100 ticks with 30% of HCUs cued."""
    return single_pop("100x100 density 0.1", 100, 100, n_patterns, train_ticks, 0, recall_ticks, 0.3, 10, seed=seed,
                      record=record, check=check)


def config4(seed=0, hcu=64, mcu=64, n_patterns=16, train_ticks=300, rest_ticks=20, recall_ticks=200,
            cue_frac=0.25, poisson_hz=20.0, record=False, check=False):
    """The network of the replicate recall workload: 64x64 HCU/MCU, full
    recurrent projection (C = 4096, 4096 x 4096 weights), 16 patterns trained
    300 ticks each with 20-tick rests, 20 Hz Poisson input noise; the recall
    segments (25% of HCUs cued, 200 ticks) are what the replicates run.  At
    300 training ticks per pattern ProcCheck's all-HCU recall is non-zero
    (the last-trained patterns are recalled, with and without the input
    noise); at 100 it is zero for every replicate."""
    return single_pop(f"{hcu}x{mcu} full recurrent", hcu, mcu, n_patterns, train_ticks, rest_ticks, recall_ticks,
                      cue_frac, hcu, seed=seed, record=record, check=check, poisson_hz=poisson_hz)


def small_scale(seed=0, hcu=20, mcu=20, src=5, n_patterns=10, train_ticks=60, recall_ticks=40, record=True,
                check=True):
    """a reduced copy of the 100x100 workload for CPU-sized parity runs."""
    return single_pop(f"{hcu}x{mcu} density {src}/{hcu}", hcu, mcu, n_patterns, train_ticks, 0, recall_ticks, 0.3,
                      src, seed=seed, record=record, check=check)


def config2(seed=0, record=True, check=True, n_patterns=50, train_ticks=80, recall_ticks=20, poisson_hz=10.0):
    """pop0 5x10 -> pop1 10x10 (MCU density 0.5) + pop1 -> pop1 (density 0.1),
    per-projection tau_z in {5, 10, 20} ms, 50 paired patterns, 10 Hz Poisson
    input noise, 5000 ticks."""
    rng = np.random.default_rng(seed)
    dt = 0.001
    pats0 = draw_patterns(rng, n_patterns, 5, 10)
    pats1 = draw_patterns(rng, n_patterns, 10, 10)
    pats = [a + b for a, b in zip(pats0, pats1)]
    n_cued = 5
    stim = stim_bytes(pats, n_cued, 15)
    conn = "\n".join(_mcu_conn(rng, 10, 50, 25, 0) + _mcu_conn(rng, 10, 100, 10, 1)) + "\n"
    t = n_patterns * train_ticks
    modes = [mode(0, t, train_ticks, 0, 1, 0, 1.0, dt),
             mode(t, t + n_patterns * recall_ticks, recall_ticks, n_patterns, 1, 1, 0.0, dt, lgexp=0, lgexp_step=1)]
    t += n_patterns * recall_ticks
    text = "\n".join([
        "gen_param {", '  stim_file: "@STIM@"', f"  dt: {fmt(dt)}", f"  eps: {fmt(1e-4)}"] + modes + ["}",
        "net_param {", pop_block(5, 10, 0.005), pop_block(10, 10, 0.005),
        proj_block(0, 1, 0.005, 0.020, 0.02, 1.0, 25), proj_block(1, 1, 0.010, 0.005, 0.02, 1.0, 10), "}",
        'rec_param { directory: "@REC@" }', procs("@CONN@", seed, poisson_hz, record=record, check=check)]) + "\n"
    meta = dict(patterns=n_patterns, ticks=t, n_cued=n_cued, seed=seed, cells=10 * 25 * 10 + 10 * 10 * 10)
    return Workload("5x10 + 10x10 two projections", text, stim, conn, meta)


def net_from_solver_param(sp):
    """Populations (pop_num copies of each PopParam, ProcUpdLazy.cpp:19-29) and
    the projections whose source and destination exist (ProcUpdLazy.cpp:35-45),
    as the dicts gsbn_b200.capi.Net takes."""
    pops = []
    for pp in sp.net_param.pop_param:
        for _ in range(pp.pop_num):
            pops.append(dict(hcu_num=pp.hcu_num, mcu_num=pp.mcu_num, taum=pp.taum, wtagain=pp.wtagain,
                             maxfq=pp.maxfq, igain=pp.igain, wgain=pp.wgain, lgbias=pp.lgbias, snoise=pp.snoise))
    projs = []
    for q in sp.net_param.proj_param:
        if q.src_pop < len(pops) and q.dest_pop < len(pops):
            projs.append(dict(src_pop=q.src_pop, dest_pop=q.dest_pop, tauzi=q.tauzi, tauzj=q.tauzj, taue=q.taue,
                              taup=q.taup, maxfq=q.maxfq, bgain=q.bgain, wgain=q.wgain,
                              tauepsc=q.tauepsc if q.HasField("tauepsc") else 0.0, slot_num=q.slot_num))
    return pops, projs


def read_conn_map(text, pops, projs):
    """(ii, di) slot tables per projection from a ProcInitConn map: every
    (src_mcu, delay) pair of line `proj,dest_hcu,...` goes to the first empty
    slot of that HCU, or is dropped when the HCU is full (ProcInitConn.cpp:48-103)."""
    tables = []
    for q in projs:
        s = pops[q["src_pop"]]
        C = min(s["hcu_num"] * s["mcu_num"], int(q["slot_num"]))
        H = pops[q["dest_pop"]]["hcu_num"]
        tables.append([np.full(H * C, -1, np.int32), np.zeros(H * C, np.int32), C, np.zeros(H, np.int64)])
    for line in text.splitlines():
        v = line.split(",")
        if len(v) <= 2:
            continue
        ii, di, C, nxt = tables[int(v[0])]
        h = int(v[1])
        for i in range(2, len(v) - 1, 2):
            src = int(v[i])
            k = nxt[h]
            while k < C and ii[h * C + k] >= 0:
                k += 1
            if k < C:
                ii[h * C + k] = src
                di[h * C + k] = int(v[i + 1])
                nxt[h] = k
    return [(t[0], t[1]) for t in tables]
