"""Shared drivers for the parity tests: the ProcExtGen schedule cut into runs
of ticks with constant stimulus and plasticity, fed identically to the CPU
oracle (one tick at a time) and to the C ABI (one call per run)."""
import numpy as np

from gsbn_b200 import schema
from oracle import sim


class Run:
    def __init__(self, first, n, prn, old_prn, lginp, wmask, cycle_flags):
        self.first, self.n, self.prn, self.old_prn = first, n, prn, old_prn
        self.lginp, self.wmask = lginp.copy(), wmask.copy()


def schedule(sp, stim, pops, logf, max_ticks=None):
    """Runs of consecutive cycle-flag-1 ticks inside one ProcExtGen segment."""
    mcu_in_hcu = [p["mcu_num"] for p in pops for _ in range(p["hcu_num"])]
    gen = sim.ExtGen(sp, stim, mcu_in_hcu, logf)
    runs, cur, cur_mode = [], None, None
    ticks = 0
    while True:
        gen.tick()
        ticks += 1
        if gen.cycle_flag < 0 or (max_ticks is not None and ticks > max_ticks):
            break
        if gen.cycle_flag != 1:
            cur = None
            continue
        if cur is not None and gen.cursor == cur_mode and not gen.lginp_changed and gen.simstep == cur.first + cur.n:
            cur.n += 1
        else:
            cur = Run(gen.simstep, 1, gen.prn, gen.old_prn, gen.lginp, gen.wmask_row(), None)
            cur_mode = gen.cursor
            runs.append(cur)
    return runs


def load_workload(w, directory):
    sp, path = w.solver_param(directory)
    pops, projs = sim.net_from_solver_param(sp)
    stim = schema.read_stim(sp.gen_param.stim_file)
    with open(sim.proc_args(sp, "ProcInitConn")[2]["conn-map-file"]) as f:
        conn = sim.parse_conn_map(f.read(), pops, projs)
    argi, argf, _ = sim.proc_args(sp, "ProcUpdLazy")
    return sp, pops, projs, stim, conn, int(argi.get("seed", 0)), float(argf.get("poisson-noise-hz", 0.0))


STATE_POP = ("dsup", "act", "epsc", "bj", "spike", ".counter")
STATE_PROJ = ("pi", "ei", "zi", "ti", "pj", "ej", "zj", "pij", "eij", "zi2", "zj2", "tij", "wij", "qi", "si",
              ".siq")


def state(net, n_pops, n_projs):
    out = {}
    for p in range(n_pops):
        for k in STATE_POP:
            out[f"{k}_{p}"] = net.read(f"{k}_{p}")
    for q in range(n_projs):
        for k in STATE_PROJ:
            out[f"{k}_{q}"] = net.read(f"{k}_{q}")
    return out


def first_mismatch(a, b):
    for k in a:
        x, y = a[k], b[k]
        if x.dtype.kind == "f":
            same = np.array_equal(x.view(np.int32), y.view(np.int32))
        else:
            same = np.array_equal(x, y)
        if not same:
            bad = np.nonzero((x != y) & ~(np.isnan(x) & np.isnan(y)) if x.dtype.kind == "f" else (x != y))[0]
            i = int(bad[0]) if len(bad) else -1
            return f"{k}: {len(bad)} differ, first at {i}: {x[i] if i >= 0 else None} vs {y[i] if i >= 0 else None}"
    return None
