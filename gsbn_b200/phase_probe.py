"""Phase breakdown of the tick kernel on the 100x100 workload.

Needs the phase-probe build of the library (python -m gsbn_b200.build
--probe, which writes gsbn_b200/libgsbn_b200_probe.so) and a GPU:

    GSBN_B200_LIB=gsbn_b200/libgsbn_b200_probe.so python -m gsbn_b200.phase_probe

Runs the first `--train` training segments and, after the switch to recall,
`--recall` recall segments of the 100x100 density-0.1 workload (100 ticks
each, one persistent launch per segment), then prints, per phase, the time
per tick of the median CTA and of the slowest CTA, in microseconds at the SM
clock given by --mhz (the counters are SM clock cycles).  The probe adds a
clock read and a store per phase boundary, so the total is a little above
the default build's time per tick.  Slots 14 and 15 count the cell and row
decays done by the div_rn fallback and by the reciprocal form.

`--variant multi` probes the ProcUpdMulti launch on the same workload
(adaptation taua 0.05, adgain 1; a spike ring of `--ring` ticks): one
thread per CTA marks the phases of its HCU's tick in order.
"""
import argparse
import os
import sys
import tempfile

import numpy as np

from gsbn_b200 import capi, extgen, schema, workloads

PHASES_A = {0: "barrier wait", 1: "support", 10: "softmax: max", 11: "softmax: exp", 2: "softmax: sum",
            12: "spikes: sampling", 3: "spikes: list, publish", 4: "j-traces", 5: "column wait + refresh",
            6: "rows", 7: "end of rows", 8: "join wait", 9: "staging next chunk"}
PHASES_B = {16: "barrier wait", 26: "column units of the grid", 19: "  units: ring, cell loads",
            20: "  units: tables, decay, store", 21: "  units: group sync", 17: "delay queue: loads, ballots",
            18: "delay queue: sync", 27: "delay queue: list", 28: "spike wait", 29: "unit publication",
            24: "join wait", 25: "staging next chunk"}
PHASES_MULTI = {0: "barrier wait (global form)", 1: "support", 2: "softmax: max, exp", 3: "softmax: sum", 4: "spikes",
                5: "staging, j-traces, row list", 6: "rows: spike now, replays", 7: "weights", 8: "epsc sums",
                9: "delay queue", 10: "wait for the delay-queue warps",
                11: "uniforms", 12: "queue warps: grid-barrier wait"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--train", type=int, default=20)
    ap.add_argument("--recall", type=int, default=20)
    ap.add_argument("--mhz", type=float, default=1965.0)
    ap.add_argument("--threads", type=int, default=0)
    ap.add_argument("--variant", choices=("lazy", "multi"), default="lazy")
    ap.add_argument("--ring", type=int, default=25)
    ap.add_argument("--critical", type=int, default=0,
                    help="also print the N CTAs with the least barrier wait (the ones that arrive last most often)")
    a = ap.parse_args()
    if "probe" not in capi.LIB_PATH:
        sys.exit("set GSBN_B200_LIB to the phase-probe build (gsbn_b200/libgsbn_b200_probe.so)")
    w = workloads.config1()
    sp, _ = w.solver_param(tempfile.mkdtemp(prefix="gsbn_probe_"))
    pops, projs = workloads.net_from_solver_param(sp)
    conn = workloads.read_conn_map(w.conn, pops, projs)
    lgidx, wmask = extgen.stim_tables(schema.read_stim(sp.gen_param.stim_file))
    runs = extgen.segments(sp)
    first_recall = next(i for i, r in enumerate(runs) if r.prn == 0.0)
    kw = dict(tick_threads=a.threads)
    if a.variant == "multi":
        pops = [dict(p, taua=0.05, adgain=1.0) for p in pops]
        kw = dict(variant=1, spike_buffer=a.ring)
    net = capi.Net(pops, projs, float(np.float32(sp.gen_param.dt)), seed=w.meta["seed"], max_ticks=128, **kw)
    for k, (ii, di) in enumerate(conn):
        net.set_conn(k, ii, di)
    net.upload_stimuli_idx(lgidx, float(np.float32(sp.gen_param.eps)), wmask)
    out, counts = {}, {}
    for name, sel in (("training", runs[1:1 + a.train]), ("recall", runs[first_recall + 1:first_recall + 1 + a.recall])):
        if not sel:
            continue
        # run up to the selection without the probe, then the selection with it
        net.reset()
        for r in runs[:runs.index(sel[0])]:
            net.use_stimulus(r.lgidx, r.wmask)
            net.run(r.first, r.n, r.prn, r.old_prn)
        net.phase_probe(reset=True)
        for r in sel:
            net.use_stimulus(r.lgidx, r.wmask)
            net.run(r.first, r.n, r.prn, r.old_prn)
        c = net.phase_probe(reset=True).astype(np.float64)
        counts[name] = c
        ticks = c[:, 31:32]
        per_tick = c / np.maximum(ticks, 1) / a.mhz  # us per tick
        out[name] = per_tick
    net.close()
    if a.variant == "multi":
        for name, pt in out.items():
            print(f"== {name} segments, ProcUpdMulti: us per tick at {a.mhz:.0f} MHz (median CTA / slowest CTA)")
            tot = 0.0
            for k, ph in PHASES_MULTI.items():
                med, mx = float(np.median(pt[:, k])), float(pt[:, k].max())
                tot += med if k != 12 else 0.0  # the queue warps' wait overlaps thread 0's phases
                print(f"  {ph:<30} {med:7.3f} {mx:7.3f}")
            print(f"  {'total (median)':<30} {tot:7.3f}")
        return
    for name, pt in out.items():
        print(f"== {name} segments: us per tick at {a.mhz:.0f} MHz (median CTA / slowest CTA)")
        tot = 0.0
        for k, ph in PHASES_A.items():
            med, mx = float(np.median(pt[:, k])), float(pt[:, k].max())
            tot += med
            print(f"  A {ph:<24} {med:7.3f} {mx:7.3f}")
        print(f"  A {'total (median)':<24} {tot:7.3f}")
        for k, ph in PHASES_B.items():
            print(f"  B {ph:<24} {float(np.median(pt[:, k])):7.3f} {float(pt[:, k].max()):7.3f}")
        if a.critical:
            order = np.argsort(pt[:, 0])[:a.critical]
            keys = list(PHASES_A)
            print(f"  CTAs with the least A barrier wait (HCU: {', '.join(PHASES_A[k] for k in keys)}):")
            for c in order:
                print(f"    {int(c):4d}: " + " ".join(f"{pt[c, k]:.2f}" for k in keys))
            print(f"  A barrier wait min {float(pt[:, 0].min()):.3f}, B barrier wait min {float(pt[:, 16].min()):.3f}")
        slow, fast = float(counts[name][:, 14].sum()), float(counts[name][:, 15].sum())
        print(f"  decays: {fast:.0f} by the reciprocal form, {slow:.0f} by the div_rn fallback "
              f"({100.0 * slow / max(1.0, slow + fast):.3f} %)")


if __name__ == "__main__":
    main()
