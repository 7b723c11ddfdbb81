"""Phase breakdown of the batch kernel on the batch workload.

Needs the phase-probe build of the library (python -m gsbn_b200.build
--probe, which writes gsbn_b200/libgsbn_b200_probe.so) and a GPU:

    GSBN_B200_LIB=gsbn_b200/libgsbn_b200_probe.so python -m gsbn_b200.batch_probe

Builds the 256-network batch (HCUs 8-64, MCUs 5-50, full recurrent), runs
the first training segments unprobed, then `--segments` more with the probe
on, for each CTA size given, and prints per tick (microseconds at the SM
clock given by --mhz; the counters are SM clock cycles): the mean warp's
time in phase A (one warp per (network, HCU) item) and phase B (column and
fan-out units), the slowest warp's of the median CTA and of the slowest
CTA, the median CTA's waits at the two grid barriers, and the units and
items per tick.
"""
import argparse
import sys

import numpy as np

from gsbn_b200 import batch, capi


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--nets", type=int, default=256)
    ap.add_argument("--segments", type=int, default=3)
    ap.add_argument("--threads", default="512,384,256")
    ap.add_argument("--mhz", type=float, default=1965.0)
    a = ap.parse_args()
    if "probe" not in capi.LIB_PATH:
        sys.exit("set GSBN_B200_LIB to the phase-probe build (gsbn_b200/libgsbn_b200_probe.so)")
    members = batch.make_members(a.nets)
    runs = batch.schedule(20, train_ticks=100, recall_ticks=50)
    for threads in (int(t) for t in a.threads.split(",")):
        eng = batch.BatchEngine(members, max_ticks=128, threads=threads)
        try:
            eng.reset()
            for r in runs[:3]:
                eng.run_segment(*r)
            eng.sync()
            eng.phase_probe(reset=True)
            for r in runs[3:3 + a.segments]:
                eng.run_segment(*r)
            eng.sync()
            c = eng.phase_probe(reset=True).astype(np.float64)
        finally:
            eng.close()
        ticks = max(c[:, 6].max(), 1.0)
        wpc = threads // 32
        us = 1.0 / (ticks * a.mhz)
        print(f"{threads} threads: {ticks:.0f} ticks, {len(c)} CTAs")
        for name, mean_slot, slow_slot in (("A", 0, 1), ("B", 2, 3)):
            print(f"  phase {name}: mean warp {c[:, mean_slot].sum() / (len(c) * wpc) * us:.1f} us, slowest warp "
                  f"(median CTA) {np.median(c[:, slow_slot]) * us:.1f} us, (slowest CTA) {c[:, slow_slot].max() * us:.1f}")
        print(f"  barrier waits (thread 0, median CTA): {np.median(c[:, 4]) * us:.1f}, {np.median(c[:, 5]) * us:.1f} us")
        print(f"  units per tick {c[:, 7].sum() / ticks:.0f}, items per tick {c[:, 8].sum() / ticks:.0f}")


if __name__ == "__main__":
    main()
