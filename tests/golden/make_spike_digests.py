"""Writes tests/golden/config1_spike_digests.json: for every stimulus segment
of one full step of the 100x100 workload (100 HCUs x 100 MCUs, recurrent HCU
density 0.1, 100 patterns: 1e4 training + 1e4 recall ticks, 200 segments),
the spike count and the SHA-256 of the segment's spike log as gsbn's own
kernels compute it.

The spike log is the layout bcpnn_get_spike_log returns: per tick one bit per
MCU, little-endian uint32 words.  The simulation is the oracle in math mode
MATH_REF, whose population and projection loops call gsbn's
update_*_kernel_cpu functions compiled from the gsbn sources (oracle/_ref),
with the Philox stream, connectivity and stimulus rows the benchmark uses
(gsbn_b200.workloads.config1, ProcExtGen's schedule from gsbn_b200.extgen,
lginp values from the host's float log).  bench.py compares the device's
spike logs of its first end-to-end step with these digests.

usage: python tests/golden/make_spike_digests.py [--math ref|shared] [--out PATH]
(about two minutes of one CPU core)
"""
import argparse
import hashlib
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from gsbn_b200 import extgen, schema, workloads  # noqa: E402
from oracle import sim  # noqa: E402

OUT = os.path.join(HERE, "config1_spike_digests.json")


def pack(spikes, n_mcu):
    """per-tick index arrays -> the spike-log bytes (uint32 words, little-endian)"""
    words = (n_mcu + 31) // 32
    bits = np.zeros((len(spikes), words * 32), np.uint8)
    for t, idx in enumerate(spikes):
        bits[t, idx] = 1
    return np.packbits(bits, axis=1, bitorder="little").tobytes()


def lginp_row(row, H, M, hit, miss):
    out = np.full(H * M, miss, np.float32)
    row = np.asarray(row[:H], np.int64)
    h = np.nonzero((row >= 0) & (row < M))[0]
    out[h * M + row[h]] = hit
    return out


def digests(math=sim.MATH_REF, max_segments=None):
    """[(first tick, ticks, spikes, sha256 hex)] per segment of the step."""
    w = workloads.config1()
    sp, _ = w.solver_param(tempfile.mkdtemp(prefix="gsbn_digest_"))
    pops, projs = workloads.net_from_solver_param(sp)
    conn = workloads.read_conn_map(w.conn, pops, projs)
    lgidx, wmask = extgen.stim_tables(schema.read_stim(sp.gen_param.stim_file))
    eps = np.float32(sp.gen_param.eps)
    H, M = pops[0]["hcu_num"], pops[0]["mcu_num"]
    hit, miss = sim.extgen_logf(np.float32(1) + eps), sim.extgen_logf(np.float32(0) + eps)
    orc = sim.OracleNet(pops, projs, float(np.float32(sp.gen_param.dt)), seed=w.meta["seed"], math=math)
    for k, (ii, di) in enumerate(conn):
        orc.set_conn(k, ii, di)
    out = []
    for r in extgen.segments(sp)[:max_segments]:
        orc.set_stimulus(lginp_row(lgidx[r.lgidx], H, M, hit, miss), wmask[r.wmask][:H])
        spikes = [t[0] for t in orc.run(r.first, r.n, r.prn, r.old_prn)]
        out.append((r.first, r.n, int(sum(len(s) for s in spikes)), hashlib.sha256(pack(spikes, H * M)).hexdigest()))
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--math", choices=["ref", "shared"], default="ref")
    ap.add_argument("--out", default=OUT)
    a = ap.parse_args()
    math = sim.MATH_REF if a.math == "ref" else sim.MATH_SHARED
    seg = digests(math)
    doc = {"workload": "100x100 HCU/MCU, recurrent HCU density 0.1 (C=1000, 1e7 cells), 100 patterns: "
                       "1e4 training + 1e4 recall ticks per step (gsbn_b200.workloads.config1, seed 0)",
           "math": {"ref": "gsbn's update_*_kernel_cpu compiled from its sources (oracle/_ref), glibc expf/logf",
                    "shared": "oracle restatement with the shared exp/log"}[a.math],
           "layout": "per tick one bit per MCU, little-endian uint32 words (bcpnn_get_spike_log)",
           "ticks": sum(s[1] for s in seg), "spikes": sum(s[2] for s in seg),
           "segments": [{"first": s[0], "ticks": s[1], "spikes": s[2], "sha256": s[3]} for s in seg]}
    with open(a.out, "w") as f:
        json.dump(doc, f, indent=0)
    print("wrote", a.out, doc["ticks"], "ticks", doc["spikes"], "spikes")


if __name__ == "__main__":
    main()
