"""Writes tests/golden/reference_fixtures.json from the reference's own data
files, decoded with the protobuf runtime (gsbn_b200.schema declares the
reference schema) and plain Python: the inputs the oracle, the schedule
expansion and the C++ engine's parsers are pinned against.

Run with the path of a gsbn source tree:
    python tests/golden/make_golden.py <gsbn source root>
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from gsbn_b200 import schema  # noqa: E402

f32 = np.float32


def modes(gp):
    """ProcExtGen's segment expansion computed directly from the fields."""
    dt = f32(gp.dt)
    out = []
    for mp in gp.mode_param:
        b = int(f32(mp.begin_time) / dt)
        e = int(f32(mp.end_time) / dt)
        lg, ex, wm = mp.begin_lgidx_id, mp.begin_lgexp_id, mp.begin_wmask_id
        while b < e:
            end = min(b + mp.time_step, e)
            out.append([b, end, lg, ex, wm, float(f32(mp.prn))])
            lg += mp.lgidx_step
            ex += mp.lgexp_step
            wm += mp.wmask_step
            b = end
    return out


def main(ref):
    data = os.path.join(ref, "data")
    out = {"prototxt": {}, "stim": {}, "conn_map": {}}
    for name in sorted(os.listdir(data)):
        path = os.path.join(data, name)
        if name.endswith(".prototxt"):
            sp = schema.parse_prototxt(open(path).read())
            pops = [[p.pop_num, p.hcu_num, p.mcu_num, float(p.taum), float(p.wtagain), float(p.maxfq), float(p.igain),
                     float(p.wgain), float(p.lgbias), float(p.snoise), p.rank] for p in sp.net_param.pop_param]
            projs = [[q.src_pop, q.dest_pop, float(q.tauzi), float(q.tauzj), float(q.taue), float(q.taup),
                      float(q.maxfq), float(q.bgain), float(q.wgain),
                      float(q.tauepsc) if q.HasField("tauepsc") else None, float(q.slot_num)]
                     for q in sp.net_param.proj_param]
            procs = [[pp.name, {a.key: a.val for a in pp.argi}, {a.key: float(a.val) for a in pp.argf},
                      {a.key: a.val for a in pp.args}] for pp in sp.proc_param]
            out["prototxt"][name] = {
                "stim_file": sp.gen_param.stim_file, "dt": float(sp.gen_param.dt), "eps": float(sp.gen_param.eps),
                "modes": modes(sp.gen_param), "pops": pops, "projs": projs, "procs": procs,
                "rec_dir": sp.rec_param.directory,
            }
        elif name.endswith(".bin"):
            st = schema.read_stim(path)
            d = np.array(st.data, dtype=np.uint32)
            m = np.array(st.mask, dtype=np.float32)
            out["stim"][name] = {
                "data_rows": st.data_rows, "data_cols": st.data_cols, "mask_rows": st.mask_rows,
                "mask_cols": st.mask_cols, "data_sha1": hashlib.sha1(d.tobytes()).hexdigest(),
                "mask_sha1": hashlib.sha1(m.tobytes()).hexdigest(), "data_head": d[:24].tolist(),
                "mask_head": m[:24].tolist(), "data_sum": int(d.astype(np.int64).sum()),
            }
        elif name.endswith(".map"):
            lines = open(path).read().splitlines()
            rows = []
            for ln in lines:
                v = ln.split(",")
                if len(v) > 2:
                    pairs = [int(x) for x in v[2:]]
                    rows.append([int(v[0]), int(v[1]), len(pairs) // 2, sum(pairs[0::2]), sum(pairs[1::2])])
            out["conn_map"][name] = {"lines": len(lines), "rows": rows}
    with open(os.path.join(HERE, "reference_fixtures.json"), "w") as f:
        json.dump(out, f, indent=0, sort_keys=True)
    print("wrote", os.path.join(HERE, "reference_fixtures.json"))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <gsbn source root>")
    main(sys.argv[1])
