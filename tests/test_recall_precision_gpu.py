"""Precision of the replicate recall engine against the FP64 oracle of the
same simulation, at full size: a 64x64 network (4096 x 4096 weights) trained
on the plain FP32 path, recalled for 200 ticks by 4096 replicates (25% cue,
20 Hz Poisson noise).  For sampled replicates the engine in both forms (BF16
tensor-core and FP32 SIMT contraction) and the plain FP32 path are compared,
tick by tick, with the oracle in double:

  - support error: max |dsup - dsup_fp64| / max |dsup_fp64| over the ticks
    before the spike trains first differ;
  - spike agreement: |S & S_fp64| / |S | S_fp64| over the run, and the first
    tick where the trains differ;
  - recall: ProcCheck's decision for the replicate.

The FP64 restatement of the recall (oracle/recall_fp64.py, which the bench
uses for its in-run fp64_error on more replicates) must give the oracle's
spike trains exactly at this size too.

The numbers are written as one JSON line to $GSBN_PRECISION_OUT when set.
"""
import json
import os

import numpy as np
import pytest

from gsbn_b200 import capi, recall, workloads
from oracle import recall_fp64, sim

pytestmark = pytest.mark.gpu

NAMES = ("pij_0", "eij_0", "zi2_0", "zj2_0", "tij_0", "wij_0", "pi_0", "ei_0", "zi_0", "ti_0", "pj_0", "ej_0", "zj_0",
         "qi_0", "ii_0", "di_0", "si_0", ".siq_0", "dsup_0", "act_0", "epsc_0", "bj_0", "spike_0", ".counter_0")


def lginp_row(lg, H, M, eps):
    hit = sim.extgen_logf(np.float32(1) + np.float32(eps))
    miss = sim.extgen_logf(np.float32(0) + np.float32(eps))
    m = np.tile(np.arange(M), H)
    return np.where(lg[np.repeat(np.arange(H), M)] == m, hit, miss).astype(np.float32)


def metrics(d, s, d64, s64):
    T = len(d)
    div = next((k for k in range(T) if not np.array_equal(s[k], s64[k])), T)
    scale = max(float(np.abs(np.asarray(d64[:max(div, 1)])).max()), 1e-30)
    err = max((float(np.abs(np.asarray(d[k], np.float64) - d64[k]).max()) for k in range(max(div, 1))), default=0.0)
    both = sum(int(np.sum((s[k] != 0) & (s64[k] != 0))) for k in range(T))
    either = sum(int(np.sum((s[k] != 0) | (s64[k] != 0))) for k in range(T))
    return dict(support_rel_err=err / scale, first_divergence_tick=div, spike_jaccard=both / max(either, 1))


def test_bf16_recall_against_fp64_oracle(tmp_path):
    work = workloads.config4()
    tr = recall.Trained(work, str(tmp_path))
    trained = tr.snapshot(NAMES)
    W, st = tr.recall_inputs()
    R, T, seed_base = 4096, 200, 1
    lg, wm, expected = tr.cues(R)
    sample = [0, 1]
    H, M, N = tr.H, tr.M, tr.H * tr.M
    ed, es, ok_eng = {}, {}, {}
    for form in ("bf16", "fp32"):
        eng = recall.Recall(tr.H, tr.M, R, tr.pops[0], tr.dt, recall.kepsc_of(tr.projs[0], tr.dt), seed_base,
                            tr.poisson_hz, contraction=form)
        eng.load_state(W, st["bj"], st["epsc"], st["dsup"], st["s_tm3"], st["s_tm2"], st["s_tm1"])
        eng.set_cues(lg, tr.eps, wm)
        ed[form] = {r: [] for r in sample}
        es[form] = {r: [] for r in sample}
        for k in range(T):
            eng.run(tr.t0 + k, 1, tr.t0, tr.t0 + T - 2)
            for r in sample:
                ed[form][r].append(eng.read("dsup", r, 1)[0])
                es[form][r].append(eng.read("spike", r, 1)[0])
        ok_eng[form] = recall.recall_decisions(eng.read("counts"), H, M, expected)
        eng.close()
    ok_bf16 = ok_eng["bf16"]
    W64, bj0, bj1, pos = recall_fp64.catchup_weights(tr.pops, tr.projs, tr.dt, tr.poisson_hz, trained, tr.t0,
                                                     tr.old_prn, lginp_row(lg[0], H, M, tr.eps), wm[0])
    rs = recall_fp64.RecallFP64(tr.pops[0], tr.dt, recall_fp64.kepsc_tau(tr.projs[0]), tr.poisson_hz, W64, bj0, bj1,
                                pos, st["epsc"], st["dsup"], (st["s_tm3"], st["s_tm2"], st["s_tm1"]), lg, wm, tr.eps,
                                seed_base, sample)
    restated = [rs.step(tr.t0 + k) for k in range(T)]

    out = {"replicates": R, "ticks": T, "sample": sample, "per_replicate": []}
    for r in sample:
        net = capi.Net(tr.pops, tr.projs, tr.dt, seed=seed_base + r, poisson_hz=tr.poisson_hz, max_ticks=T)
        orc = sim.OracleNet(tr.pops, tr.projs, tr.dt, seed=seed_base + r, poisson_hz=tr.poisson_hz, real_bits=64)
        for n, a in trained.items():
            net.write(n, a)
            orc.write(n, a)
        net.set_stimulus_idx(lg[r], tr.eps, wm[r])
        orc.set_stimulus(lginp_row(lg[r], H, M, tr.eps), wm[r])
        pd, ps, od, os_ = [], [], [], []
        for k in range(T):
            old = tr.old_prn if k == 0 else 0.0
            net.run(tr.t0 + k, 1, 0.0, old)
            orc.update(tr.t0 + k, 0.0, old)
            orc.exchange()
            pd.append(net.read("dsup_0"))
            ps.append(net.read("spike_0"))
            od.append(orc.read("dsup_0"))
            os_.append(orc.read("spike_0"))
        net.close()
        del orc

        def decision(spk):
            counts = np.sum(np.stack(spk[: T - 1]) != 0, axis=0)[None, :]
            return bool(recall.recall_decisions(counts, H, M, expected[r:r + 1])[0])

        i = sample.index(r)
        for k in range(T):
            assert np.array_equal(restated[k][1][i], os_[k]), f"replicate {r}: FP64 restatement spikes, tick {k}"
            assert np.abs(restated[k][0][i] - od[k]).max() <= 1e-12 * np.abs(od[k]).max(), (r, k)
        rec = {"replicate": r, "bf16": metrics(ed["bf16"][r], es["bf16"][r], od, os_),
               "fp32_engine": metrics(ed["fp32"][r], es["fp32"][r], od, os_), "plain_fp32": metrics(pd, ps, od, os_),
               "recall": {"bf16": bool(ok_bf16[r]), "fp32_engine": bool(ok_eng["fp32"][r]),
                          "plain_fp32": decision(ps), "fp64": decision(os_)}}
        out["per_replicate"].append(rec)
        # the plain FP32 path and the FP32 engine stay at FP32 rounding of the
        # double simulation
        assert rec["plain_fp32"]["support_rel_err"] < 1e-4, rec
        assert rec["fp32_engine"]["support_rel_err"] < 1e-4, rec
        # BF16 weights move the support by about their rounding (2^-9 relative)
        assert rec["bf16"]["support_rel_err"] < 2e-2, rec
        assert rec["bf16"]["first_divergence_tick"] >= 1, rec
    out["recall_bf16_all"] = f"{int(ok_bf16.sum())}/{R}"
    out["fp64_error"] = {
        "support_rel_err_bf16_max": max(x["bf16"]["support_rel_err"] for x in out["per_replicate"]),
        "support_rel_err_fp32_max": max(x["plain_fp32"]["support_rel_err"] for x in out["per_replicate"]),
        "support_rel_err_fp32_engine_max": max(x["fp32_engine"]["support_rel_err"] for x in out["per_replicate"]),
        "spike_jaccard_bf16_min": min(x["bf16"]["spike_jaccard"] for x in out["per_replicate"]),
        "spike_jaccard_fp32_min": min(x["plain_fp32"]["spike_jaccard"] for x in out["per_replicate"]),
        "first_divergence_bf16": [x["bf16"]["first_divergence_tick"] for x in out["per_replicate"]],
        "first_divergence_fp32": [x["plain_fp32"]["first_divergence_tick"] for x in out["per_replicate"]],
        "recall_agree_with_fp64": sum(int(x["recall"]["bf16"] == x["recall"]["fp64"]) for x in out["per_replicate"]),
        "replicates_compared": len(sample),
    }
    dest = os.environ.get("GSBN_PRECISION_OUT")
    if dest:
        with open(dest, "w") as f:
            f.write(json.dumps(out) + "\n")
