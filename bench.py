#!/usr/bin/env python
"""Throughput of the ProcUpdLazy hot path (+ spike recording) on B200.

Workload: the 100x100 HCU/MCU network with a recurrent projection at HCU
density 0.1 (C = 1000 slots per destination HCU, 1e7 synaptic cells), 100
seeded one-MCU-per-HCU patterns trained 100 ticks each (1e4 ticks, prn 1)
followed by 100 recalls of 100 ticks with 30% of the HCUs cued (1e4 ticks,
prn 0): 2e4 ticks, 200 stimulus segments.  Synthetic inputs follow the
reference's generator conventions (gsbn_b200/workloads.py); no dataset.

A step is one full pass of that schedule from the network's initial state:
bcpnn_reset, then one bcpnn_run per segment.  `value` is synaptic updates/s
(row + column + all-cells cell updates, counted by the kernels) over K steps,
timed with CUDA events on the library's stream, stimulus rows already
resident in HBM.  `e2e` is the same metric through the C ABI with host
buffers: per segment the stimulus row is copied from pinned host memory, the
segment's spike log is read back, and ProcCheck's recall counters run on the
device with their per-HCU results read back; all of it is queued behind the
runs, with one synchronisation per step.  The network state (~0.25 GB) is larger than L2, so no flush is
needed between steps.

--impl reference times gsbn's own CPU kernels (update_*_kernel_cpu of
ProcUpdLazy, compiled from the gsbn sources into oracle/_ref and driven by the
oracle's loops, single-threaded like gsbn's CPU path) over the whole step:
the schedule is cut into warmup + steps contiguous windows and the timed
windows cover everything after the warm-up ones.  The in-line cpu_baseline
times the same kernels on windows spread over the schedule (early, middle
and late segments of both phases), started from the device's state at each
window.  `parity` compares the device's spike logs of one end-to-end step,
segment by segment, with digests of gsbn's kernels running the same step
(tests/golden/config1_spike_digests.json).
"""
import argparse
import hashlib
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}
# nominal FP32 FFMA rate of one B200: 148 SMs x 128 FP32 lanes x 2 flops at
# the 1965 MHz maximum SM clock (no measured figure exists for the SIMT pipes)
FP32_SIMT_PEAK_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return p, "measured"
    except Exception:
        return PEAKS_FALLBACK, "fallback"


def profile_traffic():
    """Per-launch DRAM traffic of tick_kernel from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "tick_kernel_100x100.md")
    try:
        with open(path) as f:
            for line in f:
                if line.startswith("traffic_bytes_per_launch:"):
                    return float(line.split(":")[1])
    except OSError:
        pass
    return None


class Clocks:
    """nvidia-smi clock/throttle sampling during the timed region."""

    def __init__(self, device):
        self.samples = []
        self.proc = None
        self.device = device

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=clocks.sm,clocks.max.sm,power.draw,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples for k in range(4) if len(s) > 3 + k and s[3 + k] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def build_schedule(work_dir):
    """Workload files, network description, connectivity and the segment
    schedule (identical for every step), with product-side helpers only: the
    prototxt is parsed by the protobuf runtime, the ProcInitConn map by
    gsbn_b200.workloads, the schedule by gsbn_b200.extgen."""
    from gsbn_b200 import extgen, schema, workloads
    w = workloads.config1()
    sp, path = w.solver_param(work_dir)
    pops, projs = workloads.net_from_solver_param(sp)
    stim = schema.read_stim(sp.gen_param.stim_file)
    conn = workloads.read_conn_map(w.conn, pops, projs)
    runs = extgen.segments(sp)
    return w, sp, pops, projs, stim, conn, runs


def combine_over_ranks(seconds, units, device):
    """Whole-job figures of a replicated run: the slowest rank's time and the
    units all ranks processed (torch.distributed must be initialised when
    more than one rank runs)."""
    import torch
    if not torch.distributed.is_available() or not torch.distributed.is_initialized() or \
            torch.distributed.get_world_size() == 1:
        return seconds, units
    t = torch.tensor([float(seconds)], dtype=torch.float64, device=device)
    u = torch.tensor([float(units)], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    torch.distributed.all_reduce(u, op=torch.distributed.ReduceOp.SUM)
    return float(t[0]), float(u[0])


def algorithmic_bytes(pops, projs, row_cells, col_cells, ticks):
    """Bytes the reference algorithm must move: 44 B per row cell (read
    pij, eij, zi2, zj2, tij, write them and wij), 40 B per column cell (the
    same without wij) and, per tick, 8*dim_proj + 25 B per MCU for the
    population update (epsc and bj of every incoming projection, lginp, dsup
    read+write, act, spike, counter read+write).  The j-traces (24 B per MCU
    per projection) and the delay queue (16 B per slot) are left out: this
    build keeps them on chip, so the figure is a lower bound."""
    per_tick = 0
    for k, p in enumerate(pops):
        dim_proj = sum(1 for q in projs if q["dest_pop"] == k)
        per_tick += p["hcu_num"] * p["mcu_num"] * (8 * dim_proj + 25)
    return 44 * row_cells + 40 * col_cells + per_tick * ticks


def run_ours(args, rank, world, local_rank, cpu=False):
    import torch
    from gsbn_b200 import capi
    dev = local_rank
    torch.cuda.set_device(dev)
    work = tempfile.mkdtemp(prefix=f"gsbn_bench_{rank}_")
    from gsbn_b200 import extgen
    w, sp, pops, projs, stim, conn, runs = build_schedule(work)
    seed = w.meta["seed"]
    eps = float(np.float32(sp.gen_param.eps))
    net = capi.Net(pops, projs, float(np.float32(sp.gen_param.dt)), seed=seed, device=dev, max_ticks=128)
    for k, (ii, di) in enumerate(conn):
        net.set_conn(k, ii, di)
    # device-resident stimulus: every lgidx row -> lginp row, every wmask row
    lgidx, wmask = extgen.stim_tables(stim)
    net.upload_stimuli_idx(lgidx, eps, wmask)
    stream = torch.cuda.ExternalStream(net.stream(), device=dev)
    n_ticks = sum(r.n for r in runs)

    def step(events=None):
        net.reset()
        for i, r in enumerate(runs):
            net.use_stimulus(r.lgidx, r.wmask)
            if events is not None:
                events[i][0].record(stream)
            net.run(r.first, r.n, r.prn, r.old_prn)
            if events is not None:
                events[i][1].record(stream)

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    for _ in range(args.warmup):
        step()
    net.sync()
    c0 = sum(net.counters())
    l0 = net.kernel_launches()
    per_run = [[(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in runs]
               for _ in range(args.steps)]
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    with Clocks(dev) as clk:
        start.record(stream)
        for s in range(args.steps):
            step(per_run[s])
        stop.record(stream)
        net.sync()
        torch.cuda.synchronize()
    barrier()
    ms = start.elapsed_time(stop)
    cells = sum(net.counters()) - c0
    launches = net.kernel_launches() - l0
    row, col, allc = net.counters()
    # tick-kernel time per launch: one persistent launch per run; runs with an
    # all-cells catch-up (prn change) also launch the sweep and are left out
    tk_ms, tk_ticks, tk_launches = 0.0, 0, 0
    for s in range(args.steps):
        for i, r in enumerate(runs):
            if r.prn == r.old_prn:
                tk_ms += per_run[s][i][0].elapsed_time(per_run[s][i][1])
                tk_ticks += r.n
                tk_launches += 1
    tick_us = tk_ms * 1e3 / max(1, tk_ticks)
    launch_us = tk_ms * 1e3 / max(1, tk_launches)
    ticks_per_launch = tk_ticks / max(1, tk_launches)
    ms, cells = combine_over_ranks(ms, cells, f"cuda:{dev}")

    # e2e: host buffers through the C ABI, every segment's spike log read back
    # (ProcSpkRec's input) and ProcCheck's recall counted on the device.  The
    # step's stimulus tables (ProcExtGen's pattern-index and mask rows) are
    # copied from page-locked memory at the start of every step; each
    # segment's row selection, run, spike-log copy and recall result are
    # queued on the library stream; one sync per step.
    pin_lg = torch.empty(lgidx.shape, dtype=torch.int32, pin_memory=True).numpy()
    pin_wm = torch.empty(wmask.shape, dtype=torch.float32, pin_memory=True).numpy()
    pin_lg[:], pin_wm[:] = lgidx, wmask
    words = (pops[0]["hcu_num"] * pops[0]["mcu_num"] + 31) // 32
    pin_log = [torch.empty((r.n, words), dtype=torch.int32, pin_memory=True).numpy().view(np.uint32) for r in runs]
    h2d = pin_lg.nbytes + pin_wm.nbytes
    d2h = sum(a.nbytes for a in pin_log)
    lib = capi.load()

    check = extgen.DeviceCheck(sp, lgidx, net, [(p["hcu_num"], p["mcu_num"]) for p in pops],
                               alloc=lambda k: torch.zeros(k, dtype=torch.int32, pin_memory=True).numpy())
    d2h += sum(a.nbytes + b.nbytes for c in check.bufs for a, b in c)

    def e2e_step():
        net.reset()
        check.reset()
        net._check(lib.bcpnn_upload_stimuli_idx_async(net._h, pin_lg.shape[0], capi._ptr(pin_lg), eps,
                                                      pin_wm.shape[0], capi._ptr(pin_wm)))
        for i, r in enumerate(runs):
            net._check(lib.bcpnn_use_stimulus(net._h, r.lgidx, r.wmask))
            net.run(r.first, r.n, r.prn, r.old_prn)
            net._check(lib.bcpnn_get_spike_log_async(net._h, 0, capi._ptr(pin_log[i]), pin_log[i].size))
            check.after_run(r)
        net.sync()
        return check.result()

    recall = e2e_step()
    net.sync()
    e0 = sum(net.counters())
    barrier()
    # timed on the device (CUDA events on the library stream), like the rest;
    # each step ends with the host's synchronisation, so the gaps where the
    # device waits for the host's next calls are inside the interval
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        recall = e2e_step()
    ev1.record(stream)
    net.sync()
    torch.cuda.synchronize()
    e_s = ev0.elapsed_time(ev1) * 1e-3
    e_cells = sum(net.counters()) - e0
    e_s, e_cells = combine_over_ranks(e_s, e_cells, f"cuda:{dev}")
    # every e2e step is the same pass from the initial state: its spike logs
    # are the step's spike trains
    parity = spike_parity(pin_log)
    cpu_base = None
    if cpu:
        n = len(runs)
        first_recall = next(i for i, r in enumerate(runs) if r.prn == 0.0)
        picks = sorted({0, first_recall // 2, first_recall - 1, first_recall, (first_recall + n) // 2, n - 1})
        states = capture_states(net, runs, picks)
        v, kind, sample, _ = cpu_spread_sample(sp, pops, projs, seed, runs, states, cells / args.steps / world)
        cpu_base = {"value": v, "unit": "cell updates/s", "cores": 1, "kind": kind, "sample": sample,
                    "cpu": cpu_model()}

    out = None
    if rank == 0:
        pk, pk_kind = peaks()
        n_steps = args.warmup + args.steps + 0.0
        bytes_per_tick = algorithmic_bytes(pops, projs, row / n_steps, col / n_steps, n_ticks) / n_ticks
        bytes_per_launch = bytes_per_tick * ticks_per_launch
        achieved = bytes_per_launch / (launch_us * 1e-6) / 1e9
        traffic = profile_traffic()
        value = cells / (ms / 1e3)
        out = {
            "metric": "synaptic updates/s", "value": value, "unit": "cell updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded patterns and connectivity, gen_rnd.py conventions)",
            "config": {"workload": "100x100 HCU/MCU, recurrent HCU density 0.1 (C=1000, 1e7 cells), 100 patterns: "
                                   "1e4 training + 1e4 recall ticks per step",
                       "ticks_per_step": n_ticks, "segments_per_step": len(runs),
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                       "l2": "state 0.25 GB > 126 MB L2, no flush"},
            "ticks_per_s": n_ticks * args.steps * world / (ms / 1e3),
            "parity": parity,
            "recall": f"{recall[0]}/{recall[1]}",
            "gpu_launches": launches,
            "roofline": {"bound": "hbm", "kernel": "tick_kernel", "achieved": achieved, "peak": pk["hbm_gbs"],
                         "unit": "GB/s", "frac": achieved / pk["hbm_gbs"], "peak_kind": pk_kind,
                         "traffic": traffic, "algorithmic_bytes_per_launch": bytes_per_launch,
                         "us_per_launch": launch_us, "ticks_per_launch": ticks_per_launch,
                         "us_per_tick": tick_us,
                         "traffic_source": "profiles/tick_kernel_100x100.md (ncu dram bytes per launch)"},
            "e2e": {"value": e_cells / e_s, "unit": "cell updates/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "ms_per_step": e_s * 1e3 / args.steps},
            "clocks": clk.summary(),
        }
        if cpu_base is not None:
            out["cpu_baseline"] = cpu_base
    net.close()
    return out


RECALL_STATE = ("pij_0", "eij_0", "zi2_0", "zj2_0", "tij_0", "wij_0", "pi_0", "ei_0", "zi_0", "ti_0", "pj_0", "ej_0",
                "zj_0", "qi_0", "ii_0", "di_0", "si_0", ".siq_0", "dsup_0", "act_0", "epsc_0", "bj_0", "spike_0",
                ".counter_0")


def _recall_engine(tr, W, st, R, lg, wm, seed_base, hz, dev, contraction):
    from gsbn_b200 import recall
    eng = recall.Recall(tr.H, tr.M, R, tr.pops[0], tr.dt, recall.kepsc_of(tr.projs[0], tr.dt), seed_base, hz, dev,
                        contraction=contraction)
    eng.set_cues(lg[:R], tr.eps, wm[:R])
    eng.load_state(W, st["bj"], st["epsc"], st["dsup"], st["s_tm3"], st["s_tm2"], st["s_tm1"])
    eng.clear_counts()
    return eng


def time_recall_engine(tr, W, st, R, T, lg, wm, seed_base, dev, contraction, steps, warmup):
    """One form of the replicate engine on the recall workload: the counted
    run first (ProcCheck's counters over the ticks strictly inside the
    segment), then `warmup` untimed and `steps` timed runs of T ticks, each
    from the trained state (the state load is outside the timed region).  In
    the timed runs the engine also times every contraction launch in place
    (a CUDA event pair on its stream around each launch).  Returns (ms per
    run, counts, kernel launches per run, ms per contraction launch)."""
    import torch
    eng = _recall_engine(tr, W, st, R, lg, wm, seed_base, tr.poisson_hz, dev, contraction)
    try:
        stream = torch.cuda.ExternalStream(eng.stream(), device=dev)

        def load():
            eng.load_state(W, st["bj"], st["epsc"], st["dsup"], st["s_tm3"], st["s_tm2"], st["s_tm1"])
            eng.clear_counts()

        eng.run(tr.t0, T, tr.t0, tr.t0 + T - 2)
        counts = eng.read("counts")
        for _ in range(max(0, warmup - 1)):
            load()
            eng.run(tr.t0, T)
        times, launches = [], 0
        eng.timing(True)
        for _ in range(steps):
            load()
            l0 = eng.launches()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            eng.run(tr.t0, T)
            e1.record(stream)
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
            launches += eng.launches() - l0
        c_ms, c_n = eng.contraction_time()
    finally:
        eng.close()
    return statistics.mean(times), counts, launches / max(1, steps), c_ms / max(1, c_n)


def recall_counts(tr, W, st, R, T, lg, wm, seed_base, hz, dev, contraction):
    """ProcCheck's counters of R replicates after one T-tick recall segment"""
    eng = _recall_engine(tr, W, st, R, lg, wm, seed_base, hz, dev, contraction)
    try:
        eng.run(tr.t0, T, tr.t0, tr.t0 + T - 2)
        return eng.read("counts")
    finally:
        eng.close()


def plain_recall(tr, trained, T, lg, wm, expected, seed_base, hz, dev, n, timed):
    """The plain FP32 path (one ProcUpdLazy network per replicate, every
    trace carried) on replicates 0..n-1: ProcCheck decisions, per-HCU
    accuracy and, when timed, the device time of each replicate's run."""
    import torch
    from gsbn_b200 import capi, recall
    N = tr.H * tr.M
    ms, ok, acc, cells = [], [], [], 0
    for r in range(n):
        net = capi.Net(tr.pops, tr.projs, tr.dt, seed=seed_base + r, poisson_hz=hz, device=dev, max_ticks=T)
        try:
            for name, a in trained.items():
                net.write(name, a)
            net.set_stimulus_idx(lg[r], tr.eps, wm[r])
            ps = torch.cuda.ExternalStream(net.stream(), device=dev)
            c0 = sum(net.counters())
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(ps)
            net.run(tr.t0, T, 0.0, tr.old_prn)
            e1.record(ps)
            net.sync()
            torch.cuda.synchronize()
            if timed:
                ms.append(e0.elapsed_time(e1))
                cells += sum(net.counters()) - c0
            bits = np.unpackbits(net.spike_log(0).view(np.uint8), axis=1, bitorder="little")[:, :N]
        finally:
            net.close()
        counts = bits[: T - 1].sum(axis=0)[None, :]
        ok.append(bool(recall.recall_decisions(counts, tr.H, tr.M, expected[r:r + 1])[0]))
        acc.append(float(recall.hcu_accuracy(counts, tr.H, tr.M, expected[r:r + 1])[0]))
    return ms, ok, acc, cells


def recall_fp64_errors(tr, trained, W, st, T, lg, wm, expected, seed_base, hz, dev, K):
    """Error of both engine forms against the FP64 oracle of the same
    simulation (oracle/recall_fp64.py, pinned to the oracle in double), on
    replicates 0..K-1 of the workload -- the same Philox keys and cues as in
    the timed runs.  Each engine runs the segment tick by tick and its dsup
    and spike rows of the sample are read after every tick; the FP64 oracle
    runs the same K replicates.  Per replicate: the support error before the
    spike trains first differ, the first tick where they differ, the spike
    Jaccard over the run, and ProcCheck's decision."""
    from gsbn_b200 import recall
    from oracle import recall_fp64
    H, M = tr.H, tr.M
    R = max(128, -(-K // 128) * 128)
    lg_r = recall_fp64.lginp_rows(lg[:1], H, M, tr.eps)[0]
    W64, bj0, bj1, pos = recall_fp64.catchup_weights(tr.pops, tr.projs, tr.dt, hz, trained, tr.t0, tr.old_prn, lg_r,
                                                     wm[0])
    rs = recall_fp64.RecallFP64(tr.pops[0], tr.dt, recall_fp64.kepsc_tau(tr.projs[0]), hz, W64, bj0, bj1, pos,
                                st["epsc"], st["dsup"], (st["s_tm3"], st["s_tm2"], st["s_tm1"]), lg, wm, tr.eps,
                                seed_base, list(range(K)))
    d64, s64 = [], []
    for k in range(T):
        d, s = rs.step(tr.t0 + k)
        d64.append(d)
        s64.append(s)
    counts64 = np.sum(np.stack(s64[:T - 1]) != 0, axis=0)
    ok64 = recall.recall_decisions(counts64, H, M, expected[:K])
    out = {"replicates_compared": K, "ticks": T, "poisson_hz": hz,
           "method": "engine rows 0..K-1 read every tick vs the FP64 restatement of the same replicates "
                     "(oracle/recall_fp64.py, spike-identical to OracleNet(real_bits=64))",
           "recall_fp64": f"{int(ok64.sum())}/{K}"}
    for form in ("bf16", "fp32"):
        eng = _recall_engine(tr, W, st, R, lg, wm, seed_base, hz, dev, form)
        try:
            ds, ss = [], []
            for k in range(T):
                eng.run(tr.t0 + k, 1, tr.t0, tr.t0 + T - 2)
                ds.append(eng.read("dsup", 0, K))
                ss.append(eng.read("spike", 0, K))
            ok = recall.recall_decisions(eng.read("counts", 0, K), H, M, expected[:K])
        finally:
            eng.close()
        ms = [recall_fp64.error_metrics([ds[k][i] for k in range(T)], [ss[k][i] for k in range(T)],
                                        [d64[k][i] for k in range(T)], [s64[k][i] for k in range(T)])
              for i in range(K)]
        err = [m["support_rel_err"] for m in ms]
        div = [m["first_divergence_tick"] for m in ms]
        jac = [m["spike_jaccard"] for m in ms]
        out["bf16_engine" if form == "bf16" else "fp32_engine"] = {
            "support_rel_err_max": max(err), "support_rel_err_median": float(np.median(err)),
            "first_divergence_tick_min": min(div), "first_divergence_tick_median": float(np.median(div)),
            "replicates_identical_over_run": sum(int(d == T) for d in div),
            "spike_jaccard_min": min(jac), "spike_jaccard_mean": float(np.mean(jac)),
            "recall": f"{int(ok.sum())}/{K}",
            "recall_agree_with_fp64": f"{int(np.sum(ok == ok64))}/{K}"}
    return out


def run_recall_extension(dev, steps, warmup, replicates=4096, ticks=200, plain_sample=8, fp64_sample=32, cpu=True):
    """The precision extension: recall of a trained 64x64 network (4096 x 4096
    weights) by 4096 noise replicates (25% cue, 20 Hz Poisson noise, 200
    ticks) with the support as a BF16 tcgen05 contraction; against the same
    engine with an FP32 SIMT contraction (W in FP32), against the plain FP32
    path running replicates one network per launch, and against the FP64
    oracle of the same simulation on a sample of replicates."""
    from gsbn_b200 import recall, workloads
    work = workloads.config4()
    tr = recall.Trained(work, tempfile.mkdtemp(prefix="gsbn_recall_"), device=dev)
    trained = tr.snapshot(RECALL_STATE)
    W, st = tr.recall_inputs()
    R, T, seed_base, H, M = replicates, ticks, 1, tr.H, tr.M
    N = H * M
    lg, wm, expected = tr.cues(R)
    ms, counts, launches, k_ms = time_recall_engine(tr, W, st, R, T, lg, wm, seed_base, dev, "bf16", steps, warmup)
    ms32, counts32, launches32, k_ms32 = time_recall_engine(tr, W, st, R, T, lg, wm, seed_base, dev, "fp32", steps,
                                                            warmup)
    flops = 2.0 * R * N * N * T
    tflops, tflops32 = flops / (ms * 1e-3) / 1e12, flops / (ms32 * 1e-3) / 1e12
    k_tflops, k_tflops32 = flops / T / (k_ms * 1e-3) / 1e12, flops / T / (k_ms32 * 1e-3) / 1e12
    pk, pk_kind = peaks()
    value, value32 = R * T / (ms * 1e-3), R * T / (ms32 * 1e-3)

    def decisions(c):
        return recall.recall_decisions(c, H, M, expected), recall.hcu_accuracy(c, H, M, expected)

    ok, acc = decisions(counts)
    ok32, acc32 = decisions(counts32)
    plain_ms, plain_ok, plain_acc, plain_cells = plain_recall(tr, trained, T, lg, wm, expected, seed_base,
                                                              tr.poisson_hz, dev, plain_sample, True)
    plain_rate = T / (statistics.mean(plain_ms) * 1e-3)
    # the same trained weights recalled without the input noise
    ok_q, acc_q = decisions(recall_counts(tr, W, st, R, T, lg, wm, seed_base, 0.0, dev, "bf16"))
    ok32_q, acc32_q = decisions(recall_counts(tr, W, st, R, T, lg, wm, seed_base, 0.0, dev, "fp32"))
    _, plain_q, plain_q_acc, _ = plain_recall(tr, trained, T, lg, wm, expected, seed_base, 0.0, dev, plain_sample,
                                              False)
    fp64 = {"with_noise": recall_fp64_errors(tr, trained, W, st, T, lg, wm, expected, seed_base, tr.poisson_hz, dev,
                                             fp64_sample),
            "without_noise": recall_fp64_errors(tr, trained, W, st, T, lg, wm, expected, seed_base, 0.0, dev,
                                                fp64_sample)}

    def frac(x):
        return f"{int(np.sum(x))}/{len(x)}"

    def agree(a, b):
        return f"{int(np.sum(np.asarray(a) == np.asarray(b)))}/{len(a)}"

    def rec(o, a, o32, a32, po, pa):
        return {"bf16_all": frac(o), "fp32_engine_all": frac(o32), "decisions_agree_bf16_fp32_all": agree(o, o32),
                "bf16_sample": frac(o[:plain_sample]), "plain_fp32_sample": frac(po),
                "decisions_agree_bf16_plain_sample": agree(o[:plain_sample], po),
                "hcu_accuracy_bf16_all": float(a.mean()), "hcu_accuracy_fp32_engine_all": float(a32.mean()),
                "hcu_accuracy_plain_fp32_sample": float(np.mean(pa)),
                "hcu_accuracy_bf16_sample": float(a[:plain_sample].mean())}

    if cpu:
        try:
            v, sample = cpu_recall_sample(tr.pops, tr.projs, tr.dt, tr.poisson_hz, trained, lg[0], wm[0], tr.eps,
                                          tr.t0, tr.old_prn, T, seed_base)
            cpu_base = {"value": v, "unit": "replicate-ticks/s", "cores": 1, "kind": "port", "sample": sample,
                        "cpu": cpu_model()}
        except Exception as e:  # an auxiliary figure: the GPU numbers stand without it
            cpu_base = {"unavailable": f"{type(e).__name__}: {e}"}
    else:
        cpu_base = None
    return {
        "workload": f"64x64 HCU/MCU full recurrent (4096 x 4096 weights), {work.meta['patterns']} patterns trained "
                    f"300 ticks each, {R} noise replicates, 25% cue, 20 Hz Poisson noise, {T} recall ticks",
        "metric": "replicate ticks/s", "value": value, "unit": "replicate-ticks/s", "steps": steps,
        "ms_per_step": ms, "us_per_tick": ms * 1e3 / T, "gpu_launches_per_step": launches,
        "dtype": "bf16 weights x exact 0/1 spikes, fp32 accumulate; fp32 state",
        "roofline": {"bound": "tensor", "kernel": "recall_tick_kernel", "achieved": k_tflops,
                     "peak": pk["bf16_tflops"], "unit": "TFLOP/s", "frac": k_tflops / pk["bf16_tflops"],
                     "peak_kind": pk_kind + " (burst)", "flops_per_launch": 2.0 * R * N * N,
                     "us_per_launch": k_ms * 1e3,
                     "timing": "CUDA event pair around every contraction launch on its stream, in place beside the "
                               "population kernel of the same tick",
                     "tick_tflops": tflops, "tick_frac": tflops / pk["bf16_tflops"]},
        "fp32_engine": {"value": value32, "unit": "replicate-ticks/s", "ms_per_step": ms32,
                        "us_per_tick": ms32 * 1e3 / T, "tflops": tflops32, "gpu_launches_per_step": launches32,
                        "contraction_us_per_launch": k_ms32 * 1e3, "contraction_tflops": k_tflops32,
                        "kernel": "recall_fp32_kernel (SIMT FFMA, W in fp32)",
                        "fp32_simt_peak_tflops": FP32_SIMT_PEAK_TFLOPS,
                        "frac_of_fp32_simt_peak": k_tflops32 / FP32_SIMT_PEAK_TFLOPS},
        "speedup_bf16_vs_fp32_engine": value / value32,
        "plain_fp32": {"value": plain_rate, "unit": "replicate-ticks/s", "replicates_timed": plain_sample,
                       "ms_per_replicate": statistics.mean(plain_ms),
                       "cell_updates_per_s": plain_cells / (sum(plain_ms) * 1e-3)},
        "speedup_vs_plain_fp32": value / plain_rate,
        "recall": dict(rec(ok, acc, ok32, acc32, plain_ok, plain_acc),
                       fp64_sample=fp64["with_noise"]["recall_fp64"],
                       without_noise=dict(rec(ok_q, acc_q, ok32_q, acc32_q, plain_q, plain_q_acc),
                                          fp64_sample=fp64["without_noise"]["recall_fp64"])),
        "fp64_error": fp64,
        "cpu_baseline": cpu_base,
    }


def run_multi_extension(dev, steps, warmup, ring=25, cpu=True):
    """ProcUpdMulti (row-only updates replaying a ring of postsynaptic spikes,
    adaptation) on the 100x100 density-0.1 workload with gsbn's spike buffer
    size 25: the same 200-segment step as the headline, one persistent launch
    per run (the resident form: each HCU's state in shared memory)."""
    import torch
    from gsbn_b200 import capi, extgen
    work = tempfile.mkdtemp(prefix="gsbn_multi_")
    w, sp, pops, projs, stim, conn, runs = build_schedule(work)
    pops = [dict(p, taua=0.05, adgain=1.0) for p in pops]
    net = capi.Net(pops, projs, float(np.float32(sp.gen_param.dt)), seed=w.meta["seed"], device=dev, max_ticks=128,
                   variant=1, spike_buffer=ring)
    try:
        for k, (ii, di) in enumerate(conn):
            net.set_conn(k, ii, di)
        lgidx, wmask = extgen.stim_tables(stim)
        net.upload_stimuli_idx(lgidx, float(np.float32(sp.gen_param.eps)), wmask)
        stream = torch.cuda.ExternalStream(net.stream(), device=dev)

        def step():
            net.reset()
            for r in runs:
                net.use_stimulus(r.lgidx, r.wmask)
                net.run(r.first, r.n, r.prn, r.old_prn)

        for _ in range(max(1, warmup)):
            step()
        net.sync()
        c0, l0 = sum(net.counters()), net.kernel_launches()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            step()
        e1.record(stream)
        net.sync()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        cells = (sum(net.counters()) - c0) / steps
        ticks = sum(r.n for r in runs)
        out = {"workload": "100x100 HCU/MCU, recurrent density 0.1, ProcUpdMulti with spike buffer size 25 "
                           "(adaptation taua 0.05, adgain 1): 1e4 training + 1e4 recall ticks per step",
               "metric": "synaptic updates/s", "value": cells / (ms * 1e-3), "unit": "cell updates/s",
               "ticks_per_s": ticks / (ms * 1e-3), "us_per_tick": ms * 1e3 / ticks, "ms_per_step": ms,
               "steps": steps, "gpu_launches_per_step": (net.kernel_launches() - l0) / steps, "dtype": "f32"}
    finally:
        net.close()
    if cpu:
        try:
            v, sample = cpu_multi_sample(ring)
            out["cpu_baseline"] = {"value": v, "unit": "cell updates/s", "cores": 1, "kind": "port",
                                   "sample": sample, "cpu": cpu_model()}
        except Exception as e:  # an auxiliary figure: the GPU numbers above stand without it
            out["cpu_baseline"] = {"unavailable": f"{type(e).__name__}: {e}"}
    return out


BATCH_PARITY = ("dsup_0", "act_0", "epsc_0", "bj_0", "spike_0", ".counter_0", "pj_0", "ej_0", "zj_0", "pi_0", "ei_0",
                "zi_0", "ti_0")


def run_batch_extension(dev, steps, n_nets=256, head_ticks=500, cpu=True):
    """The batching extension: 256 independent networks of uneven size (HCUs
    8-64, MCUs 5-50, full recurrent), 20 patterns each, advanced together by
    the batch engine (one persistent kernel per run) under the launch shape its
    tuner picks, against the plain path (one network per launch, one after the
    other) on the same first ticks."""
    import torch
    from gsbn_b200 import batch
    members = batch.make_members(n_nets)
    runs = batch.schedule(20, train_ticks=100, recall_ticks=50)
    ticks = sum(r[1] for r in runs)
    eng = batch.BatchEngine(members, device=dev, max_ticks=128)
    t0 = time.perf_counter()
    shape, tune_us = eng.tune(20, train_rows=(0, 0), recall_rows=(20, 1))
    tune_s = time.perf_counter() - t0
    stream = torch.cuda.ExternalStream(eng.stream(), device=dev)

    def step():
        eng.reset()
        for r in runs:
            eng.run_segment(*r)

    step()  # warm-up: tables, the first catch-ups
    eng.sync()
    c0, l0 = eng.counters(), eng.launches()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(steps):
        step()
    e1.record(stream)
    eng.sync()
    torch.cuda.synchronize()
    sec = e0.elapsed_time(e1) * 1e-3 / steps
    c1 = eng.counters()
    row, col, allc = [(c1[k] - c0[k]) / steps for k in range(3)]
    cells = row + col + allc
    launches = (eng.launches() - l0) / steps
    head = [r for r in runs if r[0] <= head_ticks]
    n_head = sum(r[1] for r in head)
    eng.reset()
    torch.cuda.synchronize()
    h0, h1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    h0.record(stream)
    for r in head:
        eng.run_segment(*r)
    h1.record(stream)
    eng.sync()
    t_head_batch = h0.elapsed_time(h1) * 1e-3
    plain = batch.Plain(members, device=dev)
    plain.run_segment(1, 2, 1.0, 0.0, 0, 0)  # warm-up: tables, graphs
    plain.sync()
    plain.reset()
    plain.sync()
    pc0 = plain.counters()
    t0 = time.perf_counter()
    for r in head:
        for net in plain.nets:
            net.use_stimulus(r[4], r[5])
            net.run(*r[:4])
            net.sync()
    t_head_plain = time.perf_counter() - t0
    plain_cells = plain.counters() - pc0
    # every member against the same network run alone on the plain path, after
    # the same ticks: population and row-trace vectors by bit pattern
    same = 0
    for k, net in enumerate(plain.nets):
        same += all(np.array_equal(np.asarray(eng.read(k, n)).view(np.uint8), np.asarray(net.read(n)).view(np.uint8))
                    for n in BATCH_PARITY)
    eng.close()
    plain.close()
    pk, pk_kind = peaks()
    # algorithmic bytes: 44 B per row cell and all-cells cell, 40 B per column
    # cell, 8 + 25 B per MCU per tick (one projection per member)
    mcus = sum(m.H * m.M for m in members)
    algo = 44 * (row + allc) + 40 * col + 33 * mcus * ticks
    achieved = algo / sec / 1e9
    out = {
        "workload": f"{n_nets} independent networks, HCUs 8-64 x MCUs 5-50 (uniform), full recurrent, "
                    f"{sum(m.cells for m in members) / 1e6:.0f}M cells, 20 patterns each: "
                    f"{ticks} ticks (20 x 100 training + 20 x 50 recall)",
        "metric": "network ticks/s", "value": n_nets * ticks / sec, "unit": "network-ticks/s",
        "cell_updates_per_s": cells / sec, "ms_per_step": sec * 1e3, "us_per_tick": sec * 1e6 / ticks,
        "steps": steps, "gpu_launches_per_step": launches,
        "schedule": {"threads": shape[0], "cost_weights": list(shape[1:]), "tuner_us_per_tick": tune_us,
                     "tuner_s": tune_s},
        "roofline": {"bound": "hbm", "kernel": "batch_kernel", "achieved": achieved, "peak": pk["hbm_gbs"],
                     "unit": "GB/s", "frac": achieved / pk["hbm_gbs"], "peak_kind": pk_kind,
                     "algorithmic_bytes_per_step": algo},
        "plain_one_network_per_launch": {"network_ticks_per_s": n_nets * n_head / t_head_plain,
                                         "cell_updates_per_s": plain_cells / t_head_plain, "ticks_timed": n_head},
        "batched_same_ticks": {"network_ticks_per_s": n_nets * n_head / t_head_batch},
        "speedup_vs_plain_same_ticks": t_head_plain / t_head_batch,
        "parity_vs_plain": {"members_identical": f"{same}/{len(members)}", "ticks": n_head,
                            "arrays": list(BATCH_PARITY)},
    }
    if cpu:
        try:
            v, cores, sample = cpu_batch_sample(members, runs)
            out["cpu_baseline"] = {"value": v, "unit": "network-ticks/s", "cores": cores, "kind": "port",
                                   "sample": sample, "cpu": cpu_model()}
        except Exception as e:  # an auxiliary figure: the GPU numbers above stand without it
            out["cpu_baseline"] = {"unavailable": f"{type(e).__name__}: {e}"}
    return out


def _phase_sample(orc, runs, sample_ticks):
    """Time an oracle network (OracleNet or MultiNetC) on a bounded sample of
    a schedule: the first `sample_ticks` training ticks, then
    `sample_ticks // 2` recall ticks, each phase's first tick (which carries
    its all-cells pass) timed alone.  Returns (cells/s scaled to the whole
    schedule by the phase rates, training ticks run, recall ticks run,
    seconds spent)."""
    train = [r for r in runs if r.prn != 0.0]
    recall = [r for r in runs if r.prn == 0.0]

    def timed(rs, limit):
        c0, t0, done = sum(orc.counters()), time.perf_counter(), 0
        for r in rs:
            n = min(r.n, limit - done)
            if n <= 0:
                break
            orc.set_stimulus(r.lginp, r.wmask)
            orc.run(r.first, n, r.prn, r.old_prn, spikes=False)
            done += n
        return time.perf_counter() - t0, sum(orc.counters()) - c0, done

    def phase(rs, limit):
        # the first tick carries the phase's all-cells catch-up: timed alone
        head = [type(rs[0])(rs[0].first, 1, rs[0].prn, rs[0].old_prn, rs[0].lginp, rs[0].wmask, None)]
        tail = [type(rs[0])(rs[0].first + 1, rs[0].n - 1, rs[0].prn, rs[0].prn, rs[0].lginp, rs[0].wmask, None)]
        t1, c1, _ = timed(head, 1)
        t2, c2, n2 = timed(tail + rs[1:], limit - 1)
        total = sum(r.n for r in rs)
        return t1 + t2 / n2 * (total - 1), c1 + c2 / n2 * (total - 1), t1 + t2, 1 + n2

    t_tr, c_tr, s_tr, n_tr = phase(train, sample_ticks)
    t_rc, c_rc, s_rc, n_rc = phase(recall, sample_ticks // 2)
    return (c_tr + c_rc) / (t_tr + t_rc), n_tr, n_rc, s_tr + s_rc


GOLDEN_DIGESTS = os.path.join(ROOT, "tests", "golden", "config1_spike_digests.json")
ORACLE_POP = ("dsup", "act", "epsc", "bj", "spike", ".counter")
ORACLE_PROJ = ("ii", "di", "qi", "ti", "tij", "pi", "ei", "zi", "pj", "ej", "zj", "pij", "eij", "zi2", "zj2", "wij",
               "si", ".siq")


def reference_oracle(pops, projs, dt, seed):
    """gsbn's own CPU kernels (oracle/_ref, math MATH_REF) when that build
    exists, else the restatement with glibc math (MATH_LIBM, bit-identical to
    them in the CPU tests).  Returns (oracle network, kind, math description)."""
    from oracle import sim
    if sim.ref_available():
        return (sim.OracleNet(pops, projs, dt, seed=seed, math=sim.MATH_REF), "reference",
                "gsbn's update_*_kernel_cpu compiled from its sources (oracle/_ref), glibc expf/logf, 1 thread")
    return (sim.OracleNet(pops, projs, dt, seed=seed, math=sim.MATH_LIBM), "port",
            "oracle restatement with glibc expf/logf (oracle/_ref not built), 1 thread")


def host_runs(sp, pops, runs):
    """(first, n, prn, old_prn, lginp, wmask) per segment, with ProcExtGen's
    lginp values from the host's float log, as gsbn computes them"""
    from gsbn_b200 import extgen, schema
    from oracle import sim
    lgidx, wmask = extgen.stim_tables(schema.read_stim(sp.gen_param.stim_file))
    eps = np.float32(sp.gen_param.eps)
    H, M = pops[0]["hcu_num"], pops[0]["mcu_num"]
    hit, miss = sim.extgen_logf(np.float32(1) + eps), sim.extgen_logf(np.float32(0) + eps)
    return [(r.first, r.n, r.prn, r.old_prn, _lginp_row(lgidx[r.lgidx], H, M, hit, miss), wmask[r.wmask][:H])
            for r in runs]


def capture_states(net, runs, picks):
    """The device state at the start of each picked segment, from one more
    pass of the step (outside every timed region)."""
    names = [f"{k}_0" for k in ORACLE_POP + ORACLE_PROJ]
    net.reset()
    states = {}
    for i, r in enumerate(runs):
        if i in picks:
            net.sync()
            states[i] = {n: net.read(n) for n in names}
        net.use_stimulus(r.lgidx, r.wmask)
        net.run(r.first, r.n, r.prn, r.old_prn)
    net.sync()
    return states


def cpu_spread_sample(sp, pops, projs, seed, runs, states, cells_per_step):
    """gsbn's kernels on one core, on windows spread over the schedule: each
    picked segment is run from the device's state at its start.  A segment
    whose prn differs from the previous one carries the all-cells catch-up in
    its first tick, which is timed alone.  The step's CPU time is estimated as
    the catch-up ticks as measured plus the mean per-tick time of each phase
    times that phase's other ticks; the value is the device-counted cells of a
    step over that time.  Returns (cells/s, kind, sample description, seconds
    spent)."""
    orc, kind, math = reference_oracle(pops, projs, float(np.float32(sp.gen_param.dt)), seed)
    hr = host_runs(sp, pops, runs)
    per_tick = {True: [0.0, 0], False: [0.0, 0]}   # training?: [seconds, ticks]
    switch = {True: [], False: []}
    spent = 0.0
    for i in sorted(states):
        for name, a in states[i].items():
            orc.write(name, a)
        first, n, prn, old_prn, lg, wm = hr[i]
        orc.set_stimulus(lg, wm)
        train = prn != 0.0
        t0 = time.perf_counter()
        orc.run(first, 1, prn, old_prn, spikes=False)
        t1 = time.perf_counter()
        orc.run(first + 1, n - 1, prn, prn, spikes=False)
        t2 = time.perf_counter()
        if prn != old_prn:
            switch[train].append(t1 - t0)
            per_tick[train][0] += t2 - t1
            per_tick[train][1] += n - 1
        else:
            per_tick[train][0] += t2 - t0
            per_tick[train][1] += n
        spent += t2 - t0
    est = 0.0
    for train in (True, False):
        rs = [r for r in runs if (r.prn != 0.0) == train]
        n_sw = sum(1 for r in rs if r.prn != r.old_prn)
        ticks = sum(r.n for r in rs)
        sw = statistics.mean(switch[train]) if switch[train] else 0.0
        est += n_sw * sw + per_tick[train][0] / max(1, per_tick[train][1]) * (ticks - n_sw)
    picks = sorted(states)
    sample = (f"{math}; {len(picks)} segments of the step (indices {picks}, "
              f"{sum(runs[i].n for i in picks)} ticks: early, middle and late training and recall, each started "
              f"from the device's state, catch-up ticks timed alone), {spent:.1f} s of CPU; step time = catch-ups "
              f"+ per-phase tick time x phase ticks; value = device-counted cells per step / that time")
    return cells_per_step / est, kind, sample, spent


def spike_parity(pin_logs, path=GOLDEN_DIGESTS):
    """The device's spike logs of one end-to-end step, segment by segment,
    against the digests of gsbn's kernels running the same step."""
    try:
        with open(path) as f:
            gold = json.load(f)
    except OSError as e:
        return {"status": "unchecked", "why": str(e)}
    segs = gold["segments"]
    if len(segs) != len(pin_logs):
        return {"status": "unchecked", "why": f"{len(segs)} golden segments, {len(pin_logs)} device segments"}
    same, first_bad = 0, None
    for k, (g, log) in enumerate(zip(segs, pin_logs)):
        if hashlib.sha256(np.ascontiguousarray(log).tobytes()).hexdigest() == g["sha256"]:
            same += 1
        elif first_bad is None:
            got = int(np.unpackbits(log.view(np.uint8)).sum())
            first_bad = {"segment": k, "first_tick": g["first"], "device_spikes": got, "reference_spikes": g["spikes"]}
    out = {"status": "identical" if same == len(segs) else "differs", "segments_identical": f"{same}/{len(segs)}",
           "ticks": gold["ticks"], "reference_spikes": gold["spikes"], "against": gold["math"],
           "digests": "tests/golden/config1_spike_digests.json"}
    if first_bad:
        out["first_difference"] = first_bad
    return out


def cpu_multi_sample(ring, sample_ticks=1200):
    """The compiled ProcUpdMulti oracle (oracle/bcpnn_oracle_multi.cpp) on a
    bounded sample of the ProcUpdMulti workload, one core, as cpu_sample.
    Returns (cells/s, sample description)."""
    from gsbn_b200 import workloads
    from oracle import multi, sim
    from tests.harness import load_workload, schedule
    work = tempfile.mkdtemp(prefix="gsbn_cpu_multi_")
    sp, pops, projs, stim, conn, seed, phz = load_workload(workloads.config1(), work)
    pops = [dict(p, taua=0.05, adgain=1.0) for p in pops]
    orc = multi.MultiNetC(pops, projs, float(np.float32(sp.gen_param.dt)), seed=seed, spike_buffer=ring)
    for k, (ii, di) in enumerate(conn):
        orc.set_conn(k, ii, di)
    runs = schedule(sp, stim, pops, sim.extgen_logf)
    v, n_tr, n_rc, secs = _phase_sample(orc, runs, sample_ticks)
    sample = (f"{n_tr} training ticks + {n_rc} recall ticks, including both all-cells catch-ups, {secs:.1f} s "
              f"on 1 core; per-tick rates scaled to the 2e4-tick step")
    return v, sample


def _lginp_row(row, hcu, mcu, hit, miss):
    """ProcExtGen's lginp for one stimulus row (ProcExtGen.cpp:130-144): per
    HCU log(1+eps) on the indexed MCU, log(eps) elsewhere and on HCUs without
    input."""
    out = np.full(hcu * mcu, miss, np.float32)
    row = np.asarray(row[:hcu], np.int64)
    h = np.nonzero((row >= 0) & (row < mcu))[0]
    out[h * mcu + row[h]] = hit
    return out


def _batch_member_cpu(item):
    """One batch member on the oracle, in a spawned worker: its first training
    tick (with the start-of-run all-cells pass) and k_tr more training ticks,
    then its first recall tick (with the training->recall all-cells catch-up)
    and k_rc more recall ticks, each part timed alone.  Returns the member's
    CPU seconds for its whole schedule, scaled per phase, and the seconds
    actually spent."""
    (pop, proj, seed, ii, di, lg_tr, wm_tr, lg_rc, wm_rc, tr_run, rc_run, dt, eps, k_tr, k_rc) = item
    from oracle import sim
    orc = sim.OracleNet([pop], [proj], dt, seed=seed)
    orc.set_conn(0, ii, di)
    H, M = pop["hcu_num"], pop["mcu_num"]
    hit, miss = orc.logf(np.float32(1) + np.float32(eps)), orc.logf(np.float32(eps))
    total, spent = 0.0, 0.0
    for (first, n_phase, prn, old_prn), lg, wm, k in ((tr_run, lg_tr, wm_tr, k_tr), (rc_run, lg_rc, wm_rc, k_rc)):
        orc.set_stimulus(_lginp_row(lg, H, M, hit, miss), wm[:H])
        t0 = time.perf_counter()
        orc.run(first, 1, prn, old_prn, spikes=False)
        t1 = time.perf_counter()
        orc.run(first + 1, k, prn, prn, spikes=False)
        t2 = time.perf_counter()
        total += (t1 - t0) + (t2 - t1) / k * (n_phase - 1)
        spent += t2 - t0
    return total, spent


def cpu_batch_sample(members, runs, k_tr=20, k_rc=10):
    """The oracle on the batched workload: B independent networks over the
    host's cores (one spawned worker per core, largest networks first).  Every
    member runs a bounded sample of its schedule (_batch_member_cpu); the
    members' scaled CPU seconds, summed and divided by the cores, give the
    wall time of the whole batch.  Returns (network ticks/s, cores, sample
    description)."""
    import multiprocessing as mp
    train = [r for r in runs if r[2] != 0.0]
    recall = [r for r in runs if r[2] == 0.0]
    tr_run = (train[0][0], sum(r[1] for r in train), train[0][2], train[0][3])
    rc_run = (recall[0][0], sum(r[1] for r in recall), recall[0][2], recall[0][3])
    ticks = sum(r[1] for r in runs)
    items = [(m.pop, m.proj, m.seed, m.ii, m.di, m.lgidx[train[0][4]], m.wmask[train[0][5]],
              m.lgidx[recall[0][4]], m.wmask[recall[0][5]], tr_run, rc_run, 0.001, 1e-4, k_tr, k_rc)
             for m in sorted(members, key=lambda m: -m.cells)]
    from concurrent.futures import ProcessPoolExecutor
    cores = max(1, min(len(os.sched_getaffinity(0)), 64, len(items)))
    t0 = time.perf_counter()
    # spawned workers (no fork of a process that holds a CUDA context); a worker
    # that dies raises BrokenProcessPool here instead of leaving a wait behind
    with ProcessPoolExecutor(max_workers=cores, mp_context=mp.get_context("spawn")) as pool:
        res = list(pool.map(_batch_member_cpu, items, chunksize=1))
    wall = time.perf_counter() - t0
    cpu_total = sum(r[0] for r in res)
    value = len(members) * ticks / (cpu_total / cores)
    sample = (f"all {len(members)} networks, each 1+{k_tr} training and 1+{k_rc} recall ticks (both all-cells "
              f"passes included) on {cores} worker processes, {wall:.1f} s wall; per-phase tick rates scaled to "
              f"the {ticks}-tick schedule, summed CPU time divided by the cores")
    return value, cores, sample


def cpu_recall_sample(pops, projs, dt, poisson_hz, state, lg_row, wm_row, eps, t0, old_prn, ticks, seed, k=40):
    """The oracle on one recall replicate of the trained network, one core:
    the end-of-training state written in, the first recall tick (with its
    all-cells catch-up) and k more ticks timed, scaled to `ticks` ticks.
    gsbn has no recall-only path, so this is the full ProcUpdLazy per tick.
    Returns (replicate ticks/s, sample description)."""
    from oracle import sim
    orc = sim.OracleNet(pops, projs, dt, seed=seed, poisson_hz=poisson_hz)
    for name, a in state.items():
        orc.write(name, a)
    H, M = pops[0]["hcu_num"], pops[0]["mcu_num"]
    hit, miss = orc.logf(np.float32(1) + np.float32(eps)), orc.logf(np.float32(eps))
    orc.set_stimulus(_lginp_row(lg_row, H, M, hit, miss), wm_row[:H])
    s0 = time.perf_counter()
    orc.run(t0, 1, 0.0, old_prn, spikes=False)
    s1 = time.perf_counter()
    orc.run(t0 + 1, k, 0.0, 0.0, spikes=False)
    s2 = time.perf_counter()
    per_rep = (s1 - s0) + (s2 - s1) / k * (ticks - 1)
    sample = (f"one replicate, 1+{k} recall ticks on 1 core ({s2 - s0:.1f} s; the first tick carries the "
              f"all-cells catch-up), scaled to {ticks} ticks")
    return ticks / per_rep, sample


def cut_windows(hruns, n_win):
    """The runs (first, n, prn, old_prn, lginp, wmask) of a schedule cut into
    n_win contiguous windows of equal tick counts; a run split across windows
    continues with old_prn = prn, as one run of ticks does.  Returns (windows,
    tick bounds)."""
    total = sum(r[1] for r in hruns)
    bounds = [round(total * k / n_win) for k in range(n_win + 1)]
    windows = [[] for _ in range(n_win)]
    t = 0
    for first, n, prn, old_prn, lg, wm in hruns:
        k = 0
        while k < n:
            win = max(i for i in range(n_win) if bounds[i] <= t)
            take = min(n - k, bounds[win + 1] - t)
            windows[win].append((first + k, take, prn, old_prn if k == 0 else prn, lg, wm))
            k += take
            t += take
    return windows, bounds


def run_reference(args):
    """The reference arm: gsbn's own CPU kernels (reference_oracle), one
    thread like gsbn's ProcUpdLazy CPU path, on the same workload.  The step's
    2e4-tick schedule is cut into warmup + steps contiguous windows of equal
    tick counts; the warm-up windows run untimed and the timed windows cover
    the rest of the schedule, training->recall catch-up included.  value =
    cells the timed windows updated / their time."""
    from gsbn_b200 import workloads
    work = tempfile.mkdtemp(prefix="gsbn_ref_")
    w, sp, pops, projs, stim, conn, runs = build_schedule(work)
    orc, kind, math = reference_oracle(pops, projs, float(np.float32(sp.gen_param.dt)), w.meta["seed"])
    for k, (ii, di) in enumerate(conn):
        orc.set_conn(k, ii, di)
    total = sum(r.n for r in runs)
    n_win = args.warmup + args.steps
    windows, bounds = cut_windows(host_runs(sp, pops, runs), n_win)
    secs, cells = [], []
    for i, win in enumerate(windows):
        c0, t0 = sum(orc.counters()), time.perf_counter()
        for first, n, prn, old_prn, lg, wm in win:
            orc.set_stimulus(lg, wm)
            orc.run(first, n, prn, old_prn, spikes=False)
        if i >= args.warmup:
            secs.append(time.perf_counter() - t0)
            cells.append(sum(orc.counters()) - c0)
    value = sum(cells) / sum(secs)
    timed_ticks = total - bounds[args.warmup]
    sample = (f"{math}; ticks {bounds[args.warmup] + 1}..{total} of the 2e4-tick step in {args.steps} contiguous "
              f"windows of ~{total // n_win} ticks ({sum(secs):.1f} s timed) after {args.warmup} untimed warm-up "
              f"windows; value = cells updated / time over the timed windows")
    return {
        "metric": "synaptic updates/s", "value": value, "unit": "cell updates/s", "n_gpus": 0,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": sum(secs) * 1e3 / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded patterns and connectivity, gen_rnd.py conventions)", "impl": "reference",
        "config": {"workload": "100x100 HCU/MCU, recurrent HCU density 0.1 (C=1000, 1e7 cells), 100 patterns: "
                               "1e4 training + 1e4 recall ticks per step",
                   "ticks_timed": timed_ticks},
        "cpu_baseline": {"value": value, "unit": "cell updates/s", "cores": 1, "kind": kind, "sample": sample,
                         "cpu": cpu_model()},
        "e2e": {"value": value, "unit": "cell updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def extensions_summary(ext):
    """The headline figures of each extension, short enough to sit near the
    front of the JSON line (the full objects follow under "extensions")."""
    out = {}
    r = ext.get("bf16_recall")
    if r:
        f = r.get("fp64_error", {}).get("with_noise", {})
        out["bf16_recall"] = {
            "replicate_ticks_per_s": r["value"], "contraction_tflops": r["roofline"]["achieved"],
            "contraction_frac_bf16_peak": r["roofline"]["frac"], "tick_frac_bf16_peak": r["roofline"]["tick_frac"],
            "speedup_bf16_vs_fp32_engine": r.get("speedup_bf16_vs_fp32_engine"),
            "speedup_vs_plain_fp32": r.get("speedup_vs_plain_fp32"),
            "recall_bf16_fp32engine_fp64sample": [r["recall"]["bf16_all"], r["recall"]["fp32_engine_all"],
                                                 r["recall"].get("fp64_sample")],
            "recall_without_noise": [r["recall"]["without_noise"]["bf16_all"],
                                     r["recall"]["without_noise"]["fp32_engine_all"],
                                     r["recall"]["without_noise"].get("fp64_sample")],
            "fp64_support_rel_err_max_bf16_fp32": [f.get("bf16_engine", {}).get("support_rel_err_max"),
                                                   f.get("fp32_engine", {}).get("support_rel_err_max")],
            "fp64_replicates": f.get("replicates_compared")}
    b = ext.get("batched")
    if b:
        out["batched"] = {"network_ticks_per_s": b["value"], "speedup_vs_plain": b.get("speedup_vs_plain_same_ticks"),
                          "members_identical_to_plain": b.get("parity_vs_plain", {}).get("members_identical"),
                          "frac_hbm": b.get("roofline", {}).get("frac"), "cell_updates_per_s": b.get("cell_updates_per_s")}
    m = ext.get("procupdmulti")
    if m:
        out["procupdmulti"] = {"cell_updates_per_s": m["value"]}
    return out


def front(out, key, value, after="dtype"):
    """out with `key` inserted right after `after`"""
    res = {}
    for k, v in out.items():
        res[k] = v
        if k == after:
            res[key] = value
    if key not in res:
        res[key] = value
    return res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extensions", action="store_true")
    ap.add_argument("--only-extensions", action="store_true", help="run the extension workloads alone (profiling)")
    ap.add_argument("--batch-nets", type=int, default=256, help="networks of the batched extension")
    ap.add_argument("--ext", default="bf16_recall,batched,procupdmulti",
                    help="with --only-extensions: the extensions to run (comma separated)")
    ap.add_argument("--recall-replicates", type=int, default=4096)
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    cpu = world == 1 and not args.no_cpu_baseline
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args)), flush=True)
        return
    if world > 1:
        import datetime

        import torch
        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    if args.only_extensions:
        if rank == 0:
            want = args.ext.split(",")
            ext = {}
            if "bf16_recall" in want:
                ext["bf16_recall"] = run_recall_extension(local_rank, args.steps, args.warmup,
                                                          args.recall_replicates, cpu=cpu)
            if "batched" in want:
                ext["batched"] = run_batch_extension(local_rank, max(1, args.steps // 2), n_nets=args.batch_nets,
                                                     cpu=cpu)
            if "procupdmulti" in want:
                ext["procupdmulti"] = run_multi_extension(local_rank, max(1, args.steps // 2), 1, cpu=cpu)
            print(json.dumps({"extensions_summary": extensions_summary(ext), "extensions": ext}), flush=True)
        return
    out = run_ours(args, rank, world, local_rank, cpu=cpu)
    # the extensions are single-GPU measurements: under torchrun the other
    # ranks would hold their GPUs at the final barrier while rank 0 runs them
    if rank == 0 and world == 1 and not args.no_extensions:
        out["extensions"] = {"bf16_recall": run_recall_extension(local_rank, args.steps, args.warmup,
                                                                 args.recall_replicates, cpu=cpu),
                             "batched": run_batch_extension(local_rank, max(1, args.steps // 2),
                                                            n_nets=args.batch_nets, cpu=cpu),
                             "procupdmulti": run_multi_extension(local_rank, max(1, args.steps // 2), 1, cpu=cpu)}
        out = front(out, "extensions_summary", extensions_summary(out["extensions"]))
    if rank == 0:
        print(json.dumps(out), flush=True)
    if world > 1:
        import torch
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
