"""Replicate recall engine (tcgen05 BF16 support contraction + fused
population update) on the GPU, and its FP32 SIMT form.

1. Synthetic state, tick by tick, both forms: dsup and spikes must equal, bit
   for bit, a float32 restatement of gsbn's population update (shared exp,
   Philox streams); epsc must equal epsc*(1-kepsc) + S(t-3) . W computed in
   float64 (W rounded to BF16 for the BF16 form, as is for the FP32 form),
   within the FP32 accumulation bound; the spike ring must feed each
   tick's own spikes back three ticks later; counters must sum the counted
   ticks.
2. A network trained on the plain FP32 path: the first recall tick of every
   replicate matches the plain path bit for bit (it depends only on the
   trained state), epsc after it matches within the BF16 rounding of W, and
   the spike trains of sampled replicates stay close over the run.
"""
import numpy as np
import pytest

from gsbn_b200 import capi, recall, workloads
from oracle import sim

pytestmark = pytest.mark.gpu

f32 = np.float32


def bf16(x):
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16
    return (u.astype(np.uint32) << 16).view(np.float32)


class Pop:
    def __init__(self, H, M, taum=0.005, wtagain=1.0, maxfq=100.0, igain=1.0, wgain=1.0, lgbias=9.21, dt=0.001,
                 eps=1e-4, hz=20.0, kepsc=0.1, seed_base=7):
        self.H, self.M, self.N = H, M, H * M
        self.d = dict(hcu_num=H, mcu_num=M, taum=taum, wtagain=wtagain, maxfq=maxfq, igain=igain, wgain=wgain,
                      lgbias=lgbias, snoise=0.0)
        self.dt, self.eps, self.hz, self.kepsc, self.seed_base = dt, eps, hz, kepsc, seed_base

    def update(self, dsup_prev, epsc_prev, bj, lgidx, wmask, tick):
        """gsbn's population update (Pop.cpp:229-323) in float32, per replicate row"""
        H, M, N = self.H, self.M, self.N
        R = dsup_prev.shape[0]
        d = self.d
        hit = sim.extgen_logf(f32(1) + f32(self.eps))
        miss = sim.extgen_logf(f32(0) + f32(self.eps))
        m_idx = np.tile(np.arange(M), H)
        h_idx = np.repeat(np.arange(H), M)
        lginp = np.where(lgidx[:, h_idx] == m_idx[None, :], hit, miss).astype(f32)
        wsup = f32(0) + (bj[None, :] + epsc_prev)
        sup = (f32(d["lgbias"]) + f32(d["igain"]) * lginp) + f32(0)
        sup = sup + (f32(d["wgain"]) * wmask[:, h_idx]) * wsup
        taumdt = f32(self.dt) / f32(d["taum"])
        dn = (dsup_prev + (sup - dsup_prev) * taumdt).astype(f32)
        dh = dn.reshape(R, H, M)
        mx = np.maximum(dn[:, 0][:, None], dh.max(axis=2)).astype(f32)
        g = f32(d["wtagain"])
        maxact = sim.expf(g * mx)
        a = sim.expf(g * (dh - mx[:, :, None])).reshape(R, H, M)
        a = np.where(maxact[:, :, None] < 1, a * maxact[:, :, None], a).astype(f32)
        vsum = np.zeros((R, H), f32)
        for m in range(M):
            vsum = (vsum + a[:, :, m]).astype(f32)
        a = np.where(vsum[:, :, None] > 1, a / vsum[:, :, None], a).astype(f32)
        u = np.stack([sim.uniforms(self.seed_base + r, 0, tick, N) for r in range(R)]).reshape(R, H, M)
        spk = u < a * (f32(d["maxfq"]) * f32(self.dt))
        if self.hz > 0:
            up = np.stack([sim.uniforms_poisson(self.seed_base + r, 0, tick, N) for r in range(R)]).reshape(R, H, M)
            spk |= up < f32(self.hz) * f32(self.dt)
        return dn, spk.reshape(R, N).astype(np.int8)

    def engine(self, R, contraction="bf16"):
        return recall.Recall(self.H, self.M, R, self.d, self.dt, self.kepsc, self.seed_base, self.hz,
                             contraction=contraction)


def bits_equal(a, b):
    return np.array_equal(np.asarray(a, np.float32).view(np.uint32), np.asarray(b, np.float32).view(np.uint32))


@pytest.mark.parametrize("contraction", ["bf16", "fp32"])
@pytest.mark.parametrize("H,M,R", [(8, 32, 128), (16, 64, 256), (32, 16, 128)])
def test_synthetic_ticks(H, M, R, contraction):
    rng = np.random.default_rng(H * 1000 + M)
    pop = Pop(H, M)
    N = pop.N
    W = (rng.standard_normal((N, N)) * 0.5).astype(np.float32)
    bj = rng.standard_normal(N).astype(np.float32)
    epsc0 = rng.standard_normal(N).astype(np.float32)
    dsup0 = (rng.standard_normal(N) - 3).astype(np.float32)
    hist = [(rng.random(N) < 0.2).astype(np.int8) for _ in range(3)]  # t-3, t-2, t-1
    lgidx = rng.integers(-1, M, (R, H)).astype(np.int32)
    lgidx[rng.random((R, H)) < 0.3] = 0x7FFFFFFF
    wmask = (rng.random((R, H)) < 0.5).astype(np.float32)
    eng = pop.engine(R, contraction)
    eng.load_state(W, bj, epsc0, dsup0, *hist)
    eng.set_cues(lgidx, pop.eps, wmask)
    # the BF16 form multiplies W rounded once to BF16, the FP32 form W itself
    Wb = (bf16(W) if contraction == "bf16" else W).astype(np.float64)

    eng.timing(True)  # the contraction launches timed in place; results unchanged
    dsup = np.tile(dsup0, (R, 1))
    epsc = np.tile(epsc0, (R, 1))
    spikes = [np.tile(h, (R, 1)) for h in hist]
    first = 10
    counted = np.zeros((R, N), np.int64)
    for k in range(6):
        t = first + k
        eng.run(t, 1, first, first + 2)
        want_d, want_s = pop.update(dsup, epsc, bj, lgidx, wmask, t)
        got_d, got_s, got_e = eng.read("dsup"), eng.read("spike"), eng.read("epsc")
        assert bits_equal(got_d, want_d), f"dsup differs at tick {t}"
        assert np.array_equal(got_s, want_s), f"spikes differ at tick {t}"
        s_in = spikes[-3].astype(np.float64)
        want_e = epsc.astype(np.float64) * np.float64(f32(1) - f32(pop.kepsc)) + s_in @ Wb
        bound = 1e-5 * (np.abs(epsc).astype(np.float64) + s_in @ np.abs(Wb)) + 1e-6
        assert np.all(np.abs(got_e - want_e) <= bound), f"epsc differs at tick {t}: max {np.abs(got_e - want_e).max()}"
        if k < 3:
            counted += want_s
        dsup, epsc = got_d, got_e
        spikes.append(got_s)
    assert np.array_equal(eng.read("counts").astype(np.int64), counted)
    assert eng.launches() >= 6
    ms, n = eng.contraction_time()
    assert n == 6 and ms > 0
    # history rows written back are read back
    eng.write("spike_tm1", spikes[-1])
    assert np.array_equal(eng.read("spike_tm1"), spikes[-1])
    with pytest.raises(capi.BcpnnError):
        eng.read("nope")
    with pytest.raises(capi.BcpnnError):
        eng.run(100, 300, 0, 10000)  # more than 255 counted ticks


def test_rejects_bad_shapes():
    pop = Pop(8, 32)
    for H, M, R in [(8, 32, 100), (3, 32, 128), (8, 48, 128), (5, 64, 128)]:
        with pytest.raises(capi.BcpnnError):
            recall.Recall(H, M, R, dict(pop.d, hcu_num=H, mcu_num=M), 0.001, 0.1)


@pytest.mark.parametrize("contraction", ["bf16", "fp32"])
def test_trained_network_first_tick_exact(tmp_path, contraction):
    work = workloads.config4(hcu=16, mcu=16, n_patterns=6, train_ticks=60, rest_ticks=10, recall_ticks=60)
    tr = recall.Trained(work, str(tmp_path))
    names = ["pij_0", "eij_0", "zi2_0", "zj2_0", "tij_0", "wij_0", "pi_0", "ei_0", "zi_0", "ti_0", "pj_0", "ej_0",
             "zj_0", "qi_0", "ii_0", "di_0", "si_0", "dsup_0", "act_0", "epsc_0", "bj_0", "spike_0", ".counter_0",
             ".siq_0"]
    trained = tr.snapshot(names)
    W, st = tr.recall_inputs()
    R, seed_base = 128, 1000
    lg, wm, expected = tr.cues(R)
    eng = recall.Recall(tr.H, tr.M, R, tr.pops[0], tr.dt, recall.kepsc_of(tr.projs[0], tr.dt), seed_base,
                        tr.poisson_hz, contraction=contraction)
    eng.load_state(W, st["bj"], st["epsc"], st["dsup"], st["s_tm3"], st["s_tm2"], st["s_tm1"])
    eng.set_cues(lg, tr.eps, wm)
    # epsc after the first tick: within BF16 rounding of W (2^-9 relative per
    # weight) or within FP32 accumulation of the active rows
    tol = 2 ** -7 if contraction == "bf16" else 1e-5
    sample = [0, 1, 5, 77]
    plain = []
    for r in sample:
        net = capi.Net(tr.pops, tr.projs, tr.dt, seed=seed_base + r, poisson_hz=tr.poisson_hz, max_ticks=256)
        for n, a in trained.items():
            net.write(n, a)
        net.set_stimulus_idx(lg[r], tr.eps, wm[r])
        plain.append(net)
    T = 40
    agree, total = 0, 0
    for k in range(T):
        t = tr.t0 + k
        eng.run(t, 1, tr.t0, tr.t0 + T - 2)
        for i, r in enumerate(sample):
            plain[i].run(t, 1, 0.0, tr.old_prn if k == 0 else 0.0)
            pd, ps, pe = plain[i].read("dsup_0"), plain[i].read("spike_0"), plain[i].read("epsc_0")
            ed = eng.read("dsup", r, 1)[0]
            es = eng.read("spike", r, 1)[0]
            ee = eng.read("epsc", r, 1)[0]
            if k == 0:
                assert bits_equal(ed, pd), f"replicate {r}: first recall tick dsup differs"
                assert np.array_equal(es, ps), f"replicate {r}: first recall tick spikes differ"
                scale = np.abs(W).max() * 64 + np.abs(pe).max()
                assert np.abs(ee - pe).max() <= tol * scale, f"replicate {r}: epsc after tick 1"
            agree += int(np.sum((es != 0) & (ps != 0)))
            total += int(np.sum((es != 0) | (ps != 0)))
    assert total > 0
    assert agree / total > (0.8 if contraction == "bf16" else 0.95), f"spike agreement {agree}/{total}"
    counts = eng.read("counts")
    ok = recall.recall_decisions(counts, tr.H, tr.M, expected)
    assert ok.shape == (R,)
