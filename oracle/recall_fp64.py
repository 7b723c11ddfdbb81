"""FP64 restatement of the recall phase (prn = 0) of one trained population
with a full recurrent projection, for many noise replicates at once.

Test infrastructure: the tests use it, and bench.py uses it as the checker
of its fp64_error figures, outside every timed region.  Nothing in the
library calls it.

It restates OracleNet(real_bits=64) -- the oracle's ProcUpdLazy in double --
for the part of a recall tick that reaches the spikes.  With kp = 0 the
weights w_ij and biases b_j keep the values the prn-change catch-up of the
first recall tick gave them (Proj.cpp:289 recomputes w_ij there; the row and
j-trace updates rewrite them only when kp != 0, Proj.cpp:352-356, 445-451),
so the P/E/Z traces are not carried.  Per tick t, per replicate, in double:

  population update, Pop.cpp:229-323 (the oracle's sup_kernel_1..3):
    wsup = 0 + (bj + epsc);  sup = lgbias + igain*lginp + noise;
    sup += (wgain*wmask)*wsup;  dsup += (sup - dsup)*taumdt;
    softmax/WTA with the running max seeded by dsup of population MCU 0
    (Pop.cpp:270); spike = u < act*maxfqdt with the FP32 Philox uniform u,
    OR the project-defined Poisson input noise (FP32 uniform < FP32 rate);
  projection, Proj.cpp:310-363 then :445-451:
    epsc *= (1 - kepsc); epsc += w_ij for every slot whose source spiked at
    t-3 (delay 1: the exchange after t-3, the queue bit set at t-2 and read
    out at t-1, ProcExchangeSpike.cpp:94-139, Proj.cpp:621-664), added in
    slot order.

catchup_weights() takes W and b_j from the oracle itself: one FP64 oracle
tick from the trained state.  tests/test_recall_fp64.py pins the
restatement against OracleNet(real_bits=64) tick by tick (identical spike
trains, dsup to the last bits).
"""
import numpy as np

from . import sim


def _f64(x):
    """a float32 parameter as the double the oracle holds ((T)float)"""
    return float(np.float32(x))


def catchup_weights(pops, projs, dt, poisson_hz, trained, t0, old_prn, lginp, wmask_row):
    """W[source, destination] and b_j (float64) as the FP64 oracle's first
    recall tick leaves them, with b_j before that tick; also the slot order
    of every destination HCU (pos[h, i] = slot of source i)."""
    H, M = pops[0]["hcu_num"], pops[0]["mcu_num"]
    N = H * M
    orc = sim.OracleNet(pops, projs, dt, seed=0, poisson_hz=poisson_hz, real_bits=64)
    for n, a in trained.items():
        orc.write(n, a)
    bj0 = orc.read("bj_0").copy()
    orc.set_stimulus(lginp, wmask_row)
    orc.update(t0, 0.0, old_prn)
    ii = orc.read("ii_0").reshape(H, -1)
    if ii.shape[1] != N or np.any(np.sort(ii, axis=1) != np.arange(N)[None, :]):
        raise ValueError("the recall restatement needs one slot per source MCU in every destination HCU")
    if np.any(orc.read("di_0") != 1):
        raise ValueError("the recall restatement needs delay 1 on every slot")
    wij = orc.read("wij_0").reshape(H, N, M)
    W = np.empty((N, N), np.float64)
    pos = np.empty((H, N), np.int64)
    for h in range(H):
        W[ii[h], h * M:(h + 1) * M] = wij[h]
        pos[h, ii[h]] = np.arange(N)
    bj1 = orc.read("bj_0").copy()
    del orc
    return W, bj0, bj1, pos


def lginp_rows(lg, H, M, eps):
    """ProcExtGen's lginp (float log(1+eps) on the indexed MCU, log(eps)
    elsewhere) for rows of per-HCU MCU indices"""
    hit = sim.extgen_logf(np.float32(1) + np.float32(eps))
    miss = sim.extgen_logf(np.float32(0) + np.float32(eps))
    lg = np.asarray(lg).reshape(-1, H)
    m = np.tile(np.arange(M), H)
    return np.where(lg[:, np.repeat(np.arange(H), M)] == m[None, :], hit, miss).astype(np.float32)


class RecallFP64:
    """K replicates (seeds seed_base + r for r in `reps`) from one trained
    state; step() runs one tick of all of them."""

    def __init__(self, pop, dt, kepsc_tau, poisson_hz, W, bj0, bj1, pos, epsc0, dsup0, s_hist, lg, wm, eps,
                 seed_base, reps):
        self.H, self.M = pop["hcu_num"], pop["mcu_num"]
        H, M = self.H, self.M
        self.N = N = H * M
        self.W, self.bj0, self.bj1 = W, np.asarray(bj0, np.float64), np.asarray(bj1, np.float64)
        dt64 = _f64(dt)
        self.taumdt = dt64 / _f64(pop["taum"])
        self.maxfqdt = _f64(pop["maxfq"]) * dt64
        self.wtagain, self.igain = _f64(pop["wtagain"]), _f64(pop["igain"])
        self.wgain, self.lgbias, self.snoise = _f64(pop["wgain"]), _f64(pop["lgbias"]), _f64(pop["snoise"])
        # the projection's epsc rate in double: dt / tauepsc, else dt / tauzi (Proj.cpp:6-107)
        self.one_m_kepsc = 1.0 - dt64 / _f64(kepsc_tau)
        self.pr = np.float32(np.float32(poisson_hz) * np.float32(dt))
        self.poisson = poisson_hz > 0
        self.seeds = [seed_base + r for r in reps]
        K = len(reps)
        self.lginp = lginp_rows(np.asarray(lg)[list(reps)], H, M, eps).astype(np.float64)
        self.wmask = np.asarray(wm, np.float32)[list(reps)].astype(np.float64)[:, np.repeat(np.arange(H), M)]
        self.dsup = np.tile(np.asarray(dsup0, np.float32).astype(np.float64), (K, 1))
        self.epsc = np.tile(np.asarray(epsc0, np.float32).astype(np.float64), (K, 1))
        self.hist = [np.tile(np.asarray(s, np.int8) != 0, (K, 1)) for s in s_hist]  # t-3, t-2, t-1
        same = bool(np.all(pos == pos[0][None, :]))
        self.order = np.argsort(pos[0]) if same else None
        self.pos = pos
        self.ticks = 0

    def _rows(self, k, active):
        """epsc[k] += w_ij of the active sources, slot order in every HCU"""
        if self.order is not None:
            src = self.order[active[self.order]]
            e = self.epsc[k]
            for i in src:
                e += self.W[i]
            return
        M = self.M
        for h in range(self.H):
            src = np.nonzero(active)[0]
            src = src[np.argsort(self.pos[h, src])]
            e = self.epsc[k, h * M:(h + 1) * M]
            for i in src:
                e += self.W[i, h * M:(h + 1) * M]

    def step(self, simstep):
        H, M, N = self.H, self.M, self.N
        K = len(self.seeds)
        bj = self.bj0 if self.ticks == 0 else self.bj1
        wsup = 0.0 + (bj[None, :] + self.epsc)
        if self.snoise != 0:
            noise = self.snoise * np.stack([sim.normals(s, 0, simstep, N) for s in self.seeds]).astype(np.float64)
        else:
            noise = 0.0
        sup = self.lgbias + self.igain * self.lginp + noise
        sup = sup + (self.wgain * self.wmask) * wsup
        self.dsup = self.dsup + (sup - self.dsup) * self.taumdt
        dh = self.dsup.reshape(K, H, M)
        mx = np.maximum(self.dsup[:, 0][:, None], dh.max(axis=2))
        maxact = np.exp(self.wtagain * mx)
        a = np.exp(self.wtagain * (dh - mx[:, :, None]))
        a = np.where((maxact < 1)[:, :, None], a * maxact[:, :, None], a)
        vsum = np.zeros((K, H))
        for m in range(M):
            vsum = vsum + a[:, :, m]
        a = np.where((vsum > 1)[:, :, None], a / vsum[:, :, None], a).reshape(K, N)
        u = np.stack([sim.uniforms(s, 0, simstep, N) for s in self.seeds]).astype(np.float64)
        spk = u < a * self.maxfqdt
        if self.poisson:
            up = np.stack([sim.uniforms_poisson(s, 0, simstep, N) for s in self.seeds])
            spk |= up < self.pr
        self.epsc = self.epsc * self.one_m_kepsc
        active = self.hist[0]
        for k in range(K):
            if active[k].any():
                self._rows(k, active[k])
        self.hist = self.hist[1:] + [spk]
        self.ticks += 1
        return self.dsup.copy(), spk.astype(np.int8)


def kepsc_tau(proj):
    """the time constant behind the projection's epsc rate"""
    return proj["tauepsc"] if proj.get("tauepsc", 0.0) and proj["tauepsc"] > 0 else proj["tauzi"]


def error_metrics(d, s, d64, s64):
    """Per replicate: support error max|dsup - dsup64| / max|dsup64| over the
    ticks before the spike trains first differ, the first tick where they
    differ (len(d) = never), and the spike Jaccard over the run."""
    T = len(d)
    div = next((k for k in range(T) if not np.array_equal(s[k], s64[k])), T)
    upto = max(div, 1)
    scale = max(float(np.abs(np.asarray(d64[:upto])).max()), 1e-30)
    err = max(float(np.abs(np.asarray(d[k], np.float64) - d64[k]).max()) for k in range(upto))
    both = sum(int(np.sum((s[k] != 0) & (s64[k] != 0))) for k in range(T))
    either = sum(int(np.sum((s[k] != 0) | (s64[k] != 0))) for k in range(T))
    return dict(support_rel_err=err / scale, first_divergence_tick=div, spike_jaccard=both / max(either, 1))
