"""The FP64 recall restatement (oracle/recall_fp64.py) against the oracle in
double, on the CPU.

A 16x16 network with a full recurrent projection is trained on the float
oracle (4 patterns, 60 ticks each with 10-tick rests, 20 Hz Poisson input
noise).  From its end-of-training state, replicates recall with their own
Philox keys and cues: once through OracleNet(real_bits=64) -- the whole
ProcUpdLazy in double, every trace carried -- and once through the
restatement.  The spike trains must be identical tick by tick and dsup equal
to a few ulps of double; the restatement's ProcCheck decisions are then the
FP64 oracle's.
"""
import numpy as np
import pytest

from gsbn_b200 import extgen, recall, schema, workloads
from oracle import recall_fp64, sim

STATE = ("pij_0", "eij_0", "zi2_0", "zj2_0", "tij_0", "wij_0", "pi_0", "ei_0", "zi_0", "ti_0", "pj_0", "ej_0",
         "zj_0", "qi_0", "ii_0", "di_0", "si_0", ".siq_0", "dsup_0", "act_0", "epsc_0", "bj_0", "spike_0",
         ".counter_0")


class OracleTrained:
    """recall.Trained on the float oracle: a network trained up to its first
    recall segment (tick t0)"""

    def __init__(self, work, directory):
        with open(work.write(directory)) as f:
            sp = schema.parse_prototxt(f.read())
        self.pops, self.projs = workloads.net_from_solver_param(sp)
        upd = [p for p in sp.proc_param if p.name == "ProcUpdLazy"][0]
        seed = {a.key: a.val for a in upd.argi}.get("seed", 0)
        self.poisson_hz = float({a.key: a.val for a in upd.argf}.get("poisson-noise-hz", 0.0))
        self.dt = float(np.float32(sp.gen_param.dt))
        self.eps = float(np.float32(sp.gen_param.eps))
        self.H, self.M = self.pops[0]["hcu_num"], self.pops[0]["mcu_num"]
        self.net = sim.OracleNet(self.pops, self.projs, self.dt, seed=seed, poisson_hz=self.poisson_hz)
        conn = [p for p in sp.proc_param if p.name == "ProcInitConn"][0]
        with open({a.key: a.val for a in conn.args}["conn-map-file"]) as f:
            for k, (ii, di) in enumerate(workloads.read_conn_map(f.read(), self.pops, self.projs)):
                self.net.set_conn(k, ii, di)
        self.lgidx, self.wmask = extgen.stim_tables(schema.read_stim(sp.gen_param.stim_file))
        runs = extgen.segments(sp)
        k = next(i for i, r in enumerate(runs) if r.prn == 0.0)
        for r in runs[:k]:
            self.net.set_stimulus(recall_fp64.lginp_rows(self.lgidx[r.lgidx], self.H, self.M, self.eps)[0],
                                  self.wmask[r.wmask][:self.H])
            self.net.run(r.first, r.n, r.prn, r.old_prn, spikes=False)
        self.t0, self.old_prn = runs[k].first, runs[k].old_prn
        self.n_patterns = work.meta["patterns"]


@pytest.fixture(scope="module")
def trained(tmp_path_factory):
    work = workloads.config4(hcu=16, mcu=16, n_patterns=4, train_ticks=60, rest_ticks=10, recall_ticks=40)
    return OracleTrained(work, str(tmp_path_factory.mktemp("recall_fp64")))


def test_restatement_matches_the_fp64_oracle(trained):
    tr = trained
    H, M, N = tr.H, tr.M, tr.H * tr.M
    state = {n: tr.net.read(n) for n in STATE}
    st = recall.end_of_training_state(tr.net, H, M)
    P = tr.n_patterns
    reps, seed_base, T = [0, 1, 2, 5], 11, 40
    lg = np.stack([tr.lgidx[P + (r % P)] for r in range(max(reps) + 1)]).astype(np.int32)
    wm = np.stack([tr.wmask[1][:H]] * (max(reps) + 1)).astype(np.float32)
    lginp = recall_fp64.lginp_rows(lg, H, M, tr.eps)
    W, bj0, bj1, pos = recall_fp64.catchup_weights(tr.pops, tr.projs, tr.dt, tr.poisson_hz, state, tr.t0,
                                                   tr.old_prn, lginp[0], wm[0])
    rs = recall_fp64.RecallFP64(tr.pops[0], tr.dt, recall_fp64.kepsc_tau(tr.projs[0]), tr.poisson_hz, W, bj0, bj1,
                                pos, st["epsc"], st["dsup"], (st["s_tm3"], st["s_tm2"], st["s_tm1"]), lg, wm, tr.eps,
                                seed_base, reps)
    got = [rs.step(tr.t0 + k) for k in range(T)]
    spikes = 0
    for i, r in enumerate(reps):
        orc = sim.OracleNet(tr.pops, tr.projs, tr.dt, seed=seed_base + r, poisson_hz=tr.poisson_hz, real_bits=64)
        for n, a in state.items():
            orc.write(n, a)
        orc.set_stimulus(lginp[r], wm[r])
        for k in range(T):
            orc.update(tr.t0 + k, 0.0, tr.old_prn if k == 0 else 0.0)
            orc.exchange()
            d64, s64 = orc.read("dsup_0"), orc.read("spike_0")
            assert np.array_equal(got[k][1][i], s64), f"replicate {r}: spikes differ at tick {k}"
            err = np.abs(got[k][0][i] - d64).max() / np.abs(d64).max()
            assert err < 1e-13, f"replicate {r}: dsup at tick {k}, relative {err}"
            spikes += int(s64.sum())
        del orc
    assert spikes > 50


def test_error_metrics():
    d64 = [np.array([1.0, -2.0]), np.array([1.5, -2.5]), np.array([1.0, 0.0])]
    s64 = [np.array([1, 0]), np.array([0, 1]), np.array([1, 1])]
    d = [np.array([1.0, -2.0], np.float32), np.array([1.5, -2.4], np.float32), np.array([9.0, 9.0], np.float32)]
    s = [np.array([1, 0]), np.array([0, 1]), np.array([1, 0])]
    m = recall_fp64.error_metrics(d, s, d64, s64)
    assert m["first_divergence_tick"] == 2
    assert abs(m["support_rel_err"] - np.float64(np.float32(2.4) - 2.5).__abs__() / 2.5) < 1e-7
    assert m["spike_jaccard"] == 3 / 4


def test_rows_follow_each_hcus_slot_order():
    """epsc += w over the active sources in the slot order of every
    destination HCU, also when the HCUs order their slots differently"""
    rng = np.random.default_rng(3)
    H, M = 3, 4
    N = H * M
    # magnitudes spread over 16 decades across rows: the sums depend on the order
    W = rng.standard_normal((N, N)) * (10.0 ** rng.uniform(-8, 8, N))[:, None]
    pos = np.stack([rng.permutation(N) for _ in range(H)])
    pop = dict(hcu_num=H, mcu_num=M, taum=0.005, wtagain=1.0, maxfq=100.0, igain=1.0, wgain=1.0, lgbias=0.0,
               snoise=0.0)
    z = np.zeros(N, np.float32)
    rs = recall_fp64.RecallFP64(pop, 0.001, 0.005, 0.0, W, z, z, pos, z, z, (z, z, z),
                                np.zeros((1, H), np.int32), np.ones((1, H), np.float32), 1e-4, 0, [0])
    active = rng.random(N) < 0.6
    rs._rows(0, active)
    for h in range(H):
        src = [i for i in np.argsort(pos[h]) if active[i]]  # slot order of HCU h
        for m in range(M):
            want = 0.0
            for i in src:
                want += W[i, h * M + m]
            assert rs.epsc[0, h * M + m] == want
