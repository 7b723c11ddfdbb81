"""TEST INFRASTRUCTURE, NOT PART OF THE PRODUCT.

CPU restatement of gsbn's ProcUpdMulti (the row-only update that replays a
ring of postsynaptic spikes), in float32 scalar arithmetic, for networks of
config-0 size.  It follows the reference text operation by operation (paths
relative to the gsbn source tree):

  ProcUpdMulti::update_cpu   src/gsbn/procedures/ProcUpdMulti.cpp:94-125
  Pop::init_new              ProcUpdMulti/Pop.cpp:6-110 (dsup, act, ada, spike ring)
  update_sup_kernel_1..3     ProcUpdMulti/Pop.cpp:222-401
  Proj::init_new             ProcUpdMulti/Proj.cpp:6-108
  update_all_kernel_cpu      ProcUpdMulti/Proj.cpp:210-319, update_all_cpu 490-555
  update_jxx_kernel_cpu      ProcUpdMulti/Proj.cpp:321-362, update_jxx_cpu 557-583
  update_row_kernel_cpu      ProcUpdMulti/Proj.cpp:364-488, update_row_cpu 638-706
  update_que_cpu             ProcUpdMulti/Proj.cpp:620-636 (ssi: 585-594)
  ProcExchangeSpike          src/gsbn/procedures/ProcExchangeSpike.cpp:94-139

The uniform and normal draws are the project's Philox streams (the same as
the ProcUpdLazy oracle); exp and log are the shared bit-exact functions of
oracle/bcpnn_oracle.cpp (MATH_SHARED).  Parity against a gsbn binary is
unpinned (the reference cannot be built here).
"""
import ctypes

import numpy as np

from oracle import sim

f32 = np.float32


class MultiNet:
    """One network under ProcUpdMulti; the call shape of gsbn_b200.capi.Net."""

    def __init__(self, pops, projs, dt, seed=0, spike_buffer=1):
        lib = sim.load()
        lib.oracle_log_double.restype = ctypes.c_double
        lib.oracle_log_double.argtypes = [ctypes.c_int, ctypes.c_double]
        self._exp = lambda x: f32(lib.oracle_expf(sim.MATH_SHARED, float(f32(x))))
        self._log = lambda x: f32(lib.oracle_logf(sim.MATH_SHARED, float(f32(x))))
        self.dt, self.seed, self.B = f32(dt), seed, int(spike_buffer)
        self.pops, self.projs = [], []
        hcu = mcu = 0
        for p in pops:
            H, M = int(p["hcu_num"]), int(p["mcu_num"])
            n = H * M
            d = dict(H=H, M=M, n=n, hcu_start=hcu, mcu_start=mcu, dim_proj=0,
                     taumdt=f32(self.dt / f32(p["taum"])), wtagain=f32(p["wtagain"]),
                     maxfqdt=f32(f32(p["maxfq"]) * self.dt), igain=f32(p["igain"]), wgain=f32(p["wgain"]),
                     lgbias=f32(p["lgbias"]), snoise=f32(p["snoise"]),
                     tauadt=f32(self.dt / f32(p["taua"])), adgain=f32(p["adgain"]),
                     dsup=np.full(n, f32(lib.oracle_log_double(sim.MATH_SHARED, 1.0 / M)), f32), act=np.full(n, f32(1.0 / M), f32),
                     ada=np.zeros(n, f32), ring=np.zeros((self.B, n), np.int8), counter=np.zeros(n, np.int32),
                     spike=np.zeros(n, np.int8))
            self.pops.append(d)
            hcu += H
            mcu += n
        for q in projs:
            P, S = self.pops[q["dest_pop"]], self.pops[q["src_pop"]]
            C = min(S["n"], int(f32(q["slot_num"])))
            tauzi, tauzj, taue, taup = (f32(q[k]) for k in ("tauzi", "tauzj", "taue", "taup"))
            maxfq = f32(q["maxfq"])
            tauepsc = f32(q.get("tauepsc", 0.0))
            J = dict(src=q["src_pop"], dest=q["dest_pop"], H=P["H"], M=P["M"], C=C, proj_in_pop=P["dim_proj"],
                     kzi=f32(self.dt / tauzi), kzj=f32(self.dt / tauzj), ke=f32(self.dt / taue),
                     taupdt=f32(self.dt / taup), eps=f32(self.dt / taup),
                     eps2=f32(f32(self.dt / taup) * f32(self.dt / taup)),
                     kfti=f32(f32(1) / f32(maxfq * tauzi)), kftj=f32(f32(1) / f32(maxfq * tauzj)),
                     bgain=f32(q["bgain"]), wgain=f32(q["wgain"]),
                     kepsc=f32(self.dt / tauepsc) if tauepsc > 0 else f32(self.dt / tauzi))
            R = P["H"] * C
            J.update(ii=np.full(R, -1, np.int32), di=np.zeros(R, np.int32), qi=np.zeros(R, np.int32),
                     siq=np.zeros(R, np.int8), pi=np.full(R, f32(1.0 / C), f32), ei=np.zeros(R, f32),
                     zi=np.zeros(R, f32), ti=np.zeros(R, np.int32), pj=np.full(P["n"], f32(1.0 / P["M"]), f32),
                     ej=np.zeros(P["n"], f32), zj=np.zeros(P["n"], f32),
                     pij=np.full(R * P["M"], f32(1.0 / C / P["M"]), f32), eij=np.zeros(R * P["M"], f32),
                     zj2=np.zeros(R * P["M"], f32), wij=np.zeros(R * P["M"], f32), si=np.zeros(S["n"], np.int8))
            P["dim_proj"] += 1
            self.projs.append(J)
        for P in self.pops:
            P["epsc"] = np.zeros(max(1, P["dim_proj"]) * P["n"], f32)
            P["bj"] = np.zeros(max(1, P["dim_proj"]) * P["n"], f32)
        self.lginp = None
        self.wmask = None

    def set_conn(self, proj, ii, di):
        J = self.projs[proj]
        J["ii"][:] = np.asarray(ii, np.int32)
        J["di"][:] = np.asarray(di, np.int32)

    def set_stimulus(self, lginp, wmask_row):
        self.lginp = np.asarray(lginp, f32)
        self.wmask = np.asarray(wmask_row, f32)

    # ---- population, ProcUpdMulti/Pop.cpp:222-401 -------------------------
    def _pop(self, k, P, t):
        H, M, n = P["H"], P["M"], P["n"]
        normal = sim.normals(self.seed, k, t, n) if P["snoise"] != 0 else None
        uni = sim.uniforms(self.seed, k, t, n)
        spk = np.zeros(n, np.int8)
        for i in range(H):
            wm = self.wmask[P["hcu_start"] + i]
            for j in range(M):
                idx = i * M + j
                wsup = f32(0)
                off = 0
                for _ in range(P["dim_proj"]):
                    wsup = f32(wsup + f32(P["bj"][off + idx] + P["epsc"][off + idx]))
                    off += n
                noise = f32(P["snoise"] * normal[idx]) if normal is not None else f32(0)
                sup = f32(f32(P["lgbias"] + f32(P["igain"] * self.lginp[P["mcu_start"] + idx])) + noise)
                sup = f32(sup + f32(f32(P["wgain"] * wm) * wsup))
                sup = f32(sup - f32(wm * P["ada"][idx]))
                sup = f32(float(sup) + 6.9 * float(wm))
                d = P["dsup"][idx]
                P["dsup"][idx] = f32(d + f32(f32(sup - d) * P["taumdt"]))
            base = i * M
            mx = P["dsup"][base]
            for m in range(M):
                if P["dsup"][base + m] > mx:
                    mx = P["dsup"][base + m]
            maxact = self._exp(f32(P["wtagain"] * mx))
            vsum = f32(0)
            for m in range(M):
                a = self._exp(f32(P["wtagain"] * f32(P["dsup"][base + m] - mx)))
                if maxact < 1:
                    a = f32(a * maxact)
                vsum = f32(vsum + a)
                P["act"][base + m] = a
            if vsum > 1:
                for m in range(M):
                    P["act"][base + m] = f32(P["act"][base + m] / vsum)
            for j in range(M):
                idx = base + j
                s = np.int8(uni[idx] < f32(P["act"][idx] * P["maxfqdt"]))
                spk[idx] = s
                P["counter"][idx] += int(s)
                P["ada"][idx] = f32(P["ada"][idx] + f32(f32(f32(P["adgain"] * P["act"][idx]) - P["ada"][idx]) * P["tauadt"]))
        P["ring"][t % self.B] = spk
        P["spike"][:] = spk

    # ---- closed forms, ProcUpdMulti/Proj.cpp:244-251, 268-275 ------------
    def _row_traces(self, pi, ei, zi, pdt, kp, ke, kzi):
        E, fd = self._exp, f32(pdt)
        a = f32(kp * fd)
        x = f32(f32(f32(f32(ei * kp) * kzi) - f32(f32(ei * ke) * kp)) + f32(f32(ke * kp) * zi))
        t1 = f32(x / f32(ke - kp))
        t2 = f32(f32(f32(ke * kp) * zi) / f32(kp - kzi))
        pn = f32(f32(pi - f32(f32(t1 + t2) / f32(ke - kzi))) / E(a))
        u1 = f32(f32(E(f32(a - f32(ke * fd))) * x) / f32(ke - kp))
        u2 = f32(f32(f32(f32(ke * kp) * zi) * E(f32(a - f32(kzi * fd)))) / f32(kp - kzi))
        pn = f32(pn + f32(f32(u1 + u2) / f32(E(a) * f32(ke - kzi))))
        b = f32(ke * fd)
        en = f32(f32(f32(ei - f32(f32(ke * zi) / f32(ke - kzi))) / E(b)) +
                 f32(f32(f32(ke * zi) * E(f32(b - f32(kzi * fd)))) / f32(E(b) * f32(ke - kzi))))
        return pn, en

    def _cell(self, pij, eij, zi2, zj2, pdt, kp, ke, kzi, kzj):
        E, fd = self._exp, f32(pdt)
        a = f32(kp * fd)
        zz = f32(f32(f32(ke * kp) * zi2) * zj2)
        x = f32(f32(f32(f32(f32(eij * kp) * kzi) - f32(f32(eij * ke) * kp)) + f32(f32(eij * kp) * kzj)) + zz)
        d2 = f32(f32(kzi - kp) + kzj)
        d3 = f32(f32(kzi - ke) + kzj)
        pn = f32(f32(pij + f32(f32(f32(x / f32(ke - kp)) - f32(zz / d2)) / d3)) / E(a))
        v1 = f32(f32(E(f32(a - f32(ke * fd))) * x) / f32(ke - kp))
        v2 = f32(f32(zz * E(f32(f32(a - f32(kzi * fd)) - f32(kzj * fd)))) / d2)
        pn = f32(pn - f32(f32(v1 - v2) / f32(E(a) * d3)))
        w = f32(f32(ke * zi2) * zj2)
        en = f32(f32(f32(eij + f32(w / d3)) / E(f32(ke * fd))) -
                 f32(w / f32(f32(E(f32(kzi * fd)) * E(f32(kzj * fd))) * d3)))
        return pn, en

    def _replay(self, J, P, row, j, tij, zi2, simstep, kp, exclusive):
        """the cell loop of update_row/update_all_kernel_cpu; returns (pij, eij, zj2, tij)"""
        idx = row * J["M"] + j
        pij, eij, zj2 = J["pij"][idx], J["eij"][idx], J["zj2"][idx]
        mcu = (row // J["C"]) * J["M"] + j
        now = tij
        if simstep - now >= self.B:
            now = simstep - self.B + 1
        while now < simstep:
            now += 1
            if P["ring"][now % self.B][mcu] > 0 and (not exclusive or now < simstep):
                pdt = now - tij
                if pdt > 0:
                    pij, eij = self._cell(pij, eij, zi2, zj2, pdt, kp, J["ke"], J["kzi"], J["kzj"])
                    zi2 = f32(zi2 * self._exp(f32(-J["kzi"] * f32(pdt))))
                    zj2 = f32(f32(zj2 * self._exp(f32(-J["kzj"] * f32(pdt)))) + J["kftj"])
                    tij = now
        return pij, eij, zi2, zj2, tij

    # ---- projections --------------------------------------------------------
    def _all(self, J, simstep, old_prn):
        """update_all_cpu with simstep-1 (Proj.cpp:490-555)"""
        P = self.pops[J["dest"]]
        t = simstep - 1
        kp = f32(J["taupdt"] * f32(old_prn))
        for i in range(J["H"] * J["C"]):
            ti, zi = int(J["ti"][i]), J["zi"][i]
            pdt = t - ti
            if pdt > 0:
                J["pi"][i], J["ei"][i] = self._row_traces(J["pi"][i], J["ei"][i], zi, pdt, kp, J["ke"], J["kzi"])
            for j in range(J["M"]):
                pij, eij, zi2, zj2, tij = self._replay(J, P, i, j, ti, zi, t, kp, False)
                pdt2 = t - tij
                if pdt2 > 0:
                    pij, eij = self._cell(pij, eij, zi2, zj2, pdt2, kp, J["ke"], J["kzi"], J["kzj"])
                    zj2 = f32(zj2 * self._exp(f32(-J["kzj"] * f32(pdt2))))
                idx = i * J["M"] + j
                J["pij"][idx], J["eij"][idx], J["zj2"][idx] = pij, eij, zj2
                if kp != 0:
                    pj = J["pj"][(i // J["C"]) * J["M"] + j]
                    J["wij"][idx] = f32(J["wgain"] * self._log(f32(f32(pij + J["eps2"]) /
                                                                   f32(f32(J["pi"][i] + J["eps"]) * f32(pj + J["eps"])))))
            if pdt > 0:
                J["zi"][i] = f32(zi * self._exp(f32(-J["kzi"] * f32(pdt))))
            J["ti"][i] = t

    def _proj(self, J, simstep, prn):
        P = self.pops[J["dest"]]
        M, C, n = J["M"], J["C"], P["n"]
        kp = f32(J["taupdt"] * f32(prn))
        eoff = J["proj_in_pop"] * n
        sj = P["ring"][simstep % self.B]
        # update_jxx (Proj.cpp:321-362)
        for idx in range(n):
            P["epsc"][eoff + idx] = f32(P["epsc"][eoff + idx] * f32(f32(1) - J["kepsc"]))
            pj, ej, zj = J["pj"][idx], J["ej"][idx], J["zj"][idx]
            pj = f32(pj + f32(f32(ej - pj) * kp))
            ej = f32(ej + f32(f32(zj - ej) * J["ke"]))
            zj = f32(zj * f32(f32(1) - J["kzj"]))
            if sj[idx] > 0:
                zj = f32(zj + J["kftj"])
            if kp != 0:
                P["bj"][eoff + idx] = f32(J["bgain"] * self._log(f32(pj + J["eps"])))
            J["pj"][idx], J["ej"][idx], J["zj"][idx] = pj, ej, zj
        # update_ssi + update_row (Proj.cpp:585-594, 638-706)
        ssi = [r for r in range(J["H"] * C) if J["siq"][r] > 0]
        for row in ssi:
            ti, zi = int(J["ti"][row]), J["zi"][row]
            pdt = simstep - ti
            if pdt > 0:
                J["pi"][row], J["ei"][row] = self._row_traces(J["pi"][row], J["ei"][row], zi, pdt, kp, J["ke"],
                                                              J["kzi"])
            h = row // C
            for j in range(M):
                pij, eij, zi2, zj2, tij = self._replay(J, P, row, j, ti, zi, simstep, kp, True)
                pdt2 = simstep - tij
                pij, eij = self._cell(pij, eij, zi2, zj2, pdt2, kp, J["ke"], J["kzi"], J["kzj"])
                zj2 = f32(zj2 * self._exp(f32(-J["kzj"] * f32(pdt2))))
                if sj[h * M + j] > 0:
                    zj2 = f32(zj2 + J["kftj"])
                idx = row * M + j
                J["pij"][idx], J["eij"][idx], J["zj2"][idx] = pij, eij, zj2
                if kp != 0:
                    pj = J["pj"][h * M + j]
                    w = f32(J["wgain"] * self._log(f32(f32(pij + J["eps2"]) /
                                                       f32(f32(J["pi"][row] + J["eps"]) * f32(pj + J["eps"])))))
                    J["wij"][idx] = w
                else:
                    w = J["wij"][idx]
                P["epsc"][eoff + h * M + j] = f32(P["epsc"][eoff + h * M + j] + w)
            if pdt > 0:
                J["zi"][row] = f32(f32(zi * self._exp(f32(-J["kzi"] * f32(pdt)))) + J["kfti"])
            J["ti"][row] = simstep
        # update_que (Proj.cpp:620-636)
        for r in range(J["H"] * C):
            if J["ii"][r] < 0:
                continue
            J["siq"][r] = J["qi"][r] & 1
            J["qi"][r] >>= 1
            if J["si"][J["ii"][r]] > 0:
                J["qi"][r] |= 1 << (int(J["di"][r]) - 1)
        return len(ssi)

    def run(self, first, n, prn, old_prn):
        """ticks first .. first+n-1; returns the spike log [n, words] of every population"""
        logs = [np.zeros((n, (P["n"] + 31) // 32), np.uint32) for P in self.pops]
        with np.errstate(over="ignore", invalid="ignore", divide="ignore", under="ignore"):
            self._run(first, n, prn, old_prn, logs)
        return logs

    def _run(self, first, n, prn, old_prn, logs):
        for k in range(n):
            t = first + k
            for q, P in enumerate(self.pops):
                self._pop(q, P, t)
                for i in np.nonzero(P["spike"])[0]:
                    logs[q][k, i >> 5] |= np.uint32(1 << (int(i) & 31))
            for J in self.projs:
                if k == 0 and prn != old_prn:
                    self._all(J, t, old_prn)
                self._proj(J, t, prn)
            for J in self.projs:
                J["si"][:] = self.pops[J["src"]]["spike"]

    def read(self, name):
        base, _, num = name.rpartition("_")
        k = int(num)
        if base in ("dsup", "act", "ada", "spike", "epsc", "bj"):
            return self.pops[k][base].copy()
        if base == ".counter":
            return self.pops[k]["counter"].copy()
        return self.projs[k][base].copy()


POP_KEYS = ("taum", "wtagain", "maxfq", "igain", "wgain", "lgbias", "snoise", "taua", "adgain")


def _declare(lib):
    vp, i32, u32, fl, sz = ctypes.c_void_p, ctypes.c_int, ctypes.c_uint32, ctypes.c_float, ctypes.c_size_t
    lib.oracle_multi_create.restype = vp
    lib.oracle_multi_create.argtypes = [fl, u32, i32, i32, vp, vp, i32, vp, vp]
    lib.oracle_multi_destroy.argtypes = [vp]
    lib.oracle_multi_set_stimulus.argtypes = [vp, vp, vp]
    lib.oracle_multi_run.argtypes = [vp, i32, i32, fl, fl, vp]
    lib.oracle_multi_state_info.restype = ctypes.c_longlong
    lib.oracle_multi_state_info.argtypes = [vp, ctypes.c_char_p, ctypes.POINTER(i32)]
    lib.oracle_multi_read_state.argtypes = [vp, ctypes.c_char_p, vp, sz]
    lib.oracle_multi_write_state.argtypes = [vp, ctypes.c_char_p, vp, sz]
    lib.oracle_multi_counters.argtypes = [vp, ctypes.POINTER(ctypes.c_ulonglong)]
    return lib


class MultiNetC:
    """The same restatement compiled (oracle/bcpnn_oracle_multi.cpp), for
    networks beyond 10x10; the call shape of MultiNet, plus write() and
    counters() (active-row cells, 0 column cells, all-cells sweeps)."""

    def __init__(self, pops, projs, dt, seed=0, spike_buffer=1):
        self.lib = _declare(sim.load())
        dims = np.array([[p["hcu_num"], p["mcu_num"]] for p in pops], np.int32).reshape(-1)
        pf = np.array([[p.get(k, 0.0) for k in POP_KEYS] for p in pops], np.float32).reshape(-1)
        pi = np.array([[q["src_pop"], q["dest_pop"]] for q in projs] or [[0, 0]], np.int32).reshape(-1)
        qf = np.array([[q.get(k, 0.0) for k in sim.PROJ_KEYS] for q in projs] or [[0.0] * 9], np.float32).reshape(-1)
        self.h = self.lib.oracle_multi_create(float(f32(dt)), seed, int(spike_buffer), len(pops), sim._p(dims),
                                              sim._p(pf), len(projs), sim._p(pi), sim._p(qf))
        if not self.h:
            raise ValueError("oracle_multi_create refused the description")
        self.sizes = [int(p["hcu_num"]) * int(p["mcu_num"]) for p in pops]

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.oracle_multi_destroy(self.h)
            self.h = None

    def _vec(self, name):
        kind = ctypes.c_int()
        n = self.lib.oracle_multi_state_info(self.h, name.encode(), ctypes.byref(kind))
        if n < 0:
            raise KeyError(name)
        return n, {0: np.float32, 1: np.int32, 2: np.int8}[kind.value]

    def read(self, name):
        n, dt = self._vec(name)
        out = np.zeros(n, dt)
        assert self.lib.oracle_multi_read_state(self.h, name.encode(), sim._p(out), out.nbytes) == 0
        return out

    def write(self, name, arr):
        n, dt = self._vec(name)
        a = np.ascontiguousarray(arr, dtype=dt)
        assert a.size == n
        assert self.lib.oracle_multi_write_state(self.h, name.encode(), sim._p(a), a.nbytes) == 0

    def set_conn(self, proj, ii, di):
        self.write(f"ii_{proj}", ii)
        self.write(f"di_{proj}", di)

    def set_stimulus(self, lginp, wmask_row):
        self._lg = np.ascontiguousarray(lginp, np.float32)
        self._wm = np.ascontiguousarray(wmask_row, np.float32)
        self.lib.oracle_multi_set_stimulus(self.h, sim._p(self._lg), sim._p(self._wm))

    def run(self, first, n, prn, old_prn, spikes=True):
        """ticks first .. first+n-1; the spike log [n, words] of every
        population (None without `spikes`)"""
        words = [(s + 31) // 32 for s in self.sizes]
        buf = np.zeros(n * sum(words), np.uint32) if spikes else None
        rc = self.lib.oracle_multi_run(self.h, first, n, prn, old_prn, sim._p(buf) if spikes else None)
        assert rc == 0, rc
        if not spikes:
            return None
        out, off = [], 0
        for w in words:
            out.append(buf[off:off + n * w].reshape(n, w).copy())
            off += n * w
        return out

    def counters(self):
        c = (ctypes.c_ulonglong * 2)()
        self.lib.oracle_multi_counters(self.h, c)
        return [int(c[0]), 0, int(c[1])]
