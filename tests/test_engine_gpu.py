"""The host engine end to end on the GPU: prototxt network descriptions run
through the procedure registry (ProcExtGen, ProcUpdLazy, ProcExchangeSpike,
ProcInitConn, ProcSpkRec, ProcCheck, ProcSnapshot) must write the same record
files, byte for byte, as the CPU oracle's restatement of gsbn's procedures,
whether ticks run one device launch per stimulus segment or one per tick.
"""
import os
import subprocess

import numpy as np
import pytest

from gsbn_b200 import engine, schema, workloads
from oracle import sim

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GSBN_SIM = os.path.join(os.path.dirname(HERE), "gsbn_b200", "gsbn_sim")


def write(w, directory, edit=None):
    path = w.write(str(directory))
    if edit:
        with open(path) as f:
            text = edit(f.read())
        with open(path, "w") as f:
            f.write(text)
    with open(path) as f:
        sp = schema.parse_prototxt(f.read())
    return path, sp


def rec_files(sp):
    d = sp.rec_param.directory
    out = {}
    for sub in ("ProcSpkRec", "ProcCheck"):
        p = os.path.join(d, sub)
        if os.path.isdir(p):
            for name in sorted(os.listdir(p)):
                with open(os.path.join(p, name)) as f:
                    out[f"{sub}/{name}"] = f.read()
    return out


def oracle_files(sp, directory, **kw):
    ref = sim.simulate(sp, str(directory), **kw)
    files = {f"ProcSpkRec/{k}": v for k, v in ref["rec"].items()}
    if ref["check"]:
        files["ProcCheck/check_result.txt"] = "\n".join(ref["check"]) + "\n"
    return files, ref


def run(path, windows=True, snapshot=None):
    s = engine.Solver(path, snapshot)
    s.run(windows)
    st = s.stats()
    s.close()
    return st


def test_config0_matches_oracle_files(tmp_path):
    path, sp = write(workloads.config0(), tmp_path)
    st = run(path)
    got = rec_files(sp)
    want, ref = oracle_files(sp, tmp_path)
    assert set(got) == set(want)
    for name in want:
        assert got[name] == want[name], name
    assert (st["correct"], st["patterns"]) == ref["correct"]
    assert st["ticks"] == ref["simstep"]
    assert st["windows"] < st["ticks"] / 20  # one device run per segment


def test_windows_equal_ticks(tmp_path):
    w = workloads.config0()
    pa, spa = write(w, tmp_path / "a")
    pb, spb = write(w, tmp_path / "b")
    run(pa, windows=True)
    st = run(pb, windows=False)
    assert st["windows"] == 0
    fa, fb = rec_files(spa), rec_files(spb)
    assert fa == fb


def test_two_populations_poisson(tmp_path):
    w = workloads.config2(n_patterns=12, train_ticks=80, recall_ticks=20)
    path, sp = write(w, tmp_path)
    st = run(path)
    got = rec_files(sp)
    want, ref = oracle_files(sp, tmp_path)
    for name in want:
        assert got[name] == want[name], name
    assert (st["correct"], st["patterns"]) == ref["correct"]


def test_external_spike_file(tmp_path):
    rng = np.random.default_rng(11)
    lines = []
    for t in range(1, 400):
        k = int(rng.integers(0, 4))
        idx = sorted(rng.choice(100, size=k, replace=False).tolist())
        if idx:
            lines.append(",".join(str(v) for v in [t, 0] + idx))
    lines.append("5,0,1,2")  # a later line for a tick replaces the earlier one
    ext = tmp_path / "ext.csv"
    ext.write_text("\n".join(lines) + "\n")

    def edit(text):
        return text.replace('name: "ProcUpdLazy"', f'name: "ProcUpdLazy"\n  args {{ key: "external spike" val: "{ext}" }}')

    path, sp = write(workloads.config0(), tmp_path, edit)
    run(path)
    got = rec_files(sp)
    want, _ = oracle_files(sp, tmp_path)
    assert got["ProcSpkRec/spk_pop_0.csv"] == want["ProcSpkRec/spk_pop_0.csv"]
    assert "5,1,2\n" in got["ProcSpkRec/spk_pop_0.csv"]


def test_snapshot_and_restore(tmp_path):
    dt = np.float32(0.001)
    t_snap = 1650
    assert int(np.float32(np.float32(t_snap) * dt) / dt) == t_snap

    def with_snapshot(text):
        return text + f'proc_param {{ name: "ProcSnapshot" argi {{ key: "period" val: {t_snap} }} ' \
                      f'argi {{ key: "offset" val: {t_snap} }} }}\n'

    w = workloads.config0()
    path, sp = write(w, tmp_path / "full", with_snapshot)
    run(path)
    snap_dir = os.path.join(sp.rec_param.directory, "ProcSnapshot")
    names = os.listdir(snap_dir)
    assert len(names) == 1 and names[0].startswith("Snapshot_1.65")
    st = schema.SolverState()
    with open(os.path.join(snap_dir, names[0]), "rb") as f:
        st.ParseFromString(f.read())
    assert st.prn == 0.0
    vecs = {v.name: np.array(v.data, np.float32) for v in st.vector_state_f32}
    vecs.update({v.name: np.array(v.data, np.int32) for v in st.vector_state_i32})
    vecs.update({v.name: np.array(v.data, np.int8) for v in st.vector_state_i8})
    # against the oracle's state after the same tick
    ref = sim.simulate(sp, str(tmp_path / "full"), max_ticks=t_snap)
    assert ref["simstep"] == t_snap
    for name in ("pij_0", "eij_0", "zi2_0", "zj2_0", "tij_0", "wij_0", "pi_0", "ei_0", "zi_0", "ti_0", "pj_0",
                 "ej_0", "zj_0", "qi_0", "ii_0", "di_0", "si_0", "dsup_0", "act_0", "epsc_0", "bj_0", "spike_0"):
        a = ref["net"].read(name)
        b = vecs[name].astype(a.dtype)
        assert np.array_equal(a.view(np.uint8), b.view(np.uint8)), name
    # restore and run to the end: the spikes after the snapshot match the uninterrupted run
    path2, sp2 = write(w, tmp_path / "restored")
    run(path2, snapshot=os.path.join(snap_dir, names[0]))
    full = rec_files(sp)["ProcSpkRec/spk_pop_0.csv"].splitlines()
    rest = rec_files(sp2)["ProcSpkRec/spk_pop_0.csv"].splitlines()
    after = [l for l in full[1:] if int(l.split(",")[0]) > t_snap]
    assert rest[0] == full[0]
    assert rest[1:] == after
    assert len(after) > 50


def test_snapshot_and_restore_procupdmulti(tmp_path):
    """ProcSnapshot of a ProcUpdMulti network holds the vectors gsbn's
    ProcUpdMulti creates: ada_<pop> (its adaptation current) and the spike ring
    spike_<pop> (spike buffer size x H x M), no per-cell zi2 or tij
    (ProcUpdMulti/Pop.cpp:54-69, Proj.cpp:63-80).  Restored with -s, the run
    continues the uninterrupted spike train, adaptation included."""
    dt = np.float32(0.001)
    t_snap = 1650
    ring = 25

    def multi(text):
        text = text.replace('name: "ProcUpdLazy"', 'name: "ProcUpdMulti"\n  argi { key: "spike buffer size" val: %d }'
                            % ring)
        return text

    def with_snapshot(text):
        return multi(text) + f'proc_param {{ name: "ProcSnapshot" argi {{ key: "period" val: {t_snap} }} ' \
                             f'argi {{ key: "offset" val: {t_snap} }} }}\n'

    w = workloads.config0()
    path, sp = write(w, tmp_path / "full", with_snapshot)
    run(path)
    snap_dir = os.path.join(sp.rec_param.directory, "ProcSnapshot")
    names = os.listdir(snap_dir)
    assert len(names) == 1 and names[0].startswith("Snapshot_1.65")
    st = schema.SolverState()
    with open(os.path.join(snap_dir, names[0]), "rb") as f:
        st.ParseFromString(f.read())
    f32 = {v.name: np.array(v.data, np.float32) for v in st.vector_state_f32}
    i8 = {v.name: np.array(v.data, np.int8) for v in st.vector_state_i8}
    i32 = {v.name for v in st.vector_state_i32}
    assert "ada_0" in f32 and np.any(f32["ada_0"] != 0)
    assert i8["spike_0"].size == ring * 100 and i8["spike_0"].sum() > 0
    assert "zi2_0" not in f32 and "tij_0" not in i32 and "pij_0" in f32
    path2, sp2 = write(w, tmp_path / "restored", multi)
    run(path2, snapshot=os.path.join(snap_dir, names[0]))
    full = rec_files(sp)["ProcSpkRec/spk_pop_0.csv"].splitlines()
    rest = rec_files(sp2)["ProcSpkRec/spk_pop_0.csv"].splitlines()
    after = [l for l in full[1:] if int(l.split(",")[0]) > t_snap]
    assert rest[0] == full[0]
    assert rest[1:] == after
    assert len(after) > 50


def test_snapshot_lists_gsbn_vectors_in_key_order(tmp_path):
    """A ProcUpdLazy snapshot holds ada_<pop> (H x M zeros: gsbn creates it
    and never updates it) and lists each type's vectors in the order of gsbn's
    map keys "<name>_<type>" (Database.cpp:257-295)."""
    t_snap = 400
    w = workloads.config0()
    path, sp = write(w, tmp_path, lambda text: text + f'proc_param {{ name: "ProcSnapshot" argi {{ key: "period" '
                                                      f'val: {t_snap} }} argi {{ key: "offset" val: {t_snap} }} }}\n')
    run(path)
    snap_dir = os.path.join(sp.rec_param.directory, "ProcSnapshot")
    st = schema.SolverState()
    with open(os.path.join(snap_dir, os.listdir(snap_dir)[0]), "rb") as f:
        st.ParseFromString(f.read())
    for vs, suffix in ((st.vector_state_f32, "_f32"), (st.vector_state_i32, "_i32"), (st.vector_state_i8, "_i08")):
        keys = [v.name + suffix for v in vs]
        assert keys == sorted(keys)
    f32 = {v.name: np.array(v.data, np.float32) for v in st.vector_state_f32}
    assert f32["ada_0"].size == 100 and not f32["ada_0"].any()
    assert {"zi2_0", "pij_0", "wij_0"} <= set(f32)


def test_gsbn_sim_command(tmp_path):
    path, sp = write(workloads.config0(), tmp_path)
    r = subprocess.run([GSBN_SIM, "-n", path, "-m", "GPU"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert "correct pattern:" in r.stdout and "Total time for [2.2" in r.stdout
    want, _ = oracle_files(sp, tmp_path)
    assert rec_files(sp)["ProcSpkRec/spk_pop_0.csv"] == want["ProcSpkRec/spk_pop_0.csv"]
    bad = subprocess.run([GSBN_SIM, "-n", path, "-m", "CPU"], capture_output=True, text=True, timeout=300)
    assert bad.returncode == 1 and "no CPU path" in bad.stderr


@pytest.mark.parametrize("geometry", [False, True])
def test_structural_plasticity_matches_oracle(tmp_path, geometry):
    """ProcStructuralPlasticity (device pruning + host growth, seeded stream)
    against the oracle's restatement: same records, same final connectivity
    and traces.  With enable-geometry the grown rows get delays drawn from the
    HCUs' grid distance (the population laid out as a 5 x 2 grid at offset
    (1, 0, 3))."""
    def edit(text):
        text = text.replace("prn: 1.0\n    plasticity: 0", "prn: 1.0\n    plasticity: 1")
        geo = ('  argi { key: "enable-geometry" val: 1 }\n  argf { key: "d-norm" val: 0.9 }\n'
               '  argf { key: "v-cond" val: 0.25 }\n') if geometry else ""
        sp_block = ('proc_param {\n  name: "ProcStructuralPlasticity"\n  argi { key: "period" val: 50 }\n'
                    '  argi { key: "pruning-period" val: 100 }\n  argi { key: "t-th" val: 60 }\n'
                    '  argi { key: "seed" val: 7 }\n  argf { key: "wp" val: 1.5 }\n  argf { key: "wn" val: -1.5 }\n'
                    + geo + '}\n')
        if geometry:
            text = text.replace("    snoise: 0\n  }", "    snoise: 0\n    shape: 5\n    shape: 2\n    position: 1\n"
                                "    position: 0\n    position: 3\n  }", 1)
        return text.replace('proc_param {\n  name: "ProcSpkRec"', sp_block + 'proc_param {\n  name: "ProcSpkRec"')

    path, sp = write(workloads.config0(), tmp_path, edit)
    assert [p.name for p in sp.proc_param].index("ProcStructuralPlasticity") == 4
    s = engine.Solver(path)
    s.run()
    net = s.net(1, 1)
    got = {n: net.read(n) for n in ("ii_0", "di_0", "pij_0", "eij_0", "zj2_0", "ti_0", "wij_0", ".counter_0")}
    files = rec_files(sp)
    s.close()
    want_files, ref = oracle_files(sp, tmp_path)
    for name in want_files:
        assert files[name] == want_files[name], name
    for n, a in got.items():
        b = ref["net"].read(n)
        assert np.array_equal(a.view(np.uint8), b.view(np.uint8)), n
    # pruning and regrowth both happened
    assert (got["ii_0"] < 0).any() or (got["ii_0"] != np.tile(np.arange(100), 10)).any()
    if geometry:
        assert "shape: 5" in open(path).read()
        assert (got["di_0"] > 1).any(), "grown rows carry geometric delays"
