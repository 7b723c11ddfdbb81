"""Host engine checks that need no GPU: the hand-written prototxt parser and
StimRawData decoder against the protobuf runtime's own text and wire parsers
(on the gsbn schema), their error behaviour, and the procedure registry.
"""
import os
import struct

import numpy as np
import pytest

from gsbn_b200 import engine, schema, workloads
from oracle import sim

# the gsbn source tree ($GSBN_REFERENCE_ROOT, else oracle/Makefile's REF_ROOT);
# the tests that read its data files skip when it is absent
REF_DATA = os.path.join(sim.reference_root() or "", "data")

PROCEDURES = {"ProcExtGen", "ProcUpdLazy", "ProcExchangeSpike", "ProcInitConn", "ProcSpkRec", "ProcCheck",
              "ProcSnapshot", "ProcStructuralPlasticity", "ProcUpdMulti"}


def g_float(v):
    """shortest %.{6..9}g text that reads back to the same float32"""
    v = np.float32(v)
    if np.isnan(v):
        return "nan"
    for prec in range(6, 10):
        s = "%.*g" % (prec, float(v))
        if np.float32(float(s)) == v:
            return s
    return s


def py_dump(sp):
    """the engine's canonical dump, computed from a protobuf-runtime message"""
    g = sp.gen_param
    out = [f"gen.stim_file={g.stim_file}", f"gen.dt={g_float(g.dt)}", f"gen.eps={g_float(g.eps)}"]
    for i, m in enumerate(g.mode_param):
        out.append(f"mode[{i}]=" + ",".join([g_float(m.begin_time), g_float(m.end_time), str(m.begin_lgidx_id),
                                              str(m.begin_lgexp_id), str(m.begin_wmask_id), str(m.time_step),
                                              str(m.lgidx_step), str(m.lgexp_step), str(m.wmask_step),
                                              g_float(m.prn), str(m.plasticity)]))
    for i, p in enumerate(g.procedure):
        out.append(f"gen.procedure[{i}]={p}")
    for i, p in enumerate(sp.net_param.pop_param):
        vals = [str(p.pop_num), str(p.hcu_num), str(p.mcu_num), str(p.fanout_num)] + \
               [g_float(getattr(p, k)) for k in ("taum", "wtagain", "maxfq", "igain", "wgain", "lgbias", "snoise",
                                                 "adgain", "taua")] + [str(p.type), str(p.rank)]
        out.append(f"pop[{i}]=" + ",".join(vals) + ",pos" + "".join(f":{v}" for v in p.position) + ",shape" +
                   "".join(f":{v}" for v in p.shape))
    for i, q in enumerate(sp.net_param.proj_param):
        vals = [str(q.src_pop), str(q.dest_pop)] + [g_float(getattr(q, k)) for k in
                                                    ("tauzi", "tauzj", "taue", "taup", "maxfq", "bgain", "wgain")]
        vals.append(g_float(q.tauepsc) if q.HasField("tauepsc") else "-")
        vals += [g_float(q.slot_num), g_float(q.distance)]
        out.append(f"proj[{i}]=" + ",".join(vals))
    out.append(f"rec.directory={sp.rec_param.directory}")
    for i, p in enumerate(sp.proc_param):
        out.append(f"proc[{i}]={p.name}")
        out += [f"proc[{i}].argi.{a.key}={a.val}" for a in p.argi]
        out += [f"proc[{i}].argf.{a.key}={g_float(a.val)}" for a in p.argf]
        out += [f"proc[{i}].args.{a.key}={a.val}" for a in p.args]
    return "\n".join(out) + "\n"


def both(tmp_path, text):
    path = tmp_path / "net.prototxt"
    path.write_text(text)
    ours = engine.prototxt_dump(str(path))
    theirs = py_dump(schema.parse_prototxt(text))
    return ours, theirs


def test_registry_names():
    assert set(engine.procedure_names()) == PROCEDURES


@pytest.mark.parametrize("name", ["10x10_rnd", "2x5x10_rnd", "cartoon", "color", "nocol", "sp"])
def test_reference_prototxt(tmp_path, name):
    path = os.path.join(REF_DATA, name + ".prototxt")
    if not os.path.exists(path):
        pytest.skip("reference data not present")
    with open(path) as f:
        text = f.read()
    assert engine.prototxt_dump(path) == py_dump(schema.parse_prototxt(text))


@pytest.mark.parametrize("make", [workloads.config0, workloads.config2, workloads.config1])
def test_workload_prototxt(tmp_path, make):
    w = make()
    path = w.write(str(tmp_path))
    with open(path) as f:
        text = f.read()
    assert engine.prototxt_dump(path) == py_dump(schema.parse_prototxt(text))


SYNTAX = r'''
# comment line
gen_param <
  stim_file: "a" 'b' "\x41\101\n\t\"q\""   # adjacent strings, escapes
  dt: 1e-3f ; eps: .5
  mode_param { begin_time: 0 end_time: 2.5E1 time_step: 0x10 prn: -0.0 }
  mode_param: { begin_time: 1 end_time: 3, lgidx_step: 010 prn: inf }
  procedure: "x" procedure: ["y", "z"]
>
net_param {
  pop_param { pop_num: 1 hcu_num: 4294967295 mcu_num: 3 fanout_num: 0 position: [-2147483648, 5] shape: [1,2] }
  proj_param { src_pop: 0 dest_pop: 0 tauzi: 0.005 tauzj: 0.005001 taue: 0.0050002 taup: 60 slot_num: 1.5
               tauepsc: 1e-38 bgain: -3 }
}
rec_param {}
proc_param { name: "ProcUpdLazy" argi { key: "seed" val: -7 } argf: [{ key: "f" val: 3.4028235e38 }]
             args { key: "external spike" val: "x,y.csv" } }
'''


def test_syntax_forms(tmp_path):
    ours, theirs = both(tmp_path, SYNTAX)
    assert ours == theirs


def test_float_rounding(tmp_path):
    # decimal -> double -> float, including values that are not exact floats
    vals = ["0.1", "0.001", "1e-45", "3.4028234e38", "0.0050002", "123456789", "16777217", "1.00000005",
            "2.5e-8", "9.999999e-4"]
    for v in vals:
        text = f'gen_param {{ dt: {v} eps: {v} }} net_param {{}} rec_param {{}}'
        ours, theirs = both(tmp_path, text)
        assert ours == theirs, v


BAD = [
    ("unknown field", 'gen_param { dt: 1 eps: 1 bogus: 3 } net_param {} rec_param {}'),
    ("missing required", 'gen_param { eps: 1 } net_param {} rec_param {}'),
    ("missing top-level", 'gen_param { dt: 1 eps: 1 } net_param {}'),
    ("repeated optional", 'gen_param { dt: 1 dt: 2 eps: 1 } net_param {} rec_param {}'),
    ("negative uint", 'gen_param { dt: 1 eps: 1 mode_param { begin_time: 0 end_time: 1 time_step: -1 } } '
                      'net_param {} rec_param {}'),
    ("float into uint", 'gen_param { dt: 1 eps: 1 mode_param { begin_time: 0 end_time: 1 time_step: 1.5 } } '
                        'net_param {} rec_param {}'),
    ("uint out of range", 'gen_param { dt: 1 eps: 1 mode_param { begin_time: 0 end_time: 1 time_step: 4294967296 } } '
                          'net_param {} rec_param {}'),
    ("string into float", 'gen_param { dt: "1" eps: 1 } net_param {} rec_param {}'),
    ("unterminated string", 'gen_param { stim_file: "abc dt: 1 eps: 1 } net_param {} rec_param {}'),
    ("missing brace", 'gen_param { dt: 1 eps: 1 net_param {} rec_param {}'),
    ("scalar as message", 'gen_param: 3 net_param {} rec_param {}'),
    ("missing key", 'gen_param { dt: 1 eps: 1 } net_param {} rec_param {} proc_param { name: "a" argi { val: 1 } }'),
]


@pytest.mark.parametrize("what,text", BAD, ids=[b[0] for b in BAD])
def test_rejects(tmp_path, what, text):
    path = tmp_path / "bad.prototxt"
    path.write_text(text)
    # the protobuf runtime rejects it too (its Python text parser leaves the
    # required-field check to IsInitialized, which the C++ parser applies)
    try:
        msg = schema.parse_prototxt(text)
    except Exception:
        pass
    else:
        assert not msg.IsInitialized(), what
    with pytest.raises(engine.EngineError):
        engine.prototxt_dump(str(path))


# ---------------------------------------------------------------- StimRawData

def _varint(v):
    out = b""
    while v >= 0x80:
        out += bytes([(v & 0x7F) | 0x80])
        v >>= 7
    return out + bytes([v])


def _tag(field, wt):
    return _varint(field << 3 | wt)


def _stim_reference_encoding(data, mask, dr, dc, mr, mc):
    m = schema.StimRawData(data_rows=dr, data_cols=dc, mask_rows=mr, mask_cols=mc)
    m.data.extend(int(x) for x in data)
    m.mask.extend(float(x) for x in mask)
    return m.SerializeToString()


def _check_decode(tmp_path, blob, data, mask, dims):
    p = tmp_path / "stim.bin"
    p.write_bytes(blob)
    d, m = engine.stim_decode(str(p))
    assert d.shape == (dims[0], dims[1]) and m.shape == (dims[2], dims[3])
    assert np.array_equal(d.ravel(), np.asarray(data, np.uint32))
    assert np.array_equal(m.ravel().view(np.uint32), np.asarray(mask, np.float32).view(np.uint32))


def test_stim_workloads(tmp_path):
    for make in (workloads.config0, workloads.config2):
        w = make()
        path = w.write(str(tmp_path / make.__name__))
        sp = schema.parse_prototxt(open(path).read())
        ref = schema.read_stim(sp.gen_param.stim_file)
        d, m = engine.stim_decode(sp.gen_param.stim_file)
        assert np.array_equal(d.ravel(), np.asarray(ref.data, np.uint32))
        assert np.array_equal(m.ravel(), np.asarray(ref.mask, np.float32))


def test_stim_reference_file():
    path = os.path.join(REF_DATA, "stimuli_10x10_100_-1_rnd.bin")
    if not os.path.exists(path):
        pytest.skip("reference data not present")
    ref = schema.read_stim(path)
    d, m = engine.stim_decode(path)
    assert d.shape == (ref.data_rows, ref.data_cols)
    assert np.array_equal(d.ravel(), np.asarray(ref.data, np.uint32))
    assert np.array_equal(m.ravel(), np.asarray(ref.mask, np.float32))


def test_stim_wire_variants(tmp_path):
    rng = np.random.default_rng(1)
    data = rng.integers(0, 2 ** 32, 12, dtype=np.uint64).tolist() + [0x7FFFFFFF, 0xFFFFFFFF]
    data = data[:12]
    mask = rng.standard_normal(6).astype(np.float32).tolist()
    dims = (3, 4, 2, 3)
    # packed, as the protobuf runtime writes it
    _check_decode(tmp_path, _stim_reference_encoding(data, mask, *dims), data, mask, dims)
    # unpacked repeated fields, fields out of order, unknown fields of every wire type
    blob = _tag(5, 0) + _varint(3) + _tag(99, 0) + _varint(12345) + _tag(1, 0) + _varint(3)
    for x in data[:5]:
        blob += _tag(3, 0) + _varint(int(x))
    blob += _tag(98, 1) + b"\x01" * 8 + _tag(2, 0) + _varint(4)
    blob += _tag(3, 2) + _varint(len(b"".join(_varint(int(x)) for x in data[5:]))) + \
        b"".join(_varint(int(x)) for x in data[5:])
    blob += _tag(97, 2) + _varint(3) + b"abc" + _tag(4, 0) + _varint(2) + _tag(96, 5) + b"\x00" * 4
    for x in mask:
        blob += _tag(6, 5) + struct.pack("<f", x)
    _check_decode(tmp_path, blob, data, mask, dims)
    # the protobuf runtime reads the same bytes identically
    ref = schema.StimRawData()
    ref.ParseFromString(blob)
    assert list(ref.data) == [int(x) for x in data]


def test_stim_rejects(tmp_path):
    good = _stim_reference_encoding([1, 2], [0.5], 1, 2, 1, 1)
    cases = {
        "truncated": good[:-2],
        "size mismatch": _stim_reference_encoding([1, 2, 3], [0.5], 1, 2, 1, 1),
        "missing required": _tag(1, 0) + _varint(0),
        "bad wire type": _tag(1, 5) + b"\x00" * 4 + good,
    }
    for what, blob in cases.items():
        p = tmp_path / f"{what.replace(' ', '_')}.bin"
        p.write_bytes(blob)
        with pytest.raises(engine.EngineError):
            engine.stim_decode(str(p))
    with pytest.raises(engine.EngineError):
        engine.stim_decode(str(tmp_path / "does_not_exist.bin"))


def test_solver_errors_without_gpu(tmp_path):
    """errors found while reading the description come back as statuses"""
    bad = tmp_path / "bad.prototxt"
    bad.write_text('gen_param { dt: 1 eps: 1 } net_param {} rec_param {} proc_param { name: "ProcNope" }')
    with pytest.raises(engine.EngineError, match="stim|ProcNope|not found"):
        engine.Solver(str(bad))
    with pytest.raises(engine.EngineError, match="cannot open"):
        engine.Solver(str(tmp_path / "missing.prototxt"))
