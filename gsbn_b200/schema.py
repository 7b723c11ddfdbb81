"""gsbn's protobuf schema (src/gsbn/proto/gsbn.proto:1-160) declared at run time.

The reference ships the schema as a .proto file compiled by protoc into
gsbn_pb2 for its Python tools (tools/stimgen/gen_rnd.py:14-15).  protoc is not
available here, so the same messages, field numbers, labels and defaults are
declared through descriptor_pb2 and turned into message classes by the
protobuf runtime.  The field layout has to match the reference exactly: it is
the on-disk format of prototxt network descriptions, StimRawData stimulus
files and SolverState snapshots.
"""
from google.protobuf import descriptor_pb2, descriptor_pool, message_factory, text_format

_F = descriptor_pb2.FieldDescriptorProto
_OPT, _REQ, _REP = _F.LABEL_OPTIONAL, _F.LABEL_REQUIRED, _F.LABEL_REPEATED
_T = {
    "float": _F.TYPE_FLOAT, "double": _F.TYPE_DOUBLE, "uint32": _F.TYPE_UINT32, "int32": _F.TYPE_INT32,
    "int64": _F.TYPE_INT64, "string": _F.TYPE_STRING, "bytes": _F.TYPE_BYTES,
}

# message -> [(name, number, label, type or message name, default, packed)]
_MESSAGES = {
    "SolverParam": [("gen_param", 1, _REQ, "GenParam", None, False),
                    ("net_param", 2, _REQ, "NetParam", None, False),
                    ("rec_param", 3, _REQ, "RecParam", None, False),
                    ("proc_param", 4, _REP, "ProcParam", None, False)],
    "GenParam": [("stim_file", 1, _OPT, "string", None, False),
                 ("dt", 2, _REQ, "float", None, False),
                 ("eps", 3, _REQ, "float", "0.001", False),
                 ("mode_param", 4, _REP, "ModeParam", None, False),
                 ("procedure", 5, _REP, "string", None, False)],
    "ModeParam": [("begin_time", 1, _REQ, "float", None, False),
                  ("end_time", 2, _REQ, "float", None, False),
                  ("begin_lgidx_id", 3, _OPT, "uint32", "0", False),
                  ("begin_lgexp_id", 4, _OPT, "uint32", "0", False),
                  ("begin_wmask_id", 5, _OPT, "uint32", "0", False),
                  ("time_step", 6, _OPT, "uint32", "1", False),
                  ("lgidx_step", 7, _OPT, "uint32", "1", False),
                  ("lgexp_step", 8, _OPT, "uint32", "1", False),
                  ("wmask_step", 9, _OPT, "uint32", "1", False),
                  ("prn", 10, _OPT, "float", "1.0", False),
                  ("plasticity", 11, _OPT, "uint32", "1", False)],
    "NetParam": [("pop_param", 1, _REP, "PopParam", None, False),
                 ("proj_param", 2, _REP, "ProjParam", None, False)],
    "PopParam": [("pop_num", 1, _REQ, "uint32", None, False),
                 ("hcu_num", 2, _REQ, "uint32", None, False),
                 ("mcu_num", 3, _REQ, "uint32", None, False),
                 ("fanout_num", 4, _REQ, "uint32", None, False),
                 ("taum", 5, _OPT, "float", "0.01", False),
                 ("wtagain", 6, _OPT, "float", "4", False),
                 ("maxfq", 7, _OPT, "float", "100", False),
                 ("igain", 8, _OPT, "float", "1.0", False),
                 ("wgain", 9, _OPT, "float", "1.0", False),
                 ("lgbias", 10, _OPT, "float", "0", False),
                 ("snoise", 11, _OPT, "float", "0", False),
                 ("adgain", 12, _OPT, "float", "1", False),
                 ("taua", 13, _OPT, "float", "0.05", False),
                 ("position", 15, _REP, "int32", None, True),
                 ("shape", 16, _REP, "uint32", None, True),
                 ("type", 17, _OPT, "uint32", "0", False),
                 ("rank", 18, _OPT, "uint32", "0", False)],
    "ProjParam": [("src_pop", 1, _REQ, "uint32", None, False),
                  ("dest_pop", 2, _REQ, "uint32", None, False),
                  ("tauzi", 3, _REQ, "float", None, False),
                  ("tauzj", 4, _REQ, "float", None, False),
                  ("taue", 5, _REQ, "float", None, False),
                  ("taup", 6, _REQ, "float", None, False),
                  ("maxfq", 7, _OPT, "float", "100", False),
                  ("bgain", 8, _OPT, "float", "0", False),
                  ("wgain", 9, _OPT, "float", "0", False),
                  ("tauepsc", 10, _OPT, "float", None, False),
                  ("slot_num", 11, _REQ, "float", None, False),
                  ("distance", 12, _OPT, "float", "0", False)],
    "RecParam": [("directory", 1, _OPT, "string", ".", False)],
    "ProcParam": [("name", 1, _REQ, "string", None, False),
                  ("argi", 2, _REP, "ProcParamArgI", None, False),
                  ("argf", 3, _REP, "ProcParamArgF", None, False),
                  ("args", 4, _REP, "ProcParamArgS", None, False)],
    "ProcParamArgI": [("key", 1, _REQ, "string", None, False), ("val", 2, _REQ, "int32", None, False)],
    "ProcParamArgF": [("key", 1, _REQ, "string", None, False), ("val", 2, _REQ, "float", None, False)],
    "ProcParamArgS": [("key", 1, _REQ, "string", None, False), ("val", 2, _REQ, "string", None, False)],
    "SolverState": [("timestamp", 1, _REQ, "float", None, False),
                    ("prn", 2, _REQ, "float", None, False),
                    ("table_state", 3, _REP, "TableState", None, False),
                    ("vector_state_i8", 4, _REP, "VectorStateI8", None, False),
                    ("vector_state_i16", 5, _REP, "VectorStateI16", None, False),
                    ("vector_state_i32", 6, _REP, "VectorStateI32", None, False),
                    ("vector_state_i64", 7, _REP, "VectorStateI64", None, False),
                    ("vector_state_f16", 8, _REP, "VectorStateF16", None, False),
                    ("vector_state_f32", 9, _REP, "VectorStateF32", None, False),
                    ("vector_state_f64", 10, _REP, "VectorStateF64", None, False)],
    "TableState": [("name", 1, _REQ, "string", None, False), ("desc", 2, _REQ, "bytes", None, False),
                   ("data", 3, _REQ, "bytes", None, False)],
    "StimRawData": [("data_rows", 1, _REQ, "uint32", None, False),
                    ("data_cols", 2, _REQ, "uint32", None, False),
                    ("data", 3, _REP, "uint32", None, True),
                    ("mask_rows", 4, _REQ, "uint32", None, False),
                    ("mask_cols", 5, _REQ, "uint32", None, False),
                    ("mask", 6, _REP, "float", None, True)],
}
for _name, _elem in (("I8", "int32"), ("I16", "int32"), ("I32", "int32"), ("I64", "int64"),
                     ("F16", "float"), ("F32", "float"), ("F64", "double")):
    _MESSAGES["VectorState" + _name] = [("name", 1, _REQ, "string", None, False),
                                        ("ld", 2, _OPT, "uint32", "1", False),
                                        ("data", 3, _REP, _elem, None, True)]


def _build():
    fdp = descriptor_pb2.FileDescriptorProto(name="gsbn.proto", package="gsbn", syntax="proto2")
    for mname, fields in _MESSAGES.items():
        m = fdp.message_type.add(name=mname)
        for fname, num, label, ftype, default, packed in fields:
            f = m.field.add(name=fname, number=num, label=label)
            if ftype in _T:
                f.type = _T[ftype]
            else:
                f.type = _F.TYPE_MESSAGE
                f.type_name = ".gsbn." + ftype
            if default is not None:
                f.default_value = default
            if packed:
                f.options.packed = True
    pool = descriptor_pool.DescriptorPool()
    pool.Add(fdp)
    return {name: message_factory.GetMessageClass(pool.FindMessageTypeByName("gsbn." + name))
            for name in _MESSAGES}


_CLASSES = _build()
SolverParam = _CLASSES["SolverParam"]
StimRawData = _CLASSES["StimRawData"]
SolverState = _CLASSES["SolverState"]


def parse_prototxt(text):
    """Parse a protobuf text-format network description (Solver.cpp:12-15)."""
    msg = SolverParam()
    text_format.Parse(text, msg)
    return msg


def read_stim(path):
    """Decode a StimRawData file (ProcExtGen.cpp:61-89)."""
    msg = StimRawData()
    with open(path, "rb") as f:
        msg.ParseFromString(f.read())
    return msg
