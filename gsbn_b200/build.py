"""Builds libgsbn_b200.so (C ABI + sm_100a kernels + C++ engine) and the
gsbn_sim command in place, with nvcc for sm_100a only.

The plain FP32 path is compiled with -fmad=false so that no multiply-add is
fused: the kernels then perform the same IEEE operations as the reference's
CPU expressions.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INC = os.path.join(ROOT, "include")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off", "-I" + INC, "-I" + CSRC]
PLAIN = ["-fmad=false"]


def _sources(sub, ext):
    d = os.path.join(CSRC, sub)
    if not os.path.isdir(d):
        return []
    return sorted(os.path.join(d, f) for f in os.listdir(d) if f.endswith(ext))


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def _headers():
    out = []
    for d in (CSRC, os.path.join(CSRC, "engine"), INC):
        out += [os.path.join(d, f) for f in os.listdir(d) if f.endswith((".h", ".cuh", ".hpp"))]
    return out


def _stale(obj, src, force):
    """An object is rebuilt when it is missing or older than its source or
    any header of the library."""
    if force or not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(f) > t for f in [src, __file__] + _headers())


def build(verbose_ptxas=False, force=False, probe=False):
    """probe: a second library, libgsbn_b200_probe.so, with the tick kernel's
    phase probe compiled in (-DBCPNN_PHASE_PROBE); the default build has none."""
    nvcc = os.environ.get("NVCC", "nvcc")
    objdir = os.path.join(HERE, "_build_probe" if probe else "_build")
    flags = ["-DBCPNN_PHASE_PROBE"] if probe else []
    os.makedirs(objdir, exist_ok=True)
    objs = []
    for src in sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu")):
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        extra = ["-Xptxas", "-v"] if verbose_ptxas else []
        if _stale(obj, src, force or verbose_ptxas):
            _run([nvcc] + ARCH + COMMON + PLAIN + flags + extra + ["-c", src, "-o", obj])
        objs.append(obj)
    for src in _sources("engine", ".cpp"):
        obj = os.path.join(objdir, "engine_" + os.path.basename(src) + ".o")
        if _stale(obj, src, force):
            _run([nvcc] + COMMON + flags + ["-Wno-deprecated-gpu-targets", "-x", "c++", "-c", src, "-o", obj])
        objs.append(obj)
    lib = os.path.join(HERE, "libgsbn_b200_probe.so" if probe else "libgsbn_b200.so")
    _run([nvcc] + ARCH + ["-shared", "-o", lib] + objs + ["-cudart", "static"])
    main = os.path.join(CSRC, "engine", "main", "gsbn_sim.cpp")
    if os.path.exists(main) and not probe:
        exe = os.path.join(HERE, "gsbn_sim")
        _run([nvcc] + COMMON + ["-Wno-deprecated-gpu-targets", "-x", "c++", main, "-o", exe, "-L" + HERE, "-lgsbn_b200",
                                "-Xlinker", "-rpath=$ORIGIN"])
    return lib


if __name__ == "__main__":
    build(verbose_ptxas="-v" in sys.argv, force="--force" in sys.argv, probe="--probe" in sys.argv)
