"""B200-native BCPNN simulation core: the ProcUpdLazy / ProcSpkRec hot path of
gsbn behind its prototxt schema and Procedure registry.

    libgsbn_b200.so   C ABI (include/bcpnn.h) + sm_100a kernels + C++ engine
    gsbn_b200.capi    ctypes binding of the C ABI
    gsbn_b200.schema  gsbn.proto message classes (prototxt / stimulus files)
    gsbn_b200.workloads  seeded synthetic workloads in gsbn's formats
"""
import os

PACKAGE_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PACKAGE_DIR, "libgsbn_b200.so")
SIM_PATH = os.path.join(PACKAGE_DIR, "gsbn_sim")
