"""bcpnn_read_state_noalloc, the read for callers that cannot allocate device
memory (an embedder whose device memory is pre-reserved for its own pool, or
a loop that must not stall on cudaMalloc/cudaFree), against bcpnn_read_state.

It gathers the interleaved cell fields into a fixed array compiled into the
library instead of a cudaMalloc'd staging buffer; its results must be the
same bits as the allocating read, on two calls in a row.  The first call on a
device looks the array's address up: test_first_call_in_a_fresh_process
makes that first call in a new process, whatever ran before in this one.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

from gsbn_b200 import capi, workloads
from tests.harness import load_workload, schedule

pytestmark = pytest.mark.gpu

NAMES = ("pij_0", "eij_0", "zi2_0", "zj2_0", "wij_0", "tij_0", "pi_0", "dsup_0", "epsc_0", "spike_0", "si_0")


def trained_net(tmp_path):
    sp, pops, projs, stim, conn, seed, phz = load_workload(workloads.config0(), str(tmp_path))
    net = capi.Net(pops, projs, 0.001, seed=seed, max_ticks=128)
    for k, (ii, di) in enumerate(conn):
        net.set_conn(k, ii, di)
    runs = schedule(sp, stim, pops, lambda x: np.float32(np.log(np.float64(x))))
    return net, runs


def same_bits(a, b):
    if a.dtype.kind == "f":
        return np.array_equal(a.view(np.int32), b.view(np.int32))
    return np.array_equal(a, b)


def test_noalloc_read_matches_allocating_read(tmp_path):
    net, runs = trained_net(tmp_path)
    for r in runs[:3]:
        net.set_stimulus(r.lginp, r.wmask)
        net.run(r.first, r.n, r.prn, r.old_prn)
    first = {n: net.read_noalloc(n) for n in NAMES}
    second = {n: net.read_noalloc(n) for n in NAMES}
    for n in NAMES:
        ref = net.read(n)
        assert same_bits(first[n], ref), n
        assert same_bits(second[n], ref), n
    assert np.any(first["pij_0"] != first["pij_0"][0])
    # after more ticks the static array holds the previous call's values; the
    # next reads must still equal the allocating read
    r = runs[3]
    net.set_stimulus(r.lginp, r.wmask)
    net.run(r.first, r.n, r.prn, r.old_prn)
    for n in ("pij_0", "zj2_0"):
        assert same_bits(net.read_noalloc(n), net.read(n)), n
        assert same_bits(net.read_noalloc(n), net.read(n)), n
    net.close()


def test_noalloc_read_rejects_fields_beyond_the_static_array():
    # 100 HCUs x 1000 slots x 11 MCUs = 1.1e6 cells > 1048576
    pops = [dict(hcu_num=100, mcu_num=11, taum=0.005, wtagain=1.0, maxfq=100.0, igain=1.0, wgain=1.0,
                 lgbias=0.0, snoise=0.0)]
    projs = [dict(src_pop=0, dest_pop=0, tauzi=0.01, tauzj=0.01, taue=0.02, taup=1.0, maxfq=100.0, bgain=1.0,
                  wgain=1.0, tauepsc=0.0, slot_num=1000.0)]
    net = capi.Net(pops, projs, 0.001, max_ticks=8)
    with pytest.raises(capi.BcpnnError) as e:
        net.read_noalloc("pij_0")
    assert e.value.status == -4
    assert net.read("pij_0").size == 1100000
    assert same_bits(net.read_noalloc("wij_0"), net.read("wij_0"))
    net.close()


FRESH = """
import sys
import numpy as np
sys.path.insert(0, sys.argv[1])
from tests.test_zz_no_alloc import NAMES, same_bits, trained_net
net, runs = trained_net(sys.argv[2])
for r in runs[:2]:
    net.set_stimulus(r.lginp, r.wmask)
    net.run(r.first, r.n, r.prn, r.old_prn)
for n in NAMES:
    a, b, ref = net.read_noalloc(n), net.read_noalloc(n), net.read(n)
    assert same_bits(a, ref) and same_bits(b, ref), n
net.close()
print("fresh ok")
"""


def test_first_call_in_a_fresh_process(tmp_path):
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, "-c", FRESH, root, str(tmp_path)], capture_output=True, text=True,
                         timeout=600)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "fresh ok" in out.stdout
