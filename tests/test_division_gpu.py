"""The decay closed forms (Proj.cpp:409-415, 435-443, 519-527) divide on the
GPU with a warp-uniform exact division instead of `/`: zero numerators and
infinite divisors by their exact signed zero, a double-precision quotient
rounded once for subnormal or extreme operands.  It must return the same bits
as `/` for every float pair; here 2**31 pairs per seed, one in two forced into
a hard class (zero, infinite, subnormal, huge or extreme-ratio operands).  The
bit-exact parity of every state array against the oracle covers the same
division inside the kernels."""
import pytest

from gsbn_b200 import capi

pytestmark = pytest.mark.gpu

POP = dict(hcu_num=2, mcu_num=2, taum=0.005, wtagain=1.0, maxfq=100.0, igain=1.0, wgain=1.0, lgbias=0.0, snoise=0.0)


@pytest.mark.parametrize("seed", [1, 2])
def test_exact_division_matches_ieee_quotient(seed):
    net = capi.Net([POP], [], 0.001, seed=0)
    try:
        tested, bad = net.selftest_division(1 << 31, seed)
    finally:
        net.close()
    assert tested > (1 << 31) * 0.9
    assert bad == 0
