"""The shared numerics contract (include/bcpnn_numerics.h), through the CPU
oracle library that compiles it: Philox4x32-10 against the published
known-answer vectors (Salmon et al., SC'11, Random123 kat_vectors), the
stream map, and the float exp/log against correctly rounded values."""
import numpy as np

from oracle import sim

# (counter, key, expected output) -- Philox4x32-10 known answers
KAT = [
    ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
    ((0xFFFFFFFF,) * 4, (0xFFFFFFFF,) * 2, (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
    ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
     (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
]


def ulp_diff(a, b):
    ia = a.astype(np.float32).view(np.int32).astype(np.int64)
    ib = b.astype(np.float32).view(np.int32).astype(np.int64)
    ia = np.where(ia < 0, np.int64(-2 ** 31) - ia, ia)
    ib = np.where(ib < 0, np.int64(-2 ** 31) - ib, ib)
    return np.abs(ia - ib)


def test_philox_known_answers():
    for ctr, key, want in KAT:
        assert tuple(int(x) for x in sim.philox(ctr, key)) == want


def test_uniform_stream_map():
    u = sim.uniforms(0, 0, 1, 4096)
    assert u.min() >= 0.0 and u.max() < 1.0
    assert abs(u.mean() - 0.5) < 0.02
    # 24-bit grid: u * 2^24 is an integer
    assert np.all(np.floor(u * 2 ** 24) == u * 2 ** 24)
    # lane i of block i>>2 of Philox((i>>2, tick, 0, 0), (seed, pop*16))
    for i in (0, 1, 2, 3, 4, 4095):
        blk = sim.philox((i >> 2, 1, 0, 0), (0, 0))
        assert u[i] == np.float32((int(blk[i & 3]) >> 8) * 2.0 ** -24)
    assert not np.array_equal(u, sim.uniforms(0, 1, 1, 4096))
    assert not np.array_equal(u, sim.uniforms(0, 0, 2, 4096))
    assert not np.array_equal(u, sim.uniforms(1, 0, 1, 4096))


def test_normal_stream():
    z = sim.normals(3, 0, 7, 20000).astype(np.float64)
    assert abs(z.mean()) < 0.03
    assert abs(z.std() - 1.0) < 0.03


def test_expf_within_one_ulp_of_correctly_rounded():
    rng = np.random.default_rng(0)
    x = np.concatenate([rng.uniform(-104, 89, 1_000_000), rng.uniform(-1e-3, 1e-3, 100_000),
                        rng.standard_normal(100_000)]).astype(np.float32)
    got = sim.expf(x)
    with np.errstate(over="ignore"):  # x above ~88.72 rounds to inf in float32, as it should
        want = np.exp(x.astype(np.float64)).astype(np.float32)
    assert ulp_diff(got, want).max() <= 1


def test_logf_within_two_ulp_of_correctly_rounded():
    rng = np.random.default_rng(1)
    bits = rng.integers(1, 0x7F800000, 1_000_000, dtype=np.int64).astype(np.uint32)
    x = np.concatenate([bits.view(np.float32), rng.uniform(0.5, 2.0, 200_000).astype(np.float32)])
    got = sim.logf(x)
    want = np.log(x.astype(np.float64)).astype(np.float32)
    assert ulp_diff(got, want).max() <= 2


def test_special_values():
    e = sim.expf(np.array([np.nan, np.inf, -np.inf, 89.5, -110.0, 0.0, 88.72], np.float32))
    assert np.isnan(e[0]) and e[1] == np.inf and e[2] == 0.0 and e[3] == np.inf and e[4] == 0.0 and e[5] == 1.0
    assert np.isfinite(e[6])
    lg = sim.logf(np.array([np.nan, -1.0, 0.0, np.inf, 1.0, 1e-45], np.float32))
    assert np.isnan(lg[0]) and np.isnan(lg[1]) and lg[2] == -np.inf and lg[3] == np.inf and lg[4] == 0.0
    assert abs(lg[5] - np.float32(np.log(1.401298464324817e-45))) <= 1e-5


def test_shared_definition_close_to_glibc():
    rng = np.random.default_rng(2)
    x = rng.uniform(-80, 80, 200_000).astype(np.float32)
    assert ulp_diff(sim.expf(x), sim.expf(x, sim.MATH_LIBM)).max() <= 1
    y = rng.uniform(1e-6, 1e6, 200_000).astype(np.float32)
    assert ulp_diff(sim.logf(y), sim.logf(y, sim.MATH_LIBM)).max() <= 2
