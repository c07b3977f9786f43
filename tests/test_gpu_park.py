"""Park Mod-PP-MM (ccmm/park.rs:1405-1647) on the GPU against the oracle.

The oracle restates the reference's Reference backend (u128 accumulator
reduced after every term); every output word must match (tolerance zero) for
square and ragged shapes, small and full-width moduli (including 2^64 - 59,
the largest 64-bit prime, and the composite 2^64 - 1) and entries at or above
the modulus. The reference's own characterization sizes are n = 256 .. 4096;
the largest here is checked on sampled entries.
"""
import numpy as np
import pytest

import ckks_b200 as cb

pytestmark = pytest.mark.gpu

# 0x7ffff6001: the modulus of the reference's characterization (research_profile_4096, ckks/parameters.rs:249-258)
MODULI = [2, 3, 17, 65537, 0x7ffff6001, 0x3ffffffd20001, 0xfffffffffffc001, 2**64 - 59, 2**64 - 1]


def _rand(rng, shape, q, full=False):
    hi = 2**64 if full else q
    return rng.integers(0, hi, shape, dtype=np.uint64)


@pytest.mark.parametrize("q", MODULI)
@pytest.mark.parametrize("shape", [(1, 1, 1), (7, 13, 5), (64, 64, 64), (65, 17, 130)])
def test_park_matches_oracle(oracle, cuda, q, shape):
    r, k, c = shape
    rng = np.random.default_rng(r * 1000 + k * 10 + c)
    a, b = _rand(rng, (r, k), q), _rand(rng, (k, c), q)
    assert np.array_equal(cb.park_mod_pp_mm(a, b, q), oracle.park_mod_pp_mm(a, b, q))


def test_park_non_canonical_inputs(oracle, cuda):
    rng = np.random.default_rng(5)
    for q in (17, 0xfffffffffffc001, 2**64 - 59):
        a, b = _rand(rng, (33, 47), q, full=True), _rand(rng, (47, 21), q, full=True)
        assert np.array_equal(cb.park_mod_pp_mm(a, b, q), oracle.park_mod_pp_mm(a, b, q))


def test_park_device_path_and_large_square(oracle, cuda):
    import torch
    q = 0xfffffffffffc001
    n = 1024
    rng = np.random.default_rng(11)
    a, b = _rand(rng, (n, n), q), _rand(rng, (n, n), q)
    da, db = cb.as_u64_tensor(a), cb.as_u64_tensor(b)
    got = cb.to_numpy_u64(cb.park_mod_pp_mm(da, db, q))
    torch.cuda.synchronize()
    for (i, j) in [(0, 0), (n - 1, n - 1), (17, 900), (511, 3)]:
        want = oracle.park_mod_pp_mm(a[i:i + 1], b[:, j:j + 1], q)[0, 0]
        assert got[i, j] == want, (i, j)
    # a full row against the oracle
    assert np.array_equal(got[100:101], oracle.park_mod_pp_mm(a[100:101], b, q))


def test_park_rejects_empty_and_bad_modulus(cuda):
    a = np.ones((2, 2), np.uint64)
    with pytest.raises(cb.CkksError):
        cb.park_mod_pp_mm(a, a, 1)
    with pytest.raises((cb.CkksError, ValueError)):
        cb.park_mod_pp_mm(np.ones((0, 2), np.uint64), a, 17)
