"""Park Mod-PP-MM (ccmm/park.rs:1405-1647) on the GPU against the oracle.

The oracle restates the reference's Reference backend (u128 accumulator
reduced after every term); every output word of both device backends (INT8
tensor cores, 192-bit CUDA-core sums) must match (tolerance zero) for square
and ragged shapes, moduli of every byte width from 1 to 8 (including 2^64 -
59, the largest 64-bit prime, and the composite 2^64 - 1), entries at or above
the modulus, and inner sums long enough that the tensor-core form adds the
residues of several launches. The reference's own characterization sizes are
n = 256 .. 4096; n = 4096 is checked backend against backend in full and
against the oracle on sampled rows.
"""
import numpy as np
import pytest

import ckks_b200 as cb

pytestmark = pytest.mark.gpu

# 0x7ffff6001: the modulus of the reference's characterization (research_profile_4096, ckks/parameters.rs:249-258)
MODULI = [2, 3, 17, 257, 65537, 2**31 - 1, 0x7ffff6001, 2**47 - 115, 0x3ffffffd20001, 0xfffffffffffc001,
          2**64 - 59, 2**64 - 1]
BACKENDS = ["tensor_cores", "cuda_cores"]


def _rand(rng, shape, q, full=False):
    hi = 2**64 if full else q
    return rng.integers(0, hi, shape, dtype=np.uint64)


def _dev(cuda, a, b, q, backend):
    got = cb.park_mod_pp_mm(cb.as_u64_tensor(a), cb.as_u64_tensor(b), q, backend=backend)
    return cb.to_numpy_u64(got)


@pytest.mark.parametrize("backend", BACKENDS)
@pytest.mark.parametrize("q", MODULI)
@pytest.mark.parametrize("shape", [(1, 1, 1), (7, 13, 5), (64, 64, 64), (130, 70, 100)])
def test_park_matches_oracle(oracle, cuda, q, shape, backend):
    r, k, c = shape
    rng = np.random.default_rng(r * 1000 + k * 10 + c)
    a, b = _rand(rng, (r, k), q), _rand(rng, (k, c), q)
    assert np.array_equal(_dev(cuda, a, b, q, backend), oracle.park_mod_pp_mm(a, b, q))


def test_park_host_path(oracle, cuda):
    rng = np.random.default_rng(2)
    for q in (17, 0x7ffff6001, 2**64 - 59):
        a, b = _rand(rng, (65, 17), q), _rand(rng, (17, 130), q)
        assert np.array_equal(cb.park_mod_pp_mm(a, b, q), oracle.park_mod_pp_mm(a, b, q))


@pytest.mark.parametrize("backend", BACKENDS)
def test_park_non_canonical_inputs(oracle, cuda, backend):
    rng = np.random.default_rng(5)
    for q in (17, 0x7ffff6001, 0xfffffffffffc001, 2**64 - 59):
        a, b = _rand(rng, (33, 47), q, full=True), _rand(rng, (47, 21), q, full=True)
        assert np.array_equal(_dev(cuda, a, b, q, backend), oracle.park_mod_pp_mm(a, b, q))


@pytest.mark.parametrize("shape,q", [((3, 4200, 5), 2**64 - 59),      # 8 bytes: 4128 terms per launch
                                     ((5, 7000, 9), 0x7ffff6001),     # 5 bytes: 6592 terms per launch
                                     ((2, 33100, 3), 251)])           # 1 byte: 33024 terms per launch
def test_park_tensor_cores_long_inner_sums(oracle, cuda, shape, q):
    r, k, c = shape
    rng = np.random.default_rng(k)
    a, b = _rand(rng, (r, k), q, full=True), _rand(rng, (k, c), q, full=True)
    assert np.array_equal(_dev(cuda, a, b, q, "tensor_cores"), oracle.park_mod_pp_mm(a, b, q))


def test_park_backends_agree_at_n1024(oracle, cuda):
    q = 0xfffffffffffc001
    n = 1024
    rng = np.random.default_rng(11)
    a, b = _rand(rng, (n, n), q), _rand(rng, (n, n), q)
    tc = _dev(cuda, a, b, q, "tensor_cores")
    assert np.array_equal(tc, _dev(cuda, a, b, q, "cuda_cores"))
    for (i, j) in [(0, 0), (n - 1, n - 1), (17, 900), (511, 3)]:
        assert tc[i, j] == oracle.park_mod_pp_mm(a[i:i + 1], b[:, j:j + 1], q)[0, 0], (i, j)
    assert np.array_equal(tc[100:101], oracle.park_mod_pp_mm(a[100:101], b, q))


def test_park_characterization_size(oracle, cuda):
    """n = 4096 with the characterization modulus: the whole product of both
    backends word for word, two full rows against the oracle."""
    import torch
    q, n = 0x7ffff6001, 4096
    rng = np.random.default_rng(4096)
    a, b = _rand(rng, (n, n), q), _rand(rng, (n, n), q)
    da, db = cb.as_u64_tensor(a), cb.as_u64_tensor(b)
    tc = cb.park_mod_pp_mm(da, db, q, backend="tensor_cores")
    pack_ms, gemm_ms = cb.park_last_timing()
    assert pack_ms > 0 and gemm_ms > 0
    cc = cb.park_mod_pp_mm(da, db, q, backend="cuda_cores")
    torch.cuda.synchronize()
    assert torch.equal(tc, cc)
    got = cb.to_numpy_u64(tc)
    for r in (0, n - 1):
        assert np.array_equal(got[r:r + 1], oracle.park_mod_pp_mm(a[r:r + 1], b, q)), r


def test_park_rejects_empty_bad_modulus_and_backend(cuda):
    a = np.ones((2, 2), np.uint64)
    with pytest.raises(cb.CkksError):
        cb.park_mod_pp_mm(a, a, 1)
    with pytest.raises((cb.CkksError, ValueError)):
        cb.park_mod_pp_mm(np.ones((0, 2), np.uint64), a, 17)
    with pytest.raises(ValueError):
        cb.park_mod_pp_mm(cb.as_u64_tensor(a), cb.as_u64_tensor(a), 17, backend="fpga")
