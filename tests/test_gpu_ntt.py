"""GPU parity: batched negacyclic NTT / inverse vs the CPU oracle, word for word.

Mirrors the reference's differential tests: radix-2 vs O(N^2) definition
(ring/ntt_params.rs:87-141), prepared vs radix-2 (ring/prepared_ntt.rs:864-1306),
round trips (ring/ntt_radix2.rs:190-230).
"""
import numpy as np
import pytest

import ckks_b200 as cb

pytestmark = pytest.mark.gpu


def rand_polys(rng, moduli, n, npoly):
    return np.stack([np.stack([rng.integers(0, q, n, dtype=np.uint64) for q in moduli]) for _ in range(npoly)])


@pytest.mark.parametrize("log_n,bits,count", [(3, 20, 1), (4, 30, 2), (6, 40, 3), (8, 50, 2), (10, 60, 3),
                                               (12, 50, 4), (13, 55, 2), (15, 50, 3), (16, 60, 2)])
def test_ntt_matches_oracle(oracle, cuda, log_n, bits, count):
    import torch
    n = 1 << log_n
    moduli = [int(x) for x in oracle.primes_below_bits(bits, n, count)]
    ctx = cb.Context(log_n, moduli)
    assert ctx.psi == [oracle.root(q, n) for q in moduli]
    rng = np.random.default_rng(log_n * 100 + bits)
    x = rand_polys(rng, moduli, n, 3)
    ref = oracle.ntt_forward(moduli, x)
    d = cb.as_u64_tensor(x)
    out = torch.empty_like(d)
    ctx.ntt_forward(d, out=out)
    torch.cuda.synchronize()
    assert np.array_equal(cb.to_numpy_u64(out), ref)
    back = torch.empty_like(d)
    ctx.ntt_inverse(out, out=back)
    assert np.array_equal(cb.to_numpy_u64(back), x)
    # inverse against the oracle on independent input
    y = rand_polys(rng, moduli, n, 2)
    ctx_y = cb.as_u64_tensor(y)
    ctx.ntt_inverse(ctx_y)  # in place
    assert np.array_equal(cb.to_numpy_u64(ctx_y), oracle.ntt_inverse(moduli, y))


def test_ntt_matches_definition_small(oracle, cuda):
    # O(N^2) definition A[k] = a(psi^(2k+1)) (ring/ntt.rs:106-127)
    for (q, log_n) in [(97, 3), (12289, 5), (12289, 8), (40961, 9)]:
        n = 1 << log_n
        ctx = cb.Context(log_n, [q])
        rng = np.random.default_rng(q + n)
        a = rng.integers(0, q, n, dtype=np.uint64)
        got = ctx.ntt_forward_host(a.reshape(1, 1, n))[0, 0]
        assert np.array_equal(got, oracle.ntt_forward_reference(q, a))
        assert np.array_equal(ctx.ntt_inverse_host(got.reshape(1, 1, n))[0, 0], a)


def test_ntt_edge_values(oracle, cuda):
    import torch
    n = 1 << 12
    moduli = [int(x) for x in oracle.primes_below_bits(61, n, 2)]
    ctx = cb.Context(12, moduli)
    for fill in ("zero", "max", "one"):
        if fill == "zero":
            x = np.zeros((1, 2, n), np.uint64)
        elif fill == "max":
            x = np.stack([np.full(n, q - 1, np.uint64) for q in moduli])[None]
        else:
            x = np.zeros((1, 2, n), np.uint64); x[..., 0] = 1
        d = cb.as_u64_tensor(x)
        ctx.ntt_forward(d)
        assert np.array_equal(cb.to_numpy_u64(d), oracle.ntt_forward(moduli, x))


def test_ntt_limb_subrange_and_host(oracle, cuda):
    n = 1 << 11
    q = [int(x) for x in oracle.primes_below_bits(50, n, 3)]
    p = [int(x) for x in oracle.primes_below_bits(60, n, 2)]
    ctx = cb.Context(11, q, p)
    rng = np.random.default_rng(5)
    sub = q[1:] + p[:1]
    x = rand_polys(rng, sub, n, 2)
    got = ctx.ntt_forward_host(x, limb_begin=1)
    assert np.array_equal(got, oracle.ntt_forward(sub, x))
    assert np.array_equal(ctx.ntt_inverse_host(got, limb_begin=1), x)


def test_ntt_c2_shape(oracle, cuda):
    # N=2^16, 32 limbs of 50-bit primes (the batched NTT configuration), 2 polys
    import torch
    n = 1 << 16
    moduli = [int(x) for x in oracle.primes_below_bits(50, n, 32)]
    ctx = cb.Context(16, moduli)
    rng = np.random.default_rng(16)
    x = rand_polys(rng, moduli, n, 2)
    d = cb.as_u64_tensor(x)
    out = torch.empty_like(d)
    ctx.ntt_forward(d, out=out)
    assert np.array_equal(cb.to_numpy_u64(out), oracle.ntt_forward(moduli, x))
    ctx.ntt_inverse(out)
    assert torch.equal(out, d)


def test_ntt_rejects_bad_arguments(cuda):
    with pytest.raises(cb.CkksError) as e:
        cb.Context(4, [97 * 2 + 1])  # 195: not prime
    assert e.value.status == -1
    ctx = cb.Context(4, [97])
    import torch
    d = torch.zeros((1, 2, 16), dtype=torch.int64, device="cuda")
    with pytest.raises(cb.CkksError) as e:
        ctx.ntt_forward(d)  # 2 limbs requested, context has 1
    assert e.value.status == -2


@pytest.mark.parametrize("log_n", [12, 16])
def test_autotuned_ntt_stays_bit_exact(oracle, cuda, log_n):
    """The autotuner records a choice for each of the five passes, and every
    tile choice it can make gives the oracle's words (forward, inverse, digits)."""
    n = 1 << log_n
    moduli = [int(x) for x in oracle.primes_below_bits(50, n, 3)]
    ctx = cb.Context(log_n, moduli)
    assert "not tuned" in ctx.tuning_report
    rep = ctx.autotune(limbs=3, polys=4)
    assert rep.count("->") == 5, rep
    rng = np.random.default_rng(log_n)
    x = rand_polys(rng, moduli, n, 2)
    d = cb.as_u64_tensor(x)
    out = ctx.ntt_forward(d.clone())
    assert np.array_equal(cb.to_numpy_u64(out), oracle.ntt_forward(moduli, x))
    back = ctx.ntt_inverse(out)
    assert np.array_equal(cb.to_numpy_u64(back), x)
