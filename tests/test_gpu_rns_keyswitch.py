"""GPU parity of the ordinary RNS key switch without auxiliary limbs (the
reference evaluator's default rotation backend and its RNS relinearization):

  apply_rns_galois_automorphism_with_prepared_ntt   ckks/rns_galois_key.rs:439-469
  rns_key_switch_with_prepared_ntt                  grafting/rns_key_switch.rs:2438-2524
  rns_relinearize_with_ntt                          grafting/rns_key_switch.rs:1842-1905
  key generation (E_i * target over Q)              grafting/rns_key_switch.rs:1155-1258

Every output word must equal the oracle's restatement (tolerance zero), for
singleton blocks (dnum = L, the reference's RNS-native form) and multi-limb
blocks, at N=2^12 and at N=2^16.
"""
import numpy as np
import pytest

import ckks_b200 as cb

pytestmark = pytest.mark.gpu


def dev(x):
    return cb.as_u64_tensor(x)


def host(t):
    return cb.to_numpy_u64(t)


def uniform_cts(rng, q, n, count):
    return np.stack([np.stack([rng.integers(0, m, (2, n), dtype=np.uint64) for m in q], axis=1)
                     for _ in range(count)])


@pytest.mark.parametrize("log_n,L,blocks", [(12, 4, [1, 1, 1, 1]), (12, 4, [2, 2]), (12, 5, [1, 2, 2]),
                                            (16, 6, [1] * 6)])
def test_rns_rotation_bit_exact(oracle, cuda, log_n, L, blocks):
    n = 1 << log_n
    q = [int(x) for x in oracle.primes_below_bits(50, n, L)]
    ctx = cb.Context(log_n, q)  # no auxiliary limbs
    rng = np.random.default_rng(log_n * 10 + len(blocks))
    s = rng.integers(-1, 2, n).astype(np.int8)
    ks = [ctx.rotation_exponent_left(1), ctx.rotation_exponent_right(3), 2 * n - 1]
    keys = [cb.KeySwitchKey.rns_generate(ctx, L, blocks, k, s, seed=300 + i) for i, k in enumerate(ks)]
    # GPU key generation equals the oracle's word for word (reference layout, NTT domain)
    ref0 = oracle.rns_key(q, blocks, s, ks[0], seed=300)
    assert np.array_equal(keys[0].download(), ref0.ravel())
    cts = uniform_cts(rng, q, n, 3)
    for g, k in enumerate(ks):
        got = host(cb.rotate(ctx, keys[g], dev(cts)))
        key_ref = keys[g].download().reshape(len(blocks), L, 2, n)
        for c in (0, 2):
            assert np.array_equal(got[c], oracle.rns_rotate(q, blocks, key_ref, k, cts[c])), (g, c)
    # several keys through the hoisted entry point: one full key switch per key
    hoisted = host(cb.rotate_hoisted(ctx, keys, dev(cts[:2])))
    for g, k in enumerate(ks):
        key_ref = keys[g].download().reshape(len(blocks), L, 2, n)
        assert np.array_equal(hoisted[1, g], oracle.rns_rotate(q, blocks, key_ref, k, cts[1])), g
    # uploaded reference-layout key
    up = cb.KeySwitchKey.rns_upload(ctx, L, blocks, ks[0], ref0)
    assert np.array_equal(host(cb.rotate(ctx, up, dev(cts[:1])))[0], oracle.rns_rotate(q, blocks, ref0, ks[0], cts[0]))


def test_rns_rotation_decodes(oracle, cuda):
    """30-bit limbs, singleton blocks, scale 2^60: the GPU rotation decrypts to
    the rotated slots (the switch's noise is about q_i sigma sqrt(N))."""
    log_n, n = 12, 1 << 12
    q = [int(x) for x in oracle.primes_below_bits(30, n, 4)]
    ctx = cb.Context(log_n, q)
    rng = np.random.default_rng(5)
    s = rng.integers(-1, 2, n).astype(np.int8)
    scale = 2.0 ** 60
    slots = rng.uniform(-1, 1, n // 2) + 1j * rng.uniform(-1, 1, n // 2)
    ct = oracle.encrypt(q, s, oracle.encode(slots, q, scale), seed=9)
    k = ctx.rotation_exponent_left(2)
    key = cb.KeySwitchKey.rns_generate(ctx, 4, [1, 1, 1, 1], k, s, seed=10)
    got = host(cb.rotate(ctx, key, dev(ct[None])))[0]
    dec = oracle.decode(q, oracle.decrypt(q, s, got), scale)
    assert np.linalg.norm(dec - np.roll(slots, -2)) / np.linalg.norm(slots) < 1e-3


@pytest.mark.parametrize("log_n,L,blocks", [(12, 4, [1, 1, 1, 1]), (12, 4, [2, 2]), (16, 4, [1] * 4)])
def test_rns_relinearize_bit_exact(oracle, cuda, log_n, L, blocks):
    n = 1 << log_n
    q = [int(x) for x in oracle.primes_below_bits(50, n, L)]
    ctx = cb.Context(log_n, q)
    rng = np.random.default_rng(log_n + 7 * len(blocks))
    s = rng.integers(-1, 2, n).astype(np.int8)
    key = cb.KeySwitchKey.rns_relin_generate(ctx, L, blocks, s, seed=77)
    ref = oracle.rns_relin_key(q, blocks, s, seed=77)  # coefficient domain [nb][2][L][N]
    assert np.array_equal(key.download(), oracle.ntt_forward(q, ref.reshape(-1, L, n)).ravel())
    up = cb.KeySwitchKey.rns_relin_upload(ctx, L, blocks, ref)
    quads = np.stack([np.stack([np.stack([rng.integers(0, m, n, dtype=np.uint64) for m in q]) for _ in range(3)])
                      for _ in range(3)])
    for k_ in (key, up):
        got = host(cb.relinearize(ctx, k_, dev(quads)))
        for c in (0, 2):
            assert np.array_equal(got[c], oracle.rns_relinearize(q, blocks, quads[c], ref)), c
    # multiply -> relinearize -> rescale with the RNS-block key
    x, y = uniform_cts(rng, q, n, 2), uniform_cts(rng, q, n, 2)
    got = host(cb.multiply_relinearize_rescale(ctx, key, dev(x), dev(y)))
    for c in range(2):
        rel = oracle.rns_relinearize(q, blocks, oracle.tensor(q, x[c], y[c]), ref)
        assert np.array_equal(got[c], oracle.rescale(q, rel.reshape(2, L, n))), c


def test_rns_key_errors(oracle, cuda):
    n = 1 << 10
    q = [int(x) for x in oracle.primes_below_bits(50, n, 3)]
    ctx = cb.Context(10, q)
    s = np.ones(n, np.int8)
    with pytest.raises(cb.CkksError) as e:
        cb.KeySwitchKey.rns_generate(ctx, 3, [1, 1], 5, s, seed=1)  # blocks do not cover Q
    assert e.value.status == -2
    with pytest.raises(cb.CkksError) as e:
        cb.KeySwitchKey.rns_generate(ctx, 3, [1, 1, 1], 4, s, seed=1)  # even exponent
    assert e.value.status == -1
    rk = cb.KeySwitchKey.rns_relin_generate(ctx, 3, [1, 1, 1], s, seed=2)
    import torch
    ct = torch.zeros((1, 2, 3, n), dtype=torch.int64, device="cuda")
    with pytest.raises(cb.CkksError) as e:
        cb.rotate(ctx, rk, ct)  # a relinearization key is not a Galois key
    assert e.value.status == -2
