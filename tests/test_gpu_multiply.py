"""GPU parity of the ciphertext products against the CPU oracle, word for word.

Covers the tensor product (rlwe/quadratic.rs:70-140), bounded
relinearization (grafting/bounded_key_switch.rs:139-223), the fused
multiply -> relinearize -> rescale chain (ckks/rns_multiply.rs:262-300),
plaintext products (ckks/rns_plain_multiply.rs:193-260) and the plain CKKS
chain at N=2^12 with one 60-bit and two 40-bit primes plus a 60-bit special
prime: HMult -> relinearize (base 2^20) -> rescale -> rotate by one slot.
Exact integer results: tolerance zero. Decoded results are compared with the
FP64 cleartext within the relative-L2 bound stated in each test.
"""
import numpy as np
import pytest

import ckks_b200 as cb

pytestmark = pytest.mark.gpu

C1_Q = [0xfffffffffffc001, 0xfffffdc001, 0xfffffc6001]
C1_P = [0xffffffffffe8001]


def dev(x):
    return cb.as_u64_tensor(x)


def host(t):
    return cb.to_numpy_u64(t)


def rand_ct(rng, q, n, count):
    return np.stack([np.stack([np.stack([rng.integers(0, m, n, dtype=np.uint64) for m in q]) for _ in range(2)])
                     for _ in range(count)])


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def small(oracle):
    n = 1 << 10
    q = [int(x) for x in oracle.primes_below_bits(50, n, 4)]
    p = [int(x) for x in oracle.primes_below_bits(60, n, 2)]
    return n, q, p, cb.Context(10, q, p)


def test_tensor_bit_exact(oracle, cuda, small):
    n, q, p, ctx = small
    rng = np.random.default_rng(1)
    for count in (1, 3, 5):
        x, y = rand_ct(rng, q, n, count), rand_ct(rng, q, n, count)
        got = host(cb.tensor(ctx, dev(x), dev(y)))
        for c in range(count):
            assert np.array_equal(got[c], oracle.tensor(q, x[c], y[c])), c
    # lower level: the Q prefix of three limbs
    x, y = rand_ct(rng, q[:3], n, 2), rand_ct(rng, q[:3], n, 2)
    got = host(cb.tensor(ctx, dev(x), dev(y)))
    assert np.array_equal(got[1], oracle.tensor(q[:3], x[1], y[1]))


@pytest.mark.parametrize("base_log", [8, 20, 32])
def test_relinearize_bit_exact(oracle, cuda, small, base_log):
    n, q, p, ctx = small
    rng = np.random.default_rng(base_log)
    s = rng.integers(-1, 2, n).astype(np.int8)
    key_ref = oracle.relin_key(q, s, base_log, seed=3)
    key = cb.KeySwitchKey.relin_upload(ctx, len(q), base_log, key_ref)
    # 1, 4 and 6 ciphertexts: a partial and a full group of the MAC
    for count in (1, 4, 6):
        quad = np.stack([np.stack([np.stack([rng.integers(0, m, n, dtype=np.uint64) for m in q]) for _ in range(3)])
                         for _ in range(count)])
        got = host(cb.relinearize(ctx, key, dev(quad)))
        for c in range(count):
            assert np.array_equal(got[c], oracle.relinearize(q, quad[c], key_ref, base_log)), (count, c)


def test_relinearize_ccmm_shape_bit_exact(oracle, cuda):
    # N=2^15, 14 x 50-bit limbs, base 2^20 (36 digits): the CCMM configuration's
    # relinearization, whose digit transforms are finished inside the key MAC
    log_n, L, base_log = 15, 14, 20
    n = 1 << log_n
    q = [int(x) for x in oracle.primes_below_bits(50, n, L)]
    ctx = cb.Context(log_n, q)
    rng = np.random.default_rng(77)
    s = rng.integers(-1, 2, n).astype(np.int8)
    key = cb.KeySwitchKey.relin_generate(ctx, L, base_log, s, seed=5)
    key_coef = oracle.ntt_inverse(q, key.download().reshape(-1, L, n)).reshape(-1, 2, L, n)
    count = 3
    quad = np.stack([np.stack([np.stack([rng.integers(0, m, n, dtype=np.uint64) for m in q]) for _ in range(3)])
                     for _ in range(count)])
    got = host(cb.relinearize(ctx, key, dev(quad)))
    for c in (0, count - 1):
        assert np.array_equal(got[c], oracle.relinearize(q, quad[c], key_coef, base_log)), c


def test_multiply_relin_rescale_bit_exact_and_decodes(oracle, cuda, small):
    n, q, p, ctx = small
    rng = np.random.default_rng(7)
    s = rng.integers(-1, 2, n).astype(np.int8)
    scale = 2.0 ** 40
    base_log = 20
    key_ref = oracle.relin_key(q, s, base_log, seed=11)
    key = cb.KeySwitchKey.relin_generate(ctx, len(q), base_log, s, seed=11)
    count = 5
    xs, ys, cx, cy = [], [], [], []
    for c in range(count):
        a = rng.uniform(-1, 1, n // 2) + 1j * rng.uniform(-1, 1, n // 2)
        b = rng.uniform(-1, 1, n // 2) + 1j * rng.uniform(-1, 1, n // 2)
        xs.append(a)
        ys.append(b)
        cx.append(oracle.encrypt(q, s, oracle.encode(a, q, scale), seed=100 + c))
        cy.append(oracle.encrypt(q, s, oracle.encode(b, q, scale), seed=200 + c))
    cx, cy = np.stack(cx), np.stack(cy)
    got = host(cb.multiply_relinearize_rescale(ctx, key, dev(cx), dev(cy)))
    assert got.shape == (count, 2, len(q) - 1, n)
    for c in range(count):
        quad = oracle.tensor(q, cx[c], cy[c])
        rel = oracle.relinearize(q, quad, key_ref, base_log)
        want = oracle.rescale(q, rel.reshape(2, len(q), n))
        assert np.array_equal(got[c], want), c
        dec = oracle.decode(q[:-1], oracle.decrypt(q[:-1], s, got[c]), scale * scale / q[-1])
        assert rel_l2(dec, xs[c] * ys[c]) < 1e-6
    # host-buffer entry point and the unfused ops give the same words
    assert np.array_equal(cb.multiply_relinearize_rescale_host(ctx, key, cx, cy), got)
    quad = cb.tensor(ctx, dev(cx), dev(cy))
    rel = cb.relinearize(ctx, key, quad)
    assert np.array_equal(host(ctx.rescale(rel)), got)


def test_mul_plain_bit_exact(oracle, cuda, small):
    n, q, p, ctx = small
    rng = np.random.default_rng(9)
    count = 3
    ct = rand_ct(rng, q, n, count)
    plain = np.stack([rng.integers(0, m, n, dtype=np.uint64) for m in q])
    plain_ntt = oracle.ntt_forward(q, plain.copy())
    got = host(cb.multiply_plain(ctx, dev(ct), dev(plain_ntt)))
    for c in range(count):
        assert np.array_equal(got[c], oracle.mul_plain(q, ct[c], plain)), c
    # one plaintext per ciphertext, and in place
    plains = np.stack([np.stack([rng.integers(0, m, n, dtype=np.uint64) for m in q]) for _ in range(count)])
    pn = np.stack([oracle.ntt_forward(q, x.copy()) for x in plains])
    d = dev(ct)
    cb.multiply_plain(ctx, d, dev(pn), out=d)
    got = host(d)
    for c in range(count):
        assert np.array_equal(got[c], oracle.mul_plain(q, ct[c], plains[c])), c


def test_product_errors(oracle, cuda, small):
    n, q, p, ctx = small
    import torch
    rng = np.random.default_rng(2)
    s = rng.integers(-1, 2, n).astype(np.int8)
    gk = cb.KeySwitchKey.hybrid_generate(ctx, len(q), 20, ctx.rotation_exponent_left(1), s, seed=1)
    x = dev(rand_ct(rng, q, n, 1))
    with pytest.raises(cb.CkksError) as e:  # a Galois key is not a relinearization key
        cb.relinearize(ctx, gk, torch.zeros((1, 3, len(q), n), dtype=torch.int64, device="cuda"))
    assert e.value.status == -2
    k1 = cb.KeySwitchKey.relin_generate(ctx, 1, 20, s, seed=1)
    with pytest.raises(cb.CkksError) as e:  # one limb: no level to rescale to
        cb.multiply_relinearize_rescale(ctx, k1, x[:, :, :1].contiguous(), x[:, :, :1].contiguous())
    assert e.value.status == -1
    rc = cb.lib().ckks_tensor(ctx.handle, cb._dptr(x), cb._dptr(x), cb._dptr(x), 1, len(q), None)
    assert rc == -1  # output overlapping an input
    assert b"overlaps" in cb.lib().ckks_last_error_string()


def test_c1_chain_multiply_relin_rescale_rotate(oracle, cuda):
    """Plain CKKS at N=2^12: q = 60 + 40 + 40 bits, P = 60 bits, scale 2^40,
    HMult -> relinearize (bounded, base 2^20) -> rescale -> rotate by 1."""
    log_n, n = 12, 1 << 12
    ctx = cb.Context(log_n, C1_Q, C1_P)
    rng = np.random.default_rng(12)
    s = rng.integers(-1, 2, n).astype(np.int8)
    scale = 2.0 ** 40
    rk_ref = oracle.relin_key(C1_Q, s, 20, seed=21)
    rk = cb.KeySwitchKey.relin_upload(ctx, 3, 20, rk_ref)
    k = ctx.rotation_exponent_left(1)
    gk_ref = oracle.hybrid_key(C1_Q[:2], C1_P, s, k, 20, seed=22)
    gk = cb.KeySwitchKey.hybrid_upload(ctx, 2, 20, k, gk_ref)
    count = 6
    a = rng.uniform(-1, 1, (count, n // 2)) + 1j * rng.uniform(-1, 1, (count, n // 2))
    b = rng.uniform(-1, 1, (count, n // 2)) + 1j * rng.uniform(-1, 1, (count, n // 2))
    cx = np.stack([oracle.encrypt(C1_Q, s, oracle.encode(a[c], C1_Q, scale), seed=300 + c) for c in range(count)])
    cy = np.stack([oracle.encrypt(C1_Q, s, oracle.encode(b[c], C1_Q, scale), seed=400 + c) for c in range(count)])
    prod = cb.multiply_relinearize_rescale(ctx, rk, dev(cx), dev(cy))
    rot = host(cb.rotate(ctx, gk, prod))
    out_scale = scale * scale / C1_Q[-1]
    for c in (0, count - 1):
        quad = oracle.tensor(C1_Q, cx[c], cy[c])
        rel = oracle.relinearize(C1_Q, quad, rk_ref, 20)
        resc = oracle.rescale(C1_Q, rel.reshape(2, 3, n))
        want = oracle.hybrid_rotate(C1_Q[:2], C1_P, gk_ref, k, 20, resc)
        assert np.array_equal(rot[c], want), c
        dec = oracle.decode(C1_Q[:2], oracle.decrypt(C1_Q[:2], s, rot[c]), out_scale)
        assert rel_l2(dec, np.roll(a[c] * b[c], -1)) < 1e-4
