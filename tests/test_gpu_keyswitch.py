"""GPU parity of the key-switching path against the CPU oracle, word for word.

Mirrors the reference's differential tests: NTT-domain Galois permutation vs
coefficient automorphism (ring/ntt_galois_permutation.rs:38-66), ModDown vs
big-integer reference (tests/r16_5_18g1_rns_mod_down.rs), hoisted vs
re-decomposed digits (grafting/bounded_gadget.rs:428-500), prepared rotation
equivalence (ckks/hybrid_rns_galois_key.rs:873-1150) and decoded rotation error
(tests/r30_9a_13_hybrid_65536.rs:200,256-262, rel-L2 < 0.01).
"""
import numpy as np
import pytest

import ckks_b200 as cb

pytestmark = pytest.mark.gpu


def params(oracle, log_n, L, K, qbits=50, pbits=60):
    n = 1 << log_n
    q = [int(x) for x in oracle.primes_below_bits(qbits, n, L)]
    p = [int(x) for x in oracle.primes_below_bits(pbits, n, K)]
    return n, q, p


def rand_poly(rng, moduli, n, lead=()):
    return np.stack([rng.integers(0, m, lead + (n,), dtype=np.uint64) for m in moduli], axis=-2)


def dev(x):
    return cb.as_u64_tensor(x)


def host(t):
    return cb.to_numpy_u64(t)


@pytest.fixture(scope="module")
def small(oracle):
    n, q, p = params(oracle, 10, 4, 2)
    ctx = cb.Context(10, q, p)
    return n, q, p, ctx


def test_automorphisms(oracle, cuda, small):
    n, q, p, ctx = small
    rng = np.random.default_rng(1)
    x = rand_poly(rng, q, n, (2,))
    for k in [1, 3, 5, 25, 2 * n - 1, ctx.rotation_exponent_left(7), ctx.rotation_exponent_right(3)]:
        got = host(ctx.automorphism_coef(dev(x), k))
        assert np.array_equal(got, oracle.automorphism_coef(q, x, k)), k
        xn = oracle.ntt_forward(q, x)
        gotn = host(ctx.automorphism_ntt(dev(xn), k))
        assert np.array_equal(gotn, oracle.automorphism_ntt(len(q), xn, k))
        # NTT-domain permutation == NTT of the coefficient automorphism
        assert np.array_equal(gotn, oracle.ntt_forward(q, oracle.automorphism_coef(q, x, k)))


def test_pointwise_and_rescale(oracle, cuda, small):
    n, q, p, ctx = small
    rng = np.random.default_rng(2)
    a, b = rand_poly(rng, q, n, (3,)), rand_poly(rng, q, n, (3,))
    got = host(ctx.pointwise(dev(a), dev(b), "mul"))
    want = np.zeros_like(a)
    for l, m in enumerate(q):
        want[:, l] = np.array([(int(u) * int(v)) % m for u, v in zip(a[:, l].ravel(), b[:, l].ravel())],
                              np.uint64).reshape(a[:, l].shape)
    assert np.array_equal(got, want)
    assert np.array_equal(host(ctx.pointwise(dev(a), dev(b), "add")), (a + b) % np.array(q, np.uint64)[:, None])
    for limbs in [4, 3, 2]:
        x = rand_poly(rng, q[:limbs], n, (2,))
        x[0, -1, :4] = [0, q[limbs - 1] // 2, q[limbs - 1] // 2 + 1, q[limbs - 1] - 1]  # centring edges
        assert np.array_equal(host(ctx.rescale(dev(x))), oracle.rescale(q[:limbs], x))


def test_mod_down(oracle, cuda, small):
    n, q, p, ctx = small
    rng = np.random.default_rng(3)
    for q_limbs in [4, 2]:
        x = rand_poly(rng, q[:q_limbs] + p, n, (2,))
        P = p[0] * p[1]
        # centring edges on the P part: floor(P/2), floor(P/2)+1, 0, P-1
        for c, v in enumerate([P // 2, P // 2 + 1, 0, P - 1]):
            x[0, q_limbs:, c] = [v % pi for pi in p]
        assert np.array_equal(host(ctx.mod_down(dev(x))), oracle.mod_down(q[:q_limbs], p, x))


@pytest.mark.parametrize("base_log", [8, 20, 32, 62])
def test_bounded_decompose_and_hoisted(oracle, cuda, small, base_log):
    n, q, p, ctx = small
    rng = np.random.default_rng(base_log)
    x = rand_poly(rng, q, n)
    Q = 1
    for m in q:
        Q *= m
    # centring edges: 0, floor(Q/2), floor(Q/2)+1, Q-1 and a value whose digits hit -B/2
    for c, v in enumerate([0, Q // 2, Q // 2 + 1, Q - 1, Q - (1 << (base_log - 1))]):
        x[:, c] = [v % m for m in q]
    d = ctx.bounded_decompose(dev(x), base_log)
    want = oracle.bounded_decompose(q, x, base_log)
    assert ctx.digit_count(len(q), base_log) == want.shape[0]
    assert np.array_equal(d.cpu().numpy(), want)
    for k in [5, 2 * n - 1, ctx.rotation_exponent_left(3)]:
        h = ctx.bounded_digits_automorphism(d, base_log, k).cpu().numpy()
        assert np.array_equal(h, oracle.bounded_automorphism_hoisted(want, base_log, k))
        # hoisted digits equal re-decomposing sigma(a) (bounded_gadget.rs:446-500)
        sx = oracle.automorphism_coef(q, x, k)
        assert np.array_equal(h, oracle.bounded_decompose(q, sx, base_log))


def encode_encrypt(oracle, q, secret, rng, scale, seed):
    n = len(secret)
    slots = rng.uniform(-1, 1, n // 2) + 1j * rng.uniform(-1, 1, n // 2)
    ct = oracle.encrypt(q, secret, oracle.encode(slots, q, scale), seed)
    return slots, ct


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("base_log", [20, 32])
def test_hybrid_rotation_bit_exact(oracle, cuda, small, base_log):
    n, q, p, ctx = small
    rng = np.random.default_rng(10 + base_log)
    s = rng.integers(-1, 2, n).astype(np.int8)
    scale = 2.0 ** 40
    slots, ct = encode_encrypt(oracle, q, s, rng, scale, seed=5)
    k = ctx.rotation_exponent_left(1)
    # key generation on the GPU equals the oracle's restatement word for word
    key_ref = oracle.hybrid_key(q, p, s, k, base_log, seed=99)
    key = cb.KeySwitchKey.hybrid_generate(ctx, len(q), base_log, k, s, seed=99)
    assert np.array_equal(key.download(), key_ref.ravel())
    want = oracle.hybrid_rotate(q, p, key_ref, k, base_log, ct)
    got = host(cb.rotate(ctx, key, dev(ct)))
    assert np.array_equal(got, want)
    dec = oracle.decode(q, oracle.decrypt(q, s, got), scale)
    assert rel_l2(dec, np.roll(slots, -1)) < 1e-6
    # uploaded key and a batch of ciphertexts
    up = cb.KeySwitchKey.hybrid_upload(ctx, len(q), base_log, k, key_ref)
    cts = np.stack([ct, encode_encrypt(oracle, q, s, rng, scale, seed=6)[1]])
    got2 = host(cb.rotate(ctx, up, dev(cts)))
    assert np.array_equal(got2[0], want)
    assert np.array_equal(got2[1], oracle.hybrid_rotate(q, p, key_ref, k, base_log, cts[1]))


def test_hybrid_rotation_lower_level_and_hoisted(oracle, cuda, small):
    n, q, p, ctx = small
    rng = np.random.default_rng(21)
    s = rng.integers(-1, 2, n).astype(np.int8)
    scale = 2.0 ** 40
    ql = q[:3]  # a ciphertext one level down
    slots, ct = encode_encrypt(oracle, ql, s, rng, scale, seed=7)
    steps = [1, 2, 5, n // 4]
    ks = [ctx.rotation_exponent_left(r) for r in steps] + [2 * n - 1]
    keys = [cb.KeySwitchKey.hybrid_generate(ctx, 3, 20, k, s, seed=100 + i) for i, k in enumerate(ks)]
    keys_ref = [oracle.hybrid_key(ql, p, s, k, 20, seed=100 + i) for i, k in enumerate(ks)]
    got = host(cb.rotate_hoisted(ctx, keys, dev(ct)))
    want = oracle.hybrid_rotate_hoisted(ql, p, keys_ref, ks, 20, ct)
    assert np.array_equal(got[0], want)
    for g, k in enumerate(ks):
        assert np.array_equal(got[0, g], oracle.hybrid_rotate(ql, p, keys_ref[g], k, 20, ct))
    for g, r in enumerate(steps):
        dec = oracle.decode(ql, oracle.decrypt(ql, s, got[0, g]), scale)
        assert rel_l2(dec, np.roll(slots, -r)) < 1e-6
    dec = oracle.decode(ql, oracle.decrypt(ql, s, got[0, -1]), scale)
    assert rel_l2(dec, np.conj(slots)) < 1e-6
    hh = cb.rotate_hoisted_host(ctx, keys, ct)
    assert np.array_equal(hh, got)


def test_rnsblock_rotation(oracle, cuda, small):
    n, q, p, ctx = small
    rng = np.random.default_rng(31)
    s = rng.integers(-1, 2, n).astype(np.int8)
    scale = 2.0 ** 40
    slots, ct = encode_encrypt(oracle, q, s, rng, scale, seed=8)
    blocks = [2, 2]
    ks = [ctx.rotation_exponent_left(1), ctx.rotation_exponent_left(9)]
    keys = [cb.KeySwitchKey.rnsblock_generate(ctx, len(q), blocks, k, s, seed=200 + i) for i, k in enumerate(ks)]
    keys_ref = [oracle.rnsblock_key(q, p, blocks, s, k, seed=200 + i) for i, k in enumerate(ks)]
    for key, kr in zip(keys, keys_ref):
        assert np.array_equal(key.download(), kr.ravel())
    got = host(cb.rotate(ctx, keys[0], dev(ct)))
    want = oracle.rnsblock_rotate(q, p, blocks, keys_ref[0], ks[0], ct)
    assert np.array_equal(got, want)
    hoisted = host(cb.rotate_hoisted(ctx, keys, dev(ct)))
    for g, k in enumerate(ks):
        assert np.array_equal(hoisted[0, g], oracle.rnsblock_rotate(q, p, blocks, keys_ref[g], k, ct))
    dec = oracle.decode(q, oracle.decrypt(q, s, got), scale)
    assert rel_l2(dec, np.roll(slots, -1)) < 1e-6


def test_relin_key_generation(oracle, cuda, small):
    n, q, p, ctx = small
    rng = np.random.default_rng(41)
    s = rng.integers(-1, 2, n).astype(np.int8)
    key = cb.KeySwitchKey.relin_generate(ctx, len(q), 20, s, seed=7)
    ref = oracle.relin_key(q, s, 20, seed=7)  # coefficient domain [D][2][L][N]
    want = oracle.ntt_forward(q, ref.reshape(-1, len(q), n))
    assert np.array_equal(key.download(), want.ravel())
    up = cb.KeySwitchKey.relin_upload(ctx, len(q), 20, ref)
    assert np.array_equal(up.download(), want.ravel())


def test_key_errors(oracle, cuda, small):
    n, q, p, ctx = small
    s = np.ones(n, np.int8)
    with pytest.raises(cb.CkksError) as e:
        cb.KeySwitchKey.hybrid_generate(ctx, len(q), 20, 4, s, seed=1)  # even exponent
    assert e.value.status == -1
    with pytest.raises(cb.CkksError) as e:
        cb.KeySwitchKey.rnsblock_generate(ctx, len(q), [2, 1], 5, s, seed=1)  # blocks do not cover Q
    assert e.value.status == -2
    k1 = cb.KeySwitchKey.hybrid_generate(ctx, 4, 20, 5, s, seed=1)
    k2 = cb.KeySwitchKey.hybrid_generate(ctx, 3, 20, 5, s, seed=1)
    import torch
    ct = torch.zeros((2, 4, n), dtype=torch.int64, device="cuda")
    with pytest.raises(cb.CkksError) as e:
        cb.rotate_hoisted(ctx, [k1, k2], ct)
    assert e.value.status == -2


@pytest.mark.parametrize("base_log", [4, 8, 32])
def test_hoisted_ntt_domain_corrections(oracle, cuda, small, base_log):
    # NTT-domain hoisting must equal the reference's digit-level hoisting word
    # for word, including coefficients whose digits hit -B/2 (frequent for
    # small bases; base 2^4 also overflows the correction lists and takes the
    # exact fallback).
    n, q, p, ctx = small
    rng = np.random.default_rng(50 + base_log)
    s = rng.integers(-1, 2, n).astype(np.int8)
    cts = np.stack([encode_encrypt(oracle, q, s, rng, 2.0 ** 40, seed=60 + i)[1] for i in range(5)])
    Q = 1
    for m in q:
        Q *= m
    # plant values whose balanced digits contain -B/2 in the first ciphertext's a-part
    for c in range(0, n, 7):
        v = (Q - (1 << (base_log - 1)) * (1 + (c % 3) * (1 << base_log))) % Q
        cts[0, 1, :, c] = [v % m for m in q]
    ks = [ctx.rotation_exponent_left(r) for r in (1, 3, 16)] + [2 * n - 1]
    keys_ref = [oracle.hybrid_key(q, p, s, k, base_log, seed=300 + i) for i, k in enumerate(ks)]
    keys = [cb.KeySwitchKey.hybrid_upload(ctx, len(q), base_log, k, kr) for k, kr in zip(ks, keys_ref)]
    got = host(cb.rotate_hoisted(ctx, keys, dev(cts)))
    for i in range(len(cts)):
        want = oracle.hybrid_rotate_hoisted(q, p, keys_ref, ks, base_log, cts[i])
        assert np.array_equal(got[i], want), i


@pytest.mark.parametrize("base_log,q_bits", [(8, 50), (32, 50), (20, 40)])
def test_tensor_core_mac_equals_cuda_core_mac(oracle, cuda, base_log, q_bits):
    """The INT8 tensor-core key-switch MAC and the CUDA-core MAC give the same
    words: 16 ciphertexts x 40 Galois keys (two key chunks, the second partial)
    at N=2^12, plus an oracle check of a few (ciphertext, key) pairs. 40-bit
    primes take the epilogue's general 128-bit reduction, 50/60-bit ones the
    two-half form."""
    log_n, n = 12, 1 << 12
    q = [int(x) for x in oracle.primes_below_bits(q_bits, n, 6)]
    p = [int(x) for x in oracle.primes_below_bits(60, n, 2)]
    ctx = cb.Context(log_n, q, p)
    rng = np.random.default_rng(70 + base_log + q_bits)
    s = rng.integers(-1, 2, n).astype(np.int8)
    ks = [ctx.rotation_exponent_left(r) for r in range(1, 41)]
    keys = [cb.KeySwitchKey.hybrid_generate(ctx, len(q), base_log, k, s, seed=900 + i) for i, k in enumerate(ks)]
    cts = np.stack([np.stack([np.stack([rng.integers(0, m, n, dtype=np.uint64) for m in q]) for _ in range(2)])
                    for _ in range(16)])
    assert ctx.tensor_cores
    tc = host(cb.rotate_hoisted(ctx, keys, dev(cts)))
    ctx.tensor_cores = False
    assert not ctx.tensor_cores
    cc = host(cb.rotate_hoisted(ctx, keys, dev(cts)))
    ctx.tensor_cores = True
    assert np.array_equal(tc, cc)
    for c, g in ((0, 0), (15, 39), (7, 33)):
        want = oracle.hybrid_rotate(q, p, keys[g].download(), ks[g], base_log, cts[c])
        assert np.array_equal(tc[c, g], want), (c, g)


def test_tensor_core_mac_corrections_bit_exact(oracle, cuda):
    """Tensor-core path (17 keys or more) with planted -B/2 digits: the carry
    corrections of the NTT-domain hoisting are applied in the tensor-core
    epilogue and the words equal the oracle's and the CUDA-core MAC's."""
    log_n, n, base_log = 12, 1 << 12, 32
    q = [int(x) for x in oracle.primes_below_bits(50, n, 4)]
    p = [int(x) for x in oracle.primes_below_bits(60, n, 1)]
    ctx = cb.Context(log_n, q, p)
    rng = np.random.default_rng(91)
    s = rng.integers(-1, 2, n).astype(np.int8)
    cts = np.stack([np.stack([np.stack([rng.integers(0, m, n, dtype=np.uint64) for m in q]) for _ in range(2)])
                    for _ in range(3)])
    Q = 1
    for m in q:
        Q *= m
    for c in range(0, n, 5):  # a-part values whose balanced digits contain -B/2
        v = (Q - (1 << (base_log - 1)) * (1 + (c % 3) * (1 << base_log))) % Q
        cts[0, 1, :, c] = [v % m for m in q]
    ks = [ctx.rotation_exponent_left(r) for r in range(1, 18)] + [2 * n - 1]
    keys = [cb.KeySwitchKey.hybrid_generate(ctx, len(q), base_log, k, s, seed=700 + i) for i, k in enumerate(ks)]
    assert ctx.tensor_cores
    tc = host(cb.rotate_hoisted(ctx, keys, dev(cts)))
    ctx.tensor_cores = False
    cc = host(cb.rotate_hoisted(ctx, keys, dev(cts)))
    ctx.tensor_cores = True
    assert np.array_equal(tc, cc)
    for c, g in ((0, 0), (0, 17), (0, 9), (2, 3)):
        want = oracle.hybrid_rotate(q, p, keys[g].download(), ks[g], base_log, cts[c])
        assert np.array_equal(tc[c, g], want), (c, g)


def test_packed_key_sets_follow_key_lifetimes(oracle, cuda):
    """The tensor-core MAC's packed key set is rebuilt when a key of the list is
    destroyed and a new one takes its place (the cache never serves a stale set)."""
    log_n, n, base_log = 12, 1 << 12, 32
    q = [int(x) for x in oracle.primes_below_bits(50, n, 3)]
    p = [int(x) for x in oracle.primes_below_bits(60, n, 1)]
    ctx = cb.Context(log_n, q, p)
    rng = np.random.default_rng(123)
    s = rng.integers(-1, 2, n).astype(np.int8)
    cts = np.stack([np.stack([np.stack([rng.integers(0, m, n, dtype=np.uint64) for m in q]) for _ in range(2)])
                    for _ in range(2)])
    ks = [ctx.rotation_exponent_left(r) for r in range(1, 19)]
    keys = [cb.KeySwitchKey.hybrid_generate(ctx, len(q), base_log, k, s, seed=40 + i) for i, k in enumerate(ks)]
    first = host(cb.rotate_hoisted(ctx, keys, dev(cts)))
    for trial in range(2):
        keys[5].close()  # frees the key and every packed set that holds it
        keys[5] = cb.KeySwitchKey.hybrid_generate(ctx, len(q), base_log, ks[5], s, seed=1000 + trial)
        got = host(cb.rotate_hoisted(ctx, keys, dev(cts)))
        want5 = oracle.hybrid_rotate(q, p, keys[5].download(), ks[5], base_log, cts[1])
        assert np.array_equal(got[1, 5], want5)
        assert np.array_equal(got[:, :5], first[:, :5]) and np.array_equal(got[:, 6:], first[:, 6:])
