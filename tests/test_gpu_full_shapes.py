"""Word-for-word parity at the benchmarked shapes.

The other GPU tests run at N <= 2^12 with a few limbs; these run the three
headline configurations at full size and compare sampled outputs with the
oracle's restatement of the reference (tolerance zero: exact modular
arithmetic), plus every output of the tensor-core MAC against the CUDA-core
MAC on the device:

  * hoisted rotations at N=2^16, 24 x 50-bit Q + 3 x 60-bit P, bounded
    hybrid-QP gadget base 2^32 (38 digits), 16 ciphertexts x 32 Galois keys
    in one call through the tensor-core MAC
    (ckks/hybrid_rns_galois_key.rs:550-780, grafting/bounded_gadget.rs:273-312);
  * a 2 x 2 x 2 structured CCMM at N=2^15 over 14 x 50-bit limbs with the
    bounded relinearization key of base 2^20 (matrix/rns_ckks_ciphertext.rs:220-318);
  * one radix-4 diagonal stage at N=2^16, 24 + 3 limbs
    (eblas/prepared_radix4_fft256.rs:744-822).

Keys are generated on the GPU (the generator equals the oracle's word for
word, tests/test_gpu_keyswitch.py) and downloaded for the oracle.
"""
import concurrent.futures as cf

import numpy as np
import pytest

import ckks_b200 as cb

pytestmark = pytest.mark.gpu

LOG_N, L, K, BASE_LOG = 16, 24, 3, 32
STEPS = [1 << i for i in range(15)] + list(range(3, 37, 2))  # the bench's 32 Galois steps


def dev(x):
    return cb.as_u64_tensor(x)


def host(t):
    return cb.to_numpy_u64(t)


def uniform_cts(rng, q, n, count):
    return np.stack([np.stack([rng.integers(0, m, (2, n), dtype=np.uint64) for m in q], axis=1)
                     for _ in range(count)])


@pytest.fixture(scope="module")
def rot_setup(oracle):
    import torch
    n = 1 << LOG_N
    q = [int(x) for x in oracle.primes_below_bits(50, n, L)]
    p = [int(x) for x in oracle.primes_below_bits(60, n, K)]
    ctx = cb.Context(LOG_N, q, p)
    rng = np.random.default_rng(2024)
    s = rng.integers(-1, 2, n).astype(np.int8)
    exps = [ctx.rotation_exponent_left(r) for r in STEPS]
    keys = [cb.KeySwitchKey.hybrid_generate(ctx, L, BASE_LOG, k, s, seed=5000 + i) for i, k in enumerate(exps)]
    yield n, q, p, ctx, s, exps, keys
    for k in keys:
        k.close()
    ctx.close()
    torch.cuda.empty_cache()


def test_rotation_full_shape_tensor_cores_bit_exact(oracle, cuda, rot_setup):
    """16 ct x 32 keys at the benchmarked shape: tensor-core MAC == CUDA-core
    MAC on every word (compared on the device), and three sampled (ciphertext,
    key) pairs == the oracle's non-hoisted reference rotation."""
    import torch
    n, q, p, ctx, s, exps, keys = rot_setup
    rng = np.random.default_rng(7)
    cts_h = uniform_cts(rng, q, n, 16)
    cts = dev(cts_h)
    assert keys[0].info()[0] == 38
    ctx.tensor_cores = True
    tc = cb.rotate_hoisted(ctx, keys, cts)
    torch.cuda.synchronize()
    assert ctx.last_mac_path == "tensor_cores"
    pairs = [(0, 0), (9, 17), (15, 31)]
    got = {pr: host(tc[pr[0], pr[1]]) for pr in pairs}
    ctx.tensor_cores = False
    cc = cb.rotate_hoisted(ctx, keys, cts)
    torch.cuda.synchronize()
    ctx.tensor_cores = True
    assert ctx.last_mac_path is not None
    assert torch.equal(tc, cc)
    del tc, cc
    torch.cuda.empty_cache()

    def ref(pr):
        c, g = pr
        return oracle.hybrid_rotate(q, p, keys[g].download(), exps[g], BASE_LOG, cts_h[c])

    with cf.ThreadPoolExecutor(len(pairs)) as ex:
        want = list(ex.map(ref, pairs))
    for pr, w in zip(pairs, want):
        assert np.array_equal(got[pr], w), pr


def test_rotation_full_shape_back_to_back_calls(cuda, rot_setup):
    """Two hoisted calls issued back to back on one stream without a
    synchronisation in between (the call returns while its last inverse
    transforms and ModDown are in flight) give the same words as a
    synchronised call."""
    import torch
    n, q, p, ctx, s, exps, keys = rot_setup
    rng = np.random.default_rng(8)
    a, b = dev(uniform_cts(rng, q, n, 3)), dev(uniform_cts(rng, q, n, 3))
    ka = keys[:8]
    out_a = cb.rotate_hoisted(ctx, ka, a)
    out_b = cb.rotate_hoisted(ctx, ka, b)
    torch.cuda.synchronize()
    ref_a = cb.rotate_hoisted(ctx, ka, a)
    torch.cuda.synchronize()
    ref_b = cb.rotate_hoisted(ctx, ka, b)
    torch.cuda.synchronize()
    assert torch.equal(out_a, ref_a) and torch.equal(out_b, ref_b)


def test_rotation_two_groups_partial_last(oracle, cuda):
    """17 ciphertexts on the tensor-core path: one full group of 16 and a
    partial group of 1, sharing the status read-back buffer; every word equals
    the CUDA-core MAC and sampled pairs equal the oracle."""
    import torch
    log_n, n = 12, 1 << 12
    q = [int(x) for x in oracle.primes_below_bits(50, n, 4)]
    p = [int(x) for x in oracle.primes_below_bits(60, n, 2)]
    ctx = cb.Context(log_n, q, p)
    rng = np.random.default_rng(17)
    s = rng.integers(-1, 2, n).astype(np.int8)
    ks = [ctx.rotation_exponent_left(r) for r in range(1, 21)]
    keys = [cb.KeySwitchKey.hybrid_generate(ctx, len(q), 32, k, s, seed=60 + i) for i, k in enumerate(ks)]
    cts_h = uniform_cts(rng, q, n, 17)
    cts = dev(cts_h)
    tc = cb.rotate_hoisted(ctx, keys, cts)
    torch.cuda.synchronize()
    assert ctx.last_mac_path == "tensor_cores"
    ctx.tensor_cores = False
    cc = cb.rotate_hoisted(ctx, keys, cts)
    torch.cuda.synchronize()
    assert ctx.last_mac_path == "cuda_cores"
    ctx.tensor_cores = True
    assert torch.equal(tc, cc)
    for c, g in ((16, 0), (16, 19), (3, 7)):
        want = oracle.hybrid_rotate(q, p, keys[g].download(), ks[g], 32, cts_h[c])
        assert np.array_equal(host(tc[c, g]), want), (c, g)


def test_ccmm_full_ring_bit_exact(oracle, cuda):
    """2 x 2 x 2 structured CCMM at the CCMM benchmark's ring (N=2^15, 14 x
    50-bit limbs, relinearization base 2^20) == the oracle's composition of
    tensor, sum, bounded relinearization and rescale."""
    import torch
    log_n, n, Lc, base_log = 15, 1 << 15, 14, 20
    q = [int(x) for x in oracle.primes_below_bits(50, n, Lc)]
    ctx = cb.Context(log_n, q)
    rng = np.random.default_rng(15)
    s = rng.integers(-1, 2, n).astype(np.int8)
    key = cb.KeySwitchKey.relin_generate(ctx, Lc, base_log, s, seed=9)
    key_ntt = key.download().reshape(-1, Lc, n)
    key_ref = oracle.ntt_inverse(q, key_ntt).reshape(-1, 2, Lc, n)  # the reference's coefficient layout
    m = kk = nc = 2
    A, B = uniform_cts(rng, q, n, m * kk), uniform_cts(rng, q, n, kk * nc)
    got = host(cb.matmul_structured(ctx, key, dev(A), dev(B), m, kk, nc)).reshape(nc * m, 2, Lc - 1, n)
    torch.cuda.synchronize()

    def entry(rc):
        r, c = rc
        acc = None
        for t in range(kk):
            tt = oracle.tensor(q, A[r + t * m], B[t + c * kk]).astype(object)
            acc = tt if acc is None else acc + tt
        quad = np.stack([acc[:, l] % q[l] for l in range(Lc)], axis=1).astype(np.uint64)
        rel = oracle.relinearize(q, quad, key_ref, base_log)
        return oracle.rescale(q, rel.reshape(2, Lc, n))

    with cf.ThreadPoolExecutor(4) as ex:
        want = list(ex.map(entry, [(r, c) for c in range(nc) for r in range(m)]))
    for i, w in enumerate(want):
        assert np.array_equal(got[i], w), i
    ctx.close()


def test_fft_stage_full_shape_bit_exact(oracle, cuda):
    """One radix-4 diagonal stage (span 16: offsets -3..3, six rotations) at
    N=2^16 over 24 + 3 limbs with base 2^32 == the oracle's composition of
    hybrid rotations, plaintext products, sums and rescale."""
    import torch
    n = 1 << LOG_N
    q = [int(x) for x in oracle.primes_below_bits(50, n, L)]
    p = [int(x) for x in oracle.primes_below_bits(60, n, K)]
    ctx = cb.Context(LOG_N, q, p)
    rng = np.random.default_rng(33)
    s = rng.integers(-1, 2, n).astype(np.int8)
    offsets = [-12, -8, -4, 4, 8, 12]
    exps = [ctx.rotation_exponent_left(o) if o > 0 else ctx.rotation_exponent_right(-o) for o in offsets]
    keys = [cb.KeySwitchKey.hybrid_generate(ctx, L, BASE_LOG, k, s, seed=800 + i) for i, k in enumerate(exps)]
    plains = np.stack([np.stack([rng.integers(0, m, n, dtype=np.uint64) for m in q]) for _ in range(7)])
    plains_ntt = oracle.ntt_forward(q, plains)
    ct = uniform_cts(rng, q, n, 1)
    got = host(cb.fft_stage(ctx, keys, dev(plains_ntt), dev(ct)))[0]
    torch.cuda.synchronize()
    keys_ref = [k.download() for k in keys]

    def rot_term(i):
        r = oracle.hybrid_rotate(q, p, keys_ref[i], exps[i], BASE_LOG, ct[0])
        return oracle.mul_plain(q, r, plains[i])

    with cf.ThreadPoolExecutor(6) as ex:
        terms = list(ex.map(rot_term, range(6)))
    acc = oracle.mul_plain(q, ct[0], plains[6]).astype(object)
    for t in terms:
        acc = acc + t.astype(object)
    acc = np.stack([acc[:, l] % q[l] for l in range(L)], axis=1).astype(np.uint64)
    want = oracle.rescale(q, acc)
    assert np.array_equal(got, want)
    for k in keys:
        k.close()
    ctx.close()
