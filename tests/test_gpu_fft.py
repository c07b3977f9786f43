"""GPU parity of the encrypted radix-4 FFT stage (eblas/prepared_radix4_fft256.rs:744-822).

Each stage is sum_t multiply_plain(rotate(ct, offset_t), diag_t) followed by a
rescale, with the radix-4 decimation-in-time diagonals of
tests/r16_6b3_fft256_four_stage.rs:38-64 (spans 4, 16, 64, 256; offsets
{-3..3} x span/4). The GPU stage must equal the oracle's composition of the
reference's rotations, plaintext products, additions and rescale word for word;
four stages over base-4 digit-reversed input must decode to the FP64 DFT of
every 256-slot block.
"""
import numpy as np
import pytest

import ckks_b200 as cb

pytestmark = pytest.mark.gpu


def root(n, e):
    return np.exp(-2j * np.pi * e / n)


def reverse_base4(i, digits=4):
    r = 0
    for _ in range(digits):
        r = r * 4 + i % 4
        i //= 4
    return r


def stage_diagonals(slots, span):
    """Radix-4 DIT stage of span 4..256 as signed-offset slot diagonals:
    out[i] = sum_off diag_off[i] * in[i + off]."""
    quarter = span // 4
    diags = {}
    for i in range(slots):
        within = i % span
        p, j = within // quarter, within % quarter
        for qd in range(4):
            off = (j + qd * quarter) - within
            diags.setdefault(off, np.zeros(slots, complex))[i] = root(span, qd * j) * root(4, p * qd)
    return dict(sorted(diags.items()))


def dev(x):
    return cb.as_u64_tensor(x)


def host(t):
    return cb.to_numpy_u64(t)


@pytest.fixture(scope="module")
def setup(oracle):
    log_n, n = 10, 1 << 10
    q = [int(x) for x in oracle.primes_below_bits(50, n, 6)]
    p = [int(x) for x in oracle.primes_below_bits(60, n, 2)]
    ctx = cb.Context(log_n, q, p)
    rng = np.random.default_rng(5)
    s = rng.integers(-1, 2, n).astype(np.int8)
    return n, q, p, ctx, s


def prepare_stage(oracle, ctx, q, p, s, span, level_limbs, base_log, seed):
    n = ctx.n
    ql = q[:level_limbs]
    diags = stage_diagonals(n // 2, span)
    plain_scale = float(ql[-1])
    offsets = [o for o in diags if o != 0]
    exps = [ctx.rotation_exponent_left(o) if o > 0 else ctx.rotation_exponent_right(-o) for o in offsets]
    keys_ref = [oracle.hybrid_key(ql, p, s, k, base_log, seed=seed + i) for i, k in enumerate(exps)]
    keys = [cb.KeySwitchKey.hybrid_upload(ctx, level_limbs, base_log, k, kr) for k, kr in zip(exps, keys_ref)]
    plains = {o: oracle.encode(diags[o], ql, plain_scale) for o in diags}
    diag_ntt = np.stack([oracle.ntt_forward(ql, plains[o].copy()) for o in offsets + [0]])
    return offsets, exps, keys, keys_ref, plains, diag_ntt, plain_scale


def oracle_stage(oracle, ql, p, offsets, exps, keys_ref, plains, base_log, ct):
    acc = oracle.mul_plain(ql, ct, plains[0])
    for o, k, kr in zip(offsets, exps, keys_ref):
        term = oracle.mul_plain(ql, oracle.hybrid_rotate(ql, p, kr, k, base_log, ct), plains[o])
        for l, m in enumerate(ql):
            acc[:, l] = (acc[:, l].astype(object) + term[:, l].astype(object)) % m
    acc = acc.astype(np.uint64)
    return oracle.rescale(ql, acc)


def test_fft_stage_bit_exact(oracle, cuda, setup):
    n, q, p, ctx, s = setup
    rng = np.random.default_rng(8)
    L, base_log = 6, 20
    offsets, exps, keys, keys_ref, plains, diag_ntt, _ = prepare_stage(oracle, ctx, q, p, s, 16, L, base_log, 40)
    cts = np.stack([np.stack([np.stack([rng.integers(0, m, n, dtype=np.uint64) for m in q]) for _ in range(2)])
                    for _ in range(3)])
    got = host(cb.fft_stage(ctx, keys, dev(diag_ntt), dev(cts)))
    assert got.shape == (3, 2, L - 1, n)
    for c in (0, 2):
        want = oracle_stage(oracle, q, p, offsets, exps, keys_ref, plains, base_log, cts[c])
        assert np.array_equal(got[c], want), c
    # without the identity term: only the rotated diagonals
    got2 = host(cb.fft_stage(ctx, keys, dev(diag_ntt[:-1]), dev(cts[:1]), identity=False))
    acc = None
    for o, k, kr in zip(offsets, exps, keys_ref):
        term = oracle.mul_plain(q, oracle.hybrid_rotate(q, p, kr, k, base_log, cts[0]), plains[o]).astype(object)
        acc = term if acc is None else acc + term
    acc = np.stack([acc[:, l] % m for l, m in enumerate(q)], axis=1).astype(np.uint64)
    assert np.array_equal(got2[0], oracle.rescale(q, acc))


def test_fft256_four_stages_decode_to_dft(oracle, cuda, setup):
    n, q, p, ctx, s = setup
    rng = np.random.default_rng(9)
    slots = n // 2
    base_log = 20
    x = rng.uniform(0, 1, slots) + 0j
    # base-4 digit-reversed input within each 256-slot block
    xr = np.array([x[(i // 256) * 256 + reverse_base4(i % 256)] for i in range(slots)])
    scale = 2.0 ** 40
    ct = oracle.encrypt(q, s, oracle.encode(xr, q, scale), seed=3)
    cur = dev(ct[None])
    level = len(q)
    for stage, span in enumerate((4, 16, 64, 256)):
        offsets, exps, keys, keys_ref, plains, diag_ntt, plain_scale = prepare_stage(
            oracle, ctx, q, p, s, span, level, base_log, 500 + 10 * stage)
        cur = cb.fft_stage(ctx, keys, dev(diag_ntt), cur)
        level -= 1
    ql = q[:level]
    # each stage multiplies the scale by plain_scale = q_{level-1} and rescales by it
    dec = oracle.decode(ql, oracle.decrypt(ql, s, host(cur)[0]), scale)
    want = np.concatenate([np.fft.fft(x[b * 256:(b + 1) * 256]) for b in range(slots // 256)])
    err = np.linalg.norm(dec - want) / np.linalg.norm(want)
    assert err < 1e-6, err


def test_cross_ciphertext_stage_bit_exact(oracle, cuda):
    """fft_stage_multi over two ciphertexts (the last column stage of the 2-D
    FFT) equals the oracle's rotations, plaintext products, sums and rescale."""
    from ckks_b200 import fft2
    log_n, n = 12, 1 << 12
    q = [int(x) for x in oracle.primes_below_bits(50, n, 3)]
    p = [int(x) for x in oracle.primes_below_bits(60, n, 1)]
    ctx = cb.Context(log_n, q, p)
    rng = np.random.default_rng(4)
    s = rng.integers(-1, 2, n).astype(np.int8)
    k = ctx.rotation_exponent_left(n // 4)
    key_ref = oracle.hybrid_key(q, p, s, k, 20, seed=9)
    key = cb.KeySwitchKey.hybrid_upload(ctx, 3, 20, k, key_ref)
    terms = fft2.cross_stage_terms(64)
    plains = [oracle.encode(t[3], q, float(q[-1])) for t in terms]
    diag_ntt = np.stack([oracle.ntt_forward(q, x.copy()) for x in plains])
    cts = np.stack([np.stack([np.stack([rng.integers(0, m, n, dtype=np.uint64) for m in q]) for _ in range(2)])
                    for _ in range(2)])
    tl = [(a, b, 0 if rot else 1) for a, b, rot, _ in terms]
    got = host(cb.fft_stage_multi(ctx, [key], tl, dev(diag_ntt), dev(cts), 2))
    rotated = [oracle.hybrid_rotate(q, p, key_ref, k, 20, cts[b]) for b in range(2)]
    for a in range(2):
        acc = None
        for (aa, b, rot, _), pl in zip(terms, plains):
            if aa != a:
                continue
            src = rotated[b] if rot else cts[b]
            t = oracle.mul_plain(q, src, pl).astype(object)
            acc = t if acc is None else acc + t
        acc = np.stack([acc[:, l] % m for l, m in enumerate(q)], axis=1).astype(np.uint64)
        assert np.array_equal(got[a], oracle.rescale(q, acc)), a


def test_fft2_image_decodes_to_dft2(oracle, cuda):
    """64 x 64 image in two ciphertexts at N=2^12: 3 row + 3 column radix-4
    stages decode to numpy's 2-D DFT."""
    from ckks_b200 import fft2
    log_n, n, S = 12, 1 << 12, 64
    q = [int(x) for x in oracle.primes_below_bits(50, n, 8)]
    p = [int(x) for x in oracle.primes_below_bits(60, n, 2)]
    ctx = cb.Context(log_n, q, p)
    rng = np.random.default_rng(6)
    s = rng.integers(-1, 2, n).astype(np.int8)
    plan = fft2.Fft2Plan(ctx, S, len(q), s, base_log=20)
    assert plan.out_level == len(q) - 6
    img = rng.uniform(0, 1, (S, S))
    scale = 2.0 ** 40
    packed = fft2.pack_image(img)
    cts = np.stack([oracle.encrypt(q, s, oracle.encode(packed[c], q, scale), seed=20 + c) for c in range(2)])
    out = host(plan.apply(dev(cts[None]))[0])
    ql = q[:plan.out_level]
    slots = np.stack([oracle.decode(ql, oracle.decrypt(ql, s, out[c]), scale) for c in range(2)])
    spec = fft2.unpack_spectrum(slots)
    want = np.fft.fft2(img)
    err = np.linalg.norm(spec - want) / np.linalg.norm(want)
    assert err < 1e-6, err


def test_fft2_several_images_in_one_call_match_one_by_one(oracle, cuda):
    """Three images through one apply (the cross stage rotates all six
    ciphertexts in one hoisted group) give the same words as three
    single-image applies."""
    import torch
    from ckks_b200 import fft2
    log_n, n, S = 12, 1 << 12, 64
    q = [int(x) for x in oracle.primes_below_bits(50, n, 8)]
    p = [int(x) for x in oracle.primes_below_bits(60, n, 2)]
    ctx = cb.Context(log_n, q, p)
    rng = np.random.default_rng(16)
    s = rng.integers(-1, 2, n).astype(np.int8)
    plan = fft2.Fft2Plan(ctx, S, len(q), s, base_log=20)
    cts = np.stack([np.stack([np.stack([rng.integers(0, m, (2, n), dtype=np.uint64) for m in q], axis=1)
                              for _ in range(2)]) for _ in range(3)])
    together = host(plan.apply(dev(cts)))
    torch.cuda.synchronize()
    for i in range(3):
        assert np.array_equal(together[i], host(plan.apply(dev(cts[i:i + 1]))[0])), i
