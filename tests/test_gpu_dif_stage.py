"""GPU parity of the packed radix-2 DIF FFT2 stage and the modulus switch.

  execute_repeated_packed_fft2_dif_stage_cp_hybrid_prepared  eblas/fft.rs:3378-3470
      direct (x) diag_d + rotate_left(x, r) (x) diag_l + rotate_right(x, r) (x) diag_r
  ..._fused_rescale                                          eblas/fft.rs:3906-4000
  mod_switch_rns_ckks_to_next                                ckks/rns_mod_switch.rs:14-58

Both stage forms must equal the oracle's composition of the reference's
hybrid rotations, plaintext products and sum (and rescale) word for word.
"""
import numpy as np
import pytest

import ckks_b200 as cb

pytestmark = pytest.mark.gpu


def dev(x):
    return cb.as_u64_tensor(x)


def host(t):
    return cb.to_numpy_u64(t)


@pytest.mark.parametrize("log_n,L,span", [(10, 5, 4), (12, 4, 64)])
def test_packed_dif_stage_bit_exact(oracle, cuda, log_n, L, span):
    n = 1 << log_n
    q = [int(x) for x in oracle.primes_below_bits(50, n, L)]
    p = [int(x) for x in oracle.primes_below_bits(60, n, 2)]
    ctx = cb.Context(log_n, q, p)
    rng = np.random.default_rng(log_n + span)
    s = rng.integers(-1, 2, n).astype(np.int8)
    base_log = 20
    ks = [ctx.rotation_exponent_left(span), ctx.rotation_exponent_right(span)]
    keys_ref = [oracle.hybrid_key(q, p, s, k, base_log, seed=400 + i) for i, k in enumerate(ks)]
    keys = [cb.KeySwitchKey.hybrid_upload(ctx, L, base_log, k, kr) for k, kr in zip(ks, keys_ref)]
    # complex-slot diagonals as plaintexts: left, right, direct
    plains = np.stack([np.stack([rng.integers(0, m, n, dtype=np.uint64) for m in q]) for _ in range(3)])
    diag_ntt = oracle.ntt_forward(q, plains)
    cts = np.stack([np.stack([np.stack([rng.integers(0, m, n, dtype=np.uint64) for m in q]) for _ in range(2)])
                    for _ in range(2)])
    plain_sum = host(cb.diag_stage(ctx, keys, dev(diag_ntt), dev(cts), rescale=False))
    resc = host(cb.diag_stage(ctx, keys, dev(diag_ntt), dev(cts), rescale=True))
    assert plain_sum.shape == (2, 2, L, n) and resc.shape == (2, 2, L - 1, n)
    for c in range(2):
        acc = oracle.mul_plain(q, cts[c], plains[2]).astype(object)
        for g in range(2):
            r = oracle.hybrid_rotate(q, p, keys_ref[g], ks[g], base_log, cts[c])
            acc = acc + oracle.mul_plain(q, r, plains[g]).astype(object)
        want = np.stack([acc[:, l] % q[l] for l in range(L)], axis=1).astype(np.uint64)
        assert np.array_equal(plain_sum[c], want), c
        assert np.array_equal(resc[c], oracle.rescale(q, want)), c
    # the rescaled form equals ckks_fft_stage
    assert np.array_equal(resc, host(cb.fft_stage(ctx, keys, dev(diag_ntt), dev(cts))))


def test_mod_switch(oracle, cuda):
    n = 1 << 11
    q = [int(x) for x in oracle.primes_below_bits(50, n, 4)]
    ctx = cb.Context(11, q)
    rng = np.random.default_rng(3)
    s = rng.integers(-1, 2, n).astype(np.int8)
    scale = 2.0 ** 40
    slots = rng.uniform(-1, 1, n // 2) + 1j * rng.uniform(-1, 1, n // 2)
    ct = oracle.encrypt(q, s, oracle.encode(slots, q, scale), seed=5)
    got = host(ctx.mod_switch(dev(ct[None])))[0]
    assert np.array_equal(got, ct[:, :3])  # the leading limbs, scale unchanged
    dec = oracle.decode(q[:3], oracle.decrypt(q[:3], s, got), scale)
    assert np.linalg.norm(dec - slots) / np.linalg.norm(slots) < 1e-6
    two = host(ctx.mod_switch(dev(np.stack([ct, ct])), limbs_out=1))
    assert np.array_equal(two[1], ct[:, :1])
    with pytest.raises(cb.CkksError):
        ctx.mod_switch(dev(ct[None]), limbs_out=5)
