"""Keys and ciphertexts made from the reference's seeded stream, on the GPU.

One ChaCha20Rng seeded with seed_from_u64 draws the ternary secret, then a
hybrid-QP Galois key (ckks/hybrid_rns_galois_key.rs:61-170), a bounded
relinearization key (grafting/bounded_key_switch.rs:28-104) and an encryption
(grafting/rns_key_switch.rs:245-387), in the reference's draw order; the
oracle's restatement of the same stream does the same on the CPU. Every key
and ciphertext word must match (tolerance zero), and both streams must end at
the same position.
"""
import numpy as np
import pytest

import ckks_b200 as cb
from oracle_lib import OracleChaCha

pytestmark = pytest.mark.gpu


def _case(oracle, log_n, q_bits, q_count, p_count):
    n = 1 << log_n
    q = [int(x) for x in oracle.primes_below_bits(q_bits, n, q_count)]
    p = [int(x) for x in oracle.primes_below_bits(60, n, p_count)]
    return n, q, p, cb.Context(log_n, q, p)


@pytest.mark.parametrize("log_n,q_count,base_log,kind,param", [
    (12, 3, 32, cb.ChaCha20Rng.GAUSSIAN, 3.2),
    (12, 3, 20, cb.ChaCha20Rng.BOUNDED_UNIFORM, 8),
    (16, 3, 32, cb.ChaCha20Rng.GAUSSIAN, 3.2),
])
def test_seeded_keys_and_encryption_match_oracle(oracle, cuda, log_n, q_count, base_log, kind, param):
    n, q, p, ctx = _case(oracle, log_n, 50, q_count, 1)
    seed = 0x9100 + log_n
    rng = cb.ChaCha20Rng.seed_from_u64(seed)
    ora = OracleChaCha(seed=seed)
    s = rng.ternary_secret(n)
    assert np.array_equal(s, ora.ternary_secret(n))

    k = ctx.rotation_exponent_left(3)
    key = cb.KeySwitchKey.hybrid_generate_rng(ctx, q_count, base_log, k, s, rng, kind, param)
    want = ora.hybrid_key(q, p, s, k, base_log, kind, param)
    assert np.array_equal(key.download().reshape(want.shape), want)

    rk = cb.KeySwitchKey.relin_generate_rng(ctx, q_count, base_log, s, rng, kind, param)
    want_r = ora.relin_key(q, s, base_log, kind, param)  # coefficient domain [D][2][L][N]
    got_r = rk.download().reshape(want_r.shape)         # stored NTT domain
    D = want_r.shape[0]
    want_r_ntt = oracle.ntt_forward(q, want_r.reshape(D * 2, q_count, n)).reshape(want_r.shape)
    assert np.array_equal(got_r, want_r_ntt)

    msg = np.stack([np.random.default_rng(3).integers(0, m, n, dtype=np.uint64) for m in q])
    ct = cb.encrypt_rng(ctx, q_count, msg, s, rng, kind, param)
    assert np.array_equal(ct, ora.encrypt(q, s, msg, kind, param))
    # decrypts to message + e: small error in every limb
    dec = oracle.decrypt(q, s, ct)
    diff = [(int(d) - int(m)) % qq for d, m, qq in zip(dec[0][:64], msg[0][:64], [q[0]] * 64)]
    assert all(v < 1000 or qq - v < 1000 for v, qq in zip(diff, [q[0]] * 64))
    # the two streams are at the same position
    assert rng.next_u64() == ora.next_u64()


def test_seeded_key_rotates_like_any_key(oracle, cuda):
    # a key from the stream drives the rotation path like a generated or uploaded key
    n, q, p, ctx = _case(oracle, 12, 50, 3, 1)
    rng = cb.ChaCha20Rng.seed_from_u64(0x9200)
    s = rng.ternary_secret(n)
    k = ctx.rotation_exponent_left(5)
    key = cb.KeySwitchKey.hybrid_generate_rng(ctx, 3, 32, k, s, rng)
    ct = np.stack([np.stack([np.random.default_rng(9).integers(0, m, n, dtype=np.uint64) for m in q])
                   for _ in range(2)])[None]
    got = cb.to_numpy_u64(cb.rotate(ctx, key, cb.as_u64_tensor(ct)))
    want = oracle.hybrid_rotate(q, p, key.download(), k, 32, ct[0])
    assert np.array_equal(got[0], want)


def test_rejects_invalid_secret_and_distribution(oracle, cuda):
    n, q, p, ctx = _case(oracle, 12, 50, 2, 1)
    rng = cb.ChaCha20Rng.seed_from_u64(1)
    with pytest.raises(cb.CkksError):
        cb.KeySwitchKey.hybrid_generate_rng(ctx, 2, 32, 5, np.zeros(n, np.int8), rng)
    s = rng.ternary_secret(n)
    with pytest.raises(cb.CkksError):
        cb.KeySwitchKey.hybrid_generate_rng(ctx, 2, 32, 5, s, rng, cb.ChaCha20Rng.GAUSSIAN, 0.0)
    with pytest.raises(cb.CkksError):
        cb.KeySwitchKey.hybrid_generate_rng(ctx, 2, 32, 4, s, rng)
