"""The reference's seeded sampling stream, on the host (no GPU needed).

The library's ckks_rng (host code of libckks_b200.so) and the oracle's
restatement must agree word for word; the ChaCha20 keystream itself is pinned
against an independent implementation (OpenSSL through the `cryptography`
package): with the 32-byte seed as key and a zero IV (32-bit counter 0, nonce
0), its keystream is rand_chacha's ChaCha20Rng stream for stream id 0.
seed_from_u64 (PCG32) and rand's gen_range are restated from their published
algorithms; no recorded reference stream exists to pin them further.
Reference properties restated: rlwe/uniform.rs:64-95 (residues below the
modulus, reproducible, empty sample), rlwe/secret_key.rs:58-96 (ternary,
nonzero, deterministic).
"""
import sys

import numpy as np
import pytest

from oracle_lib import OracleChaCha

sys.path.insert(0, __import__("os").path.join(__import__("os").path.dirname(__file__), "..", "ccmm-rs_b200"))
import ckks_b200 as cb  # noqa: E402


def _openssl_keystream(seed32, n_words, first_block=0):
    cryptography = pytest.importorskip("cryptography")
    del cryptography
    from cryptography.hazmat.primitives.ciphers import Cipher, algorithms
    iv = int(first_block).to_bytes(4, "little") + bytes(12)
    enc = Cipher(algorithms.ChaCha20(bytes(seed32), iv), mode=None).encryptor()
    ks = enc.update(bytes(4 * n_words))
    return np.frombuffer(ks, dtype="<u4").astype(np.uint32)


@pytest.mark.parametrize("seed32", [bytes(range(32)), bytes(32), bytes([0xA5] * 32),
                                    bytes((i * 37 + 11) & 0xFF for i in range(32))])
def test_keystream_matches_openssl(seed32):
    want = _openssl_keystream(seed32, 16 * 70)  # 70 blocks: crosses the 4-block buffer many times
    lib_rng = cb.ChaCha20Rng.from_seed(seed32)
    assert np.array_equal(lib_rng.words(len(want)), want)
    ora = OracleChaCha(seed32=seed32)
    assert np.array_equal(ora.words(len(want)), want)


def test_seed_from_u64_library_equals_oracle():
    for seed in [0, 1, 7, 42, 0xE10, 0x9100, 0xE110_A001, 2**64 - 1]:
        a = cb.ChaCha20Rng.seed_from_u64(seed).words(200)
        b = OracleChaCha(seed=seed).words(200)
        assert np.array_equal(a, b), seed


def test_mixed_u32_u64_reads_follow_the_word_stream():
    # BlockRng::next_u64 joins two words (low first), also when the pair straddles a refill
    rng = cb.ChaCha20Rng.seed_from_u64(99)
    words = cb.ChaCha20Rng.seed_from_u64(99).words(400)
    ora = OracleChaCha(seed=99)
    pos = 0
    pattern = [1, 2, 2, 1, 2, 1, 1, 2] * 30
    for width in pattern:
        if width == 1:
            v = rng.next_u32()
            assert v == int(words[pos])
            assert int(ora.words(1)[0]) == v
            pos += 1
        else:
            v = rng.next_u64()
            assert v == int(words[pos]) | (int(words[pos + 1]) << 32)
            assert ora.next_u64() == v
            pos += 2
    assert rng.word_position() == pos


@pytest.mark.parametrize("modulus", [2, 3, 17, 257, 65537, 1125899906826241, 1152921504606846883, 2**64 - 1])
def test_uniform_residues(modulus):
    lib_rng = cb.ChaCha20Rng.seed_from_u64(modulus)
    a = lib_rng.uniform_residues(4096, modulus)
    b = OracleChaCha(seed=modulus).uniform_residues(4096, modulus)
    assert np.array_equal(a, b)
    assert len(a) == 4096 and (a.astype(object) < modulus).all()
    assert cb.ChaCha20Rng.seed_from_u64(7).uniform_residues(0, 17).size == 0


def test_uniform_rejection_consumes_extra_words():
    # a modulus just above 2^63 rejects about half the candidates: the stream
    # position then runs ahead of two words per residue, identically in both
    q = 2**63 + 29
    lib_rng = cb.ChaCha20Rng.seed_from_u64(5)
    ora = OracleChaCha(seed=5)
    a = lib_rng.uniform_residues(1000, q)
    b = ora.uniform_residues(1000, q)
    assert np.array_equal(a, b)
    assert lib_rng.word_position() > 2 * 1000 + 200
    assert lib_rng.next_u64() == ora.next_u64()


def test_ternary_secret():
    for seed in [7, 42, 1234]:
        a = cb.ChaCha20Rng.seed_from_u64(seed).ternary_secret(4096)
        b = OracleChaCha(seed=seed).ternary_secret(4096)
        assert np.array_equal(a, b)
        assert set(np.unique(a)) <= {-1, 0, 1} and np.any(a != 0)
        counts = np.bincount(a + 1, minlength=3)
        assert (np.abs(counts - 4096 / 3) < 5 * np.sqrt(4096 * 2 / 9)).all()
    assert np.array_equal(cb.ChaCha20Rng.seed_from_u64(42).ternary_secret(8),
                          cb.ChaCha20Rng.seed_from_u64(42).ternary_secret(8))


@pytest.mark.parametrize("kind,param", [(1, 3.2), (1, 1.0), (1, 19.2), (0, 0), (0, 1), (0, 20), (0, 2**40)])
def test_error_samplers(kind, param):
    a = cb.ChaCha20Rng.seed_from_u64(11).error(8192, kind, param)
    b = OracleChaCha(seed=11).error(8192, kind, param)
    assert np.array_equal(a, b)
    if kind == 1:
        assert np.abs(a).max() <= int(np.ceil(16 * param))
        assert abs(a.std() - param) < 0.1 * param
        assert abs(a.mean()) < 4 * param / np.sqrt(len(a))
    else:
        assert np.abs(a).max() <= param
        if param == 0:
            assert not a.any()


def test_rejects_bad_arguments():
    rng = cb.ChaCha20Rng.seed_from_u64(1)
    with pytest.raises(cb.CkksError):
        rng.error(4, 1, -1.0)
    with pytest.raises(cb.CkksError):
        rng.error(4, 0, 0.5)
    with pytest.raises(cb.CkksError):
        rng.uniform_residues(4, 1)
    with pytest.raises(ValueError):
        cb.ChaCha20Rng.from_seed(b"short")
