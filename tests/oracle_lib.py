"""ctypes loader for the CPU oracle (oracle/ckks_oracle.cpp).

Test infrastructure only: tests, the smoke check and bench.py's CPU-baseline
leg load this; the product library never does.
"""
import ctypes
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(ROOT, "oracle", "_build", "libckks_oracle.so")

u64p = ctypes.POINTER(ctypes.c_uint64)
i64p = ctypes.POINTER(ctypes.c_int64)
i8p = ctypes.POINTER(ctypes.c_int8)
u32p = ctypes.POINTER(ctypes.c_uint32)
f64p = ctypes.POINTER(ctypes.c_double)
U32, U64, I32, F64 = ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int32, ctypes.c_double

_SIGS = {
    "oracle_is_prime": (I32, [U64]),
    "oracle_find_ntt_prime_below_bits": (U64, [U32, U32]),
    "oracle_primes_below_bits": (I32, [U32, U32, U32, u64p]),
    "oracle_find_negacyclic_root": (U64, [U64, U32]),
    "oracle_pow_mod": (U64, [U64, U64, U64]),
    "oracle_shoup_quotient": (U64, [U64, U64]),
    "oracle_shoup_mul": (U64, [U64, U64, U64, U64]),
    "oracle_barrett_mul": (U64, [U64, U64, U64]),
    "oracle_ntt_forward_reference": (None, [U64, U32, u64p, u64p]),
    "oracle_ntt_inverse_reference": (None, [U64, U32, u64p, u64p]),
    "oracle_ntt_forward": (None, [u64p, U32, U32, u64p, U32]),
    "oracle_ntt_inverse": (None, [u64p, U32, U32, u64p, U32]),
    "oracle_negacyclic_mul": (None, [u64p, U32, U32, u64p, u64p, u64p]),
    "oracle_pointwise_mul": (None, [u64p, U32, U32, u64p, u64p, u64p, U32]),
    "oracle_rotation_exponent_left": (U64, [U32, U64]),
    "oracle_rotation_exponent_right": (U64, [U32, U64]),
    "oracle_automorphism_coef": (None, [u64p, U32, U32, U64, u64p, u64p, U32]),
    "oracle_automorphism_ntt": (None, [U32, U32, U64, u64p, u64p, U32]),
    "oracle_rescale": (None, [u64p, U32, U32, u64p, u64p, U32]),
    "oracle_mod_down": (None, [u64p, U32, u64p, U32, U32, u64p, u64p, U32]),
    "oracle_crt_words": (U32, [u64p, U32]),
    "oracle_crt_reconstruct": (None, [u64p, U32, U32, u64p, u64p]),
    "oracle_bounded_digit_count": (U32, [u64p, U32, U32]),
    "oracle_bounded_decompose": (None, [u64p, U32, U32, U32, u64p, i64p]),
    "oracle_bounded_automorphism_hoisted": (None, [U32, U32, U32, U64, i64p, i64p]),
    "oracle_rns_block_words": (U32, [u64p, u32p, U32]),
    "oracle_rns_block_decompose": (None, [u64p, U32, u32p, U32, U32, u64p, u64p]),
    "oracle_rng_word": (U64, [U64, U64, U64]),
    "oracle_gaussian": (ctypes.c_int64, [F64, U64, U64, U64]),
    "oracle_uniform_mod": (U64, [U64, U64, U64, U64]),
    "oracle_encrypt": (None, [u64p, U32, U32, i8p, U64, F64, u64p, u64p]),
    "oracle_decrypt": (None, [u64p, U32, U32, i8p, u64p, u64p]),
    "oracle_hybrid_key_generate": (None, [u64p, U32, u64p, U32, U32, U32, i8p, U64, U64, F64, u64p]),
    "oracle_hybrid_rotate": (None, [u64p, U32, u64p, U32, U32, U32, U64, u64p, u64p, u64p]),
    "oracle_hybrid_rotate_hoisted": (None, [u64p, U32, u64p, U32, U32, U32, U32, u64p,
                                            ctypes.POINTER(u64p), u64p, u64p]),
    "oracle_hybrid_rotate_hoisted_batch": (None, [u64p, U32, u64p, U32, U32, U32, U32, u64p,
                                                  ctypes.POINTER(u64p), U32, u64p, u64p, U32]),
    "oracle_rnsblock_key_generate": (None, [u64p, U32, u64p, U32, U32, u32p, U32, i8p, U64, U64, F64, u64p]),
    "oracle_rnsblock_rotate": (None, [u64p, U32, u64p, U32, U32, u32p, U32, U64, u64p, u64p, u64p]),
    "oracle_rns_rotate": (None, [u64p, U32, U32, u32p, U32, U64, u64p, u64p, u64p]),
    "oracle_rns_relin_key_generate": (None, [u64p, U32, U32, u32p, U32, i8p, U64, F64, u64p]),
    "oracle_rns_relinearize": (None, [u64p, U32, U32, u32p, U32, u64p, u64p, u64p]),
    "oracle_tensor": (None, [u64p, U32, U32, u64p, u64p, u64p]),
    "oracle_bounded_relin_key_generate": (None, [u64p, U32, U32, U32, i8p, U64, F64, u64p]),
    "oracle_bounded_relinearize": (None, [u64p, U32, U32, U32, u64p, u64p, u64p]),
    "oracle_mul_plain": (None, [u64p, U32, U32, u64p, u64p, u64p]),
    "oracle_chacha_new": (ctypes.c_void_p, [U64]),
    "oracle_chacha_new_from_seed": (ctypes.c_void_p, [ctypes.c_char_p]),
    "oracle_chacha_free": (None, [ctypes.c_void_p]),
    "oracle_chacha_words": (None, [ctypes.c_void_p, u32p, U64]),
    "oracle_chacha_next_u64": (U64, [ctypes.c_void_p]),
    "oracle_chacha_ternary": (None, [ctypes.c_void_p, U32, i8p]),
    "oracle_chacha_error": (None, [ctypes.c_void_p, U32, ctypes.c_int, F64, i64p]),
    "oracle_chacha_uniform": (None, [ctypes.c_void_p, U32, U64, u64p]),
    "oracle_hybrid_key_generate_chacha": (None, [u64p, U32, u64p, U32, U32, U32, i8p, U64, ctypes.c_int, F64,
                                                 ctypes.c_void_p, u64p]),
    "oracle_bounded_relin_key_generate_chacha": (None, [u64p, U32, U32, U32, i8p, ctypes.c_int, F64,
                                                        ctypes.c_void_p, u64p]),
    "oracle_encrypt_chacha": (None, [u64p, U32, U32, i8p, ctypes.c_int, F64, ctypes.c_void_p, u64p, u64p]),
    "oracle_park_mod_pp_mm": (None, [u64p, u64p, U32, U32, U32, U64, u64p]),
    "oracle_slots_to_coefficients": (None, [U32, f64p, f64p]),
    "oracle_coefficients_to_slots": (None, [U32, f64p, f64p]),
    "oracle_encode": (None, [U32, f64p, u64p, U32, F64, u64p]),
    "oracle_decode": (None, [U32, u64p, U32, u64p, F64, f64p]),
}

_lib = None


def build():
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def P(a, t=u64p):
    """Pointer to a contiguous numpy array."""
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(t)


def arr(x, dtype=np.uint64):
    return np.ascontiguousarray(np.asarray(x, dtype=dtype))


class Oracle:
    """Thin numpy-facing wrapper over the oracle's C ABI."""

    def __init__(self):
        self.L = lib()

    def primes_below_bits(self, bits, degree, count):
        out = np.zeros(count, np.uint64)
        assert self.L.oracle_primes_below_bits(bits, degree, count, P(out)) == 0
        return out

    def root(self, q, n):
        return int(self.L.oracle_find_negacyclic_root(int(q), n))

    def ntt_forward(self, moduli, data):
        moduli = arr(moduli); d = arr(data).copy()
        n = d.shape[-1]; L = len(moduli)
        self.L.oracle_ntt_forward(P(moduli), L, n, P(d), d.size // (L * n))
        return d

    def ntt_inverse(self, moduli, data):
        moduli = arr(moduli); d = arr(data).copy()
        n = d.shape[-1]; L = len(moduli)
        self.L.oracle_ntt_inverse(P(moduli), L, n, P(d), d.size // (L * n))
        return d

    def ntt_forward_reference(self, q, poly):
        poly = arr(poly); out = np.zeros_like(poly)
        self.L.oracle_ntt_forward_reference(int(q), len(poly), P(poly), P(out))
        return out

    def ntt_inverse_reference(self, q, vals):
        vals = arr(vals); out = np.zeros_like(vals)
        self.L.oracle_ntt_inverse_reference(int(q), len(vals), P(vals), P(out))
        return out

    def automorphism_coef(self, moduli, data, k):
        moduli = arr(moduli); d = arr(data); out = np.zeros_like(d)
        n = d.shape[-1]; L = len(moduli)
        self.L.oracle_automorphism_coef(P(moduli), L, n, int(k), P(d), P(out), d.size // (L * n))
        return out

    def automorphism_ntt(self, limbs, data, k):
        d = arr(data); out = np.zeros_like(d); n = d.shape[-1]
        self.L.oracle_automorphism_ntt(limbs, n, int(k), P(d), P(out), d.size // (limbs * n))
        return out

    def rescale(self, moduli, data):
        moduli = arr(moduli); d = arr(data); L = len(moduli); n = d.shape[-1]
        npoly = d.size // (L * n)
        out = np.zeros((npoly, L - 1, n), np.uint64)
        self.L.oracle_rescale(P(moduli), L, n, P(d), P(out), npoly)
        return out.reshape(d.shape[:-2] + (L - 1, n))

    def mod_down(self, q, p, data):
        q = arr(q); p = arr(p); d = arr(data); L, K = len(q), len(p); n = d.shape[-1]
        npoly = d.size // ((L + K) * n)
        out = np.zeros((npoly, L, n), np.uint64)
        self.L.oracle_mod_down(P(q), L, P(p), K, n, P(d), P(out), npoly)
        return out.reshape(d.shape[:-2] + (L, n))

    def crt(self, moduli, poly):
        moduli = arr(moduli); poly = arr(poly); L = len(moduli); n = poly.shape[-1]
        w = self.L.oracle_crt_words(P(moduli), L)
        out = np.zeros((n, w), np.uint64)
        self.L.oracle_crt_reconstruct(P(moduli), L, n, P(poly), P(out))
        return [sum(int(v) << (64 * i) for i, v in enumerate(row)) for row in out]

    def digit_count(self, moduli, base_log):
        moduli = arr(moduli)
        return int(self.L.oracle_bounded_digit_count(P(moduli), len(moduli), base_log))

    def bounded_decompose(self, moduli, poly, base_log):
        moduli = arr(moduli); poly = arr(poly); n = poly.shape[-1]
        D = self.digit_count(moduli, base_log)
        out = np.zeros((D, n), np.int64)
        self.L.oracle_bounded_decompose(P(moduli), len(moduli), n, base_log, P(poly), P(out, i64p))
        return out

    def bounded_automorphism_hoisted(self, digits, base_log, k):
        d = arr(digits, np.int64); out = np.zeros_like(d)
        self.L.oracle_bounded_automorphism_hoisted(d.shape[0], d.shape[1], base_log, int(k), P(d, i64p), P(out, i64p))
        return out

    def rns_block_decompose(self, moduli, block_sizes, poly):
        moduli = arr(moduli); bs = arr(block_sizes, np.uint32); poly = arr(poly); n = poly.shape[-1]
        w = self.L.oracle_rns_block_words(P(moduli), P(bs, u32p), len(bs))
        out = np.zeros((len(bs), n, w), np.uint64)
        self.L.oracle_rns_block_decompose(P(moduli), len(moduli), P(bs, u32p), len(bs), n, P(poly), P(out))
        return [[sum(int(v) << (64 * i) for i, v in enumerate(row)) for row in blk] for blk in out]

    def encrypt(self, moduli, secret, message, seed, sigma=3.2):
        moduli = arr(moduli); s = arr(secret, np.int8); m = arr(message); L = len(moduli); n = m.shape[-1]
        ct = np.zeros((2, L, n), np.uint64)
        self.L.oracle_encrypt(P(moduli), L, n, P(s, i8p), seed, sigma, P(m), P(ct))
        return ct

    def decrypt(self, moduli, secret, ct):
        moduli = arr(moduli); s = arr(secret, np.int8); ct = arr(ct); L = len(moduli); n = ct.shape[-1]
        m = np.zeros((L, n), np.uint64)
        self.L.oracle_decrypt(P(moduli), L, n, P(s, i8p), P(ct), P(m))
        return m

    def hybrid_key(self, q, p, secret, exponent, base_log, seed, sigma=3.2):
        q = arr(q); p = arr(p); s = arr(secret, np.int8); n = len(s)
        D = self.digit_count(q, base_log)
        key = np.zeros((D, len(q) + len(p), 2, n), np.uint64)
        self.L.oracle_hybrid_key_generate(P(q), len(q), P(p), len(p), n, base_log, P(s, i8p), int(exponent),
                                          seed, sigma, P(key))
        return key

    def hybrid_rotate(self, q, p, key, exponent, base_log, ct):
        q = arr(q); p = arr(p); key = arr(key); ct = arr(ct); n = ct.shape[-1]
        out = np.zeros((2, len(q), n), np.uint64)
        self.L.oracle_hybrid_rotate(P(q), len(q), P(p), len(p), n, base_log, int(exponent), P(key), P(ct), P(out))
        return out

    def hybrid_rotate_hoisted(self, q, p, keys, exponents, base_log, ct):
        q = arr(q); p = arr(p); ct = arr(ct); n = ct.shape[-1]
        keys = [arr(k) for k in keys]; ex = arr(exponents)
        kp = (u64p * len(keys))(*[P(k) for k in keys])
        out = np.zeros((len(keys), 2, len(q), n), np.uint64)
        self.L.oracle_hybrid_rotate_hoisted(P(q), len(q), P(p), len(p), n, base_log, len(keys), P(ex), kp,
                                            P(ct), P(out))
        return out

    def rnsblock_key(self, q, p, block_sizes, secret, exponent, seed, sigma=3.2):
        q = arr(q); p = arr(p); s = arr(secret, np.int8); bs = arr(block_sizes, np.uint32); n = len(s)
        key = np.zeros((len(bs), len(q) + len(p), 2, n), np.uint64)
        self.L.oracle_rnsblock_key_generate(P(q), len(q), P(p), len(p), n, P(bs, u32p), len(bs), P(s, i8p),
                                            int(exponent), seed, sigma, P(key))
        return key

    def rnsblock_rotate(self, q, p, block_sizes, key, exponent, ct):
        q = arr(q); p = arr(p); bs = arr(block_sizes, np.uint32); key = arr(key); ct = arr(ct); n = ct.shape[-1]
        out = np.zeros((2, len(q), n), np.uint64)
        self.L.oracle_rnsblock_rotate(P(q), len(q), P(p), len(p), n, P(bs, u32p), len(bs), int(exponent),
                                      P(key), P(ct), P(out))
        return out

    def rns_key(self, q, block_sizes, secret, exponent, seed, sigma=3.2):
        """Ordinary RNS Galois key (no P): the block key with K = 0, NTT domain [nb][L][2][N]."""
        q = arr(q); s = arr(secret, np.int8); bs = arr(block_sizes, np.uint32); n = len(s)
        key = np.zeros((len(bs), len(q), 2, n), np.uint64)
        empty = np.zeros(1, np.uint64)
        self.L.oracle_rnsblock_key_generate(P(q), len(q), P(empty), 0, n, P(bs, u32p), len(bs), P(s, i8p),
                                            int(exponent), seed, sigma, P(key))
        return key

    def rns_rotate(self, q, block_sizes, key, exponent, ct):
        q = arr(q); bs = arr(block_sizes, np.uint32); key = arr(key); ct = arr(ct); n = ct.shape[-1]
        out = np.zeros((2, len(q), n), np.uint64)
        self.L.oracle_rns_rotate(P(q), len(q), n, P(bs, u32p), len(bs), int(exponent), P(key), P(ct), P(out))
        return out

    def rns_relin_key(self, q, block_sizes, secret, seed, sigma=3.2):
        q = arr(q); s = arr(secret, np.int8); bs = arr(block_sizes, np.uint32); n = len(s)
        key = np.zeros((len(bs), 2, len(q), n), np.uint64)
        self.L.oracle_rns_relin_key_generate(P(q), len(q), n, P(bs, u32p), len(bs), P(s, i8p), seed, sigma, P(key))
        return key

    def rns_relinearize(self, q, block_sizes, quad, key):
        q = arr(q); bs = arr(block_sizes, np.uint32); quad = arr(quad); key = arr(key); n = quad.shape[-1]
        out = np.zeros((2, len(q), n), np.uint64)
        self.L.oracle_rns_relinearize(P(q), len(q), n, P(bs, u32p), len(bs), P(quad), P(key), P(out))
        return out

    def tensor(self, moduli, lhs, rhs):
        moduli = arr(moduli); lhs = arr(lhs); rhs = arr(rhs); L = len(moduli); n = lhs.shape[-1]
        out = np.zeros((3, L, n), np.uint64)
        self.L.oracle_tensor(P(moduli), L, n, P(lhs), P(rhs), P(out))
        return out

    def relin_key(self, moduli, secret, base_log, seed, sigma=3.2):
        moduli = arr(moduli); s = arr(secret, np.int8); L = len(moduli); n = len(s)
        D = self.digit_count(moduli, base_log)
        key = np.zeros((D, 2, L, n), np.uint64)
        self.L.oracle_bounded_relin_key_generate(P(moduli), L, n, base_log, P(s, i8p), seed, sigma, P(key))
        return key

    def relinearize(self, moduli, quad, key, base_log):
        moduli = arr(moduli); quad = arr(quad); key = arr(key); L = len(moduli); n = quad.shape[-1]
        out = np.zeros((2, L, n), np.uint64)
        self.L.oracle_bounded_relinearize(P(moduli), L, n, base_log, P(quad), P(key), P(out))
        return out

    def park_mod_pp_mm(self, lhs, rhs, q):
        lhs = arr(lhs); rhs = arr(rhs)
        out = np.zeros((lhs.shape[0], rhs.shape[1]), np.uint64)
        self.L.oracle_park_mod_pp_mm(P(lhs), P(rhs), lhs.shape[0], lhs.shape[1], rhs.shape[1], int(q), P(out))
        return out

    def mul_plain(self, moduli, ct, plain):
        moduli = arr(moduli); ct = arr(ct); plain = arr(plain); L = len(moduli); n = ct.shape[-1]
        out = np.zeros_like(ct)
        self.L.oracle_mul_plain(P(moduli), L, n, P(ct), P(plain), P(out))
        return out

    def encode(self, slots, moduli, scale):
        s = np.ascontiguousarray(np.stack([np.real(slots), np.imag(slots)], -1).astype(np.float64))
        moduli = arr(moduli); n = 2 * len(slots)
        out = np.zeros((len(moduli), n), np.uint64)
        self.L.oracle_encode(n, P(s, f64p), P(moduli), len(moduli), float(scale), P(out))
        return out

    def decode(self, moduli, poly, scale):
        moduli = arr(moduli); poly = arr(poly); n = poly.shape[-1]
        out = np.zeros((n // 2, 2), np.float64)
        self.L.oracle_decode(n, P(moduli), len(moduli), P(poly), float(scale), P(out, f64p))
        return out[:, 0] + 1j * out[:, 1]

    def slots_to_coefficients(self, slots):
        s = np.ascontiguousarray(np.stack([np.real(slots), np.imag(slots)], -1).astype(np.float64))
        n = 2 * len(slots); out = np.zeros(n, np.float64)
        self.L.oracle_slots_to_coefficients(n, P(s, f64p), P(out, f64p))
        return out

    def coefficients_to_slots(self, coeffs):
        c = arr(coeffs, np.float64); n = len(c); out = np.zeros((n // 2, 2), np.float64)
        self.L.oracle_coefficients_to_slots(n, P(c, f64p), P(out, f64p))
        return out[:, 0] + 1j * out[:, 1]


class OracleChaCha:
    """The oracle's restatement of the reference's ChaCha20Rng stream and samplers."""

    def __init__(self, seed=None, seed32=None):
        self.L = lib()
        self.h = self.L.oracle_chacha_new_from_seed(bytes(seed32)) if seed32 is not None else \
            self.L.oracle_chacha_new(int(seed) & (2**64 - 1))

    def words(self, n):
        out = np.zeros(n, np.uint32)
        self.L.oracle_chacha_words(self.h, P(out, u32p), n)
        return out

    def next_u64(self):
        return int(self.L.oracle_chacha_next_u64(self.h))

    def ternary_secret(self, n):
        out = np.zeros(n, np.int8)
        self.L.oracle_chacha_ternary(self.h, n, P(out, i8p))
        return out

    def error(self, n, kind, param):
        out = np.zeros(n, np.int64)
        self.L.oracle_chacha_error(self.h, n, kind, float(param), P(out, i64p))
        return out

    def uniform_residues(self, n, q):
        out = np.zeros(n, np.uint64)
        self.L.oracle_chacha_uniform(self.h, n, int(q), P(out))
        return out

    def hybrid_key(self, q, p, secret, exponent, base_log, kind=1, param=3.2):
        q = arr(q); p = arr(p); s = arr(secret, np.int8); n = len(s)
        D = int(self.L.oracle_bounded_digit_count(P(q), len(q), base_log))
        key = np.zeros((D, len(q) + len(p), 2, n), np.uint64)
        self.L.oracle_hybrid_key_generate_chacha(P(q), len(q), P(p), len(p), n, base_log, P(s, i8p), int(exponent),
                                                 kind, float(param), self.h, P(key))
        return key

    def relin_key(self, q, secret, base_log, kind=1, param=3.2):
        q = arr(q); s = arr(secret, np.int8); n = len(s)
        D = int(self.L.oracle_bounded_digit_count(P(q), len(q), base_log))
        key = np.zeros((D, 2, len(q), n), np.uint64)
        self.L.oracle_bounded_relin_key_generate_chacha(P(q), len(q), n, base_log, P(s, i8p), kind, float(param),
                                                        self.h, P(key))
        return key

    def encrypt(self, q, secret, message, kind=1, param=3.2):
        q = arr(q); s = arr(secret, np.int8); m = arr(message); n = len(s)
        ct = np.zeros((2, len(q), n), np.uint64)
        self.L.oracle_encrypt_chacha(P(q), len(q), n, P(s, i8p), kind, float(param), self.h, P(m), P(ct))
        return ct

    def __del__(self):
        try:
            self.L.oracle_chacha_free(self.h)
        except Exception:
            pass
