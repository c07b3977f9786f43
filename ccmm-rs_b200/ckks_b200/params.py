"""Parameter sets of the benchmarked configurations and the prime search
behind them (host-side, through the library's C ABI:
ckks_primes_below_bits / ckks_find_negacyclic_root / ckks_is_prime).

Prime chains follow the reference's own search: NTT-friendly primes
q = 1 mod 2N descending from 2^bits - 1 in steps of 2N, deterministic
Miller-Rabin (ring/ntt_prime.rs:65-94, security/p6a/generate_candidates.py:53-73).
A chain draws its primes of each bit size in order from one pool per size,
Q limbs first and then the auxiliary P limbs, so a 60-bit P after a 60-bit
q0 is the second 60-bit prime (ckks/parameters.rs:345-362 and the
N=4096 chain of the reference's multiply tests).
"""
from dataclasses import dataclass, field

import numpy as np

from . import check, lib, u64p


def primes_below_bits(bits, degree, count):
    """The first `count` primes q = 1 mod 2*degree below 2^bits, descending."""
    out = np.zeros(count, np.uint64)
    check(lib().ckks_primes_below_bits(bits, degree, count, out.ctypes.data_as(u64p)))
    return [int(x) for x in out]


def negacyclic_root(q, degree):
    """Smallest-generator primitive 2N-th root (ring/ntt_params.rs:16-50); 0 if none."""
    return int(lib().ckks_find_negacyclic_root(int(q), int(degree)))


def is_prime(v):
    return bool(lib().ckks_is_prime(int(v)))


def chain(degree, q_bits, p_bits=()):
    """Q and P moduli for per-limb bit sizes, drawn in order from one
    descending pool per bit size (Q limbs first, then P)."""
    need = {}
    for b in list(q_bits) + list(p_bits):
        need[b] = need.get(b, 0) + 1
    pools = {b: primes_below_bits(b, degree, c) for b, c in need.items()}
    taken = {b: 0 for b in need}

    def take(b):
        v = pools[b][taken[b]]
        taken[b] += 1
        return v

    q = [take(b) for b in q_bits]
    p = [take(b) for b in p_bits]
    return q, p


@dataclass(frozen=True)
class ParamSet:
    """One benchmarked configuration: ring degree 2^log_n, Q and P limb bit
    sizes, the bounded gadget's base 2^base_log, the CKKS scale (log2)."""
    name: str
    log_n: int
    q_bits: tuple
    p_bits: tuple = ()
    base_log: int = 32
    log_scale: int = 50
    notes: str = field(default="", compare=False)

    @property
    def degree(self):
        return 1 << self.log_n

    def moduli(self):
        return chain(self.degree, self.q_bits, self.p_bits)

    def context(self):
        """A device context over this set's Q and P limbs."""
        from . import Context
        q, p = self.moduli()
        return Context(self.log_n, q, p)


CONFIGS = {
    "multiply": ParamSet("multiply", 12, (60, 40, 40), (60,), base_log=20, log_scale=40,
                         notes="HMult -> relinearize -> rescale -> rotate by 1, 64 ciphertext pairs"),
    "ntt": ParamSet("ntt", 16, (50,) * 32, (), base_log=32, log_scale=50,
                    notes="batched NTT/iNTT, 64 polynomials per launch"),
    "rotation": ParamSet("rotation", 16, (50,) * 24, (60,) * 3, base_log=32, log_scale=50,
                         notes="hoisted rotations, 16 ciphertexts x 32 Galois steps"),
    "ccmm": ParamSet("ccmm", 15, (50,) * 14, (60,) * 2, base_log=20, log_scale=40,
                     notes="structured encrypted CCMM, d in {16, 32, 48, 64}"),
    "fft2": ParamSet("fft2", 16, (50,) * 24, (60,) * 3, base_log=32, log_scale=50,
                     notes="encrypted 256x256 FFT2, two ciphertexts per image"),
}


def config(name):
    """The named parameter set (multiply, ntt, rotation, ccmm, fft2)."""
    try:
        return CONFIGS[name]
    except KeyError:
        raise KeyError("unknown parameter set %r (have: %s)" % (name, ", ".join(CONFIGS))) from None
