"""Parameter sets of the benchmarked configurations (host-side search through
the library's C ABI: ckks_primes_below_bits / ckks_find_negacyclic_root).

Prime chains follow the reference's own search (descending from 2^bits - 1
in steps of 2N, security/p6a/generate_candidates.py:53-73).
"""
import numpy as np

from . import lib, check, u64p


def primes_below_bits(bits, degree, count):
    out = np.zeros(count, np.uint64)
    check(lib().ckks_primes_below_bits(bits, degree, count, out.ctypes.data_as(u64p)))
    return [int(x) for x in out]


def negacyclic_root(q, degree):
    return int(lib().ckks_find_negacyclic_root(int(q), int(degree)))


def is_prime(v):
    return bool(lib().ckks_is_prime(int(v)))
