"""The oracle's Mod-PP-MM (ccmm/park.rs:1405-1434) against exact Python integers.

Pins the checker of the GPU Park product to the definition: every output is
the canonical residue of the integer dot product, for moduli up to 2^64 - 1
and entries up to 2^64 - 1 (the reference's Reference backend reduces a u128
accumulator after every term, which yields exactly that).
"""
import numpy as np
import pytest

from oracle_lib import Oracle


@pytest.mark.parametrize("q", [2, 97, 65537, 0xfffffffffffc001, 2**64 - 59, 2**64 - 1])
def test_park_oracle_is_the_exact_product(q):
    o = Oracle()
    rng = np.random.default_rng(q % 1000)
    for (r, k, c), full in (((3, 4, 5), False), ((6, 9, 2), True), ((1, 31, 1), True)):
        hi = 2**64 if full else q
        a = rng.integers(0, hi, (r, k), dtype=np.uint64)
        b = rng.integers(0, hi, (k, c), dtype=np.uint64)
        got = o.park_mod_pp_mm(a, b, q)
        for i in range(r):
            for j in range(c):
                want = sum(int(a[i, t]) * int(b[t, j]) for t in range(k)) % q
                assert int(got[i, j]) == want
