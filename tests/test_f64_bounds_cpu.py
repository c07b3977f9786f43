"""CPU tests: the exact FP64 modular butterflies of the NTT passes for
primes below 2^50 (nttf:: in csrc/ntt_core.cuh), emulated word for word with
IEEE double products (numpy float64, correctly rounded like the GPU's DMUL)
and exact integer arithmetic for the fused multiply-adds (an FMA rounds the
exact a*b + c once; here every such result is an integer below 2^53 and is
exact), plus the worst-case bound propagation of the four-stage halves.

- mulmod(Y, W) = Y W - t q exactly, congruent to Y W mod q, with
  |r| <= 0.75 q (|Y| < 2^51), <= q (|Y| < 2^52), <= 1.5 q (|Y| < 2^53);
- center(v) = v - rint(v / q) q lies within q/2 + |v| 2^-52;
- Cooley-Tukey halves of four stages from inputs below q (or centred) stay
  below 4.5 q; Gentleman-Sande halves of four stages from centred inputs stay
  below 8 q + 32 < 2^53 for q < 2^50 - 4.
"""
import random

import numpy as np

TWO53 = 1 << 53


def f(x):
    return np.float64(x)


def fma_exact(a, b, c):
    """fma(a, b, c) for doubles whose exact result is an integer below 2^53."""
    from fractions import Fraction
    v = Fraction(float(a)) * Fraction(float(b)) + Fraction(float(c))
    assert v.denominator == 1 and abs(v.numerator) < TWO53
    return f(v.numerator)


def mulmod(y, w, wp, q):
    """The device's nttf::mulmod, operation for operation."""
    h = f(y) * f(w)                                  # __dmul_rn
    l_exact = int(y) * int(w) - int(h)               # __fma_rn(y, w, -h): TwoProduct, exact
    assert abs(l_exact) < TWO53
    l = f(l_exact)
    t = np.rint(f(y) * f(wp))                        # rint(__dmul_rn(y, wp))
    r0 = fma_exact(-t, q, h)                         # __fma_rn(-t, q, h)
    r = r0 + l                                       # __dadd_rn, exact (integer below 2^53)
    assert int(r) == int(r0) + int(l)
    return int(r)


def center(v, q):
    t = np.rint(f(v) * (f(1.0) / f(q)))
    return int(fma_exact(-t, q, f(v)))


PRIMES = [(1 << 50) - (1 << 17) * 23 + 1, 0x3ffffffd20001, 0x3fffffc3c0001, (1 << 40) - 87, (1 << 30) + 3]


def band(y):
    a = abs(y)
    return 0.75 if a < (1 << 51) else 1.0 if a < (1 << 52) else 1.5


def test_mulmod_exact_and_banded():
    rng = random.Random(5)
    for q in PRIMES:
        for _ in range(3000):
            w = rng.choice([1, q - 1, q // 2, rng.randrange(q), rng.randrange(1 << 20)])
            wp = float(w) / float(q)
            lim = rng.choice([q, 2 * q, 4 * q, (1 << 51) - 1, (1 << 52) - 1, TWO53 - 1])
            lim = min(lim, TWO53 - 1)
            y = rng.choice([lim, -lim, rng.randrange(-lim, lim + 1), 0, 1])
            r = mulmod(y, w, wp, q)
            assert (r - y * w) % q == 0
            assert abs(r) <= band(y) * q, (q, y, w, r)


def test_center_bound():
    rng = random.Random(6)
    for q in PRIMES:
        for _ in range(3000):
            v = rng.randrange(-(TWO53 - 1), TWO53)
            r = center(v, q)
            assert (r - v) % q == 0
            assert abs(r) <= q / 2 + abs(v) * 2.0 ** -52


def ct_half(b0, q, stages=4):
    """Worst-case magnitude after `stages` CT stages from inputs below b0."""
    b = b0
    for _ in range(stages):
        assert b < TWO53
        b = b + band(b) * q
    return b


def gs_half(b0, q, stages=4):
    b = b0
    for _ in range(stages):
        prod = band(2 * b) * q
        b = max(2 * b, prod)
        assert b < TWO53, (q, b)
    return b


def test_network_bounds():
    q = (1 << 50) - 5  # the largest odd value the FP64 networks admit (q < 2^50 - 4)
    cen = q / 2 + 2
    # forward pass 1: canonical inputs, exchange, then the twist product
    b = ct_half(q, q)
    assert b <= 4.5 * q
    b = ct_half(cen, q)
    assert b <= 3.75 * q + 8
    assert band(b) * q <= q                          # twist output below q
    # forward pass 2 from the twist output (below q)
    assert ct_half(q, q) <= 4.5 * q and ct_half(cen, q) < TWO53
    # inverse passes: centred inputs, four GS stages, centred again
    b = gs_half(cen, q)
    assert b <= 8 * q + 32 and b < TWO53
    assert band(b) * q <= 1.5 * q                    # inverse-twist output


def test_emulated_network_matches_modular_arithmetic():
    """A 16-point merged CT half then a centred 16-point GS half on random
    residues, emulated with mulmod: every value stays below 2^53 and the
    results equal the exact modular products."""
    rng = random.Random(7)
    q = 0x3ffffffd20001
    for _ in range(40):
        x = [rng.randrange(q) for _ in range(16)]
        ref = list(x)
        ws = [rng.randrange(q) for _ in range(15)]
        for s in range(4):
            half = 16 >> (s + 1)
            for blk in range(1 << s):
                w = ws[(1 << s) + blk - 1]
                for o in range(half):
                    i, j = blk * 2 * half + o, blk * 2 * half + o + half
                    r = mulmod(x[j], w, float(w) / float(q), q)
                    x[i], x[j] = x[i] + r, x[i] - r
                    rr = ref[j] * w % q
                    ref[i], ref[j] = (ref[i] + rr) % q, (ref[i] - rr) % q
                    assert abs(x[i]) < TWO53 and abs(x[j]) < TWO53
        assert [v % q for v in x] == ref
        x = [center(v, q) for v in x]
        for s in range(4):
            t = 1 << s
            for blk in range(16 >> (s + 1)):
                w = ws[blk]
                for o in range(t):
                    i, j = blk * 2 * t + o, blk * 2 * t + o + t
                    d = x[i] - x[j]
                    x[i] = x[i] + x[j]
                    x[j] = mulmod(d, w, float(w) / float(q), q)
                    rd = (ref[i] - ref[j]) % q
                    ref[i] = (ref[i] + ref[j]) % q
                    ref[j] = rd * w % q
                    assert abs(x[i]) < TWO53 and abs(x[j]) < TWO53
        assert [v % q for v in x] == ref
