"""CPU tests: the bounds that the NTT kernels' lazy arithmetic relies on,
checked with exact Python integers on the same word operations (no GPU).

- the Shoup product whose quotient comes from three of the four 32 x 32-bit
  partial products lands in [0, 4q) and is congruent to W Y mod q;
- the lazy Cooley-Tukey pass (no conditional subtraction, Y' = X - W Y + 4q)
  stays below 40 q < 2^64 for up to 9 stages from inputs below 4q, for primes
  below 2^58;
- the lazy Gentleman-Sande pass with c = 2^(s+1) q stays below 2^(m+1) q with
  the [0, 4q) product, for primes below 2^54;
- the division-free lift of a signed 64-bit digit gives d mod q.
"""
import random

M64 = (1 << 64) - 1


def shoup_quotient(w, q):
    return (w << 64) // q


def mul_shoup_lazy4(y, w, wq, q):
    y0, y1, w0, w1 = y & 0xFFFFFFFF, y >> 32, wq & 0xFFFFFFFF, wq >> 32
    hi = (y1 * w1 + ((y1 * w0) >> 32) + ((y0 * w1) >> 32)) & M64
    return (y * w - hi * q) & M64


def lift_digit(d, q):
    m = (((1 << 128) - 1) // q) >> 64  # high word of the Barrett constant floor(2^128 / q)
    a = (-d) & M64 if d < 0 else d
    r = (a - ((a * m) >> 64) * q) & M64
    assert r < 2 * q
    r = r - q if r >= q else r
    return q - r if (d < 0 and r) else r


PRIMES = [(1 << 50) - 27, (1 << 49) + 9, (1 << 53) + 5, (1 << 54) - 33, (1 << 57) + 29, (1 << 58) - 27]


def test_three_product_shoup_range():
    rng = random.Random(11)
    for q in PRIMES:
        for _ in range(20000):
            w = rng.randrange(q)
            wq = shoup_quotient(w, q)
            y = rng.choice([rng.randrange(1 << 64), M64 - rng.randrange(1 << 20), rng.randrange(64 * q)])
            r = mul_shoup_lazy4(y, w, wq, q)
            assert r < 4 * q and r % q == (y * w) % q
        for w in (0, 1, q - 1):
            for y in (0, 1, M64, M64 - 1, 1 << 63, 4 * q - 1):
                r = mul_shoup_lazy4(y, w, shoup_quotient(w, q), q)
                assert r < 4 * q and r % q == (y * w) % q


def test_lazy_ct_pass_bound():
    # worst case per stage: X' = X + t, Y' = X - t + 4q with t < 4q
    for q in PRIMES:
        if q >= 1 << 58:
            continue
        bound = 4 * q  # pass input (pass 2 reads the twist product, below 4q)
        for _ in range(9):
            bound += 4 * q
        assert bound <= 40 * q < 1 << 64


def test_lazy_gs_pass_bound():
    for q in PRIMES:
        if q >= 1 << 54:
            continue
        bound = 2 * q  # inputs below 2q
        for s in range(9):
            c = q << (s + 1)
            assert bound <= c and 4 * q <= 2 * c  # X + c - Y >= 0; Y' < 4q fits the next c
            bound = max(2 * c, 4 * q)
        assert bound <= (q << 10) < 1 << 64


def test_lazy_ct_pass_exact_on_random_networks():
    # a small merged CT network run with the lazy butterflies stays below 40q and
    # reduces to the exact network's outputs
    rng = random.Random(3)
    q = (1 << 50) - 27
    for _ in range(50):
        x = [rng.randrange(4 * q) for _ in range(512)]
        ref = [v % q for v in x]
        tw = [rng.randrange(q) for _ in range(512)]
        n, t, k = 512, 512, 0
        m = 1
        while m < n:
            t //= 2
            for i in range(m):
                w = tw[m + i]
                wq = shoup_quotient(w, q)
                for j in range(2 * i * t, 2 * i * t + t):
                    u, v = x[j], mul_shoup_lazy4(x[j + t], w, wq, q)
                    x[j], x[j + t] = (u + v) & M64, (u - v + 4 * q) & M64
                    assert x[j] < 40 * q and x[j + t] < 40 * q
                    ru, rv = ref[j], ref[j + t] * w % q
                    ref[j], ref[j + t] = (ru + rv) % q, (ru - rv) % q
            m *= 2
        assert [v % q for v in x] == ref


def test_lift_digit():
    rng = random.Random(5)
    for q in PRIMES + [3, 97, (1 << 20) + 7, (1 << 30) + 3, (1 << 60) - 93, (1 << 62) - 57]:
        for d in [0, 1, -1, q, -q, q - 1, 1 - q, 1 << 31, -(1 << 31), (1 << 63) - 1, -(1 << 63)]:
            assert lift_digit(d, q) == d % q
        for _ in range(5000):
            d = rng.randrange(-(1 << 63), 1 << 63)
            assert lift_digit(d, q) == d % q
