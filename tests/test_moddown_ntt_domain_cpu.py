"""ModDown commutes with the NTT on the Q limbs (CPU, oracle only).

ModDown (ring/auxiliary_modulus.rs:89-171) maps x over QP to
  out_i = (x_i - ([x_P] centred mod P) mod q_i) * P^-1 mod q_i.
Every step after the centred CRT of the P limbs is linear per Q limb, so the
NTT-domain form
  NTT(out_i) = (NTT(x_i) - NTT(c mod q_i)) * P^-1,  c = [x_P] centred,
needs the coefficients of the P limbs only. These tests pin that identity
against the oracle's ModDown, the form a rotation whose output is consumed in
the NTT domain (the FFT stages' diagonal products) can use to skip the
inverse transform of the Q limbs and their forward transform afterwards.
"""
import numpy as np
import pytest


def centred_crt(p, xp):
    """[x_P] in (-P/2, P/2] for each coefficient (Python integers)."""
    P = 1
    for m in p:
        P *= m
    n = xp.shape[-1]
    out = []
    for j in range(n):
        v = 0
        for m, row in zip(p, xp):
            Pm = P // m
            v += int(row[j]) * Pm * pow(Pm, -1, m)
        v %= P
        out.append(v - P if v > P // 2 else v)
    return out, P


@pytest.mark.parametrize("log_n,nq,npl", [(6, 3, 1), (8, 4, 2), (10, 5, 3)])
def test_moddown_in_the_ntt_domain_matches(oracle, log_n, nq, npl):
    n = 1 << log_n
    q = [int(x) for x in oracle.primes_below_bits(50, n, nq)]
    p = [int(x) for x in oracle.primes_below_bits(60, n, npl)]
    rng = np.random.default_rng(log_n)
    x = np.stack([rng.integers(0, m, n, dtype=np.uint64) for m in q + p])[None]
    want = oracle.ntt_forward(q, oracle.mod_down(q, p, x))[0]

    # NTT-domain form: transforms of the Q limbs as they arrive, coefficients of the P limbs
    X = oracle.ntt_forward(q, x[:, :nq])[0]
    c, P = centred_crt(p, x[0, nq:])
    corr = np.stack([np.array([v % m for v in c], dtype=np.uint64) for m in q])
    C = oracle.ntt_forward(q, corr[None])[0]
    got = np.stack([np.array([(int(a) - int(b)) * pow(P, -1, m) % m for a, b in zip(X[i], C[i])],
                             dtype=np.uint64) for i, m in enumerate(q)])
    assert np.array_equal(got, want)
