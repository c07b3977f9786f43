"""CPU check of the index arithmetic that folds the Galois automorphism
sigma_k (X^j -> X^(j k), ckks/automorphism.rs:8-48) into the two inverse NTT
passes (k_inv1 / k_inv2 with GaloisOut): pass 1 stores column j_lo of a row at
position j_lo k mod B; pass 2 reads position p as column j_lo = p k^-1 mod B
and writes element i of it to row (m + i k) mod 2A (m = floor((j_lo k mod 2N)
/ B)), negated past A rows. Every (p, i) must land on sigma_k(j_lo + B i), each
output coefficient exactly once, with the sign of the wrap past N."""


def fold_targets(log_n, k):
    lb = log_n // 2
    la = log_n - lb
    A, B, N = 1 << la, 1 << lb, 1 << log_n
    kinv = pow(k, -1, 2 * N)
    out = {}
    for p in range(B):
        # pass 1 wrote original column j_lo at position (j_lo * (k mod B)) mod B
        jl = (p * (kinv & (B - 1))) & (B - 1)
        assert (jl * (k & (B - 1))) & (B - 1) == p
        m = ((jl * k) & (2 * N - 1)) >> lb
        k2a = k & (2 * A - 1)
        for i in range(A):
            r = (m + i * k2a) & (2 * A - 1)
            neg = r >= A
            t = p + B * (r & (A - 1))
            assert t not in out
            out[t] = (jl + B * i, neg)
    return out, N


def test_fold_equals_sigma():
    for log_n in (4, 5, 10, 15, 16):
        n = 1 << log_n
        for k in (1, 3, 5, 25, 2 * n - 1, (5 ** 7) % (2 * n), (5 ** 1000) % (2 * n)):
            out, N = fold_targets(log_n, k)
            assert len(out) == N
            for j in range(N):
                s = (j * k) % (2 * N)
                t, neg = (s, False) if s < N else (s - N, True)
                assert out[t] == (j, neg), (log_n, k, j)
