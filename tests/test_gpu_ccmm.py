"""GPU parity of the structured encrypted matrix product
(matrix/rns_ckks_ciphertext.rs:204-318, matmul_structured_bounded_with_ntt).

C[r][c] = Rescale(Relinearize(sum_k tensor(A[r][k], B[k][c]))) with one
ciphertext per entry, column-major. The GPU result must equal the oracle's
composition of the reference's tensor, addition, bounded relinearization and
rescale word for word (tolerance zero), and decode to the FP64 cleartext
product within the reference's own tolerance (bin/structured_ccmm_4096.rs:20,
3e-3; each entry encrypts one scalar in every slot and decodes as the mean of
the real parts of the slots).
"""
import numpy as np
import pytest

import ckks_b200 as cb

pytestmark = pytest.mark.gpu


def dev(x):
    return cb.as_u64_tensor(x)


def host(t):
    return cb.to_numpy_u64(t)


@pytest.fixture(scope="module")
def setup(oracle):
    log_n, n = 10, 1 << 10
    q = [int(x) for x in oracle.primes_below_bits(50, n, 3)]
    ctx = cb.Context(log_n, q, [int(x) for x in oracle.primes_below_bits(60, n, 1)])
    rng = np.random.default_rng(3)
    s = rng.integers(-1, 2, n).astype(np.int8)
    key_ref = oracle.relin_key(q, s, 20, seed=17)
    key = cb.KeySwitchKey.relin_upload(ctx, len(q), 20, key_ref)
    return n, q, ctx, s, key, key_ref


def oracle_ccmm(oracle, q, key_ref, A, B, m, k, n_cols):
    L, N = len(q), A.shape[-1]
    out = []
    for c in range(n_cols):
        for r in range(m):
            acc = None
            for kk in range(k):
                t = oracle.tensor(q, A[r + kk * m], B[kk + c * k]).astype(object)
                acc = t if acc is None else acc + t
            quad = np.stack([acc[:, l] % q[l] for l in range(L)], axis=1).astype(np.uint64)
            rel = oracle.relinearize(q, quad, key_ref, 20)
            out.append(oracle.rescale(q, rel.reshape(2, L, N)))
    return np.stack(out)


@pytest.mark.parametrize("m,k,n_cols", [(2, 2, 2), (3, 2, 5), (1, 4, 1)])
def test_ccmm_bit_exact(oracle, cuda, setup, m, k, n_cols):
    n, q, ctx, s, key, key_ref = setup
    rng = np.random.default_rng(m * 100 + k * 10 + n_cols)

    def rand_mat(cnt):
        return np.stack([np.stack([np.stack([rng.integers(0, mm, n, dtype=np.uint64) for mm in q])
                                   for _ in range(2)]) for _ in range(cnt)])

    A, B = rand_mat(m * k), rand_mat(k * n_cols)
    got = host(cb.matmul_structured(ctx, key, dev(A), dev(B), m, k, n_cols))
    want = oracle_ccmm(oracle, q, key_ref, A, B, m, k, n_cols)
    assert got.shape == (n_cols, m, 2, len(q) - 1, n)
    assert np.array_equal(got.reshape(want.shape), want)


def oracle_entry(oracle, q, key_ref, A, B, m, k, r, c):
    L, N = len(q), A.shape[-1]
    acc = sum(oracle.tensor(q, A[r + kk * m], B[kk + c * k]).astype(object) for kk in range(k))
    quad = np.stack([acc[:, l] % q[l] for l in range(L)], axis=1).astype(np.uint64)
    return oracle.rescale(q, oracle.relinearize(q, quad, key_ref, 20).reshape(2, L, N))


@pytest.mark.parametrize("m,k,n_cols", [(1, 1, 1), (5, 7, 19), (64, 64, 3), (33, 5, 40), (64, 65, 2)])
def test_ccmm_tensor_cores_equal_cuda_cores(oracle, cuda, setup, m, k, n_cols):
    """The per-slot products on the INT8 tensor cores (m, k <= 64: byte planes,
    one MMA per 16 columns x 4 inner indices) give the same words as the
    CUDA-core products; ragged column blocks, one-item slots and the largest
    tile are covered, and k = 65 falls back to the CUDA cores. Sampled entries
    equal the oracle."""
    import torch
    n, q, ctx, s, key, key_ref = setup
    rng = np.random.default_rng(m + 7 * k + 31 * n_cols)
    A = np.stack([np.stack([rng.integers(0, mm, (2, n), dtype=np.uint64) for mm in q], axis=1) for _ in range(m * k)])
    B = np.stack([np.stack([rng.integers(0, mm, (2, n), dtype=np.uint64) for mm in q], axis=1)
                  for _ in range(k * n_cols)])
    dA, dB = dev(A), dev(B)
    assert ctx.tensor_cores
    tc = cb.matmul_structured(ctx, key, dA, dB, m, k, n_cols)
    torch.cuda.synchronize()
    assert ctx.last_mac_path == ("tensor_cores" if k <= 64 else "cuda_cores")
    ctx.tensor_cores = False
    try:
        cc = cb.matmul_structured(ctx, key, dA, dB, m, k, n_cols)
        torch.cuda.synchronize()
        assert ctx.last_mac_path == "cuda_cores"
    finally:
        ctx.tensor_cores = True
    assert torch.equal(tc, cc)
    got = host(tc)
    for r, c in {(0, 0), (m - 1, n_cols - 1), (m // 2, n_cols // 2)}:
        assert np.array_equal(got[c, r], oracle_entry(oracle, q, key_ref, A, B, m, k, r, c)), (r, c)


def test_ccmm_decodes_to_cleartext_gemm(oracle, cuda, setup):
    n, q, ctx, s, key, key_ref = setup
    rng = np.random.default_rng(11)
    m, k, n_cols = 3, 4, 2
    scale = 2.0 ** 40
    a = rng.uniform(-1, 1, (k, m))  # column-major: a[col][row]
    b = rng.uniform(-1, 1, (n_cols, k))

    def enc(v, seed):
        slots = np.full(n // 2, v, dtype=complex)
        return oracle.encrypt(q, s, oracle.encode(slots, q, scale), seed=seed)

    A = np.stack([enc(a[kk, r], 10 + r + kk * m) for kk in range(k) for r in range(m)])
    B = np.stack([enc(b[c, kk], 100 + kk + c * k) for c in range(n_cols) for kk in range(k)])
    got = host(cb.matmul_structured(ctx, key, dev(A), dev(B), m, k, n_cols))
    want = a.T @ b.T  # m x n
    ql = q[:-1]
    out_scale = scale * scale / q[-1]
    for c in range(n_cols):
        for r in range(m):
            dec = oracle.decode(ql, oracle.decrypt(ql, s, got[c, r]), out_scale)
            assert abs(np.mean(dec.real) - want[r, c]) < 3e-3
            assert np.max(np.abs(dec - want[r, c])) < 1e-5


def test_ccmm_errors(oracle, cuda, setup):
    n, q, ctx, s, key, key_ref = setup
    import torch
    A = torch.zeros((4, 2, len(q), n), dtype=torch.int64, device="cuda")
    gk = cb.KeySwitchKey.hybrid_generate(ctx, len(q), 20, ctx.rotation_exponent_left(1), s, seed=1)
    with pytest.raises(cb.CkksError) as e:
        cb.matmul_structured(ctx, gk, A, A, 2, 2, 2)
    assert e.value.status == -2
    rc = cb.lib().ckks_ccmm_structured(ctx.handle, key.handle, cb._dptr(A), cb._dptr(A), cb._dptr(A), 2, 2, 2, None)
    assert rc == -1  # C overlapping the inputs
