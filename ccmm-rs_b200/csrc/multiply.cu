// multiply.cu -- ciphertext products on the GPU:
//   tensor      rlwe/quadratic.rs:70-140, grafting/rns_key_switch.rs:1675-1722
//               (c0 = b_x b_y, c1 = b_x a_y + a_x b_y, c2 = a_x a_y per limb,
//               negacyclic products through the NTT);
//   relinearize grafting/bounded_key_switch.rs:139-223 (bounded balanced digits
//               of c2, b = c0 + sum_j d_j k_b[j], a = c1 + sum_j d_j k_a[j]);
//   plaintext   ckks/rns_plain_multiply.rs:119-260 (NTT(ct) * prepared NTT(pt));
//   chain       ckks/rns_multiply.rs:262-300 (tensor -> relinearize -> rescale).
//
// All products are exact modular products, and the NTT is a bijection that is
// linear mod q, so forming the key sum in the NTT domain and adding c0/c1
// there before one inverse transform gives the same residues as the
// reference's per-digit inverse transforms and coefficient-domain sums.
// Batches run as whole-batch launches: one launch per stage covers every
// ciphertext (grid z), so small rings (N = 2^12) are not launch-bound per
// ciphertext.
#include "keyswitch.cuh"

namespace {

constexpr int kT = 256;
constexpr int kRelinGroup = 4;  // ciphertexts sharing one read of a relinearization key word

// X, Y: [n][2][L][N] NTT-domain (b, a). Writes c0, c1 at out01 + c * s01
// (c0 then c1, L limbs each) and c2 at out2 + c * s2.
__global__ void __launch_bounds__(kT) k_tensor(const u64* __restrict__ X, const u64* __restrict__ Y,
                                               u64* __restrict__ out01, size_t s01, u64* __restrict__ out2,
                                               size_t s2, const NttTab* __restrict__ tabs, int L, int log_n) {
    const u32 n = 1u << log_n;
    const u32 k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int l = blockIdx.y;
    const size_t c = blockIdx.z;
    const NttTab& T = tabs[l];
    const Barrett bm{T.q, T.mu_hi, T.mu_lo};
    const size_t in0 = ((c * 2 * L + l) << log_n) + k, in1 = in0 + ((size_t)L << log_n);
    const u64 xb = X[in0], xa = X[in1], yb = Y[in0], ya = Y[in1];
    Acc128 m{0, 0};
    m.mac(xb, ya);
    m.mac(xa, yb);
    m.fold(T.q, T.mu_hi, T.mu_lo);
    const size_t o = ((size_t)l << log_n) + k;
    out01[c * s01 + o] = mul_barrett(xb, yb, bm);
    out01[c * s01 + ((size_t)L << log_n) + o] = m.lo;
    out2[c * s2 + o] = mul_barrett(xa, ya, bm);
}

// Bounded relinearization key-switch sum for a group of G ciphertexts per
// read of each key word (the key streams once per group):
//   acc[c][0][l][k] = base[c][0][l][k] + sum_j Y[c][j][l][k] kb[j][l][k]
//   acc[c][1][l][k] = base[c][1][l][k] + sum_j Y[c][j][l][k] ka[j][l][k]
// key [D][2][L][N], Y [n][D][L][N], base / acc [n][2][L][N] (may alias).
template <int G>
__global__ void __launch_bounds__(kT) k_relin_mac(const u64* __restrict__ Y, const u64* __restrict__ key,
                                                  const u64* base, u64* acc, const NttTab* __restrict__ tabs, int n_ct,
                                                  int L, int D, int log_n) {
    const u32 n = 1u << log_n;
    const u32 k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int l = blockIdx.y;
    const int c0 = blockIdx.z * G;
    const NttTab& T = tabs[l];
    const u64 q = T.q, mh = T.mu_hi, ml = T.mu_lo;
    Acc128 ab[G], aa[G];
#pragma unroll
    for (int i = 0; i < G; ++i) ab[i] = aa[i] = Acc128{0, 0};
    int since = 0;
    for (int j = 0; j < D; ++j) {
        const u64 kb = __ldcs(key + ((((size_t)j * 2 * L) + l) << log_n) + k);
        const u64 ka = __ldcs(key + ((((size_t)j * 2 + 1) * L + l) << log_n) + k);
#pragma unroll
        for (int i = 0; i < G; ++i) {
            if (c0 + i < n_ct) {
                const u64 y = Y[((((size_t)(c0 + i) * D + j) * L + l) << log_n) + k];
                ab[i].mac(y, kb);
                aa[i].mac(y, ka);
            }
        }
        if (++since == 15) {
#pragma unroll
            for (int i = 0; i < G; ++i) {
                ab[i].fold(q, mh, ml);
                aa[i].fold(q, mh, ml);
            }
            since = 0;
        }
    }
#pragma unroll
    for (int i = 0; i < G; ++i) {
        if (c0 + i >= n_ct) break;
        ab[i].fold(q, mh, ml);
        aa[i].fold(q, mh, ml);
        const size_t ob = (((size_t)(c0 + i) * 2 * L + l) << log_n) + k, oa = ob + ((size_t)L << log_n);
        u64 b = ab[i].lo, a = aa[i].lo;
        if (base) {
            b = add_mod(b, base[ob], q);
            a = add_mod(a, base[oa], q);
        }
        acc[ob] = b;
        acc[oa] = a;
    }
}

// out[c][comp][l][k] = X[c][comp][l][k] * P[c * p_stride][l][k]  (grid z = 2 n; X may be out)
__global__ void __launch_bounds__(kT) k_mul_plain(const u64* X, const u64* __restrict__ P, size_t p_stride, u64* out,
                                                  const NttTab* __restrict__ tabs, int L, int log_n) {
    const u32 n = 1u << log_n;
    const u32 k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int l = blockIdx.y;
    const size_t pc = blockIdx.z;  // (ciphertext, component)
    const NttTab& T = tabs[l];
    const Barrett bm{T.q, T.mu_hi, T.mu_lo};
    const size_t i = ((pc * L + l) << log_n) + k;
    out[i] = mul_barrett(X[i], P[(pc / 2) * p_stride + ((size_t)l << log_n) + k], bm);
}

// Ciphertexts per chunk so that a chunk's workspace stays near 2^28 words
// (2 GiB) and every launch's grid z (polys_per_ct per ciphertext) fits 65535.
u32 chunk_of(u32 n, size_t words_per_ct, u32 polys_per_ct) {
    const size_t budget = size_t(1) << 28;
    size_t c = words_per_ct ? budget / words_per_ct : n;
    if (c > 65535 / polys_per_ct) c = 65535 / polys_per_ct;
    if (c < 1) c = 1;
    return (u32)(c < n ? c : n);
}

int32_t tensor_ntt(ckks_ctx* ctx, const u64* Xh, const u64* Yh, u64* out01, size_t s01, u64* out2, size_t s2, u32 n,
                   u32 L, cudaStream_t st) {
    dim3 g((ctx->n + kT - 1) / kT, L, n);
    k_tensor<<<g, kT, 0, st>>>(Xh, Yh, out01, s01, out2, s2, ctx->d_tabs, (int)L, (int)ctx->log_n);
    CKKS_CUDA_TRY(cudaGetLastError());
    return CKKS_OK;
}

size_t relin_words_per_ct(const ckks_ctx* ctx, const ckks_ksk* key) {
    return (size_t)key->D * ctx->n * (1 + key->q_limbs);
}

}  // namespace

// c2: [n][L][N] coefficient domain; acc01: [n][2][L][N] NTT-domain c0, c1 on
// entry, the NTT-domain relinearized (b, a) on return.
int32_t relin_core_launch(ckks_ctx* ctx, const ckks_ksk* key, const u64* c2, u64* acc01, u32 n, cudaStream_t st,
                          bool relin_fused) {
    const u32 L = key->q_limbs, D = key->D, N = ctx->n;
    Workspace<i64> dg;
    Workspace<u64> Y;
    int32_t rc;
    if ((rc = Y.alloc((size_t)n * D * L * N, st))) return rc;
    if (key->kind == CKKS_KSK_RELIN_RNS_BLOCK) {
        // block digits of c2 (canonical mod Q_i, rns_key_switch.rs:1875) lifted to every Q limb
        for (u32 c = 0; c < n; ++c)
            if ((rc = rnsblock_modup_launch(ctx, key, c2 + (size_t)c * L * N, Y.p + (size_t)c * D * L * N, st)))
                return rc;
        if ((rc = ntt_forward_launch_map(ctx, Y.p, Y.p, n * D, LimbMap::range(0, L), L, st))) return rc;
    } else {
        if ((rc = dg.alloc((size_t)n * D * N, st))) return rc;
        if ((rc = bounded_decompose_launch(ctx, c2, n, L, key->base_log, dg.p, nullptr, st))) return rc;
        if (relin_fused && ntt_relin_fused_supported(ctx, L))  // digit transforms stay on chip
            return ntt_relin_fused_launch(ctx, dg.p, Y.p, key->d_entries, acc01, acc01, n, L, D, st);
        if ((rc = ntt_forward_digits_launch(ctx, dg.p, Y.p, n * D, LimbMap::range(0, L), L, st))) return rc;
    }
    dim3 g((N + kT - 1) / kT, L, (n + kRelinGroup - 1) / kRelinGroup);
    k_relin_mac<kRelinGroup><<<g, kT, 0, st>>>(Y.p, key->d_entries, acc01, acc01, ctx->d_tabs, (int)n, (int)L, (int)D,
                                               (int)ctx->log_n);
    CKKS_CUDA_TRY(cudaGetLastError());
    return CKKS_OK;
}

int32_t tensor_launch(ckks_ctx* ctx, const u64* lhs, const u64* rhs, u64* out, u32 n_ct, u32 L, cudaStream_t st) {
    const size_t ct = (size_t)2 * L * ctx->n;
    const u32 chunk = chunk_of(n_ct, 2 * ct, 3);
    for (u32 c0 = 0; c0 < n_ct; c0 += chunk) {
        const u32 m = n_ct - c0 < chunk ? n_ct - c0 : chunk;
        Workspace<u64> X;
        int32_t rc;
        if ((rc = X.alloc(2 * ct * m, st))) return rc;
        u64* Yh = X.p + ct * m;
        u64* o = out + (size_t)c0 * 3 * L * ctx->n;
        if ((rc = ntt_forward_launch(ctx, lhs + c0 * ct, X.p, 2 * m, 0, L, st))) return rc;
        if ((rc = ntt_forward_launch(ctx, rhs + c0 * ct, Yh, 2 * m, 0, L, st))) return rc;
        const size_t s3 = (size_t)3 * L * ctx->n;
        if ((rc = tensor_ntt(ctx, X.p, Yh, o, s3, o + (size_t)2 * L * ctx->n, s3, m, L, st))) return rc;
        if ((rc = ntt_inverse_launch(ctx, o, o, 3 * m, 0, L, st))) return rc;
    }
    return CKKS_OK;
}

int32_t relinearize_launch(ckks_ctx* ctx, const ckks_ksk* key, const u64* quad, u64* out, u32 n_ct, cudaStream_t st) {
    const u32 L = key->q_limbs, N = ctx->n;
    const size_t poly = (size_t)L * N;
    const u32 chunk = chunk_of(n_ct, relin_words_per_ct(ctx, key) + 3 * poly, key->D > 3 ? key->D : 3);
    for (u32 c0 = 0; c0 < n_ct; c0 += chunk) {
        const u32 m = n_ct - c0 < chunk ? n_ct - c0 : chunk;
        const u64* q = quad + (size_t)c0 * 3 * poly;
        Workspace<u64> W;
        int32_t rc;
        if ((rc = W.alloc(3 * poly * m, st))) return rc;
        u64* acc = W.p;               // [m][2][L][N]
        u64* c2 = W.p + 2 * poly * m;  // [m][L][N]
        // gather c0 c1 and c2 of every ciphertext into contiguous batches
        CKKS_CUDA_TRY(cudaMemcpy2DAsync(acc, 2 * poly * 8, q, 3 * poly * 8, 2 * poly * 8, m, cudaMemcpyDeviceToDevice, st));
        CKKS_CUDA_TRY(cudaMemcpy2DAsync(c2, poly * 8, q + 2 * poly, 3 * poly * 8, poly * 8, m, cudaMemcpyDeviceToDevice, st));
        if ((rc = ntt_forward_launch(ctx, acc, acc, 2 * m, 0, L, st))) return rc;
        if ((rc = relin_core_launch(ctx, key, c2, acc, m, st))) return rc;
        if ((rc = ntt_inverse_launch(ctx, acc, out + (size_t)c0 * 2 * poly, 2 * m, 0, L, st))) return rc;
    }
    return CKKS_OK;
}

int32_t multiply_relin_rescale_launch(ckks_ctx* ctx, const ckks_ksk* key, const u64* lhs, const u64* rhs, u64* out,
                                      u32 n_ct, cudaStream_t st) {
    const u32 L = key->q_limbs, N = ctx->n;
    const size_t poly = (size_t)L * N, ct = 2 * poly;
    const u32 chunk = chunk_of(n_ct, relin_words_per_ct(ctx, key) + 7 * poly, key->D > 3 ? key->D : 3);
    for (u32 c0 = 0; c0 < n_ct; c0 += chunk) {
        const u32 m = n_ct - c0 < chunk ? n_ct - c0 : chunk;
        Workspace<u64> W;
        int32_t rc;
        if ((rc = W.alloc(7 * poly * m, st))) return rc;
        u64* Xh = W.p;                // [m][2][L][N]
        u64* Yh = Xh + ct * m;        // [m][2][L][N]
        u64* acc = Yh + ct * m;       // [m][2][L][N]
        u64* c2 = acc + ct * m;       // [m][L][N]
        if ((rc = ntt_forward_launch(ctx, lhs + c0 * ct, Xh, 2 * m, 0, L, st))) return rc;
        if ((rc = ntt_forward_launch(ctx, rhs + c0 * ct, Yh, 2 * m, 0, L, st))) return rc;
        if ((rc = tensor_ntt(ctx, Xh, Yh, acc, ct, c2, poly, m, L, st))) return rc;
        if ((rc = ntt_inverse_launch(ctx, c2, Xh, m, 0, L, st))) return rc;  // c2 to the coefficient domain
        if ((rc = relin_core_launch(ctx, key, Xh, acc, m, st))) return rc;
        if ((rc = ntt_inverse_launch(ctx, acc, Yh, 2 * m, 0, L, st))) return rc;
        if ((rc = rescale_launch(ctx, Yh, out + (size_t)c0 * 2 * (L - 1) * N, 2 * m, L, st))) return rc;
    }
    return CKKS_OK;
}

int32_t mul_plain_launch(ckks_ctx* ctx, const u64* ct_in, const u64* plain_ntt, u64* out, u32 n_ct, u32 L,
                         bool plain_per_ct, cudaStream_t st) {
    const size_t poly = (size_t)L * ctx->n;
    const u32 chunk = chunk_of(n_ct, 2 * poly, 2);
    for (u32 c0 = 0; c0 < n_ct; c0 += chunk) {
        const u32 m = n_ct - c0 < chunk ? n_ct - c0 : chunk;
        Workspace<u64> X;
        int32_t rc;
        if ((rc = X.alloc(2 * poly * m, st))) return rc;
        if ((rc = ntt_forward_launch(ctx, ct_in + (size_t)c0 * 2 * poly, X.p, 2 * m, 0, L, st))) return rc;
        dim3 g((ctx->n + kT - 1) / kT, L, 2 * m);
        k_mul_plain<<<g, kT, 0, st>>>(X.p, plain_ntt + (plain_per_ct ? (size_t)c0 * poly : 0), plain_per_ct ? poly : 0,
                                      X.p, ctx->d_tabs, (int)L, (int)ctx->log_n);
        CKKS_CUDA_TRY(cudaGetLastError());
        if ((rc = ntt_inverse_launch(ctx, X.p, out + (size_t)c0 * 2 * poly, 2 * m, 0, L, st))) return rc;
    }
    return CKKS_OK;
}
