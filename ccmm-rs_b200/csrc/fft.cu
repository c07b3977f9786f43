// fft.cu -- one diagonal-rotation stage of the encrypted radix-4 FFT
// (eblas/prepared_radix4_fft256.rs:761-822, apply_stage_internal):
//   out = Rescale( sum_t multiply_plain(rotate(ct, offset_t), diag_t) )
// where the offset-0 term, if present, multiplies the unrotated input.
//
// B200 schedule: every nonzero offset of a ciphertext is rotated by one
// hoisted key-switch batch (one decomposition per ciphertext, bit-exact with
// the reference's independent rotations); the rotated ciphertexts are
// transformed once, multiplied by their NTT-prepared diagonals and summed in
// the NTT domain with exact 128-bit accumulation, then one inverse transform
// and one rescale. The sum of products is linear mod q, so the result equals
// the reference's per-term inverse transforms and sequential additions word
// for word.
#include <vector>

#include "keyswitch.cuh"

namespace {

constexpr int kT = 256;

// acc[c][comp][l][k] = sum_t R[c][t][comp][l][k] * P[t][l][k]   (+ X[c][comp][l][k] * P[n_rot][l][k])
// R: [n][n_rot][2][L][N], X: [n][2][L][N] (identity term, may be null), P: [n_terms][L][N].
__global__ void __launch_bounds__(kT) k_diag_mac(const u64* __restrict__ R, const u64* __restrict__ X,
                                                 const u64* __restrict__ P, u64* __restrict__ acc,
                                                 const NttTab* __restrict__ tabs, int n_rot, int L, int log_n) {
    const u32 n = 1u << log_n;
    const u32 k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int l = blockIdx.y;
    const size_t c = blockIdx.z;
    const NttTab& T = tabs[l];
    const size_t poly = (size_t)L << log_n, lk = ((size_t)l << log_n) + k;
    Acc128 ab{0, 0}, aa{0, 0};
    int since = 0;
    for (int t = 0; t < n_rot; ++t) {
        const u64 p = __ldg(P + (size_t)t * poly + lk);
        const u64* r = R + (c * n_rot + t) * 2 * poly + lk;
        ab.mac(r[0], p);
        aa.mac(r[poly], p);
        if (++since == 15) {
            ab.fold(T.q, T.mu_hi, T.mu_lo);
            aa.fold(T.q, T.mu_hi, T.mu_lo);
            since = 0;
        }
    }
    if (X) {
        const u64 p = __ldg(P + (size_t)n_rot * poly + lk);
        ab.mac(X[c * 2 * poly + lk], p);
        aa.mac(X[c * 2 * poly + poly + lk], p);
    }
    ab.fold(T.q, T.mu_hi, T.mu_lo);
    aa.fold(T.q, T.mu_hi, T.mu_lo);
    acc[c * 2 * poly + lk] = ab.lo;
    acc[c * 2 * poly + poly + lk] = aa.lo;
}

// Multi-ciphertext stage: out[a] = sum over the terms t of output a of
// R[src_t][key_t] * P[t] (key_t = n_rot: the unrotated input X[src_t]).
// terms: [n_terms][3] (output, source, key) sorted by output; first[a] .. first[a+1]
// index the terms of output a. R: [n_in][n_rot][2][L][N], X: [n_in][2][L][N].
__global__ void __launch_bounds__(kT) k_diag_mac_multi(const u64* __restrict__ R, const u64* __restrict__ X,
                                                       const u64* __restrict__ P, const u32* __restrict__ terms,
                                                       const u32* __restrict__ first, u64* __restrict__ acc,
                                                       const NttTab* __restrict__ tabs, int n_rot, int L, int log_n) {
    const u32 n = 1u << log_n;
    const u32 k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int l = blockIdx.y;
    const u32 a = blockIdx.z;
    const NttTab& T = tabs[l];
    const size_t poly = (size_t)L << log_n, lk = ((size_t)l << log_n) + k;
    Acc128 ab{0, 0}, aa{0, 0};
    int since = 0;
    for (u32 t = first[a]; t < first[a + 1]; ++t) {
        const u32 src = terms[3 * t + 1], key = terms[3 * t + 2];
        const u64 p = __ldg(P + (size_t)t * poly + lk);
        const u64* r = key < (u32)n_rot ? R + ((size_t)src * n_rot + key) * 2 * poly + lk : X + (size_t)src * 2 * poly + lk;
        ab.mac(r[0], p);
        aa.mac(r[poly], p);
        if (++since == 15) {
            ab.fold(T.q, T.mu_hi, T.mu_lo);
            aa.fold(T.q, T.mu_hi, T.mu_lo);
            since = 0;
        }
    }
    ab.fold(T.q, T.mu_hi, T.mu_lo);
    aa.fold(T.q, T.mu_hi, T.mu_lo);
    acc[(size_t)a * 2 * poly + lk] = ab.lo;
    acc[(size_t)a * 2 * poly + poly + lk] = aa.lo;
}

}  // namespace

int32_t fft_stage_multi_launch(ckks_ctx* ctx, const ckks_ksk* const* keys, u32 n_rot, const u32* terms_host,
                               u32 n_terms, const u64* diag_ntt, const u64* ct_in, u32 n_in, u64* ct_out, u32 n_out,
                               u32 L, cudaStream_t st) {
    const u32 N = ctx->n;
    const size_t poly = (size_t)L * N, ct = 2 * poly;
    std::vector<u32> first(n_out + 1, 0), tl(3 * (size_t)n_terms);
    {   // stable order by output
        u32 w = 0;
        for (u32 a = 0; a < n_out; ++a) {
            first[a] = w;
            for (u32 t = 0; t < n_terms; ++t)
                if (terms_host[3 * t] == a) {
                    for (int i = 0; i < 3; ++i) tl[3 * (size_t)w + i] = terms_host[3 * t + i];
                    ++w;
                }
        }
        first[n_out] = w;
    }
    // diagonals follow the caller's term order: remap to the sorted order
    std::vector<u32> perm(n_terms);
    {
        u32 w = 0;
        for (u32 a = 0; a < n_out; ++a)
            for (u32 t = 0; t < n_terms; ++t)
                if (terms_host[3 * t] == a) perm[w++] = t;
    }
    Workspace<u64> R, X, acc, P;
    Workspace<u32> dterms;
    int32_t rc;
    if ((rc = R.alloc(ct * n_in * (n_rot ? n_rot : 1), st)) || (rc = X.alloc(ct * n_in, st)) ||
        (rc = acc.alloc(ct * n_out, st)) || (rc = P.alloc(poly * n_terms, st)) ||
        (rc = dterms.alloc(tl.size() + first.size(), st)))
        return rc;
    for (u32 w = 0; w < n_terms; ++w)
        CKKS_CUDA_TRY(cudaMemcpyAsync(P.p + (size_t)w * poly, diag_ntt + (size_t)perm[w] * poly, poly * 8,
                                      cudaMemcpyDeviceToDevice, st));
    CKKS_CUDA_TRY(cudaMemcpyAsync(dterms.p, tl.data(), tl.size() * 4, cudaMemcpyHostToDevice, st));
    CKKS_CUDA_TRY(cudaMemcpyAsync(dterms.p + tl.size(), first.data(), first.size() * 4, cudaMemcpyHostToDevice, st));
    if (n_rot) {
        if ((rc = rotate_hoisted_ntt(ctx, keys, n_rot, ct_in, R.p, n_in, st))) return rc;
        if ((rc = ntt_forward_launch(ctx, R.p, R.p, 2 * n_in * n_rot, 0, L, st))) return rc;
    }
    if ((rc = ntt_forward_launch(ctx, ct_in, X.p, 2 * n_in, 0, L, st))) return rc;
    dim3 g((N + kT - 1) / kT, L, n_out);
    k_diag_mac_multi<<<g, kT, 0, st>>>(R.p, X.p, P.p, dterms.p, dterms.p + tl.size(), acc.p, ctx->d_tabs, (int)n_rot,
                                       (int)L, (int)ctx->log_n);
    CKKS_CUDA_TRY(cudaGetLastError());
    if ((rc = ntt_inverse_launch(ctx, acc.p, acc.p, 2 * n_out, 0, L, st))) return rc;
    return rescale_launch(ctx, acc.p, ct_out, 2 * n_out, L, st);
}

int32_t fft_stage_launch(ckks_ctx* ctx, const ckks_ksk* const* keys, u32 n_rot, bool identity, const u64* diag_ntt,
                         const u64* ct_in, u64* ct_out, u32 n_ct, u32 L, cudaStream_t st, bool rescale) {
    const u32 N = ctx->n;
    const size_t poly = (size_t)L * N, ct = 2 * poly;
    // ciphertexts per chunk: rotated copies (n_rot + 1 per ciphertext) within about 2^29 words
    size_t per = ct * (n_rot + 2);
    u32 chunk = (u32)((size_t(1) << 29) / per);
    if (chunk < 1) chunk = 1;
    if (chunk > 65535 / (2 * (n_rot + 1))) chunk = 65535 / (2 * (n_rot + 1));
    if (chunk > n_ct) chunk = n_ct;
    for (u32 c0 = 0; c0 < n_ct; c0 += chunk) {
        const u32 m = n_ct - c0 < chunk ? n_ct - c0 : chunk;
        Workspace<u64> R, X;
        int32_t rc;
        if ((rc = R.alloc(ct * m * n_rot + ct * m, st))) return rc;
        u64* acc = R.p + ct * m * n_rot;
        const u64* in = ct_in + (size_t)c0 * ct;
        if (n_rot) {
            if ((rc = rotate_hoisted_ntt(ctx, keys, n_rot, in, R.p, m, st))) return rc;
            if ((rc = ntt_forward_launch(ctx, R.p, R.p, 2 * m * n_rot, 0, L, st))) return rc;
        }
        if (identity) {
            if ((rc = X.alloc(ct * m, st))) return rc;
            if ((rc = ntt_forward_launch(ctx, in, X.p, 2 * m, 0, L, st))) return rc;
        }
        dim3 g((N + kT - 1) / kT, L, m);
        k_diag_mac<<<g, kT, 0, st>>>(R.p, identity ? X.p : nullptr, diag_ntt, acc, ctx->d_tabs, (int)n_rot, (int)L,
                                     (int)ctx->log_n);
        CKKS_CUDA_TRY(cudaGetLastError());
        if (rescale) {
            if ((rc = ntt_inverse_launch(ctx, acc, acc, 2 * m, 0, L, st))) return rc;
            if ((rc = rescale_launch(ctx, acc, ct_out + (size_t)c0 * 2 * (L - 1) * N, 2 * m, L, st))) return rc;
        } else if ((rc = ntt_inverse_launch(ctx, acc, ct_out + (size_t)c0 * ct, 2 * m, 0, L, st))) {
            return rc;
        }
    }
    return CKKS_OK;
}
