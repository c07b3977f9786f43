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

}  // namespace

int32_t fft_stage_launch(ckks_ctx* ctx, const ckks_ksk* const* keys, u32 n_rot, bool identity, const u64* diag_ntt,
                         const u64* ct_in, u64* ct_out, u32 n_ct, u32 L, cudaStream_t st) {
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
        if ((rc = ntt_inverse_launch(ctx, acc, acc, 2 * m, 0, L, st))) return rc;
        if ((rc = rescale_launch(ctx, acc, ct_out + (size_t)c0 * 2 * (L - 1) * N, 2 * m, L, st))) return rc;
    }
    return CKKS_OK;
}
