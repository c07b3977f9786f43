// ccmm.cu -- structured ciphertext-ciphertext matrix multiplication
// (matrix/rns_ckks_ciphertext.rs:220-318, matmul_structured_bounded_with_ntt):
//   C[r][c] = Rescale( Relinearize( sum_k tensor(A[r][k], B[k][c]) ) )
// with one ciphertext per matrix entry, column-major (index row + col * rows,
// matrix/rns_ckks_ciphertext.rs:9), and the bounded relinearization key.
//
// In the NTT domain the tensor sum is, for every (limb l, slot s), three small
// modular matrix products of the entries' residues:
//   C0 = Ab Bb,  C1 = Ab Ba + Aa Bb,  C2 = Aa Ba      (m x k times k x n)
// which equal the reference's per-product NTTs, inverse NTTs and additions word
// for word (the NTT is linear mod q). The schedule:
//   1. forward NTT of every entry, transposed to slot-major [l][s][comp][entry];
//   2. the three products per (l, s): on the INT8 tensor cores (ccmm_tc.cu,
//      byte planes, exact) when m, k <= 64, else one CTA per (l, s) with
//      split-operand accumulators (residues pre-split into sb-bit halves,
//      sb = ceil(bits(q-1)/2); four 32x32->64-bit multiply-adds per product);
//   3. the results go back to entry-major [entry][comp][l][s] in chunks of
//      output columns, c2 is transformed back, relinearized with the bounded
//      key (digits, digit NTTs, key MAC with c0/c1 as base), transformed back
//      and rescaled.
#include "keyswitch.cuh"

namespace {

constexpr int kT = 256;
constexpr int kTile = 32;

__device__ __forceinline__ int split_bits(u64 q) { return (65 - __clzll(q - 1)) / 2; }

// X [n_ent][2][L][N] (NTT domain) -> Xt [L][N][2][ld] at entries e0.., each word
// pre-split as (x >> sb) << 32 | (x & mask) when `split`, else canonical.
// Grid (N/32, n_ent/32 rounded up, 2 L).
__global__ void __launch_bounds__(kTile * 8) k_to_slot_major(const u64* __restrict__ X, u64* __restrict__ Xt,
                                                             const NttTab* __restrict__ tabs, int n_ent, int e0,
                                                             int ld, int L, int log_n, int split) {
    __shared__ u64 tile[kTile][kTile + 1];
    const u32 n = 1u << log_n;
    const int l = blockIdx.z >> 1, comp = blockIdx.z & 1;
    const u32 s0 = blockIdx.x * kTile;
    const int c0 = blockIdx.y * kTile;
    const u64 q = tabs[l].q;
    const int sb = split_bits(q);
    const u64 mask = (1ull << sb) - 1;
    const int tx = threadIdx.x & (kTile - 1), ty = threadIdx.x / kTile;  // 32 x 8
    for (int r = ty; r < kTile; r += 8) {
        const int e = c0 + r;
        if (e < n_ent) {
            const u64 x = X[((((size_t)e * 2 + comp) * L + l) << log_n) + s0 + tx];
            tile[r][tx] = split ? ((x >> sb) << 32) | (x & mask) : x;
        }
    }
    __syncthreads();
    for (int r = ty; r < kTile; r += 8) {
        const int e = c0 + tx;
        if (e < n_ent) Xt[((((size_t)l << log_n) + s0 + r) * 2 + comp) * ld + e0 + e] = tile[tx][r];
    }
    (void)n;
}

// Ct [L][N][3][ldc] (canonical) -> Q01 [n_ent][2][L][N] (components 0, 1) and
// C2 [n_ent][L][N] (component 2). Grid (N/32, n_ent/32 rounded up, 3 L).
__global__ void __launch_bounds__(kTile * 8) k_from_slot_major(const u64* __restrict__ Ct, u64* __restrict__ Q01,
                                                               u64* __restrict__ C2, int n_ent, int ldc, int L,
                                                               int log_n) {
    __shared__ u64 tile[kTile][kTile + 1];
    const int l = blockIdx.z / 3, comp = blockIdx.z % 3;
    const u32 s0 = blockIdx.x * kTile;
    const int c0 = blockIdx.y * kTile;
    const int tx = threadIdx.x & (kTile - 1), ty = threadIdx.x / kTile;
    for (int r = ty; r < kTile; r += 8) {
        const int e = c0 + tx;
        if (e < n_ent) tile[r][tx] = Ct[((((size_t)l << log_n) + s0 + r) * 3 + comp) * ldc + e];
    }
    __syncthreads();
    for (int r = ty; r < kTile; r += 8) {
        const int e = c0 + r;
        if (e >= n_ent) continue;
        const u64 v = tile[tx][r];
        if (comp < 2) Q01[((((size_t)e * 2 + comp) * L + l) << log_n) + s0 + tx] = v;
        else C2[((((size_t)e * L + l) << log_n) + s0 + tx)] = v;
    }
}

struct Split3 {
    u64 s0, s1, s2;
    __device__ __forceinline__ void mac(u64 x, u64 y) {  // x, y pre-split (hi << 32 | lo)
        const u32 x0 = (u32)x, x1 = (u32)(x >> 32), y0 = (u32)y, y1 = (u32)(y >> 32);
        s0 += (u64)x0 * y0;
        s1 += (u64)x0 * y1;
        s1 += (u64)x1 * y0;
        s2 += (u64)x1 * y1;
    }
};

__device__ __forceinline__ u64 split_fold(const Split3& a, u64 q, u64 one_q, u64 r1, u64 r1q, u64 r2, u64 r2q) {
    u64 t = reduce_2q(mul_shoup_lazy(a.s0, 1, one_q, q), q);
    t = add_mod(t, reduce_2q(mul_shoup_lazy(a.s1, r1, r1q, q), q), q);
    return add_mod(t, reduce_2q(mul_shoup_lazy(a.s2, r2, r2q, q), q), q);
}

// One CTA per (slot s, limb l): for the output block [m] x [nc] (columns
// c_begin ..), C0/C1/C2 = sums over k of the products of At (m x k, entry
// r + kk m) and Bt (k x n, entry kk + c k). Each thread owns one row and two
// adjacent columns (8 independent split products per k); consecutive threads
// take consecutive rows, so the A reads of a warp are contiguous and its B
// reads broadcast. Partial sums are folded into the canonical residue every
// `fold_k` terms.
__global__ void __launch_bounds__(kT, 3) k_ccmm_slot(const u64* __restrict__ At, const u64* __restrict__ Bt,
                                                  u64* __restrict__ Ct, const NttTab* __restrict__ tabs, int m,
                                                  int kd, int nd, int c_begin, int nc, int log_n) {
    extern __shared__ u64 sm[];
    const int l = blockIdx.y;
    const u32 s = blockIdx.x;
    const NttTab& T = tabs[l];
    const u64 q = T.q;
    const int sb = split_bits(q);
    const u64 fold_lim = (~0ull) >> (2 * sb + 2);  // c1 adds two products per k
    const int fold_k = fold_lim > 4096 ? 4096 : (int)(fold_lim ? fold_lim : 1);
    const u64 one_q = shoup_quotient_dev(1, q);
    const u64 r1 = (1ull << sb) % q, r2 = mul_barrett(r1, r1, Barrett{q, T.mu_hi, T.mu_lo});
    const u64 r1q = shoup_quotient_dev(r1, q), r2q = shoup_quotient_dev(r2, q);
    const size_t slot = ((size_t)l << log_n) + s;
    // stage A (both components, m x k) and the B columns of this block
    u64* a_s = sm;                  // [2][m * kd]
    u64* b_s = sm + 2 * m * kd;     // [2][kd * nc]
    const u64* asrc = At + slot * 2 * (size_t)(m * kd);
    for (int i = threadIdx.x; i < 2 * m * kd; i += blockDim.x) a_s[i] = asrc[i];
    const u64* bsrc = Bt + slot * 2 * (size_t)(kd * nd);
    for (int i = threadIdx.x; i < 2 * kd * nc; i += blockDim.x) {
        const int comp = i / (kd * nc), j = i % (kd * nc);
        b_s[i] = bsrc[(size_t)comp * kd * nd + (size_t)c_begin * kd + j];
    }
    __syncthreads();
    const int pairs = (nc + 1) / 2;
    u64* cdst = Ct + slot * 3 * (size_t)(m * nc);
    for (int item = threadIdx.x; item < m * pairs; item += blockDim.x) {
        const int r = item % m, c0 = 2 * (item / m);
        const bool c1ok = c0 + 1 < nc;
        const int cb0 = c0 * kd, cb1 = (c1ok ? c0 + 1 : c0) * kd;
        Split3 acc[3][2];
        u64 res[3][2];
#pragma unroll
        for (int t = 0; t < 3; ++t)
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                acc[t][j] = Split3{0, 0, 0};
                res[t][j] = 0;
            }
        int since = 0;
        for (int kk = 0; kk < kd; ++kk) {
            const u64 ab = a_s[kk * m + r], aa = a_s[m * kd + kk * m + r];
            const u64 bb[2] = {b_s[cb0 + kk], b_s[cb1 + kk]};
            const u64 ba[2] = {b_s[kd * nc + cb0 + kk], b_s[kd * nc + cb1 + kk]};
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                acc[0][j].mac(ab, bb[j]);
                acc[1][j].mac(ab, ba[j]);
                acc[1][j].mac(aa, bb[j]);
                acc[2][j].mac(aa, ba[j]);
            }
            if (++since == fold_k) {
#pragma unroll
                for (int t = 0; t < 3; ++t)
#pragma unroll
                    for (int j = 0; j < 2; ++j) {
                        res[t][j] = add_mod(res[t][j], split_fold(acc[t][j], q, one_q, r1, r1q, r2, r2q), q);
                        acc[t][j] = Split3{0, 0, 0};
                    }
                since = 0;
            }
        }
#pragma unroll
        for (int t = 0; t < 3; ++t)
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                if (j && !c1ok) continue;
                const u64 v = add_mod(res[t][j], split_fold(acc[t][j], q, one_q, r1, r1q, r2, r2q), q);
                cdst[(size_t)t * m * nc + (size_t)(c0 + j) * m + r] = v;
            }
    }
}

int32_t to_slot_major(ckks_ctx* ctx, const u64* X, u64* Xt, u32 n_ent, u32 e0, u32 ld, u32 L, bool split,
                      cudaStream_t st) {
    dim3 g(ctx->n / kTile, (n_ent + kTile - 1) / kTile, 2 * L);
    k_to_slot_major<<<g, kTile * 8, 0, st>>>(X, Xt, ctx->d_tabs, (int)n_ent, (int)e0, (int)ld, (int)L,
                                             (int)ctx->log_n, split ? 1 : 0);
    CKKS_CUDA_TRY(cudaGetLastError());
    return CKKS_OK;
}

// entry-major transforms of n_ent entries (NTT) written slot-major into Xt
int32_t build_slot_major(ckks_ctx* ctx, const u64* X, u64* Xt, u32 n_ent, u32 L, bool split, cudaStream_t st) {
    const size_t ct = (size_t)2 * L * ctx->n;
    u32 chunk = (u32)((size_t(1) << 28) / ct);
    if (chunk < 1) chunk = 1;
    if (chunk > 32767) chunk = 32767;
    Workspace<u64> buf;
    int32_t rc;
    const u32 m0 = chunk < n_ent ? chunk : n_ent;
    if ((rc = buf.alloc(ct * m0, st))) return rc;
    for (u32 e0 = 0; e0 < n_ent; e0 += chunk) {
        const u32 m = n_ent - e0 < chunk ? n_ent - e0 : chunk;
        if ((rc = ntt_forward_launch(ctx, X + (size_t)e0 * ct, buf.p, 2 * m, 0, L, st))) return rc;
        if ((rc = to_slot_major(ctx, buf.p, Xt, m, e0, n_ent, L, split, st))) return rc;
    }
    return CKKS_OK;
}

}  // namespace

int32_t ccmm_structured_launch(ckks_ctx* ctx, const ckks_ksk* key, const u64* A, const u64* B, u64* C, u32 m, u32 kd,
                               u32 nd, cudaStream_t st) {
    const u32 L = key->q_limbs, N = ctx->n;
    const size_t poly = (size_t)L * N, ct = 2 * poly, slots = (size_t)L * N;
    if (N < (u32)kTile) {
        ckks_set_error("ckks_ccmm_structured: ring degree below 32 is not supported");
        return CKKS_ERR_BAD_ARG;
    }
    const bool use_tc = ccmm_tc_supported(ctx, m, kd);
    Workspace<u64> At, Bt;
    Workspace<int> terr;
    int32_t rc;
    if ((rc = At.alloc(slots * 2 * m * kd, st)) || (rc = Bt.alloc(slots * 2 * kd * nd, st))) return rc;
    if (use_tc) {
        if ((rc = terr.alloc(1, st))) return rc;
        CKKS_CUDA_TRY(cudaMemsetAsync(terr.p, 0, sizeof(int), st));
    }
    if ((rc = build_slot_major(ctx, A, At.p, m * kd, L, !use_tc, st))) return rc;
    if ((rc = build_slot_major(ctx, B, Bt.p, kd * nd, L, !use_tc, st))) return rc;
    // output columns per chunk: slot-major products plus entry-major quadratic parts within about 2^31 words
    u32 cc = (u32)((size_t(1) << 31) / (slots * 3 * m * 2));
    if (cc > 2) cc &= ~1u;  // whole column pairs per thread
    if (cc > 32767 / m) cc = 32767 / m;  // grid limits of the per-chunk transforms and rescale
    if (cc < 1) cc = 1;
    if (cc > nd) cc = nd;
    const size_t smem = (size_t)2 * (m * kd + kd * cc) * sizeof(u64);
    if (!use_tc && smem > 200 * 1024) {
        ckks_set_error("ckks_ccmm_structured: matrix blocks exceed shared memory (rows * inner too large)");
        return CKKS_ERR_BAD_ARG;
    }
    CKKS_CUDA_TRY(cudaFuncSetAttribute(k_ccmm_slot, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    for (u32 c0 = 0; c0 < nd; c0 += cc) {
        const u32 nc = nd - c0 < cc ? nd - c0 : cc;
        const u32 n_out = m * nc;
        Workspace<u64> Ct, Q;
        if ((rc = Ct.alloc(slots * 3 * n_out, st)) || (rc = Q.alloc(3 * poly * n_out, st))) return rc;
        u64* Q01 = Q.p;                       // [n_out][2][L][N]
        u64* C2 = Q.p + 2 * poly * n_out;     // [n_out][L][N]
        if (use_tc) {
            if ((rc = ccmm_slot_tc_launch(ctx, At.p, Bt.p, Ct.p, L, m, kd, nd, c0, nc, terr.p, st))) return rc;
        } else {
            dim3 g(N, L);
            k_ccmm_slot<<<g, kT, smem, st>>>(At.p, Bt.p, Ct.p, ctx->d_tabs, (int)m, (int)kd, (int)nd, (int)c0,
                                             (int)nc, (int)ctx->log_n);
            CKKS_CUDA_TRY(cudaGetLastError());
        }
        dim3 gt(N / kTile, (n_out + kTile - 1) / kTile, 3 * L);
        k_from_slot_major<<<gt, kTile * 8, 0, st>>>(Ct.p, Q01, C2, (int)n_out, (int)n_out, (int)L, (int)ctx->log_n);
        CKKS_CUDA_TRY(cudaGetLastError());
        if ((rc = ntt_inverse_launch(ctx, C2, C2, n_out, 0, L, st))) return rc;
        // relinearize in sub-batches bounded by the digit-transform workspace
        const size_t per = (size_t)key->D * N * (1 + L);
        u32 sub = (u32)((size_t(1) << 28) / per);
        if (sub < 1) sub = 1;
        const u32 dmax = 65535 / (key->D > 2 ? key->D : 2);
        if (sub > dmax) sub = dmax;
        for (u32 i0 = 0; i0 < n_out; i0 += sub) {
            const u32 cnt = n_out - i0 < sub ? n_out - i0 : sub;
            if ((rc = relin_core_launch(ctx, key, C2 + (size_t)i0 * poly, Q01 + (size_t)i0 * ct, cnt, st))) return rc;
        }
        if ((rc = ntt_inverse_launch(ctx, Q01, Q01, 2 * n_out, 0, L, st))) return rc;
        if ((rc = rescale_launch(ctx, Q01, C + (size_t)c0 * m * 2 * (L - 1) * N, 2 * n_out, L, st))) return rc;
    }
    (void)ct;
    if (use_tc) {
        int h_err = 0;
        CKKS_CUDA_TRY(cudaMemcpyAsync(&h_err, terr.p, sizeof(int), cudaMemcpyDeviceToHost, st));
        CKKS_CUDA_TRY(cudaStreamSynchronize(st));
        ctx->last_mac_path = 1;
        if (h_err) {
            ckks_set_error("ckks_ccmm_structured: a tensor-core pipeline wait timed out (stage " +
                           std::to_string(h_err) + ")");
            return CKKS_ERR_TIMEOUT;
        }
    } else {
        ctx->last_mac_path = 0;
    }
    return CKKS_OK;
}
