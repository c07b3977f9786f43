// ntt.cu -- batched negacyclic NTT / inverse NTT for sm_100a.
//
// Two passes over HBM per transform (N = N1 * N2, both <= 512 for N <= 2^17):
//   forward pass 1: per column j1, a merged Cooley-Tukey negacyclic N2-point
//                   transform along j2 (psi2 = psi^N1), times psi^((2k2+1) j1);
//                   written as rows [j1][k2];
//   forward pass 2: per column k2, a cyclic N1-point DIT transform along j1
//                   (w1 = psi^(2 N2)); written in natural order k2 + N2 k1.
// The inverse runs the mirror image (Gentleman-Sande).
// Each CTA stages a tile of C (<= 16) columns in shared memory; butterflies
// keep values lazily reduced in [0, 4q) with Shoup multiplication
// (__umul64hi); outputs are canonical. Result values equal the reference's
// PreparedNttPlan::forward (ring/prepared_ntt.rs:200-231) word for word:
// both compute the unique A[k] = a(psi^(2k+1)) mod q.
#include "kernels.cuh"

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ u32 bitrev(u32 x, int bits) { return __brev(x) >> (32 - bits); }

// Row-dependent XOR swizzle of the column index inside a [rows][C] tile so
// that reading one column across bit-reversed rows is bank-conflict free.
__device__ __forceinline__ int swz(u32 row, int log_rows, int C) { return (int)(bitrev(row, log_rows) & (C - 1)); }

// Forward pass 1: tile of C columns j1, N2 rows j2. With kDigits the input is
// a signed digit polynomial [D][N] (int64) shared by every limb, lifted to
// [0, q) on load (signed_mod, hybrid_rns_galois_key.rs:55-57); blockIdx.z
// then indexes the digit.
template <bool kDigits>
__global__ void __launch_bounds__(kThreads) k_ntt_fwd_pass1(const void* __restrict__ in_, u64* __restrict__ out,
                                                            const NttTab* __restrict__ tabs, LimbMap lm,
                                                            int limb_count, int log_n1, int log_n2, int log_c) {
    extern __shared__ u64 sm[];
    const int N2 = 1 << log_n2, C = 1 << log_c;
    const int limb = blockIdx.y;
    const NttTab T = tabs[lm(limb)];
    const u64 q = T.q, q2 = q << 1;
    const size_t base = ((size_t)blockIdx.z * limb_count + limb) << (log_n1 + log_n2);
    const int j1_0 = blockIdx.x << log_c;

    if (kDigits) {
        const i64* in = (const i64*)in_ + ((size_t)blockIdx.z << (log_n1 + log_n2));
        for (int idx = threadIdx.x; idx < (N2 << log_c); idx += blockDim.x) {
            int j2 = idx >> log_c, c = idx & (C - 1);
            i64 d = in[j1_0 + c + ((size_t)j2 << log_n1)];
            u64 a = d < 0 ? (u64)(-d) : (u64)d;
            a = a >= q ? a % q : a;
            sm[(j2 << log_c) + (c ^ swz(j2, log_n2, C))] = (d < 0 && a) ? q - a : a;
        }
    } else {
        const u64* in = (const u64*)in_;
        for (int idx = threadIdx.x; idx < (N2 << log_c); idx += blockDim.x) {
            int j2 = idx >> log_c, c = idx & (C - 1);
            sm[(j2 << log_c) + (c ^ swz(j2, log_n2, C))] = in[base + j1_0 + c + ((size_t)j2 << log_n1)];
        }
    }
    __syncthreads();
    // merged CT: natural in -> bit-reversed out (psi_rev holds psi2^bitrev(i))
    for (int m = 1, lt = log_n2 - 1; m < N2; m <<= 1, --lt) {
        for (int idx = threadIdx.x; idx < ((N2 >> 1) << log_c); idx += blockDim.x) {
            int c = idx & (C - 1), b = idx >> log_c;
            int i = b >> lt;
            int r0 = (i << (lt + 1)) + (b & ((1 << lt) - 1)), r1 = r0 + (1 << lt);
            u64 S = __ldg(T.psi_rev + m + i), Sq = __ldg(T.psi_rev_q + m + i);
            u64* p0 = &sm[(r0 << log_c) + (c ^ swz(r0, log_n2, C))];
            u64* p1 = &sm[(r1 << log_c) + (c ^ swz(r1, log_n2, C))];
            u64 X = *p0, Y = *p1;
            X = X >= q2 ? X - q2 : X;
            u64 t = mul_shoup_lazy(Y, S, Sq, q);
            *p0 = X + t;
            *p1 = X - t + q2;
        }
        __syncthreads();
    }
    // twiddle psi^((2k2+1) j1), store rows [j1][k2] (lazy, [0, 2q))
    for (int idx = threadIdx.x; idx < (N2 << log_c); idx += blockDim.x) {
        int k2 = idx & (N2 - 1), c = idx >> log_n2;
        u32 r = bitrev(k2, log_n2);
        u64 v = sm[(r << log_c) + (c ^ (k2 & (C - 1)))];
        size_t t = ((size_t)(j1_0 + c) << log_n2) + k2;
        out[base + t] = mul_shoup_lazy(v, __ldg(T.mid + t), __ldg(T.mid_q + t), q);
    }
}

// Forward pass 2: tile of C columns k2, N1 rows j1. The CTA reads its whole
// tile before writing the same addresses, so src may equal dst.
__global__ void __launch_bounds__(kThreads) k_ntt_fwd_pass2(const u64* src, u64* dst, const NttTab* __restrict__ tabs,
                                                            LimbMap lm, int limb_count, int log_n1, int log_n2,
                                                            int log_c) {
    extern __shared__ u64 sm[];
    const int N1 = 1 << log_n1, N2 = 1 << log_n2, C = 1 << log_c;
    const int limb = blockIdx.y;
    const NttTab T = tabs[lm(limb)];
    const u64 q = T.q, q2 = q << 1;
    const size_t base = ((size_t)blockIdx.z * limb_count + limb) << (log_n1 + log_n2);
    const int k2_0 = blockIdx.x << log_c;

    for (int idx = threadIdx.x; idx < (N1 << log_c); idx += blockDim.x) {
        int j1 = idx >> log_c, c = idx & (C - 1);
        sm[(bitrev(j1, log_n1) << log_c) + c] = src[base + ((size_t)j1 << log_n2) + k2_0 + c];
    }
    __syncthreads();
    // cyclic DIT: bit-reversed in -> natural out
    for (int lh = 0; lh < log_n1; ++lh) {
        const int half = 1 << lh;
        const int tw_shift = log_n1 - lh - 1;  // w1^(o * N1/len), len = 2*half
        for (int idx = threadIdx.x; idx < ((N1 >> 1) << log_c); idx += blockDim.x) {
            int c = idx & (C - 1), b = idx >> log_c;
            int o = b & (half - 1), blk = b >> lh;
            int r0 = (blk << (lh + 1)) + o, r1 = r0 + half;
            int ti = o << tw_shift;
            u64 W = __ldg(T.w + ti), Wq = __ldg(T.w_q + ti);
            u64* p0 = &sm[(r0 << log_c) + c];
            u64* p1 = &sm[(r1 << log_c) + c];
            u64 X = *p0, Y = *p1;
            X = X >= q2 ? X - q2 : X;
            u64 t = mul_shoup_lazy(Y, W, Wq, q);
            *p0 = X + t;
            *p1 = X - t + q2;
        }
        __syncthreads();
    }
    for (int idx = threadIdx.x; idx < (N1 << log_c); idx += blockDim.x) {
        int k1 = idx >> log_c, c = idx & (C - 1);
        dst[base + ((size_t)k1 << log_n2) + k2_0 + c] = reduce_4q(sm[(k1 << log_c) + c], q);
    }
}

// Inverse pass A: tile of C columns k2; cyclic GS over k1 (natural in ->
// bit-reversed out), times N^-1 psi^-((2k2+1) j1), stored as rows [k2][j1].
__global__ void __launch_bounds__(kThreads) k_ntt_inv_passA(const u64* __restrict__ in, u64* __restrict__ out,
                                                            const NttTab* __restrict__ tabs, LimbMap lm,
                                                            int limb_count, int log_n1, int log_n2, int log_c) {
    extern __shared__ u64 sm[];
    const int N1 = 1 << log_n1, C = 1 << log_c;
    const int limb = blockIdx.y;
    const NttTab T = tabs[lm(limb)];
    const u64 q = T.q, q2 = q << 1;
    const size_t base = ((size_t)blockIdx.z * limb_count + limb) << (log_n1 + log_n2);
    const int k2_0 = blockIdx.x << log_c;

    for (int idx = threadIdx.x; idx < (N1 << log_c); idx += blockDim.x) {
        int k1 = idx >> log_c, c = idx & (C - 1);
        sm[(k1 << log_c) + (c ^ swz(k1, log_n1, C))] = in[base + ((size_t)k1 << log_n2) + k2_0 + c];
    }
    __syncthreads();
    for (int lh = log_n1 - 1; lh >= 0; --lh) {
        const int half = 1 << lh;
        const int tw_shift = log_n1 - lh - 1;
        for (int idx = threadIdx.x; idx < ((N1 >> 1) << log_c); idx += blockDim.x) {
            int c = idx & (C - 1), b = idx >> log_c;
            int o = b & (half - 1), blk = b >> lh;
            int r0 = (blk << (lh + 1)) + o, r1 = r0 + half;
            int ti = o << tw_shift;
            u64 W = __ldg(T.w_inv + ti), Wq = __ldg(T.w_inv_q + ti);
            u64* p0 = &sm[(r0 << log_c) + (c ^ swz(r0, log_n1, C))];
            u64* p1 = &sm[(r1 << log_c) + (c ^ swz(r1, log_n1, C))];
            u64 X = *p0, Y = *p1;
            u64 s = X + Y;
            *p0 = s >= q2 ? s - q2 : s;
            *p1 = mul_shoup_lazy(X - Y + q2, W, Wq, q);
        }
        __syncthreads();
    }
    for (int idx = threadIdx.x; idx < (N1 << log_c); idx += blockDim.x) {
        int j1 = idx & (N1 - 1), c = idx >> log_n1;
        u32 r = bitrev(j1, log_n1);
        u64 v = sm[(r << log_c) + (c ^ (j1 & (C - 1)))];
        size_t t = ((size_t)(k2_0 + c) << log_n1) + j1;
        out[base + t] = mul_shoup_lazy(v, __ldg(T.imid + t), __ldg(T.imid_q + t), q);
    }
}

// Inverse pass B: tile of C columns j1; merged GS negacyclic over k2
// (bit-reversed in -> natural out). src may equal dst (same address set per CTA).
__global__ void __launch_bounds__(kThreads) k_ntt_inv_passB(const u64* src, u64* dst, const NttTab* __restrict__ tabs,
                                                            LimbMap lm, int limb_count, int log_n1, int log_n2,
                                                            int log_c) {
    extern __shared__ u64 sm[];
    const int N2 = 1 << log_n2, C = 1 << log_c;
    const int limb = blockIdx.y;
    const NttTab T = tabs[lm(limb)];
    const u64 q = T.q, q2 = q << 1;
    const size_t base = ((size_t)blockIdx.z * limb_count + limb) << (log_n1 + log_n2);
    const int j1_0 = blockIdx.x << log_c;

    for (int idx = threadIdx.x; idx < (N2 << log_c); idx += blockDim.x) {
        int k2 = idx >> log_c, c = idx & (C - 1);
        sm[(bitrev(k2, log_n2) << log_c) + c] = src[base + ((size_t)k2 << log_n1) + j1_0 + c];
    }
    __syncthreads();
    for (int lt = 0, h = N2 >> 1; h >= 1; ++lt, h >>= 1) {
        for (int idx = threadIdx.x; idx < ((N2 >> 1) << log_c); idx += blockDim.x) {
            int c = idx & (C - 1), b = idx >> log_c;
            int i = b >> lt;
            int r0 = (i << (lt + 1)) + (b & ((1 << lt) - 1)), r1 = r0 + (1 << lt);
            u64 S = __ldg(T.psi_inv_rev + h + i), Sq = __ldg(T.psi_inv_rev_q + h + i);
            u64* p0 = &sm[(r0 << log_c) + c];
            u64* p1 = &sm[(r1 << log_c) + c];
            u64 X = *p0, Y = *p1;
            u64 s = X + Y;
            *p0 = s >= q2 ? s - q2 : s;
            *p1 = mul_shoup_lazy(X - Y + q2, S, Sq, q);
        }
        __syncthreads();
    }
    for (int idx = threadIdx.x; idx < (N2 << log_c); idx += blockDim.x) {
        int j2 = idx >> log_c, c = idx & (C - 1);
        dst[base + j1_0 + c + ((size_t)j2 << log_n1)] = reduce_2q(sm[(j2 << log_c) + c], q);
    }
}

int log2_min(int log_dim, int log_cmax) { return log_dim < log_cmax ? log_dim : log_cmax; }

}  // namespace

void ntt_set_smem_limits() {
    static bool done = false;
    if (done) return;
    int bytes = 96 * 1024;
    cudaFuncSetAttribute(k_ntt_fwd_pass1<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    cudaFuncSetAttribute(k_ntt_fwd_pass1<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    cudaFuncSetAttribute(k_ntt_fwd_pass2, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    cudaFuncSetAttribute(k_ntt_inv_passA, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    cudaFuncSetAttribute(k_ntt_inv_passB, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    done = true;
}

int32_t ntt_forward_launch(ckks_ctx* ctx, const u64* in, u64* out, u32 n_polys, u32 limb_begin, u32 limb_count,
                           cudaStream_t st) {
    return ntt_forward_launch_map(ctx, in, out, n_polys, LimbMap::range(limb_begin, limb_count), limb_count, st);
}

int32_t ntt_inverse_launch(ckks_ctx* ctx, const u64* in, u64* out, u32 n_polys, u32 limb_begin, u32 limb_count,
                           cudaStream_t st) {
    return ntt_inverse_launch_map(ctx, in, out, n_polys, LimbMap::range(limb_begin, limb_count), limb_count, st);
}

int32_t ntt_forward_launch_map(ckks_ctx* ctx, const u64* in, u64* out, u32 n_polys, LimbMap lm, u32 limb_count,
                               cudaStream_t st) {
    if (n_polys == 0 || limb_count == 0) return CKKS_OK;
    const int l1 = ctx->log_n1, l2 = ctx->log_n2;
    u64* mid = out;
    Workspace<u64> tmp;
    if (in == out) {  // pass 1 reads columns and writes rows: stage through a workspace
        if (int32_t rc = tmp.alloc((size_t)n_polys * limb_count * ctx->n, st)) return rc;
        mid = tmp.p;
    }
    int lc1 = log2_min(l1, 4), lc2 = log2_min(l2, 4);
    dim3 g1(1u << (l1 - lc1), limb_count, n_polys), g2(1u << (l2 - lc2), limb_count, n_polys);
    k_ntt_fwd_pass1<false><<<g1, kThreads, (sizeof(u64) << (l2 + lc1)), st>>>(in, mid, ctx->d_tabs, lm, limb_count,
                                                                       l1, l2, lc1);
    k_ntt_fwd_pass2<<<g2, kThreads, (sizeof(u64) << (l1 + lc2)), st>>>(mid, out, ctx->d_tabs, lm,
                                                                       limb_count, l1, l2, lc2);
    CKKS_CUDA_TRY(cudaGetLastError());
    return CKKS_OK;
}

int32_t ntt_inverse_launch_map(ckks_ctx* ctx, const u64* in, u64* out, u32 n_polys, LimbMap lm, u32 limb_count,
                               cudaStream_t st) {
    if (n_polys == 0 || limb_count == 0) return CKKS_OK;
    const int l1 = ctx->log_n1, l2 = ctx->log_n2;
    u64* mid = out;
    Workspace<u64> tmp;
    if (in == out) {
        if (int32_t rc = tmp.alloc((size_t)n_polys * limb_count * ctx->n, st)) return rc;
        mid = tmp.p;
    }
    int lcA = log2_min(l2, 4), lcB = log2_min(l1, 4);
    dim3 gA(1u << (l2 - lcA), limb_count, n_polys), gB(1u << (l1 - lcB), limb_count, n_polys);
    k_ntt_inv_passA<<<gA, kThreads, (sizeof(u64) << (l1 + lcA)), st>>>(in, mid, ctx->d_tabs, lm, limb_count,
                                                                       l1, l2, lcA);
    k_ntt_inv_passB<<<gB, kThreads, (sizeof(u64) << (l2 + lcB)), st>>>(mid, out, ctx->d_tabs, lm,
                                                                       limb_count, l1, l2, lcB);
    CKKS_CUDA_TRY(cudaGetLastError());
    return CKKS_OK;
}

int32_t ntt_forward_digits_launch(ckks_ctx* ctx, const i64* digits, u64* out, u32 D, LimbMap lm, u32 limbs,
                                  cudaStream_t st) {
    if (D == 0 || limbs == 0) return CKKS_OK;
    const int l1 = ctx->log_n1, l2 = ctx->log_n2;
    int lc1 = log2_min(l1, 4), lc2 = log2_min(l2, 4);
    dim3 g1(1u << (l1 - lc1), limbs, D), g2(1u << (l2 - lc2), limbs, D);
    k_ntt_fwd_pass1<true><<<g1, kThreads, (sizeof(u64) << (l2 + lc1)), st>>>(digits, out, ctx->d_tabs, lm, limbs, l1,
                                                                             l2, lc1);
    k_ntt_fwd_pass2<<<g2, kThreads, (sizeof(u64) << (l1 + lc2)), st>>>(out, out, ctx->d_tabs, lm, limbs, l1, l2, lc2);
    CKKS_CUDA_TRY(cudaGetLastError());
    return CKKS_OK;
}
