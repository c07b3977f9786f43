// elementwise.cu -- limb-parallel kernels: Galois automorphisms (coefficient
// and NTT domain), NTT-domain products and sums, rescale, and the exact
// QP -> Q ModDown. One thread per (limb, coefficient); grids are
// (N / 256, limbs, polys), coalesced on the contiguous coefficient axis.
#include "context.cuh"
#include "kernels.cuh"
#include "ntt_core.cuh"
#include "moddown_f64.cuh"

namespace {

constexpr int kT = 256;

// ckks/automorphism.rs:8-48, output-driven: out[t] = +-in[s], s = t * k^-1 mod 2N
__global__ void k_automorphism_coef(const u64* __restrict__ in, u64* __restrict__ out, const NttTab* __restrict__ tabs,
                                    LimbMap lm, int limbs, int log_n, u64 k_inv) {
    const u32 n = 1u << log_n;
    const u32 t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int limb = blockIdx.y;
    const size_t base = ((size_t)blockIdx.z * limbs + limb) << log_n;
    const u64 s = ((u64)t * k_inv) & (2ull * n - 1);
    const u64 q = tabs[lm(limb)].q;
    u64 v = in[base + (s & (n - 1))];
    out[base + t] = s >= n ? neg_mod(v, q) : v;
}

// ring/ntt_galois_permutation.rs:5-19: out[i] = in[((k (2i+1)) mod 2N - 1) / 2]
__global__ void k_automorphism_ntt(const u64* __restrict__ in, u64* __restrict__ out, int limbs, int log_n, u64 k) {
    const u32 n = 1u << log_n;
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const size_t base = ((size_t)blockIdx.z * limbs + blockIdx.y) << log_n;
    out[base + i] = in[base + (galois_src(i, k, log_n))];
}

// op: 0 mul, 1 add, 2 sub (ring/ntt_polynomial.rs:186-236, ring/polynomial.rs add/sub)
__global__ void k_pointwise(const u64* __restrict__ a, const u64* __restrict__ b, u64* __restrict__ out,
                            const NttTab* __restrict__ tabs, LimbMap lm, int limbs, int log_n, int op) {
    const u32 n = 1u << log_n;
    const u32 c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    const int limb = blockIdx.y;
    const size_t i = (((size_t)blockIdx.z * limbs + limb) << log_n) + c;
    const NttTab& T = tabs[lm(limb)];
    Barrett m{T.q, T.mu_hi, T.mu_lo};
    u64 x = a[i], y = b[i];
    out[i] = op == 0 ? mul_barrett(x, y, m) : op == 1 ? add_mod(x, y, T.q) : sub_mod(x, y, T.q);
}

// ckks/rns_rescale.rs:107-167: ((x - centered(x mod q_d)) * q_d^-1) mod q_i
__global__ void k_rescale(const u64* __restrict__ in, u64* __restrict__ out, const NttTab* __restrict__ tabs,
                          const u64* __restrict__ inv, const u64* __restrict__ inv_q, int limbs_in, int log_n) {
    const u32 n = 1u << log_n;
    const u32 c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    const int i = blockIdx.y, drop = limbs_in - 1;
    const u64 qd = tabs[drop].q, qi = tabs[i].q;
    const size_t src = (size_t)blockIdx.z * limbs_in << log_n;
    const size_t dst = (size_t)blockIdx.z * (limbs_in - 1) << log_n;
    u64 r = in[src + ((size_t)drop << log_n) + c];
    u64 rq;
    if (r > qd / 2) {
        u64 mag = qd - r;
        mag = mag >= qi ? mag % qi : mag;
        rq = neg_mod(mag, qi);
    } else {
        rq = r >= qi ? r % qi : r;
    }
    u64 d = sub_mod(in[src + ((size_t)i << log_n) + c], rq, qi);
    out[dst + ((size_t)i << log_n) + c] = mul_shoup(d, inv[i], inv_q[i], qi);
}

// ring/auxiliary_modulus.rs:89-171: centered CRT over P from the K auxiliary
// residues (mixed-radix Garner, exact), then (x_i - r) * P^-1 mod q_i for every
// Q limb. One thread per output coefficient t; with exps_inv, the output is
// the coefficient automorphism X -> X^k of the ModDown result
// (k^-1 = exps_inv[(poly / 2) % n_keys]): out[t] = +-value[s] with
// s = t k^-1 mod 2N (negated when s >= N), so the stores are coalesced and the
// reads gather within one polynomial. ModDown commutes exactly with that
// signed permutation because P is odd.
// KT > 0 fixes the number of auxiliary limbs at compile time (KT == 0: md.K at
// run time). The Q-limb gathers are issued kBatch at a time so each thread keeps
// several independent loads in flight (the reads are scattered under sigma).
// Per-limb constants are staged in shared memory: q, (P^-1 mod q, Shoup),
// -P mod q, (2K+1) q, then (p_0..p_{j-1} mod q, Shoup) for j < K. kLazy (every Q
// prime below 2^59): the K products are summed lazily in [0, 2q) each and the
// difference x - r is formed as x + (2K+1) q - r < (2K+2) q < 2^64, with one
// reduction at the end; the result is the same canonical residue.
template <int KT, bool kLazy>
__global__ void __launch_bounds__(kT) k_mod_down(const u64* __restrict__ in, u64* __restrict__ out, ModDownConst md,
                                                 int q_limbs, int log_n, const u64* __restrict__ exps_inv, int n_keys) {
    constexpr int kBatch = 8;
    extern __shared__ u64 cs[];
    const int K = KT > 0 ? KT : md.K;
    constexpr int KM = KT > 0 ? KT : kMaxAux;
    const int W = 5 + 2 * K;
    for (int idx = threadIdx.x; idx < q_limbs * W; idx += blockDim.x) {
        const int i = idx / W, f = idx - i * W;
        const u64 qi = md.q[i];
        u64 v;
        if (f == 0) v = qi;
        else if (f == 1) v = md.pinv_mod_q[i];
        else if (f == 2) v = md.pinv_mod_q_q[i];
        else if (f == 3) v = qi - md.p_mod_q[i];  // P mod q is in [1, q): distinct primes
        else if (f == 4) v = (u64)(2 * K + 1) * qi;
        else if (f < 5 + K) v = md.pre[(size_t)i * kMaxAux + (f - 5)];
        else v = md.pre_q[(size_t)i * kMaxAux + (f - 5 - K)];
        cs[idx] = v;
    }
    __syncthreads();
    const u32 n = 1u << log_n;
    const u32 t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const size_t src = (size_t)blockIdx.y * (q_limbs + K) << log_n;
    const size_t dst = (size_t)blockIdx.y * q_limbs << log_n;
    u32 c = t;
    bool flip = false;
    if (exps_inv) {
        const u64 s = ((u64)t * exps_inv[(blockIdx.y >> 1) % n_keys]) & (2ull * n - 1);
        flip = s >= n;
        c = (u32)(s & (n - 1));
    }
    const u64* x = in + src + c;
    u64 v[KM];
#pragma unroll
    for (int i = 0; i < KM; ++i)
        if (i < K) v[i] = __ldg(x + ((size_t)(q_limbs + i) << log_n));
#pragma unroll
    for (int i = 0; i < KM; ++i) {
        if (i < K) {
            const u64 p = md.p[i];
            u64 acc = 0;
#pragma unroll
            for (int j = 0; j < i; ++j) acc = add_mod(acc, mul_shoup(v[j], md.pp[i][j], md.pp_q[i][j], p), p);
            v[i] = mul_shoup(sub_mod(v[i], acc, p), md.pinv[i], md.pinv_q[i], p);
        }
    }
    // centered: value > floor(P/2) -> negative (lexicographic mixed-radix compare)
    bool neg = false, decided = false;
#pragma unroll
    for (int i = KM - 1; i >= 0; --i) {
        if (i < K && !decided && v[i] != md.half[i]) {
            neg = v[i] > md.half[i];
            decided = true;
        }
    }
    u64* o = out + dst + t;
    for (int i0 = 0; i0 < q_limbs; i0 += kBatch) {
        u64 xin[kBatch];
#pragma unroll
        for (int u = 0; u < kBatch; ++u)
            if (i0 + u < q_limbs) xin[u] = __ldg(x + ((size_t)(i0 + u) << log_n));
#pragma unroll
        for (int u = 0; u < kBatch; ++u) {
            const int i = i0 + u;
            if (i < q_limbs) {
                const u64* ci = cs + i * W;
                const u64 qi = ci[0];
                u64 r = neg ? ci[3] : 0;  // r == centred CRT_P(x_P) mod q, lazily
                u64 w;
                if (kLazy) {
#pragma unroll
                    for (int j = 0; j < KM; ++j)
                        if (j < K) r += mul_shoup_lazy(v[j], ci[5 + j], ci[5 + K + j], qi);
                    w = reduce_2q(mul_shoup_lazy(xin[u] + ci[4] - r, ci[1], ci[2], qi), qi);
                } else {
#pragma unroll
                    for (int j = 0; j < KM; ++j)
                        if (j < K) r = add_mod(r, mul_shoup(v[j], ci[5 + j], ci[5 + K + j], qi), qi);
                    w = mul_shoup(sub_mod(xin[u], r, qi), ci[1], ci[2], qi);
                }
                o[(size_t)i << log_n] = flip ? neg_mod(w, qi) : w;
            }
        }
    }
}

// ModDown on the FP64 pipe, for Q primes below 2^50 and K <= 3 auxiliary limbs
// (the integer form above is instruction-bound on the ALU and FMA pipes while
// the FP64 pipe idles). The centred CRT value y_c of the auxiliary residues is
// rebuilt exactly from its mixed-radix digits as three 64-bit words
// (|y_c| < P/2 < 2^187) and its magnitude split into four 47-bit words w_k;
// then per Q limb, with s the sign of y_c,
//   out = x P^-1 - s sum_k w_k (2^(47 k) P^-1 mod q)   (mod q):
// five exact FP64 modular products (nttf::mulmod, multiplicands below 2^51, so
// each result is below 0.75 q in magnitude and the sum below 3.75 q) and one
// exact reduction. The words equal k_mod_down's. sigma as there.
template <int KT>
__global__ void __launch_bounds__(kT) k_mod_down_f64(const u64* __restrict__ in, u64* __restrict__ out,
                                                     ModDownConst md, int q_limbs, int log_n,
                                                     const u64* __restrict__ exps_inv, int n_keys) {
    extern __shared__ double fcs[];  // [q_limbs][12]: q, 1/q, (P^-1, /q), (2^(47k) P^-1, /q) k = 0..3
    for (int idx = threadIdx.x; idx < q_limbs * 12; idx += blockDim.x) fcs[idx] = md.f64c[idx];
    __syncthreads();
    const u32 n = 1u << log_n;
    const u32 t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const size_t src = (size_t)blockIdx.y * (q_limbs + KT) << log_n;
    const size_t dst = (size_t)blockIdx.y * q_limbs << log_n;
    u32 c = t;
    bool flip = false;
    if (exps_inv) {
        const u64 sg = ((u64)t * exps_inv[(blockIdx.y >> 1) % n_keys]) & (2ull * n - 1);
        flip = sg >= n;
        c = (u32)(sg & (n - 1));
    }
    const u64* x = in + src + c;
    u64 v[KT];
#pragma unroll
    for (int i = 0; i < KT; ++i) v[i] = __ldg(x + ((size_t)(q_limbs + i) << log_n));
    double w[4];
    bool neg;
    mdf::crt_words<KT>(v, md, w, neg);
    u64* o = out + dst + t;
    for (int i = 0; i < q_limbs; ++i)
        o[(size_t)i << log_n] = mdf::limb(nttf::from_u52(__ldg(x + ((size_t)i << log_n))), w, neg, fcs + i * 12, flip);
}

}  // namespace

// ------------------------------------------------------------------ launchers
int32_t automorphism_coef_launch(ckks_ctx* ctx, const u64* in, u64* out, u32 n_polys, LimbMap lm, u32 limbs, u64 k,
                                 cudaStream_t st) {
    if (!n_polys || !limbs) return CKKS_OK;
    const u64 two_n = 2ull * ctx->n;
    k %= two_n;
    u64 k_inv = 1;  // inverse of k modulo 2N (odd k): k^(N/2 * 2 - 1) via repeated squaring in Z/2N
    {
        u64 e = ctx->n - 1, b = k;  // group (Z/2NZ)^* has exponent N/2; k^(N-1) = k^-1
        while (e) {
            if (e & 1) k_inv = (k_inv * b) % two_n;
            b = (b * b) % two_n;
            e >>= 1;
        }
    }
    dim3 g((ctx->n + kT - 1) / kT, limbs, n_polys);
    k_automorphism_coef<<<g, kT, 0, st>>>(in, out, ctx->d_tabs, lm, limbs, ctx->log_n, k_inv);
    CKKS_CUDA_TRY(cudaGetLastError());
    return CKKS_OK;
}

int32_t automorphism_ntt_launch(ckks_ctx* ctx, const u64* in, u64* out, u32 n_polys, u32 limbs, u64 k,
                                cudaStream_t st) {
    if (!n_polys || !limbs) return CKKS_OK;
    dim3 g((ctx->n + kT - 1) / kT, limbs, n_polys);
    k_automorphism_ntt<<<g, kT, 0, st>>>(in, out, limbs, ctx->log_n, k % (2ull * ctx->n));
    CKKS_CUDA_TRY(cudaGetLastError());
    return CKKS_OK;
}

int32_t pointwise_launch(ckks_ctx* ctx, const u64* a, const u64* b, u64* out, u32 n_polys, LimbMap lm, u32 limbs,
                         int op, cudaStream_t st) {
    if (!n_polys || !limbs) return CKKS_OK;
    dim3 g((ctx->n + kT - 1) / kT, limbs, n_polys);
    k_pointwise<<<g, kT, 0, st>>>(a, b, out, ctx->d_tabs, lm, limbs, ctx->log_n, op);
    CKKS_CUDA_TRY(cudaGetLastError());
    return CKKS_OK;
}

int32_t rescale_launch(ckks_ctx* ctx, const u64* in, u64* out, u32 n_polys, u32 limbs_in, cudaStream_t st) {
    if (!n_polys) return CKKS_OK;
    const u64* inv = ctx->d_rescale_inv + (size_t)(limbs_in - 1) * 2 * ctx->L;
    dim3 g((ctx->n + kT - 1) / kT, limbs_in - 1, n_polys);
    k_rescale<<<g, kT, 0, st>>>(in, out, ctx->d_tabs, inv, inv + ctx->L, limbs_in, ctx->log_n);
    CKKS_CUDA_TRY(cudaGetLastError());
    return CKKS_OK;
}

int32_t mod_down_launch(ckks_ctx* ctx, const u64* in, u64* out, u32 n_polys, u32 q_limbs, cudaStream_t st) {
    return mod_down_sigma_multi(ctx, in, out, n_polys, q_limbs, nullptr, 1, st);
}

int32_t mod_down_sigma_multi(ckks_ctx* ctx, const u64* in, u64* out, u32 n_polys, u32 q_limbs,
                             const u64* d_exps_inv, u32 n_keys, cudaStream_t st) {
    if (!n_polys) return CKKS_OK;
    // lazy differences need (2K + 2) q < 2^64: every Q prime below 2^59 (K <= 8)
    bool lazy = true, f64 = ctx->K >= 1 && ctx->K <= 3;
    for (u32 i = 0; i < q_limbs; ++i) {
        lazy = lazy && ctx->moduli[i] < (1ull << 59);
        f64 = f64 && ctx->moduli[i] < (1ull << 50);
    }
    for (u32 k = 0; k < ctx->K; ++k) f64 = f64 && ctx->moduli[ctx->L + k] < (1ull << 62);
    // grid.y limit: chunks are multiples of 2 * n_keys so (poly / 2) % n_keys pairs stay aligned
    const u32 unit = 2 * (n_keys ? n_keys : 1);
    const u32 chunk = (65535 / unit) * unit;
    for (u32 p0 = 0; p0 < n_polys; p0 += chunk) {
        const u32 cnt = (n_polys - p0) < chunk ? (n_polys - p0) : chunk;
        dim3 g((ctx->n + kT - 1) / kT, cnt);
        const u64* pin = in + ((size_t)p0 * (q_limbs + ctx->K) << ctx->log_n);
        u64* pout = out + ((size_t)p0 * q_limbs << ctx->log_n);
        const int nk = n_keys ? (int)n_keys : 1;
        const size_t smem = (size_t)q_limbs * (5 + 2 * ctx->K) * sizeof(u64);
#define CKKS_MD(KK, LZ) k_mod_down<KK, LZ><<<g, kT, smem, st>>>(pin, pout, ctx->mod_down, q_limbs, ctx->log_n, d_exps_inv, nk)
#define CKKS_MDF(KK) k_mod_down_f64<KK><<<g, kT, (size_t)q_limbs * 12 * sizeof(double), st>>>(pin, pout, ctx->mod_down, \
                                                                                          q_limbs, ctx->log_n, d_exps_inv, nk)
        if (f64) {
            switch (ctx->K) {
                case 1: CKKS_MDF(1); break;
                case 2: CKKS_MDF(2); break;
                default: CKKS_MDF(3);
            }
        } else if (lazy) {
            switch (ctx->K) {
                case 1: CKKS_MD(1, true); break;
                case 2: CKKS_MD(2, true); break;
                case 3: CKKS_MD(3, true); break;
                default: CKKS_MD(0, true);
            }
        } else {
            switch (ctx->K) {
                case 1: CKKS_MD(1, false); break;
                case 2: CKKS_MD(2, false); break;
                case 3: CKKS_MD(3, false); break;
                default: CKKS_MD(0, false);
            }
        }
#undef CKKS_MD
#undef CKKS_MDF
    }
    CKKS_CUDA_TRY(cudaGetLastError());
    return CKKS_OK;
}
