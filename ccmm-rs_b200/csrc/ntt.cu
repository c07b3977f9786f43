// ntt.cu -- batched negacyclic NTT / inverse NTT for sm_100a.
//
// Twisted four-step form, N = A * B (A = 2^ceil(logN/2), B = 2^floor(logN/2)),
// input index j = j_lo + B i, output index k = k_a + A k_b:
//   A[k_a + A k_b] = sum_{j_lo} psi_2B^((2k_b+1) j_lo) * [psi^((2k_a+1-A) j_lo)
//                    * sum_i a[j_lo + B i] psi_A^((2k_a+1) i)]
// with psi_A = psi^B and psi_2B = psi^A, which is the reference definition
// A[k] = a(psi^(2k+1)) (ring/ntt.rs:101-127) regrouped.
//   forward pass 1 (column j_lo): A-point negacyclic merged CT, twist, store
//     row j_lo (A contiguous words);
//   forward pass 2 (unit k_a): B-point negacyclic merged CT over {k_a + A j_lo},
//     written back to the same addresses in natural order (in-place safe).
//   The inverse runs the merged GS networks in the opposite order with the
//   inverse twist (N^-1 folded in).
// Both passes use small tables (A or B entries of psi^bitrev with Shoup
// companions, staged in shared memory); the twist is one coalesced N-entry
// table. Each CTA handles C columns (or units); a thread holds R1 points in
// registers for the first half of the stages and R2 for the second, with one
// shared-memory exchange, and every global access is a 128-byte segment.
// Butterflies are Harvey-lazy with Shoup multiplication (primes below 2^58 /
// 2^54 skip the conditional subtractions and estimate the Shoup quotient from
// three 32-bit partial products); outputs are canonical.
#include <cstdio>

#include "ntt_core.cuh"
#include "moddown_f64.cuh"

namespace {

using nttc::brev;

constexpr int kMaxThreads = 256;

// Resident CTAs of kMaxThreads per SM asked of the register allocator: 3 caps a
// thread at 80 registers, 4 at 64. Tiles of up to 2^8 points fit those caps with
// at most a few words of spill, and the extra resident warps hide the global
// loads (forward pass 1 over digits: 1157 -> 953 us for 27 limbs x 64 polys of
// N = 2^16 at 64 registers; the inverse passes gain about 3 % at 80). 2^9-point
// tiles spill hundreds of bytes at either cap and keep the compiler's own
// allocation (a minimum of 0 leaves the count unspecified).
template <int LOG_M>
constexpr int min_ctas(int want) {
    return LOG_M <= 8 ? want : 0;
}

template <int LOG_M>
struct Split {
    static constexpr int M = 1 << LOG_M;
    static constexpr int LR1 = (LOG_M + 1) / 2, LR2 = LOG_M / 2;
    static constexpr int R1 = 1 << LR1, R2 = 1 << LR2;
    static constexpr int RMAX = R1 > R2 ? R1 : R2;
};

// Signed digit -> residue mod q without a division: m = floor(2^64 / q) (the
// high word of the Barrett constant floor(2^128 / q)) makes umulhi(|d|, m)
// floor(|d| / q) or one less, so one conditional subtraction finishes |d| mod q
// for every 64-bit |d|.
__device__ __forceinline__ u64 lift_digit(i64 d, u64 q, u64 m) {
    const u64 a = d < 0 ? 0 - (u64)d : (u64)d;
    u64 r = a - __umul64hi(a, m) * q;
    r = r >= q ? r - q : r;
    return (d < 0 && r) ? q - r : r;
}

// Stage a small (W, W/q) table of the FP64 networks in shared memory (16-byte
// entries: one 128-bit shared load per twiddle).
__device__ __forceinline__ const double2* stage_table_f64(u64* at, const double2* __restrict__ v, int M) {
    double2* st = reinterpret_cast<double2*>(at);
    for (int i = threadIdx.x; i < M; i += blockDim.x) st[i] = __ldg(v + i);
    return st;
}

// Stage a small twiddle table (M values then M Shoup companions) in shared memory.
__device__ __forceinline__ void stage_table(u64* st, const u64* __restrict__ v, const u64* __restrict__ vq, int M) {
    for (int i = threadIdx.x; i < M; i += blockDim.x) {
        st[i] = __ldg(v + i);
        st[M + i] = __ldg(vq + i);
    }
}

// Forward pass 1 over columns j_lo: negacyclic A-point merged CT with
// psi_A = psi^B (natural in, bit-reversed out), times the twist
// psi^((2k_a+1-A) j_lo), stored as row j_lo in natural k_a order.
// kDigits: the input is a signed digit polynomial [D][N] shared by every limb
// (blockIdx.z = digit), lifted on load (signed_mod, hybrid_rns_galois_key.rs:55-57).
template <int LOG_M, bool kDigits>
__global__ void __launch_bounds__(kMaxThreads, min_ctas<LOG_M>(4))
k_fwd1(const void* __restrict__ in_, u64* __restrict__ out,
       const NttTab* __restrict__ tabs, LimbMap lm, int limb_count,
       int log_b, int log_c) {
    using S = Split<LOG_M>;
    extern __shared__ u64 sm[];
    const int C = 1 << log_c, tid = threadIdx.x;
    const int limb = blockIdx.y;
    const NttTab& T = tabs[lm(limb)];
    const u64 q = T.q;
    const size_t base = ((size_t)blockIdx.z * limb_count + limb) << (LOG_M + log_b);
    const int c0 = blockIdx.x << log_c;
    if (LOG_M <= 8 && T.f64) {  // FP64 network: inputs in [0, q), twist output below q in magnitude
        // Phase 2 runs the row group g = tid % R1 in the low lanes, so a warp reads 16
        // different blocks (g << ls) + b of a stage s = LR1 + ls: they are staged at
        // (1 << s) + (b << LR1) + g (consecutive in g) instead of 2^ls entries apart,
        // which cost up to 16-way shared-memory bank conflicts per twiddle load.
        double2* tab = reinterpret_cast<double2*>(sm + (S::M << log_c));
        for (int i = tid; i < S::M; i += blockDim.x) {
            int pos = i;
            if (i >= (1 << S::LR1)) {
                const int s = 31 - __clz(i), ls = s - S::LR1, blk = i - (1 << s);
                pos = (1 << s) + ((blk & ((1 << ls) - 1)) << S::LR1) + (blk >> ls);
            }
            tab[pos] = __ldg(T.fA + i);
        }
        const double qd = T.qd, qinv = T.qinv;
        double* smd = reinterpret_cast<double*>(sm);
        auto twf = [&](int s, u32 blk) { return tab[(1u << s) + blk]; };  // stages below LR1: natural order
        auto twf2 = [&](int s, u32 blk) {
            const int ls = s - S::LR1;
            return tab[(1u << s) + ((blk & ((1u << ls) - 1)) << S::LR1) + (blk >> ls)];
        };
        __syncthreads();
        if (tid < (C << S::LR2)) {
            const int c = tid & (C - 1), i0 = tid >> log_c;
            double x[S::R1];
            if (kDigits) {
                const i64* in = (const i64*)in_ + ((size_t)blockIdx.z << (LOG_M + log_b));
#pragma unroll
                for (int e = 0; e < S::R1; ++e)
                    x[e] = nttf::from_u52(lift_digit(in[c0 + c + ((size_t)(i0 + S::R2 * e) << log_b)], q, T.mu_hi));
            } else {
                const u64* in = (const u64*)in_ + base;
#pragma unroll
                for (int e = 0; e < S::R1; ++e) x[e] = nttf::from_u52(in[c0 + c + ((size_t)(i0 + S::R2 * e) << log_b)]);
            }
            nttf::ct_stages<S::LR1>(x, 0, 0, twf, qd);
#pragma unroll
            for (int e = 0; e < S::R1; ++e)
                smd[((i0 + S::R2 * e) << log_c) + (c ^ (e & (C - 1)))] = nttf::center(x[e], qd, qinv);
        }
        __syncthreads();
        if (tid < (C << S::LR1)) {
            const int g = tid & (S::R1 - 1), c = tid >> S::LR1;
            double y[S::R2];
#pragma unroll
            for (int e = 0; e < S::R2; ++e) y[e] = smd[((S::R2 * g + e) << log_c) + (c ^ (g & (C - 1)))];
            nttf::ct_stages<S::LR2>(y, S::LR1, g, twf2, qd);
            const size_t row = (size_t)(c0 + c) << LOG_M;
#pragma unroll
            for (int e = 0; e < S::R2; ++e) {
                const size_t p = row + brev(S::R2 * g + e, LOG_M);
                const double2 w = __ldg(T.fmid + p);
                out[base + p] = (u64)__double_as_longlong(nttf::mulmod(y[e], w.x, w.y, qd));
            }
        }
        return;
    }
    u64* st = sm + (S::M << log_c);
    stage_table(st, T.psiA, T.psiA_q, S::M);
    auto tw = [&](int s, u32 blk, u64& W, u64& Wq) {
        u32 idx = (1u << s) + blk;
        W = st[idx];
        Wq = st[S::M + idx];
    };
    __syncthreads();
    if (tid < (C << S::LR2)) {
        const int c = tid & (C - 1), i0 = tid >> log_c;
        u64 x[S::R1];
        if (kDigits) {
            const i64* in = (const i64*)in_ + ((size_t)blockIdx.z << (LOG_M + log_b));
#pragma unroll
            for (int e = 0; e < S::R1; ++e) x[e] = lift_digit(in[c0 + c + ((size_t)(i0 + S::R2 * e) << log_b)], q, T.mu_hi);
        } else {
            const u64* in = (const u64*)in_ + base;
#pragma unroll
            for (int e = 0; e < S::R1; ++e) x[e] = in[c0 + c + ((size_t)(i0 + S::R2 * e) << log_b)];
        }
        if (q < nttc::kLazyCtBound) nttc::ct_stages<S::LR1, false>(x, 0, 0, tw, q);
        else nttc::ct_stages<S::LR1, true>(x, 0, 0, tw, q);
#pragma unroll
        for (int e = 0; e < S::R1; ++e) sm[((i0 + S::R2 * e) << log_c) + (c ^ (e & (C - 1)))] = x[e];
    }
    __syncthreads();
    if (tid < (C << S::LR1)) {
        const int g = tid & (S::R1 - 1), c = tid >> S::LR1;
        u64 y[S::R2];
#pragma unroll
        for (int e = 0; e < S::R2; ++e) y[e] = sm[((S::R2 * g + e) << log_c) + (c ^ (g & (C - 1)))];
        if (q < nttc::kLazyCtBound) nttc::ct_stages<S::LR2, false>(y, S::LR1, g, tw, q);
        else nttc::ct_stages<S::LR2, true>(y, S::LR1, g, tw, q);
        const size_t row = (size_t)(c0 + c) << LOG_M;
#pragma unroll
        for (int e = 0; e < S::R2; ++e) {
            const size_t p = row + brev(S::R2 * g + e, LOG_M);
            out[base + p] = mul_shoup_lazy(y[e], __ldg(T.mid + p), __ldg(T.mid_q + p), q);
        }
    }
}

// Forward pass 2 over units k_a: negacyclic B-point merged CT with
// psi_2B = psi^A on {k_a + A j_lo}; output k_b = brev(r) stored at k_a + A k_b
// (natural order). src may equal dst; values < 4q in, canonical out.
template <int LOG_M>
__global__ void __launch_bounds__(kMaxThreads, min_ctas<LOG_M>(4))
k_fwd2(const u64* src, u64* dst, const NttTab* __restrict__ tabs,
       LimbMap lm, int limb_count, int log_a, int log_c) {
    using S = Split<LOG_M>;
    extern __shared__ u64 sm[];
    const int C = 1 << log_c, tid = threadIdx.x;
    const int limb = blockIdx.y;
    const NttTab& T = tabs[lm(limb)];
    const u64 q = T.q;
    const size_t base = ((size_t)blockIdx.z * limb_count + limb) << (LOG_M + log_a);
    const int b0 = blockIdx.x << log_c;
    const int c = tid & (C - 1);
    if (LOG_M <= 8 && T.f64) {  // FP64 network: pass-1 doubles (below q in magnitude) in, canonical out
        const double2* tab = stage_table_f64(sm + (S::M << log_c), T.fB, S::M);
        const double qd = T.qd, qinv = T.qinv;
        double* smd = reinterpret_cast<double*>(sm);
        auto twf = [&](int s, u32 blk) { return tab[(1u << s) + blk]; };
        __syncthreads();
        if (tid < (C << S::LR2)) {
            const int i0 = tid >> log_c;
            double x[S::R1];
#pragma unroll
            for (int e = 0; e < S::R1; ++e)
                x[e] = __longlong_as_double((long long)src[base + ((size_t)(i0 + S::R2 * e) << log_a) + b0 + c]);
            nttf::ct_stages<S::LR1>(x, 0, 0, twf, qd);
#pragma unroll
            for (int e = 0; e < S::R1; ++e) smd[((i0 + S::R2 * e) << log_c) + c] = nttf::center(x[e], qd, qinv);
        }
        __syncthreads();
        if (tid < (C << S::LR1)) {
            const int g = tid >> log_c;
            double y[S::R2];
#pragma unroll
            for (int e = 0; e < S::R2; ++e) y[e] = smd[((S::R2 * g + e) << log_c) + c];
            nttf::ct_stages<S::LR2>(y, S::LR1, g, twf, qd);
#pragma unroll
            for (int e = 0; e < S::R2; ++e)
                dst[base + ((size_t)brev(S::R2 * g + e, LOG_M) << log_a) + b0 + c] = nttf::to_canonical(y[e], qd, qinv);
        }
        return;
    }
    u64* st = sm + (S::M << log_c);
    stage_table(st, T.psiB, T.psiB_q, S::M);
    auto tw = [&](int s, u32 blk, u64& W, u64& Wq) {
        u32 idx = (1u << s) + blk;
        W = st[idx];
        Wq = st[S::M + idx];
    };
    __syncthreads();
    if (tid < (C << S::LR2)) {
        const int i0 = tid >> log_c;
        u64 x[S::R1];
#pragma unroll
        for (int e = 0; e < S::R1; ++e) x[e] = src[base + ((size_t)(i0 + S::R2 * e) << log_a) + b0 + c];
        if (q < nttc::kLazyCtBound) nttc::ct_stages<S::LR1, false>(x, 0, 0, tw, q);
        else nttc::ct_stages<S::LR1, true>(x, 0, 0, tw, q);
#pragma unroll
        for (int e = 0; e < S::R1; ++e) sm[((i0 + S::R2 * e) << log_c) + c] = x[e];
    }
    __syncthreads();
    if (tid < (C << S::LR1)) {
        const int g = tid >> log_c;
        u64 y[S::R2];
#pragma unroll
        for (int e = 0; e < S::R2; ++e) y[e] = sm[((S::R2 * g + e) << log_c) + c];
        if (q < nttc::kLazyCtBound) {
            nttc::ct_stages<S::LR2, false>(y, S::LR1, g, tw, q);
            const u64 one_q = (~0ull) / q;  // floor(2^64 / q) for odd q
#pragma unroll
            for (int e = 0; e < S::R2; ++e)
                dst[base + ((size_t)brev(S::R2 * g + e, LOG_M) << log_a) + b0 + c] =
                    reduce_2q(mul_shoup_lazy(y[e], 1, one_q, q), q);
        } else {
            nttc::ct_stages<S::LR2, true>(y, S::LR1, g, tw, q);
#pragma unroll
            for (int e = 0; e < S::R2; ++e)
                dst[base + ((size_t)brev(S::R2 * g + e, LOG_M) << log_a) + b0 + c] = reduce_4q(y[e], q);
        }
    }
}

// Inverse pass 1 over units k_a: negacyclic B-point merged GS with psi_2B^-1
// on the bit-reversed input {k_a + A brev(r)}, times the inverse twist
// N^-1 psi^-((2k_a+1-A) j_lo), stored as row k_a (lazy, [0, 2q); limbs on the
// FP64 network: doubles below 1.5 q in magnitude). in != out.
// With go.exps (sigma_k folded in), column j_lo of the row is stored at
// position j_lo k mod B, so pass 2 reads the columns of each output column
// together.
template <int LOG_M>
__global__ void __launch_bounds__(kMaxThreads, min_ctas<LOG_M>(3))
k_inv1(const u64* __restrict__ in, u64* __restrict__ out,
       const NttTab* __restrict__ tabs, LimbMap lm, int limb_count,
       int log_a, int log_c, GaloisOut go) {
    using S = Split<LOG_M>;
    extern __shared__ u64 sm[];
    const int C = 1 << log_c, tid = threadIdx.x;
    const int limb = blockIdx.y;
    const NttTab& T = tabs[lm(limb)];
    const u64 q = T.q;
    const size_t base = ((size_t)blockIdx.z * limb_count + limb) << (LOG_M + log_a);
    const int b0 = blockIdx.x << log_c;
    const bool f64 = LOG_M <= 8 && T.f64;
    u64* st = sm + (S::M << log_c);
    if (f64) stage_table_f64(st, T.fB_inv, S::M);
    else stage_table(st, T.psiB_inv, T.psiB_inv_q, S::M);
    const double2* tabf = reinterpret_cast<const double2*>(st);
    const double qd = T.qd, qinv = T.qinv;
    double* smd = reinterpret_cast<double*>(sm);
    auto tw = [&](int s, u32 blk, u64& W, u64& Wq) {
        u32 idx = (S::M >> (s + 1)) + blk;
        W = st[idx];
        Wq = st[S::M + idx];
    };
    auto twf = [&](int s, u32 blk) { return tabf[(S::M >> (s + 1)) + blk]; };
    __syncthreads();
    if (tid < (C << S::LR1)) {
        const int c = tid & (C - 1), g = tid >> log_c;
        if (f64) {  // centred inputs, four GS stages (below 8 q), centred at the exchange
            double x[S::R2];
#pragma unroll
            for (int e = 0; e < S::R2; ++e)
                x[e] = nttf::center(nttf::from_u52(in[base + ((size_t)brev(S::R2 * g + e, LOG_M) << log_a) + b0 + c]),
                                    qd, qinv);
            nttf::gs_stages<S::LR2>(x, 0, g, twf, qd);
#pragma unroll
            for (int e = 0; e < S::R2; ++e) {
                const int r = S::R2 * g + e;
                smd[(r << log_c) + (c ^ (r & (C - 1)))] = nttf::center(x[e], qd, qinv);
            }
        } else {
            u64 x[S::R2];
#pragma unroll
            for (int e = 0; e < S::R2; ++e) x[e] = in[base + ((size_t)brev(S::R2 * g + e, LOG_M) << log_a) + b0 + c];
            if (q < nttc::kLazyGsBound) nttc::gs_stages<S::LR2, true>(x, 0, g, tw, q);
            else nttc::gs_stages<S::LR2, false>(x, 0, g, tw, q);
#pragma unroll
            for (int e = 0; e < S::R2; ++e) {
                const int r = S::R2 * g + e;
                sm[(r << log_c) + (c ^ (r & (C - 1)))] = x[e];
            }
        }
    }
    __syncthreads();
    const bool act = tid < (C << S::LR2);
    const int i0 = tid & (S::R2 - 1), c = tid >> S::LR2;
    const size_t row = (size_t)(b0 + c) << LOG_M;
    u64 v[S::R1];
    if (act) {
        if (f64) {
            double y[S::R1];
#pragma unroll
            for (int e = 0; e < S::R1; ++e) {
                const int r = i0 + S::R2 * e;
                y[e] = smd[(r << log_c) + (c ^ (r & (C - 1)))];
            }
            nttf::gs_stages<S::LR1>(y, S::LR2, 0, twf, qd);
#pragma unroll
            for (int e = 0; e < S::R1; ++e) {
                const double2 w = __ldg(T.fmidi + row + i0 + S::R2 * e);
                v[e] = (u64)__double_as_longlong(nttf::mulmod(y[e], w.x, w.y, qd));
            }
        } else {
            u64 y[S::R1];
#pragma unroll
            for (int e = 0; e < S::R1; ++e) {
                const int r = i0 + S::R2 * e;
                y[e] = sm[(r << log_c) + (c ^ (r & (C - 1)))];
            }
            if (q < nttc::kLazyGsBound) nttc::gs_stages<S::LR1, true>(y, S::LR2, 0, tw, q);
            else nttc::gs_stages<S::LR1, false>(y, S::LR2, 0, tw, q);
#pragma unroll
            for (int e = 0; e < S::R1; ++e) {
                const size_t p = row + i0 + S::R2 * e;
                v[e] = mul_shoup_lazy(y[e], __ldg(T.midi + p), __ldg(T.midi_q + p), q);
            }
        }
    }
    if (go.exps) {  // columns of the row permuted: j_lo -> j_lo k mod B (B = M)
        const u32 k = (u32)(go.exps[(blockIdx.z >> 1) % go.n_keys] & (S::M - 1));
        __syncthreads();
        if (act) {
#pragma unroll
            for (int e = 0; e < S::R1; ++e) sm[(c << LOG_M) + (((u32)(i0 + S::R2 * e) * k) & (S::M - 1))] = v[e];
        }
        __syncthreads();
        if (act) {
#pragma unroll
            for (int e = 0; e < S::R1; ++e) v[e] = sm[(c << LOG_M) + i0 + S::R2 * e];
        }
    }
    if (act) {
#pragma unroll
        for (int e = 0; e < S::R1; ++e) out[base + row + i0 + S::R2 * e] = v[e];
    }
}

// Inverse pass 2 over columns j_lo: negacyclic A-point merged GS with
// psi_A^-1 on {j_lo + B brev(r)}; natural output j_lo + B i, canonical.
// src may equal dst.
// With ib.b, the b components of key-switch accumulators get P b added (InvBase).
// With go.exps (pass 1 stored permuted columns), position p holds column
// j_lo = p k^-1 mod B, and element i of it goes to coefficient
// sigma_k(j_lo + B i) = p + B ((m + i k) mod 2A), m = floor((j_lo k mod 2N) / B),
// negated past A rows; ib.b must then be null.
template <int LOG_M>
__global__ void __launch_bounds__(kMaxThreads, min_ctas<LOG_M>(3))
k_inv2(const u64* src, u64* dst, const NttTab* __restrict__ tabs,
       LimbMap lm, int limb_count, int log_b, int log_c, InvBase ib, GaloisOut go) {
    using S = Split<LOG_M>;
    extern __shared__ u64 sm[];
    const int C = 1 << log_c, tid = threadIdx.x;
    const int limb = blockIdx.y;
    const NttTab& T = tabs[lm(limb)];
    const u64 q = T.q;
    const size_t base = ((size_t)blockIdx.z * limb_count + limb) << (LOG_M + log_b);
    const int c0 = blockIdx.x << log_c;
    const int c = tid & (C - 1);
    const bool f64 = LOG_M <= 8 && T.f64;
    u64* st = sm + (S::M << log_c);
    if (f64) stage_table_f64(st, T.fA_inv, S::M);
    else stage_table(st, T.psiA_inv, T.psiA_inv_q, S::M);
    const double2* tabf = reinterpret_cast<const double2*>(st);
    const double qd = T.qd, qinv = T.qinv;
    double* smd = reinterpret_cast<double*>(sm);
    auto tw = [&](int s, u32 blk, u64& W, u64& Wq) {
        u32 idx = (S::M >> (s + 1)) + blk;
        W = st[idx];
        Wq = st[S::M + idx];
    };
    auto twf = [&](int s, u32 blk) { return tabf[(S::M >> (s + 1)) + blk]; };
    __syncthreads();
    if (tid < (C << S::LR1)) {
        const int g = tid >> log_c;
        if (f64) {  // pass-1 doubles (below 1.5 q) centred, four GS stages, centred at the exchange
            double x[S::R2];
#pragma unroll
            for (int e = 0; e < S::R2; ++e)
                x[e] = nttf::center(
                    __longlong_as_double((long long)src[base + c0 + c + ((size_t)brev(S::R2 * g + e, LOG_M) << log_b)]),
                    qd, qinv);
            nttf::gs_stages<S::LR2>(x, 0, g, twf, qd);
#pragma unroll
            for (int e = 0; e < S::R2; ++e) smd[((S::R2 * g + e) << log_c) + c] = nttf::center(x[e], qd, qinv);
        } else {
            u64 x[S::R2];
#pragma unroll
            for (int e = 0; e < S::R2; ++e) x[e] = src[base + c0 + c + ((size_t)brev(S::R2 * g + e, LOG_M) << log_b)];
            if (q < nttc::kLazyGsBound) nttc::gs_stages<S::LR2, true>(x, 0, g, tw, q);
            else nttc::gs_stages<S::LR2, false>(x, 0, g, tw, q);
#pragma unroll
            for (int e = 0; e < S::R2; ++e) sm[((S::R2 * g + e) << log_c) + c] = x[e];
        }
    }
    __syncthreads();
    const bool act = tid < (C << S::LR2);
    const int i0 = tid >> log_c;
    u64 v[S::R1];
    if (act) {
        if (f64) {
            double y[S::R1];
#pragma unroll
            for (int e = 0; e < S::R1; ++e) y[e] = smd[((i0 + S::R2 * e) << log_c) + c];
            nttf::gs_stages<S::LR1>(y, S::LR2, 0, twf, qd);
#pragma unroll
            for (int e = 0; e < S::R1; ++e) v[e] = nttf::to_canonical(y[e], qd, qinv);
        } else {
#pragma unroll
            for (int e = 0; e < S::R1; ++e) v[e] = sm[((i0 + S::R2 * e) << log_c) + c];
            if (q < nttc::kLazyGsBound) {
                nttc::gs_stages<S::LR1, true>(v, S::LR2, 0, tw, q);
                const u64 one_q = (~0ull) / q;  // floor(2^64 / q) for odd q
#pragma unroll
                for (int e = 0; e < S::R1; ++e) v[e] = reduce_2q(mul_shoup_lazy(v[e], 1, one_q, q), q);
            } else {
                nttc::gs_stages<S::LR1, false>(v, S::LR2, 0, tw, q);
#pragma unroll
                for (int e = 0; e < S::R1; ++e) v[e] = reduce_2q(v[e], q);
            }
        }
        const u32 poly = blockIdx.z;
        if (ib.b && !(poly & 1) && (u32)limb < ib.q_limbs) {
            const u64* bb = ib.b + (size_t)(poly / (2 * ib.n_keys)) * ib.b_stride + ((size_t)limb << (LOG_M + log_b));
            const u64 pf = ib.pf[limb], pfq = ib.pf_q[limb];
#pragma unroll
            for (int e = 0; e < S::R1; ++e)
                v[e] = add_mod(v[e], mul_shoup(__ldg(bb + c0 + c + ((size_t)(i0 + S::R2 * e) << log_b)), pf, pfq, q), q);
        }
    }
    if (go.exps) {  // every element to its image row (through shared memory: stores stay row-coalesced)
        const u32 gk = (blockIdx.z >> 1) % go.n_keys;
        const u64 k = go.exps[gk], kinv = go.exps_inv[gk];
        const u32 bmask = (1u << log_b) - 1, amask2 = (2u << LOG_M) - 1;
        const u32 jl = (u32)(((u64)(c0 + c) * (kinv & bmask)) & bmask);
        const u32 m = (u32)((((u64)jl * k) & ((2ull << (LOG_M + log_b)) - 1)) >> log_b);
        const u32 k2a = (u32)(k & amask2);
        __syncthreads();
        if (act) {
#pragma unroll
            for (int e = 0; e < S::R1; ++e) {
                const u32 r = (m + (u32)(i0 + S::R2 * e) * k2a) & amask2;
                const bool neg = r >= (u32)S::M;
                sm[((r & (S::M - 1)) << log_c) + c] = neg ? neg_mod(v[e], q) : v[e];
            }
        }
        __syncthreads();
        if (act) {
#pragma unroll
            for (int e = 0; e < S::R1; ++e) v[e] = sm[((i0 + S::R2 * e) << log_c) + c];
        }
    }
    if (act) {
#pragma unroll
        for (int e = 0; e < S::R1; ++e) dst[base + c0 + c + ((size_t)(i0 + S::R2 * e) << log_b)] = v[e];
    }
}

// ----------------------------------------------------------------------------
// Inverse pass 2 fused with ModDown (hoisted rotations; ring/auxiliary_modulus.rs:89-171).
// Pass 1 ran with sigma_k folded in (GaloisOut), so every column tile of pass 2
// holds the same output coefficients in every limb. k_inv2_pcrt finishes the
// K auxiliary limbs of a tile and writes, per coefficient, the four 47-bit
// words of the centred P-CRT value with its sign folded in (mdf::crt_words:
// the ModDown products are odd in the words, so negating them negates each
// product exactly); k_inv2_moddown finishes one Q limb of a tile and applies
// mdf::limb with those words, writing the ModDown output. The inverse
// transform's Q-limb output never reaches HBM, and the same canonical residues
// as k_inv2 followed by k_mod_down_f64 come out.

// Pass 2 of one limb of a column tile, sigma folded (k_inv2 with go.exps):
// thread (i0, c) ends with v[e] = output row i0 + R2 e, column c0 + c.
template <int LOG_M>
__device__ __forceinline__ void inv2_tile_folded(const u64* __restrict__ src, const NttTab& T, u64* sm, int log_b,
                                                 int log_c, int c0, u32 poly, const GaloisOut& go, bool act,
                                                 u64 (&v)[Split<LOG_M>::R1]) {
    using S = Split<LOG_M>;
    const int C = 1 << log_c, tid = threadIdx.x;
    const int c = tid & (C - 1);
    const u64 q = T.q;
    const bool f64 = T.f64;
    u64* st = sm + (S::M << log_c);
    if (f64) stage_table_f64(st, T.fA_inv, S::M);
    else stage_table(st, T.psiA_inv, T.psiA_inv_q, S::M);
    const double2* tabf = reinterpret_cast<const double2*>(st);
    const double qd = T.qd, qinv = T.qinv;
    double* smd = reinterpret_cast<double*>(sm);
    auto tw = [&](int s, u32 blk, u64& W, u64& Wq) {
        u32 idx = (S::M >> (s + 1)) + blk;
        W = st[idx];
        Wq = st[S::M + idx];
    };
    auto twf = [&](int s, u32 blk) { return tabf[(S::M >> (s + 1)) + blk]; };
    __syncthreads();
    if (tid < (C << S::LR1)) {
        const int g = tid >> log_c;
        if (f64) {
            double x[S::R2];
#pragma unroll
            for (int e = 0; e < S::R2; ++e)
                x[e] = nttf::center(
                    __longlong_as_double((long long)src[c0 + c + ((size_t)brev(S::R2 * g + e, LOG_M) << log_b)]), qd,
                    qinv);
            nttf::gs_stages<S::LR2>(x, 0, g, twf, qd);
#pragma unroll
            for (int e = 0; e < S::R2; ++e) smd[((S::R2 * g + e) << log_c) + c] = nttf::center(x[e], qd, qinv);
        } else {
            u64 x[S::R2];
#pragma unroll
            for (int e = 0; e < S::R2; ++e) x[e] = src[c0 + c + ((size_t)brev(S::R2 * g + e, LOG_M) << log_b)];
            if (q < nttc::kLazyGsBound) nttc::gs_stages<S::LR2, true>(x, 0, g, tw, q);
            else nttc::gs_stages<S::LR2, false>(x, 0, g, tw, q);
#pragma unroll
            for (int e = 0; e < S::R2; ++e) sm[((S::R2 * g + e) << log_c) + c] = x[e];
        }
    }
    __syncthreads();
    const int i0 = tid >> log_c;
    if (act) {
        if (f64) {
            double y[S::R1];
#pragma unroll
            for (int e = 0; e < S::R1; ++e) y[e] = smd[((i0 + S::R2 * e) << log_c) + c];
            nttf::gs_stages<S::LR1>(y, S::LR2, 0, twf, qd);
#pragma unroll
            for (int e = 0; e < S::R1; ++e) v[e] = nttf::to_canonical(y[e], qd, qinv);
        } else {
#pragma unroll
            for (int e = 0; e < S::R1; ++e) v[e] = sm[((i0 + S::R2 * e) << log_c) + c];
            if (q < nttc::kLazyGsBound) {
                nttc::gs_stages<S::LR1, true>(v, S::LR2, 0, tw, q);
                const u64 one_q = (~0ull) / q;
#pragma unroll
                for (int e = 0; e < S::R1; ++e) v[e] = reduce_2q(mul_shoup_lazy(v[e], 1, one_q, q), q);
            } else {
                nttc::gs_stages<S::LR1, false>(v, S::LR2, 0, tw, q);
#pragma unroll
                for (int e = 0; e < S::R1; ++e) v[e] = reduce_2q(v[e], q);
            }
        }
    }
    {  // every element to its image row (as k_inv2)
        const u32 gk = (poly >> 1) % go.n_keys;
        const u64 k = go.exps[gk], kinv = go.exps_inv[gk];
        const u32 bmask = (1u << log_b) - 1, amask2 = (2u << LOG_M) - 1;
        const u32 jl = (u32)(((u64)(c0 + c) * (kinv & bmask)) & bmask);
        const u32 m = (u32)((((u64)jl * k) & ((2ull << (LOG_M + log_b)) - 1)) >> log_b);
        const u32 k2a = (u32)(k & amask2);
        __syncthreads();
        if (act) {
#pragma unroll
            for (int e = 0; e < S::R1; ++e) {
                const u32 r = (m + (u32)(i0 + S::R2 * e) * k2a) & amask2;
                const bool neg = r >= (u32)S::M;
                sm[((r & (S::M - 1)) << log_c) + c] = neg ? neg_mod(v[e], q) : v[e];
            }
        }
        __syncthreads();
        if (act) {
#pragma unroll
            for (int e = 0; e < S::R1; ++e) v[e] = sm[((i0 + S::R2 * e) << log_c) + c];
        }
    }
}

// One auxiliary limb (grid y: k, local limb q_limbs + k of the [polys][LK][N]
// pass-1 output, table L_ctx + k) of a column tile, sigma folded, into
// zp [polys][K][N] (canonical).
template <int LOG_M>
__global__ void __launch_bounds__(kMaxThreads, min_ctas<LOG_M>(3))
k_inv2_p(const u64* __restrict__ src, u64* __restrict__ zp, const NttTab* __restrict__ tabs, int q_limbs,
         int L_ctx, int LK, int K, int log_b, int log_c, GaloisOut go) {
    using S = Split<LOG_M>;
    extern __shared__ u64 sm[];
    const int C = 1 << log_c, tid = threadIdx.x;
    const int c0 = blockIdx.x << log_c;
    const int k = blockIdx.y;
    const u32 poly = blockIdx.z;
    const int log_n = LOG_M + log_b;
    const bool act = tid < (C << S::LR2);
    const int c = tid & (C - 1), i0 = tid >> log_c;
    u64 v[S::R1];
    inv2_tile_folded<LOG_M>(src + (((size_t)poly * LK + q_limbs + k) << log_n), tabs[L_ctx + k], sm, log_b, log_c,
                            c0, poly, go, act, v);
    if (act) {
        u64* o = zp + (((size_t)poly * K + k) << log_n);
#pragma unroll
        for (int e = 0; e < S::R1; ++e) o[c0 + c + ((size_t)(i0 + S::R2 * e) << log_b)] = v[e];
    }
}

// Per coefficient of zp [polys][KT][N]: the four 47-bit words of the centred
// P-CRT value, sign folded in, as words [polys][N][4] (doubles).
template <int KT>
__global__ void __launch_bounds__(256) k_pwords(const u64* __restrict__ zp, double* __restrict__ words,
                                                ModDownConst md, int log_n) {
    const u32 n = 1u << log_n;
    const u32 t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const size_t poly = blockIdx.y;
    u64 v[KT];
#pragma unroll
    for (int k = 0; k < KT; ++k) v[k] = __ldg(zp + ((poly * KT + k) << log_n) + t);
    double w[4];
    bool neg;
    mdf::crt_words<KT>(v, md, w, neg);
    double2* o = reinterpret_cast<double2*>(words + (((poly << log_n) + t) << 2));
    o[0] = neg ? make_double2(-w[0], -w[1]) : make_double2(w[0], w[1]);
    o[1] = neg ? make_double2(-w[2], -w[3]) : make_double2(w[2], w[3]);
}

// One Q limb (grid x, fastest: the tile's words are reused from L2 by every
// limb) of a column tile: pass 2, then ModDown into dst [polys][q_limbs][N].
template <int LOG_M>
__global__ void __launch_bounds__(kMaxThreads, min_ctas<LOG_M>(3))
k_inv2_moddown(const u64* __restrict__ src, u64* __restrict__ dst, const double* __restrict__ words,
               const NttTab* __restrict__ tabs, const double* __restrict__ f64c, int q_limbs, int LK, int log_b,
               int log_c, GaloisOut go) {
    using S = Split<LOG_M>;
    extern __shared__ u64 sm[];
    const int C = 1 << log_c, tid = threadIdx.x;
    const int limb = blockIdx.x;
    const int c0 = blockIdx.y << log_c;
    const u32 poly = blockIdx.z;
    const int log_n = LOG_M + log_b;
    const bool act = tid < (C << S::LR2);
    const int c = tid & (C - 1), i0 = tid >> log_c;
    u64 v[S::R1];
    inv2_tile_folded<LOG_M>(src + (((size_t)poly * LK + limb) << log_n), tabs[limb], sm, log_b, log_c, c0, poly, go,
                            act, v);
    if (act) {
        double ci[12];
#pragma unroll
        for (int k = 0; k < 12; ++k) ci[k] = __ldg(f64c + limb * 12 + k);
        u64* o = dst + (((size_t)poly * q_limbs + limb) << log_n);
#pragma unroll
        for (int e = 0; e < S::R1; ++e) {
            const size_t pos = c0 + c + ((size_t)(i0 + S::R2 * e) << log_b);
            const double2* wp = reinterpret_cast<const double2*>(words + ((((size_t)poly << log_n) + pos) << 2));
            const double2 wa = __ldg(wp), wb = __ldg(wp + 1);
            const double w[4] = {wa.x, wa.y, wb.x, wb.y};
            o[pos] = mdf::limb(nttf::from_u52(v[e]), w, false, ci, false);
        }
    }
}

// Forward pass 2 of relinearization digit transforms fused with the key sum
// (grafting/bounded_key_switch.rs:139-223): for ciphertext c (grid x, so
// consecutive CTAs share the key tile in L2), a tile of C units and limb l,
// every digit j's pass-1 output is finished in registers (FP64 network) and
// multiplied by the key's b and a words at the same NTT positions. The exact
// products (nttf::mulmod, Wp = fl(W fl(1/q)): |W/q - Wp| <= 2^-52, so for a
// centred |v| < 2^49 the quotient is off by under 0.9 and |r| < 0.9 q) are
// summed in doubles, centred every 8 digits (|sum| < 0.5 q + 8 * 0.9 q < 2^53),
// and base (c0, c1 in the NTT domain) is added once: the same canonical
// residues as k_fwd2 followed by k_relin_mac, with the digit transforms never
// written to HBM.
//   mid  [n_ct][D][L][N]  pass-1 outputs of the digits (k_fwd1<_, true>)
//   key  [D][2][L][N]     NTT-domain relinearization key
//   base, acc [n_ct][2][L][N] (may alias)
template <int LOG_M>
__global__ void __launch_bounds__(kMaxThreads, LOG_M <= 5 ? 3 : 2)
k_fwd2_relin(const u64* __restrict__ mid, const u64* __restrict__ key, const u64* base, u64* acc,
             const NttTab* __restrict__ tabs, int L, int D, int log_a, int log_c) {
    using S = Split<LOG_M>;
    extern __shared__ u64 sm[];
    const int C = 1 << log_c, tid = threadIdx.x;
    const size_t ct = blockIdx.x;
    const int b0 = blockIdx.y << log_c;
    const int limb = blockIdx.z;
    const int log_n = LOG_M + log_a;
    const NttTab& T = tabs[limb];
    const double2* tab = stage_table_f64(sm + (S::M << log_c), T.fB, S::M);
    const double qd = T.qd, qinv = T.qinv;
    double* smd = reinterpret_cast<double*>(sm);
    auto twf = [&](int s, u32 blk) { return tab[(1u << s) + blk]; };
    const int c = tid & (C - 1);
    const bool act_b = tid < (C << S::LR1);
    const int g = tid >> log_c;
    double sb[S::R2], sa[S::R2];
#pragma unroll
    for (int e = 0; e < S::R2; ++e) sb[e] = sa[e] = 0.0;
    __syncthreads();
    for (int j = 0; j < D; ++j) {
        const size_t in_j = ((ct * D + j) * L + limb) << log_n;
        if (tid < (C << S::LR2)) {
            const int i0 = tid >> log_c;
            double x[S::R1];
#pragma unroll
            for (int e = 0; e < S::R1; ++e)
                x[e] = __longlong_as_double((long long)mid[in_j + ((size_t)(i0 + S::R2 * e) << log_a) + b0 + c]);
            nttf::ct_stages<S::LR1>(x, 0, 0, twf, qd);
#pragma unroll
            for (int e = 0; e < S::R1; ++e) smd[((i0 + S::R2 * e) << log_c) + c] = nttf::center(x[e], qd, qinv);
        }
        __syncthreads();
        if (act_b) {
            double y[S::R2];
#pragma unroll
            for (int e = 0; e < S::R2; ++e) y[e] = smd[((S::R2 * g + e) << log_c) + c];
            nttf::ct_stages<S::LR2>(y, S::LR1, g, twf, qd);
            const u64* kb = key + ((((size_t)j * 2) * L + limb) << log_n) + b0 + c;
            const u64* ka = kb + ((size_t)L << log_n);
#pragma unroll
            for (int e = 0; e < S::R2; ++e) {
                const size_t pos = (size_t)brev(S::R2 * g + e, LOG_M) << log_a;
                const double v = nttf::center(y[e], qd, qinv);
                const double wb = nttf::from_u52(__ldg(kb + pos)), wa = nttf::from_u52(__ldg(ka + pos));
                sb[e] = __dadd_rn(sb[e], nttf::mulmod(v, wb, __dmul_rn(wb, qinv), qd));
                sa[e] = __dadd_rn(sa[e], nttf::mulmod(v, wa, __dmul_rn(wa, qinv), qd));
            }
            if ((j & 7) == 7) {
#pragma unroll
                for (int e = 0; e < S::R2; ++e) {
                    sb[e] = nttf::center(sb[e], qd, qinv);
                    sa[e] = nttf::center(sa[e], qd, qinv);
                }
            }
        }
        __syncthreads();  // smd is rewritten by the next digit
    }
    if (act_b) {
        const size_t ob0 = ((ct * 2 * L + limb) << log_n) + b0 + c, oa0 = ob0 + ((size_t)L << log_n);
#pragma unroll
        for (int e = 0; e < S::R2; ++e) {
            const size_t pos = (size_t)brev(S::R2 * g + e, LOG_M) << log_a;
            double vb = sb[e], va = sa[e];
            if (base) {
                vb = __dadd_rn(vb, nttf::from_u52(base[ob0 + pos]));
                va = __dadd_rn(va, nttf::from_u52(base[oa0 + pos]));
            }
            acc[ob0 + pos] = nttf::to_canonical(vb, qd, qinv);
            acc[oa0 + pos] = nttf::to_canonical(va, qd, qinv);
        }
    }
}

// columns per CTA: min(16, available, 256 / RMAX), or the tuned choice `pref`
// when it is within those limits
template <int LOG_M>
int max_log_c(int log_avail) {
    int lc = 4;
    while ((Split<LOG_M>::RMAX << lc) > kMaxThreads) --lc;
    return lc < log_avail ? lc : log_avail;
}
template <int LOG_M>
int pick_log_c(int log_avail, int pref) {
    const int mx = max_log_c<LOG_M>(log_avail);
    return pref >= 0 && pref <= mx ? pref : mx;
}

template <int LOG_M>
int32_t launch_pass(int which, const void* in, u64* out, const NttTab* tabs, LimbMap lm, u32 limbs, u32 polys,
                    int log_other, cudaStream_t st, const InvBase& ib, int lc_pref, const GaloisOut& go) {
    const int lc = pick_log_c<LOG_M>(log_other, lc_pref);
    const int threads = Split<LOG_M>::RMAX << lc;
    const size_t smem = (sizeof(u64) << (LOG_M + lc)) + 2 * sizeof(u64) * (1u << LOG_M);
    dim3 grid(1u << (log_other - lc), limbs, polys);
    switch (which) {
        case 0: k_fwd1<LOG_M, false><<<grid, threads, smem, st>>>(in, out, tabs, lm, limbs, log_other, lc); break;
        case 1: k_fwd1<LOG_M, true><<<grid, threads, smem, st>>>(in, out, tabs, lm, limbs, log_other, lc); break;
        case 2: k_fwd2<LOG_M><<<grid, threads, smem, st>>>((const u64*)in, out, tabs, lm, limbs, log_other, lc); break;
        case 3: k_inv1<LOG_M><<<grid, threads, smem, st>>>((const u64*)in, out, tabs, lm, limbs, log_other, lc, go); break;
        default: k_inv2<LOG_M><<<grid, threads, smem, st>>>((const u64*)in, out, tabs, lm, limbs, log_other, lc, ib, go); break;
    }
    return CKKS_OK;
}

int32_t pass(int which, int log_m, const void* in, u64* out, const NttTab* tabs, LimbMap lm, u32 limbs, u32 polys,
             int log_other, cudaStream_t st, const InvBase& ib = InvBase{}, int lc_pref = -1,
             const GaloisOut& go = GaloisOut{}) {
    if (polys > 65535 || limbs > 65535) {  // grid y / z limits
        ckks_set_error("NTT: more than 65535 polynomials or limbs in one launch");
        return CKKS_ERR_BAD_ARG;
    }
    switch (log_m) {
        case 1: return launch_pass<1>(which, in, out, tabs, lm, limbs, polys, log_other, st, ib, lc_pref, go);
        case 2: return launch_pass<2>(which, in, out, tabs, lm, limbs, polys, log_other, st, ib, lc_pref, go);
        case 3: return launch_pass<3>(which, in, out, tabs, lm, limbs, polys, log_other, st, ib, lc_pref, go);
        case 4: return launch_pass<4>(which, in, out, tabs, lm, limbs, polys, log_other, st, ib, lc_pref, go);
        case 5: return launch_pass<5>(which, in, out, tabs, lm, limbs, polys, log_other, st, ib, lc_pref, go);
        case 6: return launch_pass<6>(which, in, out, tabs, lm, limbs, polys, log_other, st, ib, lc_pref, go);
        case 7: return launch_pass<7>(which, in, out, tabs, lm, limbs, polys, log_other, st, ib, lc_pref, go);
        case 8: return launch_pass<8>(which, in, out, tabs, lm, limbs, polys, log_other, st, ib, lc_pref, go);
        case 9: return launch_pass<9>(which, in, out, tabs, lm, limbs, polys, log_other, st, ib, lc_pref, go);
        default: ckks_set_error("NTT: unsupported transform size"); return CKKS_ERR_BAD_ARG;
    }
}

}  // namespace

void ntt_set_smem_limits() {}

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
    const int la = ctx->log_n1, lb = ctx->log_n2;
    u64* mid = out;
    Workspace<u64> tmp;
    if (in == out) {  // pass 1 reads columns and writes rows: stage through a workspace
        if (int32_t rc = tmp.alloc((size_t)n_polys * limb_count * ctx->n, st)) return rc;
        mid = tmp.p;
    }
    if (int32_t rc = pass(0, la, in, mid, ctx->d_tabs, lm, limb_count, n_polys, lb, st, InvBase{}, ctx->ntt_log_c[0])) return rc;
    if (int32_t rc = pass(2, lb, mid, out, ctx->d_tabs, lm, limb_count, n_polys, la, st, InvBase{}, ctx->ntt_log_c[2])) return rc;
    CKKS_CUDA_TRY(cudaGetLastError());
    return CKKS_OK;
}

int32_t ntt_inverse_launch_map(ckks_ctx* ctx, const u64* in, u64* out, u32 n_polys, LimbMap lm, u32 limb_count,
                               cudaStream_t st) {
    return ntt_inverse_base_launch(ctx, in, out, n_polys, lm, limb_count, InvBase{}, st);
}

int32_t ntt_inverse_base_launch(ckks_ctx* ctx, const u64* in, u64* out, u32 n_polys, LimbMap lm, u32 limb_count,
                                const InvBase& ib, cudaStream_t st, const GaloisOut& go) {
    if (go.exps && ib.b) {
        ckks_set_error("inverse NTT: a folded Galois automorphism cannot take a base term");
        return CKKS_ERR_BAD_ARG;
    }
    if (n_polys == 0 || limb_count == 0) return CKKS_OK;
    const int la = ctx->log_n1, lb = ctx->log_n2;
    u64* mid = out;
    Workspace<u64> tmp;
    if (in == out) {
        if (int32_t rc = tmp.alloc((size_t)n_polys * limb_count * ctx->n, st)) return rc;
        mid = tmp.p;
    }
    if (int32_t rc = pass(3, lb, in, mid, ctx->d_tabs, lm, limb_count, n_polys, la, st, InvBase{}, ctx->ntt_log_c[3], go)) return rc;
    if (int32_t rc = pass(4, la, mid, out, ctx->d_tabs, lm, limb_count, n_polys, lb, st, ib, ctx->ntt_log_c[4], go)) return rc;
    CKKS_CUDA_TRY(cudaGetLastError());
    return CKKS_OK;
}

int32_t ntt_forward_digits_launch(ckks_ctx* ctx, const i64* digits, u64* out, u32 D, LimbMap lm, u32 limbs,
                                  cudaStream_t st) {
    if (D == 0 || limbs == 0) return CKKS_OK;
    const int la = ctx->log_n1, lb = ctx->log_n2;
    if (int32_t rc = pass(1, la, digits, out, ctx->d_tabs, lm, limbs, D, lb, st, InvBase{}, ctx->ntt_log_c[1])) return rc;
    if (int32_t rc = pass(2, lb, out, out, ctx->d_tabs, lm, limbs, D, la, st, InvBase{}, ctx->ntt_log_c[2])) return rc;
    CKKS_CUDA_TRY(cudaGetLastError());
    return CKKS_OK;
}

// Units per CTA of the fused relinearization pass (log2); -1 follows the
// forward pass 2's tuned choice.
#ifndef CKKS_RELIN_LOG_C
#define CKKS_RELIN_LOG_C -1
#endif
constexpr int kRelinLogC = CKKS_RELIN_LOG_C;

bool ntt_relin_fused_supported(const ckks_ctx* ctx, u32 L) {
    if (ctx->log_n2 < 2 || ctx->log_n2 > 8) return false;
    for (u32 l = 0; l < L; ++l)
        if (!ctx->h_tabs[l].f64) return false;
    return true;
}

// Bounded relinearization key sum of n_ct ciphertexts from their signed digits
// [n_ct][D][N]: digit lift + forward pass 1 into mid, then k_fwd2_relin.
int32_t ntt_relin_fused_launch(ckks_ctx* ctx, const i64* digits, u64* mid, const u64* key, const u64* base, u64* acc,
                               u32 n_ct, u32 L, u32 D, cudaStream_t st) {
    if (n_ct == 0) return CKKS_OK;
    const int la = ctx->log_n1, lb = ctx->log_n2;
    const LimbMap lm = LimbMap::range(0, L);
    if (int32_t rc = pass(1, la, digits, mid, ctx->d_tabs, lm, L, n_ct * D, lb, st, InvBase{}, ctx->ntt_log_c[1]))
        return rc;
    if (n_ct > 0x7FFFFFFFu || L > 65535) {
        ckks_set_error("relinearization: batch outside the launch limits");
        return CKKS_ERR_BAD_ARG;
    }
#define CKKS_RELIN_FUSED(LM)                                                                                  \
    do {                                                                                                      \
        const int lc = pick_log_c<LM>(la, kRelinLogC >= 0 ? kRelinLogC : ctx->ntt_log_c[2]);                  \
        const size_t smem = (sizeof(u64) << (LM + lc)) + 2 * sizeof(u64) * (1u << LM);                        \
        dim3 grid(n_ct, 1u << (la - lc), L);                                                                  \
        k_fwd2_relin<LM><<<grid, Split<LM>::RMAX << lc, smem, st>>>(mid, key, base, acc, ctx->d_tabs, (int)L, \
                                                                    (int)D, la, lc);                         \
    } while (0)
    switch (lb) {
        case 2: CKKS_RELIN_FUSED(2); break;
        case 3: CKKS_RELIN_FUSED(3); break;
        case 4: CKKS_RELIN_FUSED(4); break;
        case 5: CKKS_RELIN_FUSED(5); break;
        case 6: CKKS_RELIN_FUSED(6); break;
        case 7: CKKS_RELIN_FUSED(7); break;
        default: CKKS_RELIN_FUSED(8); break;
    }
#undef CKKS_RELIN_FUSED
    CKKS_CUDA_TRY(cudaGetLastError());
    return CKKS_OK;
}

bool ntt_inverse_moddown_supported(const ckks_ctx* ctx, u32 q_limbs) {
    if (ctx->K < 1 || ctx->K > 3 || ctx->log_n1 > 8 || ctx->log_n2 < 1) return false;
    for (u32 l = 0; l < q_limbs; ++l)
        if (!ctx->h_tabs[l].f64 || ctx->moduli[l] >= (1ull << 50)) return false;
    for (u32 k = 0; k < ctx->K; ++k)
        if (ctx->moduli[ctx->L + k] >= (1ull << 62)) return false;
    return true;
}

// Inverse NTT of key-switch accumulators [polys][LK][N] (LK = q_limbs + K) with
// sigma folded, and ModDown into out [polys][q_limbs][N]. mid: workspace for
// pass 1 ([polys][LK][N]); words: workspace of polys * N * 4 doubles and zp of
// polys * K * N words (both may lie in `in`, which pass 1 has consumed).
int32_t ntt_inverse_moddown_launch(ckks_ctx* ctx, const u64* in, u64* mid, double* words, u64* zp, u64* out,
                                   u32 polys, u32 q_limbs, const GaloisOut& go, cudaStream_t st) {
    if (polys == 0) return CKKS_OK;
    if (!go.exps || !go.exps_inv || polys > 65535) {
        ckks_set_error("inverse NTT + ModDown: needs a Galois exponent table and at most 65535 polynomials");
        return CKKS_ERR_BAD_ARG;
    }
    const int la = ctx->log_n1, lb = ctx->log_n2;
    const u32 LK = q_limbs + ctx->K;
    const LimbMap lm = LimbMap::qp(ctx, q_limbs);
    if (int32_t rc = pass(3, lb, in, mid, ctx->d_tabs, lm, LK, polys, la, st, InvBase{}, ctx->ntt_log_c[3], go))
        return rc;
#define CKKS_INV_MD(LM)                                                                                            \
    do {                                                                                                           \
        const int lc = pick_log_c<LM>(lb, ctx->ntt_log_c[4]);                                                      \
        const int threads = Split<LM>::RMAX << lc;                                                                 \
        const size_t smem = (sizeof(u64) << (LM + lc)) + 2 * sizeof(u64) * (1u << LM);                            \
        k_inv2_p<LM><<<dim3(1u << (lb - lc), ctx->K, polys), threads, smem, st>>>(                                  \
            mid, zp, ctx->d_tabs, (int)q_limbs, (int)ctx->L, (int)LK, (int)ctx->K, lb, lc, go);                    \
        const dim3 gw((ctx->n + 255) / 256, polys);                                                                \
        if (ctx->K == 1) k_pwords<1><<<gw, 256, 0, st>>>(zp, words, ctx->mod_down, (int)ctx->log_n);              \
        else if (ctx->K == 2) k_pwords<2><<<gw, 256, 0, st>>>(zp, words, ctx->mod_down, (int)ctx->log_n);         \
        else k_pwords<3><<<gw, 256, 0, st>>>(zp, words, ctx->mod_down, (int)ctx->log_n);                          \
        k_inv2_moddown<LM><<<dim3(q_limbs, 1u << (lb - lc), polys), threads, smem, st>>>(                          \
            mid, out, words, ctx->d_tabs, ctx->mod_down.f64c, (int)q_limbs, (int)LK, lb, lc, go);                  \
    } while (0)
    switch (la) {
        case 1: CKKS_INV_MD(1); break;
        case 2: CKKS_INV_MD(2); break;
        case 3: CKKS_INV_MD(3); break;
        case 4: CKKS_INV_MD(4); break;
        case 5: CKKS_INV_MD(5); break;
        case 6: CKKS_INV_MD(6); break;
        case 7: CKKS_INV_MD(7); break;
        default: CKKS_INV_MD(8); break;
    }
#undef CKKS_INV_MD
    CKKS_CUDA_TRY(cudaGetLastError());
    return CKKS_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free in-place forward NTT.
//
// Some callers cannot let a library allocate device memory: processes whose
// device memory is reserved up front by their own arena or by a serving
// framework (a cudaMalloc from inside the library would fail or fragment that
// budget), and deployments that forbid device allocation after start-up.
// For them the in-place forward transform below stages its pass-1
// intermediate in a fixed file-scope device array instead of a workspace from
// the stream-ordered allocator. The array holds kStaticNttScratchWords words
// (16 MiB), is resident on every device that loads this library until the
// process exits, and is shared by every call: concurrent calls whose work
// overlaps on the GPU race on it. Pass 1 writes every word of the range it
// uses before pass 2 reads it, so nothing has to be cleared between calls.
namespace {

constexpr size_t kStaticNttScratchWords = size_t(1) << 21;
static __device__ __align__(256) u64 g_static_ntt_scratch[kStaticNttScratchWords];

std::mutex g_static_scratch_mutex;
u64* g_static_scratch_addr[128] = {};

// Device address of the array on the current device, looked up once per
// device (the host-side symbol is only a stand-in and must not reach a kernel).
int32_t static_scratch_address(u64** out) {
    int dev = 0;
    CKKS_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 128) {
        ckks_set_error("ckks_ntt_forward_inplace_static: device ordinal out of range");
        return CKKS_ERR_BAD_ARG;
    }
    std::lock_guard<std::mutex> lock(g_static_scratch_mutex);
    if (!g_static_scratch_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_static_ntt_scratch);
        if (e != cudaSuccess || !p) {
            ckks_set_error(std::string("ckks_ntt_forward_inplace_static: cudaGetSymbolAddress: ") +
                           cudaGetErrorString(e));
            return CKKS_ERR_CUDA;
        }
        g_static_scratch_addr[dev] = (u64*)p;
    }
    *out = g_static_scratch_addr[dev];
    return CKKS_OK;
}

}  // namespace

extern "C" int32_t ckks_ntt_forward_inplace_static(ckks_ctx* ctx, uint64_t* data, uint32_t n_polys,
                                                   uint32_t limb_begin, uint32_t limb_count, void* stream) {
    if (int32_t rc = ckks_require_device(ctx, "ckks_ntt_forward_inplace_static")) return rc;
    if (!data) {
        ckks_set_error("ckks_ntt_forward_inplace_static: null argument");
        return CKKS_ERR_BAD_ARG;
    }
    if ((size_t)limb_begin + limb_count > ctx->moduli.size()) {
        ckks_set_error("ckks_ntt_forward_inplace_static: limb range outside the context basis");
        return CKKS_ERR_BASIS_MISMATCH;
    }
    const size_t words = (size_t)n_polys * limb_count * ctx->n;
    if (words > kStaticNttScratchWords) {
        ckks_set_error("ckks_ntt_forward_inplace_static: n_polys * limb_count * N = " + std::to_string(words) +
                       " words exceeds the fixed scratch of " + std::to_string(kStaticNttScratchWords) +
                       " words (16 MiB); split the batch or use ckks_ntt_forward");
        return CKKS_ERR_BAD_ARG;
    }
    if (words == 0) return CKKS_OK;
    u64* scratch = nullptr;
    if (int32_t rc = static_scratch_address(&scratch)) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    const LimbMap lm = LimbMap::range(limb_begin, limb_count);
    const int la = ctx->log_n1, lb = ctx->log_n2;
    if (int32_t rc = pass(0, la, data, scratch, ctx->d_tabs, lm, limb_count, n_polys, lb, st, InvBase{}, ctx->ntt_log_c[0])) return rc;
    if (int32_t rc = pass(2, lb, scratch, data, ctx->d_tabs, lm, limb_count, n_polys, la, st, InvBase{}, ctx->ntt_log_c[2])) return rc;
    CKKS_CUDA_TRY(cudaGetLastError());
    return CKKS_OK;
}

// ---------------------------------------------------------------------------
// Autotuner: columns per CTA of every NTT pass.
//
// For each of the five passes (forward pass 1, forward pass 1 of signed digits,
// forward pass 2, inverse pass 1, inverse pass 2) every admissible number of
// columns per CTA (2^lc, lc = 1 .. the register/thread limit) is timed with CUDA
// events on a scratch batch of polys x limbs zero polynomials (the passes'
// running time does not depend on the data) and the fastest is kept in the
// context; every later transform of that context uses it. The report lists
// each pass's candidates and times (microseconds per launch) and the choice.
namespace {

template <int LOG_M>
int max_lc_for(int log_other) { return max_log_c<LOG_M>(log_other); }

int max_lc(int log_m, int log_other) {
    switch (log_m) {
        case 1: return max_lc_for<1>(log_other);
        case 2: return max_lc_for<2>(log_other);
        case 3: return max_lc_for<3>(log_other);
        case 4: return max_lc_for<4>(log_other);
        case 5: return max_lc_for<5>(log_other);
        case 6: return max_lc_for<6>(log_other);
        case 7: return max_lc_for<7>(log_other);
        case 8: return max_lc_for<8>(log_other);
        default: return max_lc_for<9>(log_other);
    }
}

}  // namespace

int32_t ntt_autotune(ckks_ctx* ctx, u32 limbs, u32 polys, cudaStream_t st) {
    if (limbs == 0 || polys == 0 || limbs > ctx->L + ctx->K) {
        ckks_set_error("ckks_ctx_autotune: limbs must be in [1, L + K] and polys >= 1");
        return CKKS_ERR_BAD_ARG;
    }
    const int la = ctx->log_n1, lb = ctx->log_n2;
    const LimbMap lm = LimbMap::range(0, limbs);
    const size_t words = (size_t)polys * limbs * ctx->n;
    Workspace<u64> a, b;
    int32_t rc;
    if ((rc = a.alloc(words, st)) || (rc = b.alloc(words, st))) return rc;
    CKKS_CUDA_TRY(cudaMemsetAsync(a.p, 0, words * sizeof(u64), st));
    cudaEvent_t e0, e1;
    CKKS_CUDA_TRY(cudaEventCreate(&e0));
    CKKS_CUDA_TRY(cudaEventCreate(&e1));
    static const char* names[5] = {"forward pass 1", "forward pass 1 (digits)", "forward pass 2", "inverse pass 1",
                                   "inverse pass 2"};
    // pass: log_m, log_other, polys (digit pass: polys digits of one polynomial)
    const int log_m[5] = {la, la, lb, lb, la}, log_o[5] = {lb, lb, la, la, lb};
    std::string rep;
    rc = CKKS_OK;
    for (int w = 0; w < 5 && rc == CKKS_OK; ++w) {
        const int mx = max_lc(log_m[w], log_o[w]);
        int best = -1;
        float best_ms = 0;
        rep += names[w];
        rep += ":";
        for (int lc = mx < 1 ? mx : 1; lc <= mx && rc == CKKS_OK; ++lc) {
            float ms = 0;
            for (int it = 0; it < 4 && rc == CKKS_OK; ++it) {  // first launch untimed
                if (it == 1) cudaEventRecord(e0, st);
                rc = pass(w, log_m[w], a.p, b.p, ctx->d_tabs, lm, limbs, polys, log_o[w], st, InvBase{}, lc);
            }
            if (rc != CKKS_OK) break;
            cudaEventRecord(e1, st);
            if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
                rc = CKKS_ERR_CUDA;
                ckks_set_error("ckks_ctx_autotune: event timing failed");
                break;
            }
            ms /= 3;
            char buf[64];
            snprintf(buf, sizeof buf, " C=%d %.1f us", 1 << lc, 1000.0 * ms);
            rep += buf;
            if (best < 0 || ms < best_ms) {
                best = lc;
                best_ms = ms;
            }
        }
        if (rc == CKKS_OK) {
            ctx->ntt_log_c[w] = best;
            char buf[64];
            snprintf(buf, sizeof buf, " -> C=%d\n", 1 << best);
            rep += buf;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc == CKKS_OK) {
        char head[96];
        snprintf(head, sizeof head, "NTT autotune N=2^%u, %u limbs x %u polys per launch\n", ctx->log_n, limbs, polys);
        ctx->tuning_report = head + rep;
    }
    return rc;
}
