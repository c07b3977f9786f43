// ntt_core.cuh -- register-tiled radix-2 networks used by the NTT passes.
//
// The forward transform is the merged Cooley-Tukey network over all N points
// (natural in, bit-reversed out) with twiddles psi^bitrev(i) (the SEAL/
// Longa-Naehrig form); the inverse is the merged Gentleman-Sande network
// (bit-reversed in, natural out) with psi^-bitrev(i). A pass runs the stages
// that touch one "column" (or "row") of the N = A x B index matrix: M = A or
// B points, held R1 per thread in registers for the first log R1 stages and
// R2 per thread for the rest, with one shared-memory exchange in between.
#pragma once
#include "kernels.cuh"

namespace nttc {

__device__ __forceinline__ u32 brev(u32 x, int bits) { return bits ? (__brev(x) >> (32 - bits)) : 0; }

// Shoup product W Y with the quotient's high word built from three of the four
// 32 x 32-bit partial products of Y and Wq: the dropped parts (the low halves
// of Y_hi Wq_lo and Y_lo Wq_hi over 2^32, and Y_lo Wq_lo over 2^64) sum to less
// than 3, so the estimate is floor(Y Wq / 2^64) or up to 2 less and the
// result Y W - hi q lies in [0, 4q) for any 64-bit Y and W < q (one extra q per
// unit of the estimate's shortfall over the exact form's [0, 2q)).
__device__ __forceinline__ u64 mul_shoup_lazy4(u64 Y, u64 W, u64 Wq, u64 q) {
    const u32 y0 = (u32)Y, y1 = (u32)(Y >> 32), w0 = (u32)Wq, w1 = (u32)(Wq >> 32);
    const u64 hi = (u64)y1 * w1 + __umulhi(y1, w0) + __umulhi(y0, w1);
    return Y * W - hi * q;
}

// Harvey butterflies on lazily reduced values.
// CT (kRed): X, Y in [0, 4q) -> X' = X + W Y, Y' = X - W Y, both in [0, 4q)
// (q2 = 2q).
// CT (!kRed): no conditional subtraction and the three-product Shoup form, W Y
// in [0, 4q) for any 64-bit Y, Y' = X - W Y + q4 (q4 = 4q); each stage adds
// less than 4q to the bound, so a pass of s stages from [0, B) ends below
// B + 4 s q. Used for q < 2^58, where a pass of up to 9 stages from inputs
// below 4q stays below 40 q < 2^64 (each pass ends in an exact reduction).
template <bool kRed = true>
__device__ __forceinline__ void ct_bfly(u64& X, u64& Y, u64 W, u64 Wq, u64 q, u64 q2) {
    if (kRed) {
        u64 x = X >= q2 ? X - q2 : X;
        u64 t = mul_shoup_lazy(Y, W, Wq, q);
        X = x + t;
        Y = x - t + q2;
    } else {
        u64 x = X;
        u64 t = mul_shoup_lazy4(Y, W, Wq, q);
        X = x + t;
        Y = x - t + q2;
    }
}
constexpr u64 kLazyCtBound = 1ull << 58;  // primes below this take the !kRed network
// GS (kLazy false): X, Y in [0, 2q) -> X' = X + Y, Y' = (X - Y) W, both in [0, 2q).
// GS (kLazy): X, Y in [0, c) with c a multiple of q (passed as q2) -> X' = X + Y
// in [0, 2c), Y' = (X + c - Y) W in [0, 4q) (three-product Shoup form); no
// conditional subtraction. Global stage s of a network whose inputs are below
// 2q uses c = 2^(s+1) q (Y' < 4q <= 2c as well), so a pass of m stages stays
// below 2^(m+1) q < 2^64 for m <= 9 (N <= 2^18) and q < 2^54.
template <bool kLazy = false>
__device__ __forceinline__ void gs_bfly(u64& X, u64& Y, u64 W, u64 Wq, u64 q, u64 q2) {
    if (kLazy) {
        const u64 d = X + q2 - Y;
        X = X + Y;
        Y = mul_shoup_lazy4(d, W, Wq, q);
    } else {
        u64 s = X + Y;
        u64 d = X - Y + q2;
        X = s >= q2 ? s - q2 : s;
        Y = mul_shoup_lazy(d, W, Wq, q);
    }
}
constexpr u64 kLazyGsBound = 1ull << 54;  // primes below this take the lazy GS network

// Merged CT stages s0 .. s0 + LR - 1 on R = 2^LR register values with pair
// distance R/2, R/4, .., 1; the twiddle block of register e at stage ls is
// (base << ls) + (e >> (LR - ls)); tw(stage, block, W, Wq) supplies the twiddle.
// Compile-time recursion keeps every register index static.
template <int LR, int LS, bool kRed, typename TW>
__device__ __forceinline__ void ct_stage(u64 (&x)[1 << LR], int s0, u32 base, TW& tw, u64 q, u64 q2) {
    if constexpr (LS < LR) {
        constexpr int half = (1 << LR) >> (LS + 1);
#pragma unroll
        for (int b = 0; b < (1 << LS); ++b) {
            u64 W, Wq;
            tw(s0 + LS, (base << LS) + b, W, Wq);
#pragma unroll
            for (int o = 0; o < half; ++o)
                ct_bfly<kRed>(x[b * 2 * half + o], x[b * 2 * half + o + half], W, Wq, q, q2);
        }
        ct_stage<LR, LS + 1, kRed>(x, s0, base, tw, q, q2);
    }
}

template <int LR, bool kRed = true, typename TW>
__device__ __forceinline__ void ct_stages(u64 (&x)[1 << LR], int s0, u32 base, TW tw, u64 q) {
    ct_stage<LR, 0, kRed>(x, s0, base, tw, q, kRed ? q << 1 : q << 2);
}

template <int LR, int LS, bool kLazy, typename TW>
__device__ __forceinline__ void gs_stage(u64 (&x)[1 << LR], int s0, u32 blk0, TW& tw, u64 q, u64 q2) {
    if constexpr (LS < LR) {
        constexpr int t = 1 << LS;
        constexpr int nblk = (1 << LR) >> (LS + 1);
        const u64 c = kLazy ? q << (s0 + LS + 1) : q2;  // lazy: 2^(s+1) q at global stage s
#pragma unroll
        for (int b = 0; b < nblk; ++b) {
            u64 W, Wq;
            tw(s0 + LS, (blk0 << (LR - LS - 1)) + b, W, Wq);
#pragma unroll
            for (int o = 0; o < t; ++o) gs_bfly<kLazy>(x[b * 2 * t + o], x[b * 2 * t + o + t], W, Wq, q, c);
        }
        gs_stage<LR, LS + 1, kLazy>(x, s0, blk0, tw, q, q2);
    }
}

// Merged GS stages with register distance t = 1, 2, .., 2^(LR-1) (local stages
// s0 .. s0 + LR - 1 of the network whose t = 2^s); block of register e at
// stage ls is (blk0 << (LR - ls - 1)) + (e >> (ls + 1)).
template <int LR, bool kLazy = false, typename TW>
__device__ __forceinline__ void gs_stages(u64 (&x)[1 << LR], int s0, u32 blk0, TW tw, u64 q) {
    gs_stage<LR, 0, kLazy>(x, s0, blk0, tw, q, q << 1);
}

}  // namespace nttc

// ---------------------------------------------------------------------------
// Exact modular butterflies on the FP64 pipe, for primes q < 2^50.
//
// Values are integers held in doubles, signed, of magnitude below 2^53 (so
// every one is exact). The product Y W (up to 2^103) is split error-free into
// h = fl(Y W) and l = Y W - h (one FMA, exact: Dekker/Ogita TwoProduct); the
// quotient estimate t = rint(fl(Y Wp)) with Wp = fl(W / q) differs from
// Y W / q by at most 1/2 + |Y| 2^-54 + ulp(Y Wp)/2; then h - t q (one FMA)
// is an integer below 2^53 in magnitude and exact, and r = (h - t q) + l =
// Y W - t q exactly. Hence r = Y W (mod q) with
//   |r| <= 0.75 q for |Y| < 2^51, <= q for |Y| < 2^52, <= 1.5 q for |Y| < 2^53.
// No result depends on a rounding: the residues are the same integers the
// Shoup network produces, up to a multiple of q, and every pass ends in an
// exact reduction to [0, q).
//
// Cooley-Tukey (X, Y) -> (X + r, X - r): a stage adds at most |r| to the
// bound. From inputs below q (or the centred reduction's q/2 + tiny), four
// stages stay below 4.5 q. Gentleman-Sande (X, Y) -> (X + Y, (X - Y) W) doubles
// the sum path: four stages from centred inputs stay below 8 q <= 2^53 - 8.
// The passes therefore reduce once at their shared-memory exchange (every
// four stages) and once at the end; the tests of lazy_bounds_cpu restate
// these bounds.
namespace nttf {

constexpr u64 kF64Bound = 1ull << 50;  // primes below this take the FP64 networks
constexpr double kTwo52 = 4503599627370496.0;

// Y W mod q as a signed integer (bounds above).
__device__ __forceinline__ double mulmod(double y, double w, double wp, double q) {
    const double h = __dmul_rn(y, w);
    const double l = __fma_rn(y, w, -h);
    const double t = rint(__dmul_rn(y, wp));
    return __dadd_rn(__fma_rn(-t, q, h), l);
}
// v - rint(v / q) q: |result| <= q/2 + |v| 2^-52 for |v| < 2^53 (exact).
__device__ __forceinline__ double center(double v, double q, double qinv) {
    return __fma_rn(-rint(__dmul_rn(v, qinv)), q, v);
}
// u64 below 2^52 -> double (exact): bits 0x433 | v is 2^52 + v.
__device__ __forceinline__ double from_u52(u64 v) {
    return __dsub_rn(__longlong_as_double((long long)(v | 0x4330000000000000ull)), kTwo52);
}
// |v| < 2^53 -> its residue in [0, q) as u64.
__device__ __forceinline__ u64 to_canonical(double v, double q, double qinv) {
    double r = center(v, q, qinv);
    r = r < 0.0 ? __dadd_rn(r, q) : r;
    return (u64)__double_as_longlong(__dadd_rn(r, kTwo52)) & 0xFFFFFFFFFFFFFull;
}

__device__ __forceinline__ void ct_bfly(double& X, double& Y, double W, double Wp, double q) {
    const double r = mulmod(Y, W, Wp, q);
    const double x = X;
    X = __dadd_rn(x, r);
    Y = __dsub_rn(x, r);
}
__device__ __forceinline__ void gs_bfly(double& X, double& Y, double W, double Wp, double q) {
    const double d = __dsub_rn(X, Y);
    X = __dadd_rn(X, Y);
    Y = mulmod(d, W, Wp, q);
}

// Merged CT / GS stages with the register and twiddle indexing of
// nttc::ct_stages / nttc::gs_stages; tw(stage, block) returns (W, Wp).
template <int LR, int LS, typename TW>
__device__ __forceinline__ void ct_stage(double (&x)[1 << LR], int s0, u32 base, TW& tw, double q) {
    if constexpr (LS < LR) {
        constexpr int half = (1 << LR) >> (LS + 1);
#pragma unroll
        for (int b = 0; b < (1 << LS); ++b) {
            const double2 w = tw(s0 + LS, (base << LS) + b);
#pragma unroll
            for (int o = 0; o < half; ++o) ct_bfly(x[b * 2 * half + o], x[b * 2 * half + o + half], w.x, w.y, q);
        }
        ct_stage<LR, LS + 1>(x, s0, base, tw, q);
    }
}
template <int LR, typename TW>
__device__ __forceinline__ void ct_stages(double (&x)[1 << LR], int s0, u32 base, TW tw, double q) {
    ct_stage<LR, 0>(x, s0, base, tw, q);
}
template <int LR, int LS, typename TW>
__device__ __forceinline__ void gs_stage(double (&x)[1 << LR], int s0, u32 blk0, TW& tw, double q) {
    if constexpr (LS < LR) {
        constexpr int t = 1 << LS;
        constexpr int nblk = (1 << LR) >> (LS + 1);
#pragma unroll
        for (int b = 0; b < nblk; ++b) {
            const double2 w = tw(s0 + LS, (blk0 << (LR - LS - 1)) + b);
#pragma unroll
            for (int o = 0; o < t; ++o) gs_bfly(x[b * 2 * t + o], x[b * 2 * t + o + t], w.x, w.y, q);
        }
        gs_stage<LR, LS + 1>(x, s0, blk0, tw, q);
    }
}
template <int LR, typename TW>
__device__ __forceinline__ void gs_stages(double (&x)[1 << LR], int s0, u32 blk0, TW tw, double q) {
    gs_stage<LR, 0>(x, s0, blk0, tw, q);
}

}  // namespace nttf
