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
