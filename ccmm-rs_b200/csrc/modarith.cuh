// modarith.cuh -- u64 modular arithmetic for sm_100a.
//
// Residues live in [0, q) at every kernel boundary; inside a kernel the NTT
// butterflies keep values lazily reduced in [0, 2q) or [0, 4q) (Harvey), which
// needs q < 2^62 (checked when a context is created).
#pragma once
#include <cstdint>

typedef uint64_t u64;
typedef int64_t i64;
typedef uint32_t u32;

#ifdef __CUDACC__
#define CKKS_HD __host__ __device__ __forceinline__
#else
#define CKKS_HD inline
#endif

// Shoup companion floor(w * 2^64 / q) (the reference's ShoupMultiplier,
// ring/modulus.rs:97-104). Host only.
inline u64 shoup_quotient_host(u64 w, u64 q) {
    return (u64)(((unsigned __int128)w << 64) / q);
}

#ifdef __CUDACC__
// x * w mod q, lazily reduced to [0, 2q); valid for any x < 2^64.
__device__ __forceinline__ u64 mul_shoup_lazy(u64 x, u64 w, u64 wq, u64 q) {
    u64 hi = __umul64hi(x, wq);
    return x * w - hi * q;
}
__device__ __forceinline__ u64 mul_shoup(u64 x, u64 w, u64 wq, u64 q) {
    u64 r = mul_shoup_lazy(x, w, wq, q);
    return r >= q ? r - q : r;
}
__device__ __forceinline__ u64 reduce_2q(u64 x, u64 q) { return x >= q ? x - q : x; }
// floor(w * 2^64 / q) on the device (w < q): one 128-by-64 division, setup use only.
__device__ __forceinline__ u64 shoup_quotient_dev(u64 w, u64 q) {
    return (u64)(((unsigned __int128)w << 64) / q);
}
__device__ __forceinline__ u64 reduce_4q(u64 x, u64 q) {
    u64 q2 = q << 1;
    x = x >= q2 ? x - q2 : x;
    return x >= q ? x - q : x;
}
__device__ __forceinline__ u64 add_mod(u64 a, u64 b, u64 q) {
    u64 s = a + b;
    return s >= q ? s - q : s;
}
__device__ __forceinline__ u64 sub_mod(u64 a, u64 b, u64 q) { return a >= b ? a - b : a + q - b; }
__device__ __forceinline__ u64 neg_mod(u64 a, u64 q) { return a ? q - a : 0; }

// Generic a * b mod q for canonical operands (both < q < 2^62) via a Barrett
// reduction of the 128-bit product with mu = floor(2^124 / q):
// quotient estimate floor(hi*2^4 ... ) -- implemented on 128-bit halves.
struct Barrett {
    u64 q;
    u64 mu_hi, mu_lo;  // floor(2^128 / q) as two 64-bit words (q > 2^32 so it fits 96 bits)
};
__device__ __forceinline__ u64 mul_barrett(u64 a, u64 b, const Barrett& m) {
    // x = a*b (< 2^124); estimate floor(x * mu / 2^128) with a <= 2 error
    u64 xlo = a * b, xhi = __umul64hi(a, b);
    // t = x * mu >> 128, mu = mu_hi*2^64 + mu_lo
    u64 p1_hi = __umul64hi(xlo, m.mu_hi);
    u64 p1_lo = xlo * m.mu_hi;
    u64 p2_hi = __umul64hi(xhi, m.mu_lo);
    u64 p2_lo = xhi * m.mu_lo;
    u64 p0_hi = __umul64hi(xlo, m.mu_lo);
    // sum of middle words with carries
    u64 mid = p0_hi + p1_lo;
    u64 c = mid < p0_hi;
    u64 mid2 = mid + p2_lo;
    c += mid2 < mid;
    u64 qt = xhi * m.mu_hi + p1_hi + p2_hi + c;
    u64 r = xlo - qt * m.q;
    while (r >= m.q) r -= m.q;
    return r;
}

// x = xhi * 2^64 + xlo (xhi < q) modulo q, Barrett with mu = floor(2^128 / q).
__device__ __forceinline__ u64 reduce_wide(u64 xhi, u64 xlo, u64 q, u64 mu_hi, u64 mu_lo) {
    u64 p0_hi = __umul64hi(xlo, mu_lo);
    u64 p1_lo = xlo * mu_hi, p1_hi = __umul64hi(xlo, mu_hi);
    u64 p2_lo = xhi * mu_lo, p2_hi = __umul64hi(xhi, mu_lo);
    u64 mid = p0_hi + p1_lo;
    u64 c = mid < p0_hi;
    u64 mid2 = mid + p2_lo;
    c += mid2 < mid;
    u64 qt = xhi * mu_hi + p1_hi + p2_hi + c;
    u64 r = xlo - qt * q;
    while (r >= q) r -= q;
    return r;
}

// Exact 128-bit sum of products of canonical residues (each < q^2 < 2^124):
// fold() reduces it to the canonical residue in lo; at most 15 products may
// be added between folds.
struct Acc128 {
    u64 hi, lo;
    __device__ __forceinline__ void mac(u64 a, u64 b) {
        u64 pl = a * b, ph = __umul64hi(a, b);
        lo += pl;
        hi += ph + (lo < pl);
    }
    __device__ __forceinline__ void fold(u64 q, u64 mu_hi, u64 mu_lo) {
        u64 h = hi >= q ? reduce_wide(0, hi, q, mu_hi, mu_lo) : hi;
        lo = reduce_wide(h, lo, q, mu_hi, mu_lo);
        hi = 0;
    }
};
#endif

inline void barrett_host(u64 q, u64* mu_hi, u64* mu_lo) {
    unsigned __int128 max = ~(unsigned __int128)0;
    unsigned __int128 mu = max / q;
    if (max % q == q - 1) mu += 1;
    *mu_hi = (u64)(mu >> 64);
    *mu_lo = (u64)mu;
}
