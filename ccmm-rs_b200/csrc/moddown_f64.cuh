// moddown_f64.cuh -- the FP64 ModDown arithmetic (ring/auxiliary_modulus.rs:89-171)
// shared by the streaming ModDown kernel (elementwise.cu) and the inverse-NTT
// pass fused with it (ntt.cu).
//
// For Q primes below 2^50 and K <= 3 auxiliary limbs: the centred CRT value
// y_c of the auxiliary residues is rebuilt exactly from its mixed-radix
// digits as three 64-bit words (|y_c| < P/2 < 2^187), its magnitude split into
// four 47-bit words w_k, and per Q limb, with s the sign of y_c,
//   out = x P^-1 - s sum_k w_k (2^(47 k) P^-1 mod q)   (mod q):
// five exact FP64 modular products (nttf::mulmod, multiplicands below 2^51,
// so each result is below 0.75 q in magnitude and the sum below 3.75 q) and
// one exact reduction.
#pragma once
#include "context.cuh"
#include "ntt_core.cuh"

namespace mdf {

// Mixed-radix digits (Garner) of the K auxiliary residues v (in place), the
// sign of the centred value (value > floor(P/2) -> negative) and the four
// 47-bit words of its magnitude.
template <int KT>
__device__ __forceinline__ void crt_words(u64 (&v)[KT], const ModDownConst& md, double (&w)[4], bool& neg) {
#pragma unroll
    for (int i = 0; i < KT; ++i) {
        const u64 p = md.p[i];
        u64 acc = 0;
#pragma unroll
        for (int j = 0; j < i; ++j) acc = add_mod(acc, mul_shoup(v[j], md.pp[i][j], md.pp_q[i][j], p), p);
        v[i] = mul_shoup(sub_mod(v[i], acc, p), md.pinv[i], md.pinv_q[i], p);
    }
    neg = false;
    bool decided = false;
#pragma unroll
    for (int i = KT - 1; i >= 0; --i) {
        if (!decided && v[i] != md.half[i]) {
            neg = v[i] > md.half[i];
            decided = true;
        }
    }
    // y = v0 + p0 (v1 + p1 v2) in three words
    typedef unsigned __int128 u128;
    u64 y0, y1 = 0, y2 = 0;
    if (KT == 1) {
        y0 = v[0];
    } else if (KT == 2) {
        const u128 a = (u128)v[1] * md.p[0] + v[0];
        y0 = (u64)a;
        y1 = (u64)(a >> 64);
    } else {
        const u128 tt = (u128)v[KT - 1] * md.p[1] + v[1];
        const u128 a = (u128)(u64)tt * md.p[0] + v[0];
        const u128 b = (u128)(u64)(tt >> 64) * md.p[0] + (u64)(a >> 64);
        y0 = (u64)a;
        y1 = (u64)b;
        y2 = (u64)(b >> 64);
    }
    if (neg) {  // |y - P| = P - y
        const u64 d0 = md.P3[0] - y0, b0 = md.P3[0] < y0;
        const u64 t1 = md.P3[1] - y1, b1 = md.P3[1] < y1;
        const u64 d1 = t1 - b0, b1b = t1 < b0;
        const u64 d2 = md.P3[2] - y2 - (b1 | b1b);
        y0 = d0;
        y1 = d1;
        y2 = d2;
    }
    const u64 m47 = (1ull << 47) - 1;
    w[0] = nttf::from_u52(y0 & m47);
    w[1] = nttf::from_u52(((y0 >> 47) | (y1 << 17)) & m47);
    w[2] = nttf::from_u52(((y1 >> 30) | (y2 << 34)) & m47);
    w[3] = nttf::from_u52((y2 >> 13) & m47);
}

// One Q limb: ci = [q, 1/q, (P^-1, /q), (2^(47 k) P^-1, /q) k = 0..3]; flip
// negates the result (the sign of a folded Galois automorphism). Canonical.
__device__ __forceinline__ u64 limb(double xd, const double (&w)[4], bool neg, const double* ci, bool flip) {
    const double q = ci[0], qinv = ci[1];
    const double r = nttf::mulmod(xd, ci[2], ci[3], q);
    const double sm = __dadd_rn(__dadd_rn(nttf::mulmod(w[0], ci[4], ci[5], q), nttf::mulmod(w[1], ci[6], ci[7], q)),
                                __dadd_rn(nttf::mulmod(w[2], ci[8], ci[9], q), nttf::mulmod(w[3], ci[10], ci[11], q)));
    double rr = nttf::center(neg ? __dadd_rn(r, sm) : __dsub_rn(r, sm), q, qinv);
    if (flip) rr = -rr;
    rr = rr < 0.0 ? __dadd_rn(rr, q) : rr;
    return (u64)__double_as_longlong(__dadd_rn(rr, nttf::kTwo52)) & 0xFFFFFFFFFFFFFull;
}

}  // namespace mdf
