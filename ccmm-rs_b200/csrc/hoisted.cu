// hoisted.cu -- NTT-domain hoisting of the bounded hybrid-QP rotation.
//
// The reference hoists at the digit level (BoundedGadgetDecomposition::
// automorphism_hoisted, grafting/bounded_gadget.rs:273-312) and transforms the
// re-normalised digits for every Galois element. Those digits equal the
// signed automorphism of the digits of a, sigma(d_j), except at coefficients
// whose source value is negated and holds a digit equal to -B/2: there the
// carry re-normalisation changes a few digits by Delta. Since
// NTT(sigma(d_j)) is the NTT-domain permutation of NTT(d_j)
// (ring/ntt_galois_permutation.rs:5-19), the exact key-switch sum is
//   sum_j NTT(d_j)[pi(k)] K_j[k] + sum_{(t,j,Delta)} Delta psi^((2k+1) t) K_j[k],
// so the digit transforms are done once per ciphertext, and every Galois
// element costs one MAC pass plus the (rare, sparse) correction terms. A
// (ciphertext, Galois element) pair whose corrections exceed the list
// capacity is recomputed by the non-hoisted path, so every output word equals
// the reference's.
//
// The MAC streams each key slice once per group of G ciphertexts (evict-first
// loads) while the hoisted digit transforms of the group stay L2-resident
// and are gathered through the permutation.
#include "keyswitch.cuh"

namespace {

constexpr int kT = 256;

struct Exc {
    u32 t, j;
    i64 delta;
};


__device__ __forceinline__ u64 pow_mod_dev(u64 b, u64 e, const Barrett& m) {
    u64 r = 1;
    while (e) {
        if (e & 1) r = mul_barrett(r, b, m);
        b = mul_barrett(b, b, m);
        e >>= 1;
    }
    return r;
}

// Flagged source coefficients (a digit equals -B/2) of G ciphertexts ->
// exception lists per (ciphertext, key): entries (t, j, Delta) where the
// reference's re-normalised digit differs from -d_j[s].
__global__ void k_hoist_exceptions(const i64* __restrict__ digits, size_t dig_stride, const u32* __restrict__ flags,
                                   size_t flag_stride, const u64* __restrict__ exps, int n_keys, int D, int base_log,
                                   int log_n, Exc* __restrict__ exc, u32* __restrict__ exc_count, int cap) {
    const int c = blockIdx.z, g = blockIdx.y;
    const u32* fl = flags + c * flag_stride;
    const u32 nflag = fl[0];
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nflag) return;
    const u32 n = 1u << log_n;
    const u32 s = fl[1 + i];
    const u64 mapped = ((u64)s * exps[g]) & (2ull * n - 1);
    if (mapped < n) return;  // not negated: digits move unchanged
    const u32 t = (u32)(mapped - n);
    const i64* d = digits + c * dig_stride;
    const i64 B = (i64)1 << base_log, half = B >> 1;
    i64 carry = 0;
    Exc* list = exc + ((size_t)c * n_keys + g) * cap;
    u32* cnt = exc_count + (size_t)c * n_keys + g;
    for (int j = 0; j < D; ++j) {
        i64 dj = d[((size_t)j << log_n) + s];
        i64 value = -dj + carry;
        i64 m = (value + half) & (B - 1);
        i64 normalized = m - half;
        carry = (value - normalized) >> base_log;
        i64 delta = normalized + dj;  // reference digit minus the naive -d_j
        if (delta != 0) {
            u32 slot = atomicAdd(cnt, 1u);
            if ((int)slot < cap) list[slot] = Exc{t, (u32)j, delta};
        }
    }
}

// MAC in the permuted index s = pi_g(k) (keys are stored permuted):
// acc'[c][g][0][l][s] = pf_l Bhat_c[l][s] + sum_j Yhat_c[j][l][s] key'_g[j][l][0][s] + corrections
// acc'[c][g][1][l][s] =                      sum_j Yhat_c[j][l][s] key'_g[j][l][1][s] + corrections
// so acc = perm_g(acc'); the caller applies sigma_g after the inverse transform.
// Every load is contiguous: keys stream once per group (evict-first), the
// group's digit transforms are re-read from L2 by every key.
template <int G>
__global__ void __launch_bounds__(kT) k_mac_hoisted(const u64* __restrict__ Yhat, size_t y_stride,
                                                    const u64* __restrict__ Bhat, size_t b_stride,
                                                    const u64* const* __restrict__ keys,
                                                    const u64* __restrict__ exps_inv, const u64* __restrict__ pf,
                                                    const u64* __restrict__ pf_q, u64* __restrict__ acc,
                                                    const NttTab* __restrict__ tabs, LimbMap lm, int n_ct, int n_keys,
                                                    int Lq, int LK, int D, int log_n, const Exc* __restrict__ exc,
                                                    const u32* __restrict__ exc_count, int cap,
                                                    const u64* __restrict__ psi) {
    const u32 n = 1u << log_n;
    const u32 s = blockIdx.x * blockDim.x + threadIdx.x;
    const int g = blockIdx.y, l = blockIdx.z;
    if (s >= n) return;
    const NttTab& T = tabs[lm(l)];
    const u64 q = T.q, mh = T.mu_hi, ml = T.mu_lo;
    const u64* key = keys[g];
    Acc128 ab[G], aa[G];
#pragma unroll
    for (int c = 0; c < G; ++c) ab[c] = aa[c] = Acc128{0, 0};
    int since = 0;
    for (int j = 0; j < D; ++j) {
        const size_t kofs = (((size_t)j * LK + l) * 2) << log_n;
        const u64 kb = __ldcs(key + kofs + s), ka = __ldcs(key + kofs + n + s);
        const size_t yofs = (((size_t)j * LK + l) << log_n) + s;
#pragma unroll
        for (int c = 0; c < G; ++c) {
            if (c < n_ct) {
                u64 y = __ldg(Yhat + c * y_stride + yofs);
                ab[c].mac(y, kb);
                aa[c].mac(y, ka);
            }
        }
        if (++since == 15) {
#pragma unroll
            for (int c = 0; c < G; ++c) {
                ab[c].fold(q, mh, ml);
                aa[c].fold(q, mh, ml);
            }
            since = 0;
        }
    }
    const Barrett bm{q, mh, ml};
#pragma unroll
    for (int c = 0; c < G; ++c) {
        if (c >= n_ct) break;
        ab[c].fold(q, mh, ml);
        aa[c].fold(q, mh, ml);
        u64 b = ab[c].lo, a = aa[c].lo;
        if (l < Lq) b = add_mod(b, mul_shoup(__ldg(Bhat + c * b_stride + ((size_t)l << log_n) + s), pf[l], pf_q[l], q), q);
        const u32 cnt = min(exc_count[(size_t)c * n_keys + g], (u32)cap);
        if (cnt) {
            const Exc* list = exc + ((size_t)c * n_keys + g) * cap;
            const u64 ps = psi[lm(l)];
            const u32 k = galois_src(s, exps_inv[g], log_n);  // unpermuted slot of s
            for (u32 e = 0; e < cnt; ++e) {
                const Exc x = list[e];
                // NTT of Delta * X^t at slot k: Delta * psi^((2k+1) t)
                u64 w = pow_mod_dev(ps, ((2ull * k + 1) * x.t) & (2ull * n - 1), bm);
                u64 dm = x.delta < 0 ? (u64)(-x.delta) % q : (u64)x.delta % q;
                if (x.delta < 0 && dm) dm = q - dm;
                u64 v = mul_barrett(w, dm, bm);
                const size_t kofs = (((size_t)x.j * LK + l) * 2) << log_n;
                b = add_mod(b, mul_barrett(v, key[kofs + s], bm), q);
                a = add_mod(a, mul_barrett(v, key[kofs + n + s], bm), q);
            }
        }
        const size_t obase = (((size_t)c * n_keys + g) * 2 * LK) << log_n;
        acc[obase + ((size_t)l << log_n) + s] = b;
        acc[obase + (((size_t)LK + l) << log_n) + s] = a;
    }
}

u64 galois_inverse_host(u64 k, u32 n) {
    const u64 two_n = 2ull * n;
    k %= two_n;
    u64 r = 1, b = k, e = n - 1;
    while (e) {
        if (e & 1) r = (r * b) % two_n;
        b = (b * b) % two_n;
        e >>= 1;
    }
    return r;
}

// Split-operand accumulator: with sb = ceil(bits(q - 1) / 2), an operand
// x < q is x1 * 2^sb + x0 (x0, x1 < 2^sb) and a product is
// x0 y0 + (x0 y1 + x1 y0) 2^sb + x1 y1 2^(2 sb). Three 64-bit partial sums
// take each 32 x 32 -> 64 multiply with accumulate (IMAD.WIDE.U32) without
// carry handling; they are reduced mod q every `fold` terms (chosen so the
// middle sum cannot overflow) and combined with 2^sb, 2^2sb mod q. The value
// is the canonical residue of the same exact sum of products.
struct SplitAcc {
    u64 s0, s1, s2;
    __device__ __forceinline__ void mac(u32 x0, u32 x1, u32 y0, u32 y1) {
        s0 += (u64)x0 * y0;
        s1 += (u64)x0 * y1;
        s1 += (u64)x1 * y0;
        s2 += (u64)x1 * y1;
    }
    // Reduce to the canonical residue, kept in s0 (s0 stays below
    // q + fold * 2^(2 sb) < 2^64 until the next fold).
    __device__ __forceinline__ void fold(u64 q, u64 one_q, u64 r1, u64 r1q, u64 r2, u64 r2q) {
        u64 t = reduce_2q(mul_shoup_lazy(s0, 1, one_q, q), q);
        t = add_mod(t, reduce_2q(mul_shoup_lazy(s1, r1, r1q, q), q), q);
        t = add_mod(t, reduce_2q(mul_shoup_lazy(s2, r2, r2q, q), q), q);
        s0 = t;
        s1 = s2 = 0;
    }
};

// Tiled MAC: one CTA owns (limb l, slot tile of kS slots) for G ciphertexts
// and every Galois key. The G x D x kS digit-transform tile is staged in
// shared memory once (pre-split into its two sb-bit halves); keys stream from
// HBM exactly once per group (evict-first), kU digits of key loads in flight
// per thread. Thread (s, lane) accumulates keys g = lane, lane + kLanes, ..
// for all G ciphertexts. Same sums as k_mac_hoisted.
constexpr int kS = 64, kLanes = 4, kU = 4;

template <int G>
__global__ void __launch_bounds__(kS * kLanes, 2) k_mac_tiled(const u64* __restrict__ Yhat, size_t y_stride,
                                                           const u64* __restrict__ Bhat, size_t b_stride,
                                                           const u64* const* __restrict__ keys,
                                                           const u64* __restrict__ exps_inv,
                                                           const u64* __restrict__ pf, const u64* __restrict__ pf_q,
                                                           u64* __restrict__ acc, const NttTab* __restrict__ tabs,
                                                           LimbMap lm, int n_ct, int n_keys, int Lq, int LK, int D,
                                                           int log_n, const Exc* __restrict__ exc,
                                                           const u32* __restrict__ exc_count, int cap,
                                                           const u64* __restrict__ psi) {
    extern __shared__ u64 ytile[];  // [G][D][kS], each word (y >> sb) << 32 | (y & mask)
    const u32 n = 1u << log_n;
    const int l = blockIdx.y;
    const u32 s0 = blockIdx.x * kS;
    const int tid = threadIdx.x, si = tid % kS, lane = tid / kS;
    const u32 s = s0 + si;
    const NttTab& T = tabs[lm(l)];
    const u64 q = T.q, mh = T.mu_hi, ml = T.mu_lo;
    const int sb = (65 - __clzll(q - 1)) / 2;  // ceil(bits(q - 1) / 2)
    const u64 mask = (1ull << sb) - 1;
    // middle sum grows by < 2^(2 sb + 1) per product: fold before 2^64
    const u64 fold_lim = (~0ull) >> (2 * sb + 1);
    const int fold_every = fold_lim > 8191 ? 8191 : (int)fold_lim;
    const u64 one_q = shoup_quotient_dev(1, q);
    const u64 r1 = (1ull << sb) % q, r2 = mul_barrett(r1, r1, Barrett{q, mh, ml});
    const u64 r1q = shoup_quotient_dev(r1, q), r2q = shoup_quotient_dev(r2, q);
    for (int c = 0; c < G; ++c)
        for (int idx = tid; idx < D * kS; idx += blockDim.x) {
            const int j = idx / kS, x = idx % kS;
            u64 y = c < n_ct ? __ldg(Yhat + c * y_stride + (((size_t)j * LK + l) << log_n) + s0 + x) : 0;
            ytile[c * D * kS + idx] = ((y >> sb) << 32) | (y & mask);
        }
    __syncthreads();
    const Barrett bm{q, mh, ml};
    u64 bterm[G];
#pragma unroll
    for (int c = 0; c < G; ++c)
        bterm[c] = (c < n_ct && l < Lq)
                       ? mul_shoup(__ldg(Bhat + c * b_stride + ((size_t)l << log_n) + s), pf[l], pf_q[l], q)
                       : 0;
    const size_t jstride = ((size_t)LK * 2) << log_n;
    for (int g = lane; g < n_keys; g += kLanes) {
        const u64* key = keys[g];
        const u64* kp = key + ((((size_t)l * 2) << log_n) + s);
        SplitAcc ab[G], aa[G];
#pragma unroll
        for (int c = 0; c < G; ++c) ab[c] = aa[c] = SplitAcc{0, 0, 0};
        int since = 0;
        for (int j0 = 0; j0 < D; j0 += kU) {
            u64 kb[kU], ka[kU];
#pragma unroll
            for (int u = 0; u < kU; ++u) {
                if (j0 + u < D) {
                    kb[u] = __ldcs(kp + (j0 + u) * jstride);
                    ka[u] = __ldcs(kp + (j0 + u) * jstride + n);
                }
            }
#pragma unroll
            for (int u = 0; u < kU; ++u) {
                if (j0 + u < D) {
                    const u32 b0 = (u32)(kb[u] & mask), b1 = (u32)(kb[u] >> sb);
                    const u32 a0 = (u32)(ka[u] & mask), a1 = (u32)(ka[u] >> sb);
#pragma unroll
                    for (int c = 0; c < G; ++c) {
                        const u64 y = ytile[(c * D + j0 + u) * kS + si];
                        const u32 y0 = (u32)y, y1 = (u32)(y >> 32);
                        ab[c].mac(y0, y1, b0, b1);
                        aa[c].mac(y0, y1, a0, a1);
                    }
                    if (++since == fold_every) {
#pragma unroll
                        for (int c = 0; c < G; ++c) {
                            ab[c].fold(q, one_q, r1, r1q, r2, r2q);
                            aa[c].fold(q, one_q, r1, r1q, r2, r2q);
                        }
                        since = 0;
                    }
                }
            }
        }
#pragma unroll
        for (int c = 0; c < G; ++c) {
            if (c >= n_ct) break;
            ab[c].fold(q, one_q, r1, r1q, r2, r2q);
            aa[c].fold(q, one_q, r1, r1q, r2, r2q);
            u64 b = add_mod(ab[c].s0, bterm[c], q), a = aa[c].s0;
            const u32 cnt = min(exc_count[(size_t)c * n_keys + g], (u32)cap);
            if (cnt) {
                const Exc* list = exc + ((size_t)c * n_keys + g) * cap;
                const u64 ps = psi[lm(l)];
                const u32 k = galois_src(s, exps_inv[g], log_n);
                for (u32 e = 0; e < cnt; ++e) {
                    const Exc x = list[e];
                    u64 w = pow_mod_dev(ps, ((2ull * k + 1) * x.t) & (2ull * n - 1), bm);
                    u64 dm = x.delta < 0 ? (u64)(-x.delta) % q : (u64)x.delta % q;
                    if (x.delta < 0 && dm) dm = q - dm;
                    u64 v = mul_barrett(w, dm, bm);
                    const size_t kofs = (((size_t)x.j * LK + l) * 2) << log_n;
                    b = add_mod(b, mul_barrett(v, key[kofs + s], bm), q);
                    a = add_mod(a, mul_barrett(v, key[kofs + n + s], bm), q);
                }
            }
            const size_t obase = (((size_t)c * n_keys + g) * 2 * LK) << log_n;
            acc[obase + ((size_t)l << log_n) + s] = b;
            acc[obase + (((size_t)LK + l) << log_n) + s] = a;
        }
    }
}

// CUDA-event phase timer (the analogue of the reference's HybridRotationTiming,
// ckks/hybrid_rns_galois_key.rs:323-336). Phases accumulate over groups.
struct PhaseTimer {
    double* out = nullptr;
    cudaStream_t st = nullptr;
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> spans;
    cudaEvent_t open_ev = nullptr;
    int open_phase = -1;
    void begin(int phase) {
        if (!out) return;
        cudaEventCreate(&open_ev);
        cudaEventRecord(open_ev, st);
        open_phase = phase;
    }
    void end() {
        if (!out || open_phase < 0) return;
        cudaEvent_t e;
        cudaEventCreate(&e);
        cudaEventRecord(e, st);
        spans.push_back({open_phase, {open_ev, e}});
        open_phase = -1;
    }
    void finish() {
        if (!out) return;
        for (auto& sp : spans) {
            float ms = 0;
            cudaEventSynchronize(sp.second.second);
            cudaEventElapsedTime(&ms, sp.second.first, sp.second.second);
            out[sp.first] += ms;
            cudaEventDestroy(sp.second.first);
            cudaEventDestroy(sp.second.second);
        }
        spans.clear();
    }
};

}  // namespace

// Hoisted hybrid rotations of n_ct ciphertexts by n_keys Galois keys (bounded
// or RNS-block gadget), out [n_ct][n_keys][2][Lq][N]. Ciphertexts are
// processed in groups of up to 4 sharing each streamed key slice.
int32_t rotate_hoisted_ntt(ckks_ctx* ctx, const ckks_ksk* const* keys, u32 n_keys, const u64* ct_in,
                                   u64* ct_out, u32 n_ct, cudaStream_t st, double* phase_ms) {
    PhaseTimer pt;
    pt.out = phase_ms;
    pt.st = st;
    const ckks_ksk* k0 = keys[0];
    const u32 Lq = k0->q_limbs, LK = ksk_limbs(k0), D = k0->D, n = ctx->n;
    const size_t ct_words = (size_t)2 * Lq * n;
    const bool bounded = k0->kind == CKKS_KSK_HYBRID_BOUNDED;
    const u32 G = n_ct >= 4 ? 4 : n_ct;
    const int cap = 1024;
    const LimbMap lq = LimbMap::range(0, Lq), lqp = LimbMap::qp(ctx, Lq);
    const size_t y_stride = (size_t)D * LK * n, b_stride = (size_t)Lq * n, d_stride = (size_t)D * n,
                 f_stride = (size_t)n + 1;
    Workspace<u64> Y, Bh, acc, Z, karr;
    Workspace<i64> dig;
    Workspace<u32> flags, cnt;
    Workspace<Exc> exc;
    int32_t rc;
    if ((rc = Y.alloc(G * y_stride, st)) || (rc = Bh.alloc(G * b_stride, st)) ||
        (rc = acc.alloc((size_t)G * n_keys * 2 * LK * n, st)) || (rc = Z.alloc((size_t)G * n_keys * 2 * LK * n, st)) ||
        (rc = karr.alloc(3 * (size_t)n_keys + ctx->moduli.size(), st)) || (rc = dig.alloc(G * d_stride, st)) ||
        (rc = flags.alloc(G * f_stride, st)) || (rc = cnt.alloc((size_t)G * n_keys, st)) ||
        (rc = exc.alloc((size_t)G * n_keys * cap, st)))
        return rc;
    // key pointers, exponents and psi per modulus
    std::vector<u64> hk(3 * (size_t)n_keys + ctx->moduli.size());
    for (u32 g = 0; g < n_keys; ++g) {
        hk[g] = (u64)(uintptr_t)keys[g]->d_entries;
        hk[n_keys + g] = keys[g]->exponent;
        hk[2 * n_keys + ctx->moduli.size() + g] = galois_inverse_host(keys[g]->exponent, n);
    }
    for (size_t i = 0; i < ctx->moduli.size(); ++i) hk[2 * n_keys + i] = ctx->psi[i];
    CKKS_CUDA_TRY(cudaMemcpyAsync(karr.p, hk.data(), hk.size() * 8, cudaMemcpyHostToDevice, st));
    const u64* const* d_keys = (const u64* const*)karr.p;
    const u64* d_exps = karr.p + n_keys;
    const u64* d_psi = karr.p + 2 * n_keys;
    const u64* d_exps_inv = karr.p + 2 * n_keys + ctx->moduli.size();
    std::vector<u32> overflow;
    std::vector<u32> h_cnt((size_t)G * n_keys);
    for (u32 c0 = 0; c0 < n_ct; c0 += G) {
        const u32 gn = (n_ct - c0) < G ? (n_ct - c0) : G;
        CKKS_CUDA_TRY(cudaMemsetAsync(flags.p, 0, G * f_stride * sizeof(u32), st));
        CKKS_CUDA_TRY(cudaMemsetAsync(cnt.p, 0, (size_t)G * n_keys * sizeof(u32), st));
        pt.begin(0);
        for (u32 c = 0; c < gn; ++c) {
            const u64* in = ct_in + (size_t)(c0 + c) * ct_words;
            if (bounded) {
                if ((rc = bounded_decompose_launch(ctx, in + (size_t)Lq * n, 1, Lq, k0->base_log, dig.p + c * d_stride,
                                                   flags.p + c * f_stride, st)))
                    return rc;
                if ((rc = ntt_forward_digits_launch(ctx, dig.p + c * d_stride, Y.p + c * y_stride, D, lqp, LK, st)))
                    return rc;
            } else {  // RNS blocks: ModUp of a, then transform (the permutation is the whole automorphism)
                if ((rc = rnsblock_modup_launch(ctx, k0, in + (size_t)Lq * n, Y.p + c * y_stride, st))) return rc;
                if ((rc = ntt_forward_launch_map(ctx, Y.p + c * y_stride, Y.p + c * y_stride, D, lqp, LK, st))) return rc;
            }
            if ((rc = ntt_forward_launch_map(ctx, in, Bh.p + c * b_stride, 1, lq, Lq, st))) return rc;
        }
        pt.end();
        pt.begin(2);
        if (bounded) {
            dim3 g((n + kT - 1) / kT, n_keys, gn);
            k_hoist_exceptions<<<g, kT, 0, st>>>(dig.p, d_stride, flags.p, f_stride, d_exps, n_keys, D,
                                                 k0->base_log, ctx->log_n, exc.p, cnt.p, cap);
        }
        pt.end();
        pt.begin(3);
        {
            const size_t smem = (size_t)(G >= 3 ? 4 : G) * D * kS * sizeof(u64);
            if (n >= (u32)kS && smem <= 200 * 1024) {
                dim3 g(n / kS, LK);
#define CKKS_MACT(GG)                                                                                              \
    do {                                                                                                           \
        cudaFuncSetAttribute(k_mac_tiled<GG>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);            \
        k_mac_tiled<GG><<<g, kS * kLanes, (size_t)GG * D * kS * sizeof(u64), st>>>(                              \
            Y.p, y_stride, Bh.p, b_stride, d_keys, d_exps_inv, ctx->d_pmodq, ctx->d_pmodq + ctx->L, acc.p,        \
            ctx->d_tabs, lqp, gn, n_keys, Lq, LK, D, ctx->log_n, exc.p, cnt.p, cap, d_psi);                        \
    } while (0)
                if (G >= 3) CKKS_MACT(4);
                else if (G == 2) CKKS_MACT(2);
                else CKKS_MACT(1);
#undef CKKS_MACT
            } else {
                dim3 g((n + kT - 1) / kT, n_keys, LK);
#define CKKS_MAC(GG)                                                                                               \
    k_mac_hoisted<GG><<<g, kT, 0, st>>>(Y.p, y_stride, Bh.p, b_stride, d_keys, d_exps_inv, ctx->d_pmodq,            \
                                        ctx->d_pmodq + ctx->L, acc.p, ctx->d_tabs, lqp, gn, n_keys, Lq, LK, D,      \
                                        ctx->log_n, exc.p, cnt.p, cap, d_psi)
                if (G >= 3) CKKS_MAC(4);
                else if (G == 2) CKKS_MAC(2);
                else CKKS_MAC(1);
#undef CKKS_MAC
            }
        }
        CKKS_CUDA_TRY(cudaGetLastError());
        pt.end();
        pt.begin(4);
        if ((rc = ntt_inverse_launch_map(ctx, acc.p, Z.p, gn * n_keys * 2, lqp, LK, st))) return rc;
        pt.end();
        pt.begin(5);
        // ModDown of every (ciphertext, key) pair, then sigma_g, straight into the output
        if ((rc = mod_down_sigma_multi(ctx, Z.p, ct_out + (size_t)c0 * n_keys * ct_words, gn * n_keys * 2, Lq, d_exps,
                                       n_keys, st)))
            return rc;
        pt.end();
        // pairs whose correction lists overflowed are recomputed exactly
        CKKS_CUDA_TRY(cudaMemcpyAsync(h_cnt.data(), cnt.p, (size_t)G * n_keys * sizeof(u32), cudaMemcpyDeviceToHost, st));
        CKKS_CUDA_TRY(cudaStreamSynchronize(st));
        for (u32 c = 0; c < gn; ++c)
            for (u32 g = 0; g < n_keys; ++g)
                if (h_cnt[(size_t)c * n_keys + g] > (u32)cap) overflow.push_back(((c0 + c) << 16) | g);
    }
    pt.finish();
    for (u32 code : overflow) {
        const u32 c = code >> 16, g = code & 0xffff;
        if ((rc = rotate_hybrid(ctx, keys[g], ct_in + (size_t)c * ct_words,
                                ct_out + ((size_t)c * n_keys + g) * ct_words, 1, st)))
            return rc;
    }
    return CKKS_OK;
}
