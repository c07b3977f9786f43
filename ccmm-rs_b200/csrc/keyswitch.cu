// keyswitch.cu -- hybrid-QP key switching, Galois rotations and key generation.
//
// Rotation (ckks/hybrid_rns_galois_key.rs:550-780), per ciphertext and
// Galois element k:
//   sigma_k on (b, a)                         coefficient-domain automorphism
//   digits of sigma(a)                        bounded gadget (exact CRT) or RNS blocks
//   Y[j][l] = NTT_l(lift(d_j))                one fused lift + forward NTT launch
//   acc_b[l] = (P mod q_l) NTT(sigma b)[l] + sum_j Y[j][l] key_b[j][l]
//   acc_a[l] =                               sum_j Y[j][l] key_a[j][l]
//   INTT, exact ModDown by P                  (ring/auxiliary_modulus.rs:89-171)
// The MAC accumulates exact 128-bit sums of products and reduces once per
// 15 terms, so the result is the canonical residue of the same sum the
// reference forms with pointwise_mul_add_assign (ring/ntt_polynomial.rs:222-236).
#include <algorithm>
#include <cmath>
#include <vector>

#include "keyswitch.cuh"

namespace {

constexpr int kT = 256;

// acc[0][l][k] = (l < Lq ? pf_l * base[l][pb(k)] : 0) + sum_j Y[j][l][py(k)] * key[j][l][0][k]
// acc[1][l][k] =                                         sum_j Y[j][l][py(k)] * key[j][l][1][k]
// py / pb: NTT-domain Galois source maps (k = 0: identity). blockIdx.z batches
// ciphertexts: Y, base and acc advance by y_stride, b_stride, a_stride words.
__global__ void __launch_bounds__(kT) k_ks_mac(const u64* __restrict__ Y, const u64* __restrict__ key,
                                               const u64* __restrict__ base, const u64* __restrict__ pf,
                                               const u64* __restrict__ pf_q, u64* __restrict__ acc,
                                               const NttTab* __restrict__ tabs, LimbMap lm, int Lq, int LK, int D,
                                               int log_n, u64 perm_y, u64 perm_b, u64 perm_key, size_t y_stride,
                                               size_t b_stride, size_t a_stride) {
    const u32 n = 1u << log_n;
    const u32 k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int l = blockIdx.y;
    Y += blockIdx.z * y_stride;
    if (base) base += blockIdx.z * b_stride;
    acc += blockIdx.z * a_stride;
    const NttTab& T = tabs[lm(l)];
    const u64 q = T.q, mu_hi = T.mu_hi, mu_lo = T.mu_lo;
    const u32 ky = perm_y ? galois_src(k, perm_y, log_n) : k;
    const u32 kk = perm_key ? galois_src(k, perm_key, log_n) : k;  // key slot of k in permuted storage
    Acc128 ab{0, 0}, aa{0, 0};
    int since = 0;
    for (int j = 0; j < D; ++j) {
        u64 y = Y[(((size_t)j * LK + l) << log_n) + ky];
        const u64* kp = key + ((((size_t)j * LK + l) * 2) << log_n);
        ab.mac(y, kp[kk]);
        aa.mac(y, kp[n + kk]);
        if (++since == 15) {
            ab.fold(q, mu_hi, mu_lo);
            aa.fold(q, mu_hi, mu_lo);
            since = 0;
        }
    }
    ab.fold(q, mu_hi, mu_lo);
    aa.fold(q, mu_hi, mu_lo);
    u64 b = ab.lo;
    if (base && l < Lq) {  // P b with auxiliary limbs, b without (ordinary RNS key switch)
        const u32 kb = perm_b ? galois_src(k, perm_b, log_n) : k;
        const u64 bv = base[((size_t)l << log_n) + kb];
        b = add_mod(b, pf ? mul_shoup(bv, pf[l], pf_q[l], q) : bv, q);
    }
    acc[((size_t)l << log_n) + k] = b;
    acc[(((size_t)LK + l) << log_n) + k] = aa.lo;
}

// ------------------------------------------------------------- sampling
// Counter-based generator: splitmix64 finaliser over (seed, stream, index).
__host__ __device__ __forceinline__ u64 mix64(u64 z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
__host__ __device__ __forceinline__ u64 rng_word(u64 seed, u64 stream, u64 index) {
    return mix64(mix64(seed ^ mix64(stream + 0x9E3779B97F4A7C15ull)) + index * 0x9E3779B97F4A7C15ull);
}
__device__ __forceinline__ u64 uniform_mod(u64 q, u64 seed, u64 stream, u64 index) {
    unsigned __int128 v = ((unsigned __int128)rng_word(seed, stream, 2 * index) << 64) | rng_word(seed, stream, 2 * index + 1);
    return (u64)(v % q);
}
__device__ __forceinline__ i64 gaussian(const u64* cdt, int len, u64 word) {
    u64 v = word >> 1;
    int k = 0;
    while (k + 1 < len && v >= cdt[k]) ++k;
    return (word & 1) ? -(i64)k : (i64)k;
}

// T[j][l][c] = factor[j][l] * s'[c] + e_j[c] mod m_l (coefficient domain)
// (t_limbs, when non-null, is a per-limb target [LK][N] replacing the ternary s_t)
__global__ void k_keygen_target(u64* __restrict__ T, const int8_t* __restrict__ s_t, const u64* __restrict__ t_limbs,
                                const u64* __restrict__ fac, const u64* __restrict__ fac_q,
                                const NttTab* __restrict__ tabs, LimbMap lm, int LK, int log_n, u64 seed, u64 tag_e,
                                const u64* __restrict__ cdt, int cdt_len, const i64* __restrict__ e_arr) {
    const u32 n = 1u << log_n;
    const u32 c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    const int l = blockIdx.y, j = blockIdx.z;
    const u64 m = tabs[lm(l)].q;
    // e_arr: the caller's sampled errors [D][N] (one logical error polynomial per entry)
    const i64 e = e_arr ? e_arr[((size_t)j << log_n) + c] : gaussian(cdt, cdt_len, rng_word(seed, tag_e | (u64)j, c));
    u64 su;
    if (t_limbs) {
        su = t_limbs[((size_t)l << log_n) + c];
    } else {
        int8_t sv = s_t[c];
        su = sv < 0 ? m - 1 : (u64)sv;
    }
    u64 t = mul_shoup(su, fac[(size_t)j * LK + l], fac_q[(size_t)j * LK + l], m);
    const u64 mag = e < 0 ? 0 - (u64)e : (u64)e;  // signed_mod (hybrid_rns_galois_key.rs:55-57)
    u64 eu = mag >= m ? mag % m : mag;
    eu = (e < 0 && eu) ? m - eu : eu;
    T[(((size_t)j * LK + l) << log_n) + c] = add_mod(t, eu, m);
}

// entries[j][l][0] = That - a * s_hat, entries[j][l][1] = a (a uniform, sampled in the NTT domain)
__global__ void k_keygen_finish(const u64* __restrict__ That, const u64* __restrict__ s_hat, u64* __restrict__ entries,
                                const NttTab* __restrict__ tabs, LimbMap lm, int LK, int log_n, u64 seed, u64 tag_a,
                                int comp_major, u64 perm, const u64* __restrict__ a_arr) {
    const u32 n = 1u << log_n;
    const u32 c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    const int l = blockIdx.y, j = blockIdx.z;
    const NttTab& T = tabs[lm(l)];
    Barrett bm{T.q, T.mu_hi, T.mu_lo};
    // a_arr: NTT of the caller's sampled uniform a [D][LK][N]
    const u64 a = a_arr ? a_arr[(((size_t)j * LK + l) << log_n) + c]
                        : uniform_mod(T.q, seed, tag_a | ((u64)j << 16) | (u64)l, c);
    u64 b = sub_mod(That[(((size_t)j * LK + l) << log_n) + c], mul_barrett(a, s_hat[((size_t)l << log_n) + c], bm), T.q);
    if (comp_major) {  // [j][2][LK][N] (relinearization key layout)
        entries[((((size_t)j * 2 + 0) * LK + l) << log_n) + c] = b;
        entries[((((size_t)j * 2 + 1) * LK + l) << log_n) + c] = a;
    } else {  // [j][LK][2][N] (Galois key layout), stored at the permuted slot
        const u32 sl = perm ? galois_src(c, perm, log_n) : c;
        entries[((((size_t)j * LK + l) * 2 + 0) << log_n) + sl] = b;
        entries[((((size_t)j * LK + l) * 2 + 1) << log_n) + sl] = a;
    }
}

// secret lifted to every limb (coefficient domain)
__global__ void k_lift_ternary(const int8_t* __restrict__ s, u64* __restrict__ out, const NttTab* __restrict__ tabs,
                               LimbMap lm, int log_n) {
    const u32 n = 1u << log_n;
    const u32 c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    const int l = blockIdx.y;
    const u64 m = tabs[lm(l)].q;
    int8_t v = s[c];
    out[((size_t)l << log_n) + c] = v < 0 ? m - 1 : (u64)v;
}

typedef unsigned __int128 u128;
u64 h_mulmod(u64 a, u64 b, u64 q) { return (u64)((u128)a * b % q); }

std::vector<u64> cdt_table(double sigma) {
    int T = (int)std::ceil(12.0 * sigma);
    std::vector<double> rho(T + 1);
    double S = 0;
    for (int k = 0; k <= T; ++k) {
        rho[k] = std::exp(-(double)k * k / (2.0 * sigma * sigma));
        S += k ? 2.0 * rho[k] : rho[k];
    }
    std::vector<u64> cdt(T + 1);
    double c = 0;
    for (int k = 0; k <= T; ++k) {
        c += (k ? 2.0 * rho[k] : rho[k]) / S;
        double v = std::ldexp(c, 63);
        cdt[k] = v >= 9223372036854775807.0 ? (1ull << 63) : (u64)v;
    }
    cdt[T] = 1ull << 63;
    return cdt;
}

// ternary secret automorphism (hybrid_rns_galois_key.rs:29-53)
std::vector<int8_t> secret_automorphism(const int8_t* s, u32 n, u64 k) {
    std::vector<int8_t> o(n, 0);
    for (u32 i = 0; i < n; ++i) {
        u64 mapped = ((u64)i * k) % (2ull * n);
        if (mapped < n) o[mapped] = s[i];
        else o[mapped - n] = (int8_t)-s[i];
    }
    return o;
}

}  // namespace

// ---------------------------------------------------------------- keys
u32 ksk_limbs(const ckks_ksk* k) { return k->with_p ? k->q_limbs + k->ctx->K : k->q_limbs; }

int32_t ksk_generate(ckks_ctx* ctx, ckks_ksk* key, const int8_t* secret, u64 seed, double sigma,
                     const std::vector<u64>& factors /*[D][LK] host*/, const std::vector<int8_t>& s_target,
                     bool comp_major, u64 tag_a, u64 tag_e, cudaStream_t st, const u64* d_target_limbs,
                     const KeySamples& smp) {
    const u32 LK = ksk_limbs(key), D = key->D, n = ctx->n;
    const LimbMap lm = key->with_p ? LimbMap::qp(ctx, key->q_limbs) : LimbMap::range(0, key->q_limbs);
    std::vector<u64> fq(factors.size());
    for (size_t i = 0; i < factors.size(); ++i) fq[i] = shoup_quotient_host(factors[i], ctx->moduli[lm((int)(i % LK))]);
    auto cdt = cdt_table(sigma);
    Workspace<u64> d_fac, d_cdt, d_T, d_That, d_s;
    Workspace<int8_t> d_st, d_sec;
    int32_t rc;
    if ((rc = d_fac.alloc(2 * factors.size(), st)) || (rc = d_cdt.alloc(cdt.size(), st)) ||
        (rc = d_T.alloc((size_t)D * LK * n, st)) || (rc = d_That.alloc((size_t)D * LK * n, st)) ||
        (rc = d_s.alloc((size_t)2 * LK * n, st)) || (rc = d_st.alloc(n, st)) || (rc = d_sec.alloc(n, st)))
        return rc;
    std::vector<u64> fac2(factors);
    fac2.insert(fac2.end(), fq.begin(), fq.end());
    CKKS_CUDA_TRY(cudaMemcpyAsync(d_fac.p, fac2.data(), fac2.size() * 8, cudaMemcpyHostToDevice, st));
    CKKS_CUDA_TRY(cudaMemcpyAsync(d_cdt.p, cdt.data(), cdt.size() * 8, cudaMemcpyHostToDevice, st));
    if (!d_target_limbs) CKKS_CUDA_TRY(cudaMemcpyAsync(d_st.p, s_target.data(), n, cudaMemcpyHostToDevice, st));
    CKKS_CUDA_TRY(cudaMemcpyAsync(d_sec.p, secret, n, cudaMemcpyHostToDevice, st));
    Workspace<i64> d_e;
    Workspace<u64> d_a;
    if (smp.e) {
        if ((rc = d_e.alloc((size_t)D * n, st))) return rc;
        CKKS_CUDA_TRY(cudaMemcpyAsync(d_e.p, smp.e, (size_t)D * n * 8, cudaMemcpyHostToDevice, st));
    }
    if (smp.a) {  // a_ntt = NTT(a) (grafting/rns_key_switch.rs:844-850)
        if ((rc = d_a.alloc((size_t)D * LK * n, st))) return rc;
        CKKS_CUDA_TRY(cudaMemcpyAsync(d_a.p, smp.a, (size_t)D * LK * n * 8, cudaMemcpyHostToDevice, st));
        if ((rc = ntt_forward_launch_map(ctx, d_a.p, d_a.p, D, lm, LK, st))) return rc;
    }
    dim3 g((n + kT - 1) / kT, LK, D);
    k_keygen_target<<<g, kT, 0, st>>>(d_T.p, d_st.p, d_target_limbs, d_fac.p, d_fac.p + factors.size(), ctx->d_tabs, lm, LK,
                                      ctx->log_n, seed, tag_e, d_cdt.p, (int)cdt.size(), d_e.p);
    if ((rc = ntt_forward_launch_map(ctx, d_T.p, d_That.p, D, lm, LK, st))) return rc;
    dim3 gs((n + kT - 1) / kT, LK, 1);
    k_lift_ternary<<<gs, kT, 0, st>>>(d_sec.p, d_s.p, ctx->d_tabs, lm, ctx->log_n);
    if ((rc = ntt_forward_launch_map(ctx, d_s.p, d_s.p + (size_t)LK * n, 1, lm, LK, st))) return rc;
    k_keygen_finish<<<g, kT, 0, st>>>(d_That.p, d_s.p + (size_t)LK * n, key->d_entries, ctx->d_tabs, lm, LK,
                                      ctx->log_n, seed, tag_a, comp_major ? 1 : 0, comp_major ? 0 : key->exponent,
                                      d_a.p);
    CKKS_CUDA_TRY(cudaGetLastError());
    return CKKS_OK;
}

int32_t ksk_alloc(ckks_ctx* ctx, ckks_ksk* key) {
    size_t words = (size_t)key->D * ksk_limbs(key) * 2 * ctx->n;
    if (cudaMalloc(&key->d_entries, words * sizeof(u64)) != cudaSuccess) {
        cudaGetLastError();
        key->d_entries = nullptr;
        ckks_set_error("out of device memory for key-switching key");
        return CKKS_ERR_OOM;
    }
    key->words = words;
    return CKKS_OK;
}

// Hybrid-QP bounded key factors: (P mod m) * (B^j mod m) (hybrid_rns_galois_key.rs:94-160)
std::vector<u64> hybrid_factors(ckks_ctx* ctx, const ckks_ksk* key) {
    const u32 LK = ksk_limbs(key);
    const LimbMap lm = LimbMap::qp(ctx, key->q_limbs);
    std::vector<u64> f((size_t)key->D * LK);
    for (u32 l = 0; l < LK; ++l) {
        u64 m = ctx->moduli[lm((int)l)], pf = 1 % m, g = 1 % m;
        for (u32 k = 0; k < ctx->K; ++k) pf = h_mulmod(pf, ctx->moduli[ctx->L + k] % m, m);
        u64 b = (u64)(((u128)1 << key->base_log) % m);
        for (u32 j = 0; j < key->D; ++j) {
            f[(size_t)j * LK + l] = h_mulmod(pf, g, m);
            g = h_mulmod(g, b, m);
        }
    }
    return f;
}

// RNS-block factors: (P mod m) on the limbs of block i, 0 elsewhere (E_i mod q_j, rns_gadget.rs:92-135)
std::vector<u64> rnsblock_factors(ckks_ctx* ctx, const ckks_ksk* key) {
    const u32 LK = ksk_limbs(key);
    std::vector<u64> f((size_t)key->D * LK, 0);
    u32 start = 0;
    for (u32 i = 0; i < key->D; ++i) {
        for (u32 l = start; l < start + key->blocks[i]; ++l) {
            u64 m = ctx->moduli[l], pf = 1 % m;
            for (u32 k = 0; k < ctx->K; ++k) pf = h_mulmod(pf, ctx->moduli[ctx->L + k] % m, m);
            f[(size_t)i * LK + l] = pf;
        }
        start += key->blocks[i];
    }
    return f;
}

// Block factors without P: E_i mod q_l = [l in block i] (rns_gadget.rs:77-135,
// crt_idempotent_residue / crt_idempotent reduced per limb).
std::vector<u64> rns_factors(ckks_ctx* ctx, const ckks_ksk* key) {
    const u32 LK = ksk_limbs(key);
    std::vector<u64> f((size_t)key->D * LK, 0);
    u32 start = 0;
    for (u32 i = 0; i < key->D; ++i) {
        for (u32 l = start; l < start + key->blocks[i]; ++l) f[(size_t)i * LK + l] = 1;
        start += key->blocks[i];
    }
    return f;
}

// Relinearization factors B^j mod q (bounded_key_switch.rs:63-79), target s^2.
std::vector<u64> relin_factors(ckks_ctx* ctx, const ckks_ksk* key) {
    const u32 L = key->q_limbs;
    std::vector<u64> f((size_t)key->D * L);
    for (u32 l = 0; l < L; ++l) {
        u64 m = ctx->moduli[l], g = 1 % m, b = (u64)(((u128)1 << key->base_log) % m);
        for (u32 j = 0; j < key->D; ++j) {
            f[(size_t)j * L + l] = g;
            g = h_mulmod(g, b, m);
        }
    }
    return f;
}

// Bounded relinearization key: entry j encrypts B^j * s^2 over Q
// (bounded_key_switch.rs:28-104); s^2 formed in the NTT domain.
int32_t relin_generate(ckks_ctx* ctx, ckks_ksk* key, const int8_t* secret, u64 seed, double sigma, cudaStream_t st,
                       const KeySamples& smp) {
    const u32 L = key->q_limbs, n = ctx->n;
    const LimbMap lm = LimbMap::range(0, L);
    Workspace<u64> S;
    Workspace<int8_t> sec;
    int32_t rc;
    if ((rc = S.alloc((size_t)2 * L * n, st)) || (rc = sec.alloc(n, st))) return rc;
    CKKS_CUDA_TRY(cudaMemcpyAsync(sec.p, secret, n, cudaMemcpyHostToDevice, st));
    dim3 gs((n + kT - 1) / kT, L, 1);
    k_lift_ternary<<<gs, kT, 0, st>>>(sec.p, S.p, ctx->d_tabs, lm, ctx->log_n);
    u64* S2 = S.p + (size_t)L * n;
    if ((rc = ntt_forward_launch_map(ctx, S.p, S2, 1, lm, L, st))) return rc;
    if ((rc = pointwise_launch(ctx, S2, S2, S2, 1, lm, L, 0, st))) return rc;
    if ((rc = ntt_inverse_launch_map(ctx, S2, S.p, 1, lm, L, st))) return rc;
    std::vector<int8_t> none;
    return ksk_generate(ctx, key, secret, seed, sigma,
                        key->kind == CKKS_KSK_RELIN_RNS_BLOCK ? rns_factors(ctx, key) : relin_factors(ctx, key), none,
                        true, TAG_RLK_A, TAG_RLK_E, st, S.p, smp);
}

std::vector<int8_t> host_secret_automorphism(const int8_t* s, u32 n, u64 k) { return secret_automorphism(s, n, k); }

// --------------------------------------------------------------- pipelines
int32_t ks_mac_launch(ckks_ctx* ctx, const u64* Y, const u64* key, const u64* base, u64* acc, u32 q_limbs, u32 D,
                      bool with_p, u64 perm_y, u64 perm_b, cudaStream_t st, u64 perm_key, u32 n_ct, size_t b_stride) {
    const u32 LK = with_p ? q_limbs + ctx->K : q_limbs;
    const LimbMap lm = with_p ? LimbMap::qp(ctx, q_limbs) : LimbMap::range(0, q_limbs);
    if (n_ct > 65535) {
        ckks_set_error("key-switch MAC: more than 65535 ciphertexts in one launch");
        return CKKS_ERR_BAD_ARG;
    }
    dim3 g((ctx->n + kT - 1) / kT, LK, n_ct);
    k_ks_mac<<<g, kT, 0, st>>>(Y, key, base, with_p ? ctx->d_pmodq : nullptr, with_p ? ctx->d_pmodq + ctx->L : nullptr,
                               acc, ctx->d_tabs, lm, q_limbs, LK,
                               D, ctx->log_n, perm_y, perm_b, perm_key, ((size_t)D * LK) << ctx->log_n, b_stride,
                               ((size_t)2 * LK) << ctx->log_n);
    CKKS_CUDA_TRY(cudaGetLastError());
    return CKKS_OK;
}

// Non-hoisted bounded rotation in the reference's order (sigma on (b, a),
// decompose sigma(a), transform every digit): the exact fallback of the hoisted
// path. The permuted key storage is read through the permutation.
int32_t rotate_hybrid(ckks_ctx* ctx, const ckks_ksk* key, const u64* ct_in, u64* ct_out, u32 n_ct, cudaStream_t st) {
    if (key->kind == CKKS_KSK_RNS_BLOCK)
        return rotate_rns(ctx, key, ct_in, ct_out, n_ct, (size_t)2 * key->q_limbs * ctx->n, st);
    if (key->kind != CKKS_KSK_HYBRID_BOUNDED) {
        const ckks_ksk* keys[1] = {key};
        for (u32 i = 0; i < n_ct; ++i) {
            const size_t ct_words = (size_t)2 * key->q_limbs * ctx->n;
            if (int32_t rc = rotate_hoisted_ntt(ctx, keys, 1, ct_in + i * ct_words, ct_out + i * ct_words, 1, st))
                return rc;
        }
        return CKKS_OK;
    }
    const u32 Lq = key->q_limbs, LK = ksk_limbs(key), D = key->D, n = ctx->n;
    const size_t ct_words = (size_t)2 * Lq * n;
    // ciphertexts are batched through every launch, as many per batch as a few GB allow
    const size_t per_ct = ct_words * 2 + (size_t)D * LK * n + 4 * (size_t)LK * n + (size_t)D * n;  // words
    const u32 m_max = (u32)std::max<size_t>(1, std::min<size_t>({(size_t)n_ct, (size_t)65535,
                                                                   ((size_t)4 << 30) / (per_ct * 8)}));
    Workspace<u64> ws;
    Workspace<i64> dg;
    int32_t rc;
    if ((rc = ws.alloc((size_t)m_max * (per_ct - (size_t)D * n), st)) || (rc = dg.alloc((size_t)m_max * D * n, st)))
        return rc;
    u64* sct = ws.p;                               // sigma(ct) [m][2][Lq][N]
    u64* s_hat = sct + (size_t)m_max * ct_words;   // NTT(sigma(ct)) [m][2][Lq][N]; the b parts are the base
    u64* Y = s_hat + (size_t)m_max * ct_words;     // [m][D][LK][N]
    u64* acc = Y + (size_t)m_max * D * LK * n;     // [m][2][LK][N]
    u64* Z = acc + (size_t)m_max * 2 * LK * n;     // [m][2][LK][N]
    const LimbMap lq = LimbMap::range(0, Lq), lqp = LimbMap::qp(ctx, Lq);
    for (u32 c0 = 0; c0 < n_ct; c0 += m_max) {
        const u32 m = n_ct - c0 < m_max ? n_ct - c0 : m_max;
        const u64* in = ct_in + (size_t)c0 * ct_words;
        u64* out = ct_out + (size_t)c0 * ct_words;
        if ((rc = automorphism_coef_launch(ctx, in, sct, 2 * m, lq, Lq, key->exponent, st))) return rc;
        if ((rc = bounded_decompose_launch(ctx, sct + (size_t)Lq * n, m, Lq, key->base_log, dg.p, nullptr, st,
                                           ct_words)))
            return rc;
        if ((rc = ntt_forward_digits_launch(ctx, dg.p, Y, D * m, lqp, LK, st))) return rc;
        if ((rc = ntt_forward_launch_map(ctx, sct, s_hat, 2 * m, lq, Lq, st))) return rc;
        if ((rc = ks_mac_launch(ctx, Y, key->d_entries, s_hat, acc, Lq, D, true, 0, 0, st, key->exponent, m,
                                ct_words)))
            return rc;
        if ((rc = ntt_inverse_launch_map(ctx, acc, Z, 2 * m, lqp, LK, st))) return rc;
        if ((rc = mod_down_launch(ctx, Z, out, 2 * m, Lq, st))) return rc;
    }
    return CKKS_OK;
}

int32_t rotate_hybrid_hoisted(ckks_ctx* ctx, const ckks_ksk* const* keys, u32 n_keys, const u64* ct_in, u64* ct_out,
                              u32 n_ct, cudaStream_t st) {
    if (keys[0]->kind == CKKS_KSK_RNS_BLOCK) {
        // the reference decomposes sigma(a) for every Galois element
        // (rns_galois_key.rs:439-469): one full key switch per key, outputs
        // interleaved as [n_ct][n_keys][2][Lq][N]
        const size_t ct_words = (size_t)2 * keys[0]->q_limbs * ctx->n;
        for (u32 g = 0; g < n_keys; ++g)
            if (int32_t rc = rotate_rns(ctx, keys[g], ct_in, ct_out + g * ct_words, n_ct, n_keys * ct_words, st))
                return rc;
        return CKKS_OK;
    }
    return rotate_hoisted_ntt(ctx, keys, n_keys, ct_in, ct_out, n_ct, st);
}

int32_t rotate_rns(ckks_ctx* ctx, const ckks_ksk* key, const u64* ct_in, u64* ct_out, u32 n_ct, size_t out_stride,
                   cudaStream_t st) {
    const u32 Lq = key->q_limbs, D = key->D, n = ctx->n;
    const size_t ct_words = (size_t)2 * Lq * n, y_words = (size_t)D * Lq * n;
    const size_t per_ct = 3 * ct_words + y_words;  // sigma(ct), NTT(sigma(ct)), accumulators, digits
    const u32 m_max = (u32)std::max<size_t>(1, std::min<size_t>({(size_t)n_ct, (size_t)(65535 / (D > 2 ? D : 2)),
                                                                   ((size_t)4 << 30) / (per_ct * 8)}));
    Workspace<u64> ws;
    int32_t rc;
    if ((rc = ws.alloc((size_t)m_max * per_ct, st))) return rc;
    u64* sct = ws.p;                              // [m][2][Lq][N]
    u64* s_hat = sct + (size_t)m_max * ct_words;  // [m][2][Lq][N]
    u64* acc = s_hat + (size_t)m_max * ct_words;  // [m][2][Lq][N]
    u64* Y = acc + (size_t)m_max * ct_words;      // [m][D][Lq][N]
    const LimbMap lq = LimbMap::range(0, Lq);
    for (u32 c0 = 0; c0 < n_ct; c0 += m_max) {
        const u32 m = n_ct - c0 < m_max ? n_ct - c0 : m_max;
        // sigma_k on (b, a) in the coefficient domain (apply_rns_automorphism)
        if ((rc = automorphism_coef_launch(ctx, ct_in + (size_t)c0 * ct_words, sct, 2 * m, lq, Lq, key->exponent, st)))
            return rc;
        // block digits of sigma(a) (RnsGadgetLayout::decompose), lifted to every Q limb
        for (u32 c = 0; c < m; ++c)
            if ((rc = rnsblock_modup_launch(ctx, key, sct + c * ct_words + (size_t)Lq * n, Y + c * y_words, st)))
                return rc;
        if ((rc = ntt_forward_launch_map(ctx, Y, Y, D * m, lq, Lq, st))) return rc;
        if ((rc = ntt_forward_launch_map(ctx, sct, s_hat, 2 * m, lq, Lq, st))) return rc;
        // b' = NTT(sigma(b)) + sum_i NTT(d_i) k_b[i], a' = sum_i NTT(d_i) k_a[i]
        if ((rc = ks_mac_launch(ctx, Y, key->d_entries, s_hat, acc, Lq, D, false, 0, 0, st, key->exponent, m, ct_words)))
            return rc;
        if (out_stride == ct_words) {
            if ((rc = ntt_inverse_launch_map(ctx, acc, ct_out + (size_t)c0 * ct_words, 2 * m, lq, Lq, st))) return rc;
        } else {
            for (u32 c = 0; c < m; ++c)  // inverse transform into each (interleaved) output slot
                if ((rc = ntt_inverse_launch_map(ctx, acc + c * ct_words, ct_out + (size_t)(c0 + c) * out_stride, 2, lq,
                                                 Lq, st)))
                    return rc;
        }
    }
    return CKKS_OK;
}

// Galois key entries [polys][N] (each poly one (digit, limb, component)):
// storage[pi_g(k)] = reference[k] (to_storage) or the inverse.
namespace {
__global__ void k_permute_entries(const u64* __restrict__ src, u64* __restrict__ dst, int log_n, u64 g, int to_storage) {
    const u32 n = 1u << log_n;
    const u32 k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const size_t base = (size_t)blockIdx.y << log_n;
    const u32 s = galois_src(k, g, log_n);
    if (to_storage) dst[base + s] = src[base + k];
    else dst[base + k] = src[base + s];
}
}  // namespace

int32_t ksk_permute_entries(ckks_ctx* ctx, const u64* src, u64* dst, size_t polys, u64 exponent, bool to_storage,
                            cudaStream_t st) {
    for (size_t p0 = 0; p0 < polys; p0 += 65535) {
        const u32 cnt = (u32)((polys - p0) < 65535 ? (polys - p0) : 65535);
        dim3 g((ctx->n + kT - 1) / kT, cnt);
        k_permute_entries<<<g, kT, 0, st>>>(src + (p0 << ctx->log_n), dst + (p0 << ctx->log_n), ctx->log_n, exponent,
                                            to_storage ? 1 : 0);
    }
    CKKS_CUDA_TRY(cudaGetLastError());
    return CKKS_OK;
}
