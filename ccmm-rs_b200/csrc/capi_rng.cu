// capi_rng.cu -- C ABI of the seeded ChaCha20 stream (rng.cu) and of the key
// generation and encryption that consume it in the reference's order.
//
// Sampling is sequential and runs on the host; every product, transform and
// sum of the keys and ciphertexts runs on the GPU (keyswitch.cu kernels).
#include <cstring>
#include <new>
#include <vector>

#include "keyswitch.cuh"
#include "rng.cuh"

namespace {

// signed_mod of a ternary secret into every limb of lm (coefficient domain)
__global__ void k_lift_secret(const int8_t* __restrict__ s, u64* __restrict__ out, const NttTab* __restrict__ tabs,
                              LimbMap lm, int log_n) {
    const u32 n = 1u << log_n;
    const u32 c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    const int l = blockIdx.y;
    const u64 m = tabs[lm(l)].q;
    const int8_t v = s[c];
    out[((size_t)l << log_n) + c] = v < 0 ? m - 1 : (u64)v;
}

// b = m + e - a s (grafting/rns_key_switch.rs:364-366), e projected by rem_euclid
__global__ void k_encrypt_finish(const u64* __restrict__ msg, const i64* __restrict__ e, const u64* __restrict__ as,
                                 u64* __restrict__ b, const NttTab* __restrict__ tabs, LimbMap lm, int log_n) {
    const u32 n = 1u << log_n;
    const u32 c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    const int l = blockIdx.y;
    const u64 q = tabs[lm(l)].q;
    const size_t i = ((size_t)l << log_n) + c;
    const i64 ev = e[c];
    const u64 mag = ev < 0 ? 0 - (u64)ev : (u64)ev;
    u64 eu = mag >= q ? mag % q : mag;
    eu = (ev < 0 && eu) ? q - eu : eu;
    b[i] = sub_mod(add_mod(msg[i], eu, q), as[i], q);
}

int32_t check_rng(ckks_rng* rng, const char* who) {
    if (!rng) {
        ckks_set_error(std::string(who) + ": null rng");
        return CKKS_ERR_BAD_ARG;
    }
    return CKKS_OK;
}

int32_t check_secret(const int8_t* s, u32 n, const char* who) {
    if (!s) {
        ckks_set_error(std::string(who) + ": null secret");
        return CKKS_ERR_BAD_ARG;
    }
    bool any = false;
    for (u32 i = 0; i < n; ++i) {
        if (s[i] < -1 || s[i] > 1) {
            ckks_set_error(std::string(who) + ": secret must be ternary");
            return CKKS_ERR_BAD_ARG;
        }
        any = any || s[i] != 0;
    }
    if (!any) {
        ckks_set_error(std::string(who) + ": secret must be nonzero");
        return CKKS_ERR_BAD_ARG;
    }
    return CKKS_OK;
}

int32_t check_dist(int32_t kind, double param, const char* who) {
    if (kind == CKKS_DIST_GAUSSIAN && param > 0 && param < 1e6) return CKKS_OK;
    if (kind == CKKS_DIST_BOUNDED_UNIFORM && param >= 0 && param < 9.2e18 && (double)(i64)param == param)
        return CKKS_OK;
    ckks_set_error(std::string(who) + ": error distribution must be bounded-uniform (integer bound >= 0) or "
                                      "discrete Gaussian (sigma > 0)");
    return CKKS_ERR_BAD_ARG;
}

// Draws of one key in the reference's order: per entry j, one logical error
// polynomial (sample_error_coefficients), then one uniform polynomial per limb
// of lm in basis order (sample_uniform_residues): hybrid_rns_galois_key.rs:124-144
// with rns_key_switch.rs:818-850, and bounded_key_switch.rs:64-96 with
// rns_key_switch.rs:278-350.
void sample_key(ckks_rng* rng, ckks_ctx* ctx, LimbMap lm, u32 LK, u32 D, int32_t kind, double param,
                std::vector<i64>& e, std::vector<u64>& a) {
    const u32 n = ctx->n;
    e.resize((size_t)D * n);
    a.resize((size_t)D * LK * n);
    for (u32 j = 0; j < D; ++j) {
        rng->error(n, kind, param, e.data() + (size_t)j * n);
        for (u32 l = 0; l < LK; ++l) rng->uniform(n, ctx->moduli[lm((int)l)], a.data() + ((size_t)j * LK + l) * n);
    }
}

int32_t finish_sync(int32_t rc, const char* who) {
    if (rc == CKKS_OK) {
        cudaError_t e = cudaDeviceSynchronize();
        if (e != cudaSuccess) {
            ckks_set_error(std::string(who) + ": " + cudaGetErrorString(e));
            return CKKS_ERR_CUDA;
        }
    }
    return rc;
}

}  // namespace

extern "C" {

int32_t ckks_rng_create(uint64_t seed, ckks_rng** out) {
    CKKS_CHECK_ARG(out != nullptr, "ckks_rng_create: out is null");
    auto* r = new (std::nothrow) ckks_rng();
    if (!r) {
        ckks_set_error("ckks_rng_create: out of host memory");
        return CKKS_ERR_OOM;
    }
    r->seed_u64(seed);
    *out = r;
    return CKKS_OK;
}

int32_t ckks_rng_create_from_seed(const uint8_t* seed, ckks_rng** out) {
    CKKS_CHECK_ARG(out != nullptr && seed != nullptr, "ckks_rng_create_from_seed: null argument");
    auto* r = new (std::nothrow) ckks_rng();
    if (!r) {
        ckks_set_error("ckks_rng_create_from_seed: out of host memory");
        return CKKS_ERR_OOM;
    }
    r->seed_bytes(seed);
    *out = r;
    return CKKS_OK;
}

int32_t ckks_rng_destroy(ckks_rng* rng) {
    delete rng;
    return CKKS_OK;
}

int32_t ckks_rng_next_u32(ckks_rng* rng, uint32_t* out) {
    if (int32_t rc = check_rng(rng, "ckks_rng_next_u32")) return rc;
    CKKS_CHECK_ARG(out != nullptr, "ckks_rng_next_u32: out is null");
    *out = rng->next_u32();
    return CKKS_OK;
}

int32_t ckks_rng_next_u64(ckks_rng* rng, uint64_t* out) {
    if (int32_t rc = check_rng(rng, "ckks_rng_next_u64")) return rc;
    CKKS_CHECK_ARG(out != nullptr, "ckks_rng_next_u64: out is null");
    *out = rng->next_u64();
    return CKKS_OK;
}

int32_t ckks_rng_fill_u32(ckks_rng* rng, uint32_t* out, uint64_t n) {
    if (int32_t rc = check_rng(rng, "ckks_rng_fill_u32")) return rc;
    CKKS_CHECK_ARG(out != nullptr || n == 0, "ckks_rng_fill_u32: out is null");
    rng->fill_u32(out, (size_t)n);
    return CKKS_OK;
}

int32_t ckks_rng_word_position(const ckks_rng* rng, uint64_t* out) {
    CKKS_CHECK_ARG(rng != nullptr && out != nullptr, "ckks_rng_word_position: null argument");
    *out = rng->pos;
    return CKKS_OK;
}

int32_t ckks_rng_ternary_secret(ckks_rng* rng, uint32_t n, int8_t* out) {
    if (int32_t rc = check_rng(rng, "ckks_rng_ternary_secret")) return rc;
    CKKS_CHECK_ARG(out != nullptr && n > 0, "ckks_rng_ternary_secret: empty secret");
    rng->ternary(n, out);
    return CKKS_OK;
}

int32_t ckks_rng_error(ckks_rng* rng, uint32_t n, int32_t kind, double param, int64_t* out) {
    if (int32_t rc = check_rng(rng, "ckks_rng_error")) return rc;
    if (int32_t rc = check_dist(kind, param, "ckks_rng_error")) return rc;
    CKKS_CHECK_ARG(out != nullptr || n == 0, "ckks_rng_error: out is null");
    return rng->error(n, kind, param, out);
}

int32_t ckks_rng_uniform_residues(ckks_rng* rng, uint32_t n, uint64_t modulus, uint64_t* out) {
    if (int32_t rc = check_rng(rng, "ckks_rng_uniform_residues")) return rc;
    CKKS_CHECK_ARG(modulus >= 2, "ckks_rng_uniform_residues: modulus must be at least 2");
    CKKS_CHECK_ARG(out != nullptr || n == 0, "ckks_rng_uniform_residues: out is null");
    rng->uniform(n, modulus, out);
    return CKKS_OK;
}

int32_t ckks_hybrid_key_generate_rng(ckks_ctx* ctx, uint32_t q_limbs, uint32_t base_log, uint64_t exponent,
                                     const int8_t* secret_host, int32_t dist_kind, double dist_param, ckks_rng* rng,
                                     ckks_ksk** out) {
    const char* who = "ckks_hybrid_key_generate_rng";
    CKKS_CHECK_ARG(out != nullptr, std::string(who) + ": out is null");
    *out = nullptr;
    if (int32_t rc = ckks_require_device(ctx, who)) return rc;
    if (int32_t rc = check_rng(rng, who)) return rc;
    if (int32_t rc = check_secret(secret_host, ctx->n, who)) return rc;
    if (int32_t rc = check_dist(dist_kind, dist_param, who)) return rc;
    CKKS_CHECK_ARG((exponent & 1) == 1, std::string(who) + ": Galois exponent must be odd modulo 2N");
    ckks_ksk* k = nullptr;
    if (int32_t rc = ksk_new(ctx, CKKS_KSK_HYBRID_BOUNDED, q_limbs, base_log, exponent, &k, who)) return rc;
    const u32 LK = ksk_limbs(k);
    std::vector<i64> e;
    std::vector<u64> a;
    sample_key(rng, ctx, LimbMap::qp(ctx, q_limbs), LK, k->D, dist_kind, dist_param, e, a);
    KeySamples smp;
    smp.e = e.data();
    smp.a = a.data();
    auto st_secret = host_secret_automorphism(secret_host, ctx->n, k->exponent);
    int32_t rc = ksk_generate(ctx, k, secret_host, 0, 1.0, hybrid_factors(ctx, k), st_secret, false, TAG_KEY_A,
                              TAG_KEY_E, nullptr, nullptr, smp);
    rc = finish_sync(rc, who);
    if (rc != CKKS_OK) {
        ckks_ksk_destroy(k);
        return rc;
    }
    *out = k;
    return CKKS_OK;
}

int32_t ckks_relin_key_generate_rng(ckks_ctx* ctx, uint32_t q_limbs, uint32_t base_log, const int8_t* secret_host,
                                    int32_t dist_kind, double dist_param, ckks_rng* rng, ckks_ksk** out) {
    const char* who = "ckks_relin_key_generate_rng";
    CKKS_CHECK_ARG(out != nullptr, std::string(who) + ": out is null");
    *out = nullptr;
    if (int32_t rc = ckks_require_device(ctx, who)) return rc;
    if (int32_t rc = check_rng(rng, who)) return rc;
    if (int32_t rc = check_secret(secret_host, ctx->n, who)) return rc;
    if (int32_t rc = check_dist(dist_kind, dist_param, who)) return rc;
    ckks_ksk* k = nullptr;
    if (int32_t rc = ksk_new(ctx, CKKS_KSK_RELIN_BOUNDED, q_limbs, base_log, 1, &k, who)) return rc;
    std::vector<i64> e;
    std::vector<u64> a;
    sample_key(rng, ctx, LimbMap::range(0, q_limbs), q_limbs, k->D, dist_kind, dist_param, e, a);
    KeySamples smp;
    smp.e = e.data();
    smp.a = a.data();
    int32_t rc = finish_sync(relin_generate(ctx, k, secret_host, 0, 1.0, nullptr, smp), who);
    if (rc != CKKS_OK) {
        ckks_ksk_destroy(k);
        return rc;
    }
    *out = k;
    return CKKS_OK;
}

int32_t ckks_encrypt_rng_host(ckks_ctx* ctx, uint32_t q_limbs, const uint64_t* message_host, const int8_t* secret_host,
                              int32_t dist_kind, double dist_param, ckks_rng* rng, uint64_t* ct_host) {
    const char* who = "ckks_encrypt_rng_host";
    if (int32_t rc = ckks_require_device(ctx, who)) return rc;
    if (int32_t rc = check_rng(rng, who)) return rc;
    if (int32_t rc = check_secret(secret_host, ctx->n, who)) return rc;
    if (int32_t rc = check_dist(dist_kind, dist_param, who)) return rc;
    CKKS_CHECK_ARG(message_host && ct_host, std::string(who) + ": null buffer");
    CKKS_CHECK_ARG(q_limbs >= 1 && q_limbs <= ctx->L, std::string(who) + ": q_limbs outside the Q basis");
    const u32 n = ctx->n, L = q_limbs;
    const LimbMap lm = LimbMap::range(0, L);
    // grafting/rns_key_switch.rs:278-387: one logical error, then a uniform a per limb
    std::vector<i64> e(n);
    std::vector<u64> a((size_t)L * n);
    rng->error(n, dist_kind, dist_param, e.data());
    for (u32 l = 0; l < L; ++l) rng->uniform(n, ctx->moduli[l], a.data() + (size_t)l * n);
    cudaStream_t st = ctx->own_stream;
    Workspace<u64> d_m, d_a, d_s, d_b;
    Workspace<i64> d_e;
    Workspace<int8_t> d_sec;
    int32_t rc;
    if ((rc = d_m.alloc((size_t)L * n, st)) || (rc = d_a.alloc((size_t)L * n, st)) ||
        (rc = d_s.alloc((size_t)L * n, st)) || (rc = d_b.alloc((size_t)L * n, st)) || (rc = d_e.alloc(n, st)) ||
        (rc = d_sec.alloc(n, st)))
        return rc;
    CKKS_CUDA_TRY(cudaMemcpyAsync(d_m.p, message_host, (size_t)L * n * 8, cudaMemcpyHostToDevice, st));
    CKKS_CUDA_TRY(cudaMemcpyAsync(d_a.p, a.data(), (size_t)L * n * 8, cudaMemcpyHostToDevice, st));
    CKKS_CUDA_TRY(cudaMemcpyAsync(d_e.p, e.data(), (size_t)n * 8, cudaMemcpyHostToDevice, st));
    CKKS_CUDA_TRY(cudaMemcpyAsync(d_sec.p, secret_host, n, cudaMemcpyHostToDevice, st));
    dim3 g((n + 255) / 256, L);
    k_lift_secret<<<g, 256, 0, st>>>(d_sec.p, d_s.p, ctx->d_tabs, lm, ctx->log_n);
    // a s as a negacyclic product (exact): NTT, pointwise, inverse NTT; a stays in coefficients
    if ((rc = ntt_forward_launch_map(ctx, d_s.p, d_s.p, 1, lm, L, st))) return rc;
    if ((rc = ntt_forward_launch_map(ctx, d_a.p, d_b.p, 1, lm, L, st))) return rc;
    if ((rc = pointwise_launch(ctx, d_b.p, d_s.p, d_b.p, 1, lm, L, 0, st))) return rc;
    if ((rc = ntt_inverse_launch_map(ctx, d_b.p, d_s.p, 1, lm, L, st))) return rc;
    k_encrypt_finish<<<g, 256, 0, st>>>(d_m.p, d_e.p, d_s.p, d_b.p, ctx->d_tabs, lm, ctx->log_n);
    CKKS_CUDA_TRY(cudaGetLastError());
    CKKS_CUDA_TRY(cudaMemcpyAsync(ct_host, d_b.p, (size_t)L * n * 8, cudaMemcpyDeviceToHost, st));
    CKKS_CUDA_TRY(cudaStreamSynchronize(st));
    std::memcpy(ct_host + (size_t)L * n, a.data(), (size_t)L * n * 8);
    return CKKS_OK;
}

}  // extern "C"
