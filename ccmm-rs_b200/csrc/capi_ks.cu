// capi_ks.cu -- C ABI: ring ops, gadgets, key-switching keys and rotations.
#include <cstring>

#include "keyswitch.cuh"

namespace {

int32_t need_ctx(ckks_ctx* ctx, const char* who) { return ckks_require_device(ctx, who); }

int32_t limb_range(ckks_ctx* ctx, u32 begin, u32 count, const char* who) {
    if (int32_t rc = need_ctx(ctx, who)) return rc;
    if ((size_t)begin + count > ctx->moduli.size()) {
        ckks_set_error(std::string(who) + ": limb range outside the context basis");
        return CKKS_ERR_BASIS_MISMATCH;
    }
    return CKKS_OK;
}

int32_t check_exponent(ckks_ctx* ctx, u64 k, const char* who) {
    if ((k & 1) == 0) {
        ckks_set_error(std::string(who) + ": Galois exponent must be odd modulo 2N");
        return CKKS_ERR_BAD_ARG;
    }
    return CKKS_OK;
}

u64 galois_pow5(u32 degree, u64 steps) {
    u64 two_n = 2ull * degree, slots = degree / 2;
    steps %= slots;
    u64 r = 1, b = 5 % two_n;
    while (steps) {
        if (steps & 1) r = r * b % two_n;
        b = b * b % two_n;
        steps >>= 1;
    }
    return r;
}

int32_t new_key(ckks_ctx* ctx, int kind, u32 q_limbs, u32 base_log, u64 exponent, const std::vector<u32>& blocks,
                ckks_ksk** out, const char* who) {
    if (int32_t rc = need_ctx(ctx, who)) return rc;
    CKKS_CHECK_ARG(out != nullptr, std::string(who) + ": out is null");
    *out = nullptr;
    CKKS_CHECK_ARG(q_limbs >= 1 && q_limbs <= ctx->L, std::string(who) + ": q_limbs outside the context Q basis");
    auto* k = new ckks_ksk();
    k->ctx = ctx;
    k->kind = kind;
    k->q_limbs = q_limbs;
    k->base_log = base_log;
    k->exponent = exponent % (2ull * ctx->n);
    k->with_p = kind == CKKS_KSK_HYBRID_BOUNDED || kind == CKKS_KSK_HYBRID_RNS_BLOCK;
    if (k->with_p && ctx->K == 0) {
        delete k;
        ckks_set_error(std::string(who) + ": hybrid keys need auxiliary limbs in the context");
        return CKKS_ERR_BASIS_MISMATCH;
    }
    if (kind == CKKS_KSK_HYBRID_RNS_BLOCK || kind == CKKS_KSK_RNS_BLOCK || kind == CKKS_KSK_RELIN_RNS_BLOCK) {
        k->blocks = blocks;
        k->D = (u32)blocks.size();
        if (int32_t rc = rnsblock_prepare(ctx, k)) {
            delete k;
            return rc;
        }
    } else {
        if (int32_t rc = bounded_digit_count(ctx, q_limbs, base_log, &k->D)) {
            delete k;
            return rc;
        }
    }
    if (int32_t rc = ksk_alloc(ctx, k)) {
        if (k->d_block_const) cudaFree(k->d_block_const);
        delete k;
        return rc;
    }
    *out = k;
    return CKKS_OK;
}

}  // namespace

int32_t ksk_new(ckks_ctx* ctx, int kind, u32 q_limbs, u32 base_log, u64 exponent, ckks_ksk** out, const char* who) {
    return new_key(ctx, kind, q_limbs, base_log, exponent, {}, out, who);
}

namespace {

int32_t finish_key(ckks_ksk* k, int32_t rc, ckks_ksk** out) {
    if (rc == CKKS_OK) {
        cudaError_t e = cudaDeviceSynchronize();
        if (e != cudaSuccess) {
            ckks_set_error(std::string("key generation: ") + cudaGetErrorString(e));
            rc = CKKS_ERR_CUDA;
        }
    }
    if (rc != CKKS_OK) {
        ckks_ksk_destroy(k);
        *out = nullptr;
    }
    return rc;
}

// Reference layout [D][LK][2][N] from the host into the permuted storage.
int32_t upload_galois(ckks_ctx* ctx, ckks_ksk* k, const uint64_t* entries_host) {
    Workspace<u64> tmp;
    if (int32_t rc = tmp.alloc(k->words, nullptr)) return rc;
    CKKS_CUDA_TRY(cudaMemcpy(tmp.p, entries_host, k->words * 8, cudaMemcpyHostToDevice));
    return ksk_permute_entries(ctx, tmp.p, k->d_entries, k->words / ctx->n, k->exponent, true, nullptr);
}

}  // namespace

extern "C" {

int32_t ckks_automorphism_coef(ckks_ctx* ctx, const uint64_t* in, uint64_t* out, uint32_t n_polys,
                               uint32_t limb_begin, uint32_t limbs, uint64_t exponent, void* stream) {
    if (int32_t rc = limb_range(ctx, limb_begin, limbs, "ckks_automorphism_coef")) return rc;
    if (int32_t rc = check_exponent(ctx, exponent, "ckks_automorphism_coef")) return rc;
    CKKS_CHECK_ARG(in && out && in != out, "ckks_automorphism_coef: buffers must be distinct and non-null");
    return automorphism_coef_launch(ctx, in, out, n_polys, LimbMap::range(limb_begin, limbs), limbs, exponent,
                                    ckks_stream(ctx, stream));
}

int32_t ckks_automorphism_ntt(ckks_ctx* ctx, const uint64_t* in, uint64_t* out, uint32_t n_polys,
                              uint32_t limb_begin, uint32_t limbs, uint64_t exponent, void* stream) {
    if (int32_t rc = limb_range(ctx, limb_begin, limbs, "ckks_automorphism_ntt")) return rc;
    if (int32_t rc = check_exponent(ctx, exponent, "ckks_automorphism_ntt")) return rc;
    CKKS_CHECK_ARG(in && out && in != out, "ckks_automorphism_ntt: buffers must be distinct and non-null");
    return automorphism_ntt_launch(ctx, in, out, n_polys, limbs, exponent, ckks_stream(ctx, stream));
}

uint64_t ckks_rotation_exponent_left(uint32_t degree, uint64_t steps) {
    if (degree < 2 || (degree & (degree - 1))) return 0;
    return galois_pow5(degree, steps);
}

uint64_t ckks_rotation_exponent_right(uint32_t degree, uint64_t steps) {
    if (degree < 2 || (degree & (degree - 1))) return 0;
    u64 slots = degree / 2;
    steps %= slots;
    return galois_pow5(degree, (slots - steps) % slots);
}

uint64_t ckks_conjugation_exponent(uint32_t degree) { return 2ull * degree - 1; }

int32_t ckks_pointwise(ckks_ctx* ctx, const uint64_t* a, const uint64_t* b, uint64_t* out, uint32_t n_polys,
                       uint32_t limb_begin, uint32_t limbs, int32_t op, void* stream) {
    if (int32_t rc = limb_range(ctx, limb_begin, limbs, "ckks_pointwise")) return rc;
    CKKS_CHECK_ARG(a && b && out && op >= 0 && op <= 2, "ckks_pointwise: bad arguments");
    return pointwise_launch(ctx, a, b, out, n_polys, LimbMap::range(limb_begin, limbs), limbs, op,
                            ckks_stream(ctx, stream));
}

int32_t ckks_rescale(ckks_ctx* ctx, const uint64_t* in, uint64_t* out, uint32_t n_polys, uint32_t limbs_in,
                     void* stream) {
    if (int32_t rc = need_ctx(ctx, "ckks_rescale")) return rc;
    CKKS_CHECK_ARG(limbs_in >= 2 && limbs_in <= ctx->L, "ckks_rescale: need 2..L limbs (cannot rescale the last level)");
    CKKS_CHECK_ARG(in && out && in != out, "ckks_rescale: buffers must be distinct and non-null");
    return rescale_launch(ctx, in, out, n_polys, limbs_in, ckks_stream(ctx, stream));
}

int32_t ckks_mod_down(ckks_ctx* ctx, const uint64_t* in, uint64_t* out, uint32_t n_polys, uint32_t q_limbs,
                      void* stream) {
    if (int32_t rc = need_ctx(ctx, "ckks_mod_down")) return rc;
    CKKS_CHECK_ARG(ctx->K > 0, "ckks_mod_down: the context has no auxiliary limbs");
    CKKS_CHECK_ARG(q_limbs >= 1 && q_limbs <= ctx->L, "ckks_mod_down: q_limbs outside the Q basis");
    CKKS_CHECK_ARG(in && out && in != out, "ckks_mod_down: buffers must be distinct and non-null");
    return mod_down_launch(ctx, in, out, n_polys, q_limbs, ckks_stream(ctx, stream));
}

int32_t ckks_mod_switch(ckks_ctx* ctx, const uint64_t* in, uint64_t* out, uint32_t n_ct, uint32_t limbs_in,
                        uint32_t limbs_out, void* stream) {
    if (int32_t rc = need_ctx(ctx, "ckks_mod_switch")) return rc;
    CKKS_CHECK_ARG(in && out, "ckks_mod_switch: null buffer");
    CKKS_CHECK_ARG(limbs_out >= 1 && limbs_out <= limbs_in && limbs_in <= ctx->L,
                   "ckks_mod_switch: need 1 <= limbs_out <= limbs_in <= L");
    if (!n_ct) return CKKS_OK;
    const size_t n = ctx->n;
    // the limbs of the lower level are the leading ones (ring/modulus_chain.rs:19-27)
    CKKS_CUDA_TRY(cudaMemcpy2DAsync(out, limbs_out * n * 8, in, limbs_in * n * 8, limbs_out * n * 8, 2 * (size_t)n_ct,
                                    cudaMemcpyDeviceToDevice, ckks_stream(ctx, stream)));
    return CKKS_OK;
}

int32_t ckks_bounded_digit_count(ckks_ctx* ctx, uint32_t q_limbs, uint32_t base_log, uint32_t* out) {
    if (int32_t rc = need_ctx(ctx, "ckks_bounded_digit_count")) return rc;
    CKKS_CHECK_ARG(out != nullptr, "ckks_bounded_digit_count: out is null");
    return bounded_digit_count(ctx, q_limbs, base_log, out);
}

int32_t ckks_bounded_decompose(ckks_ctx* ctx, const uint64_t* poly, uint32_t n_polys, uint32_t q_limbs,
                               uint32_t base_log, int64_t* digits, void* stream) {
    if (int32_t rc = need_ctx(ctx, "ckks_bounded_decompose")) return rc;
    CKKS_CHECK_ARG(poly && digits, "ckks_bounded_decompose: null buffer");
    return bounded_decompose_launch(ctx, poly, n_polys, q_limbs, base_log, digits, nullptr, ckks_stream(ctx, stream));
}

int32_t ckks_bounded_digits_automorphism(ckks_ctx* ctx, const int64_t* in, int64_t* out, uint32_t n_polys,
                                         uint32_t digit_count, uint32_t base_log, uint64_t exponent, void* stream) {
    if (int32_t rc = need_ctx(ctx, "ckks_bounded_digits_automorphism")) return rc;
    CKKS_CHECK_ARG(in && out && in != out, "ckks_bounded_digits_automorphism: buffers must be distinct");
    return digits_automorphism_launch(ctx, in, out, n_polys, digit_count, base_log, exponent % (2ull * ctx->n),
                                      ckks_stream(ctx, stream));
}

int32_t ckks_hybrid_key_generate(ckks_ctx* ctx, uint32_t q_limbs, uint32_t base_log, uint64_t exponent,
                                 const int8_t* secret_host, uint64_t seed, double sigma, ckks_ksk** out) {
    if (int32_t rc = need_ctx(ctx, "ckks_hybrid_key_generate")) return rc;
    CKKS_CHECK_ARG(secret_host && sigma > 0, "ckks_hybrid_key_generate: bad secret or sigma");
    if (int32_t rc = check_exponent(ctx, exponent, "ckks_hybrid_key_generate")) return rc;
    ckks_ksk* k;
    if (int32_t rc = new_key(ctx, CKKS_KSK_HYBRID_BOUNDED, q_limbs, base_log, exponent, {}, &k, "ckks_hybrid_key_generate"))
        return rc;
    *out = k;
    auto st_secret = host_secret_automorphism(secret_host, ctx->n, k->exponent);
    int32_t rc = ksk_generate(ctx, k, secret_host, seed, sigma, hybrid_factors(ctx, k), st_secret, false, TAG_KEY_A,
                              TAG_KEY_E, nullptr);
    return finish_key(k, rc, out);
}

int32_t ckks_hybrid_key_upload(ckks_ctx* ctx, uint32_t q_limbs, uint32_t base_log, uint64_t exponent,
                               const uint64_t* entries_host, ckks_ksk** out) {
    CKKS_CHECK_ARG(entries_host != nullptr, "ckks_hybrid_key_upload: null entries");
    if (int32_t rc = check_exponent(ctx, exponent, "ckks_hybrid_key_upload")) return rc;
    ckks_ksk* k;
    if (int32_t rc = new_key(ctx, CKKS_KSK_HYBRID_BOUNDED, q_limbs, base_log, exponent, {}, &k, "ckks_hybrid_key_upload"))
        return rc;
    *out = k;
    return finish_key(k, upload_galois(ctx, k, entries_host), out);
}

int32_t ckks_rnsblock_key_generate(ckks_ctx* ctx, uint32_t q_limbs, const uint32_t* block_sizes, uint32_t n_blocks,
                                   uint64_t exponent, const int8_t* secret_host, uint64_t seed, double sigma,
                                   ckks_ksk** out) {
    CKKS_CHECK_ARG(block_sizes && n_blocks && secret_host && sigma > 0, "ckks_rnsblock_key_generate: bad arguments");
    if (int32_t rc = check_exponent(ctx, exponent, "ckks_rnsblock_key_generate")) return rc;
    ckks_ksk* k;
    std::vector<u32> bs(block_sizes, block_sizes + n_blocks);
    if (int32_t rc = new_key(ctx, CKKS_KSK_HYBRID_RNS_BLOCK, q_limbs, 0, exponent, bs, &k, "ckks_rnsblock_key_generate"))
        return rc;
    *out = k;
    auto st_secret = host_secret_automorphism(secret_host, ctx->n, k->exponent);
    int32_t rc = ksk_generate(ctx, k, secret_host, seed, sigma, rnsblock_factors(ctx, k), st_secret, false, TAG_KEY_A,
                              TAG_KEY_E, nullptr);
    return finish_key(k, rc, out);
}

int32_t ckks_rnsblock_key_upload(ckks_ctx* ctx, uint32_t q_limbs, const uint32_t* block_sizes, uint32_t n_blocks,
                                 uint64_t exponent, const uint64_t* entries_host, ckks_ksk** out) {
    CKKS_CHECK_ARG(block_sizes && n_blocks && entries_host, "ckks_rnsblock_key_upload: bad arguments");
    if (int32_t rc = check_exponent(ctx, exponent, "ckks_rnsblock_key_upload")) return rc;
    ckks_ksk* k;
    std::vector<u32> bs(block_sizes, block_sizes + n_blocks);
    if (int32_t rc = new_key(ctx, CKKS_KSK_HYBRID_RNS_BLOCK, q_limbs, 0, exponent, bs, &k, "ckks_rnsblock_key_upload"))
        return rc;
    *out = k;
    return finish_key(k, upload_galois(ctx, k, entries_host), out);
}

int32_t ckks_rns_key_generate(ckks_ctx* ctx, uint32_t q_limbs, const uint32_t* block_sizes, uint32_t n_blocks,
                              uint64_t exponent, const int8_t* secret_host, uint64_t seed, double sigma,
                              ckks_ksk** out) {
    if (int32_t rc = need_ctx(ctx, "ckks_rns_key_generate")) return rc;
    CKKS_CHECK_ARG(out && block_sizes && n_blocks && secret_host && sigma > 0, "ckks_rns_key_generate: bad arguments");
    if (int32_t rc = check_exponent(ctx, exponent, "ckks_rns_key_generate")) return rc;
    ckks_ksk* k;
    std::vector<u32> bs(block_sizes, block_sizes + n_blocks);
    if (int32_t rc = new_key(ctx, CKKS_KSK_RNS_BLOCK, q_limbs, 0, exponent, bs, &k, "ckks_rns_key_generate")) return rc;
    *out = k;
    auto st_secret = host_secret_automorphism(secret_host, ctx->n, k->exponent);
    int32_t rc = ksk_generate(ctx, k, secret_host, seed, sigma, rns_factors(ctx, k), st_secret, false, TAG_KEY_A,
                              TAG_KEY_E, nullptr);
    return finish_key(k, rc, out);
}

int32_t ckks_rns_key_upload(ckks_ctx* ctx, uint32_t q_limbs, const uint32_t* block_sizes, uint32_t n_blocks,
                            uint64_t exponent, const uint64_t* entries_host, ckks_ksk** out) {
    if (int32_t rc = need_ctx(ctx, "ckks_rns_key_upload")) return rc;
    CKKS_CHECK_ARG(out && block_sizes && n_blocks && entries_host, "ckks_rns_key_upload: bad arguments");
    if (int32_t rc = check_exponent(ctx, exponent, "ckks_rns_key_upload")) return rc;
    ckks_ksk* k;
    std::vector<u32> bs(block_sizes, block_sizes + n_blocks);
    if (int32_t rc = new_key(ctx, CKKS_KSK_RNS_BLOCK, q_limbs, 0, exponent, bs, &k, "ckks_rns_key_upload")) return rc;
    *out = k;
    return finish_key(k, upload_galois(ctx, k, entries_host), out);
}

int32_t ckks_rns_relin_key_generate(ckks_ctx* ctx, uint32_t q_limbs, const uint32_t* block_sizes, uint32_t n_blocks,
                                    const int8_t* secret_host, uint64_t seed, double sigma, ckks_ksk** out) {
    if (int32_t rc = need_ctx(ctx, "ckks_rns_relin_key_generate")) return rc;
    CKKS_CHECK_ARG(out && block_sizes && n_blocks && secret_host && sigma > 0,
                   "ckks_rns_relin_key_generate: bad arguments");
    ckks_ksk* k;
    std::vector<u32> bs(block_sizes, block_sizes + n_blocks);
    if (int32_t rc = new_key(ctx, CKKS_KSK_RELIN_RNS_BLOCK, q_limbs, 0, 1, bs, &k, "ckks_rns_relin_key_generate"))
        return rc;
    *out = k;
    return finish_key(k, relin_generate(ctx, k, secret_host, seed, sigma, nullptr), out);
}

int32_t ckks_rns_relin_key_upload(ckks_ctx* ctx, uint32_t q_limbs, const uint32_t* block_sizes, uint32_t n_blocks,
                                  const uint64_t* entries_host, ckks_ksk** out) {
    if (int32_t rc = need_ctx(ctx, "ckks_rns_relin_key_upload")) return rc;
    CKKS_CHECK_ARG(out && block_sizes && n_blocks && entries_host, "ckks_rns_relin_key_upload: bad arguments");
    ckks_ksk* k;
    std::vector<u32> bs(block_sizes, block_sizes + n_blocks);
    if (int32_t rc = new_key(ctx, CKKS_KSK_RELIN_RNS_BLOCK, q_limbs, 0, 1, bs, &k, "ckks_rns_relin_key_upload"))
        return rc;
    *out = k;
    cudaError_t e = cudaMemcpy(k->d_entries, entries_host, k->words * 8, cudaMemcpyHostToDevice);
    int32_t rc = e == cudaSuccess ? CKKS_OK : CKKS_ERR_CUDA;
    if (e != cudaSuccess) ckks_set_error(cudaGetErrorString(e));
    // coefficient domain [dnum][2][q_limbs][N] in, NTT domain stored
    if (rc == CKKS_OK) rc = ntt_forward_launch_map(ctx, k->d_entries, k->d_entries, 2 * k->D, LimbMap::range(0, q_limbs),
                                                   q_limbs, nullptr);
    return finish_key(k, rc, out);
}

int32_t ckks_relin_key_generate(ckks_ctx* ctx, uint32_t q_limbs, uint32_t base_log, const int8_t* secret_host,
                                uint64_t seed, double sigma, ckks_ksk** out) {
    CKKS_CHECK_ARG(secret_host && sigma > 0, "ckks_relin_key_generate: bad secret or sigma");
    ckks_ksk* k;
    if (int32_t rc = new_key(ctx, CKKS_KSK_RELIN_BOUNDED, q_limbs, base_log, 1, {}, &k, "ckks_relin_key_generate"))
        return rc;
    *out = k;
    int32_t rc = relin_generate(ctx, k, secret_host, seed, sigma, nullptr);
    return finish_key(k, rc, out);
}

int32_t ckks_relin_key_upload(ckks_ctx* ctx, uint32_t q_limbs, uint32_t base_log, const uint64_t* entries_host,
                              ckks_ksk** out) {
    CKKS_CHECK_ARG(entries_host != nullptr, "ckks_relin_key_upload: null entries");
    ckks_ksk* k;
    if (int32_t rc = new_key(ctx, CKKS_KSK_RELIN_BOUNDED, q_limbs, base_log, 1, {}, &k, "ckks_relin_key_upload"))
        return rc;
    *out = k;
    cudaError_t e = cudaMemcpy(k->d_entries, entries_host, k->words * 8, cudaMemcpyHostToDevice);
    int32_t rc = e == cudaSuccess ? CKKS_OK : CKKS_ERR_CUDA;
    if (e != cudaSuccess) ckks_set_error(cudaGetErrorString(e));
    // reference layout is coefficient domain [D][2][q_limbs][N]: transform in place
    if (rc == CKKS_OK) rc = ntt_forward_launch_map(ctx, k->d_entries, k->d_entries, 2 * k->D, LimbMap::range(0, q_limbs),
                                                   q_limbs, nullptr);
    return finish_key(k, rc, out);
}

int32_t ckks_ksk_info(const ckks_ksk* key, uint32_t* digits, uint64_t* words) {
    CKKS_CHECK_ARG(key != nullptr, "ckks_ksk_info: null key");
    if (digits) *digits = key->D;
    if (words) *words = key->words;
    return CKKS_OK;
}

int32_t ckks_ksk_download(const ckks_ksk* key, uint64_t* entries_host) {
    CKKS_CHECK_ARG(key && entries_host, "ckks_ksk_download: null argument");
    if (key->kind == CKKS_KSK_RELIN_BOUNDED || key->kind == CKKS_KSK_RELIN_RNS_BLOCK) {
        CKKS_CUDA_TRY(cudaMemcpy(entries_host, key->d_entries, key->words * 8, cudaMemcpyDeviceToHost));
        return CKKS_OK;
    }
    int32_t rc;
    {
        Workspace<u64> tmp;
        if ((rc = tmp.alloc(key->words, nullptr))) return rc;
        if ((rc = ksk_permute_entries(key->ctx, key->d_entries, tmp.p, key->words / key->ctx->n, key->exponent, false,
                                      nullptr)))
            return rc;
        CKKS_CUDA_TRY(cudaMemcpy(entries_host, tmp.p, key->words * 8, cudaMemcpyDeviceToHost));
    }
    CKKS_CUDA_TRY(cudaDeviceSynchronize());
    return CKKS_OK;
}

int32_t ckks_ksk_destroy(ckks_ksk* key) {
    if (!key) return CKKS_OK;
    keyset_forget_key(key);
    if (key->d_entries) cudaFree(key->d_entries);
    if (key->d_block_const) cudaFree(key->d_block_const);
    delete key;
    return CKKS_OK;
}

int32_t ckks_rotate(ckks_ctx* ctx, const ckks_ksk* key, const uint64_t* ct_in, uint64_t* ct_out, uint32_t n_ct,
                    void* stream) {
    if (int32_t rc = need_ctx(ctx, "ckks_rotate")) return rc;
    CKKS_CHECK_ARG(key && ct_in && ct_out && ct_in != ct_out, "ckks_rotate: bad arguments");
    if (key->ctx != ctx || key->kind == CKKS_KSK_RELIN_BOUNDED || key->kind == CKKS_KSK_RELIN_RNS_BLOCK) {
        ckks_set_error("ckks_rotate: key is not a Galois key of this context");
        return CKKS_ERR_BASIS_MISMATCH;
    }
    return rotate_hybrid(ctx, key, ct_in, ct_out, n_ct, ckks_stream(ctx, stream));
}

int32_t ckks_rotate_hoisted(ckks_ctx* ctx, const ckks_ksk* const* keys, uint32_t n_keys, const uint64_t* ct_in,
                            uint64_t* ct_out, uint32_t n_ct, void* stream) {
    if (int32_t rc = need_ctx(ctx, "ckks_rotate_hoisted")) return rc;
    CKKS_CHECK_ARG(keys && n_keys && ct_in && ct_out && ct_in != ct_out, "ckks_rotate_hoisted: bad arguments");
    const ckks_ksk* k0 = keys[0];
    for (u32 g = 0; g < n_keys; ++g) {
        const ckks_ksk* k = keys[g];
        if (!k || k->ctx != ctx || k->kind != k0->kind || k->kind == CKKS_KSK_RELIN_BOUNDED ||
            k->kind == CKKS_KSK_RELIN_RNS_BLOCK ||
            k->q_limbs != k0->q_limbs || k->base_log != k0->base_log || k->D != k0->D || k->blocks != k0->blocks) {
            ckks_set_error("ckks_rotate_hoisted: keys must be Galois keys of one kind, level and gadget");
            return CKKS_ERR_BASIS_MISMATCH;
        }
    }
    return rotate_hybrid_hoisted(ctx, keys, n_keys, ct_in, ct_out, n_ct, ckks_stream(ctx, stream));
}

int32_t ckks_rotate_hoisted_timed(ckks_ctx* ctx, const ckks_ksk* const* keys, uint32_t n_keys, const uint64_t* ct_in,
                                  uint64_t* ct_out, uint32_t n_ct, void* stream, double* phase_ms) {
    if (int32_t rc = need_ctx(ctx, "ckks_rotate_hoisted_timed")) return rc;
    CKKS_CHECK_ARG(keys && n_keys && ct_in && ct_out && ct_in != ct_out && phase_ms,
                   "ckks_rotate_hoisted_timed: bad arguments");
    const ckks_ksk* k0 = keys[0];
    for (u32 g = 0; g < n_keys; ++g) {
        const ckks_ksk* k = keys[g];
        if (!k || k->ctx != ctx || k->kind != k0->kind || k->kind == CKKS_KSK_RELIN_BOUNDED ||
            k->kind == CKKS_KSK_RELIN_RNS_BLOCK ||
            k->q_limbs != k0->q_limbs || k->base_log != k0->base_log || k->D != k0->D || k->blocks != k0->blocks) {
            ckks_set_error("ckks_rotate_hoisted_timed: keys must be Galois keys of one kind, level and gadget");
            return CKKS_ERR_BASIS_MISMATCH;
        }
    }
    for (int i = 0; i < 8; ++i) phase_ms[i] = 0;
    if (k0->kind == CKKS_KSK_RNS_BLOCK) {
        ckks_set_error("ckks_rotate_hoisted_timed: keys without auxiliary limbs have no hoisted phases");
        return CKKS_ERR_BAD_ARG;
    }
    return rotate_hoisted_ntt(ctx, keys, n_keys, ct_in, ct_out, n_ct, ckks_stream(ctx, stream), phase_ms);
}

int32_t ckks_rotate_hoisted_host(ckks_ctx* ctx, const ckks_ksk* const* keys, uint32_t n_keys,
                                 const uint64_t* ct_in_host, uint64_t* ct_out_host, uint32_t n_ct) {
    if (int32_t rc = need_ctx(ctx, "ckks_rotate_hoisted_host")) return rc;
    CKKS_CHECK_ARG(keys && n_keys && keys[0] && ct_in_host && ct_out_host, "ckks_rotate_hoisted_host: bad arguments");
    const size_t ct_words = (size_t)2 * keys[0]->q_limbs * ctx->n;
    cudaStream_t st = ctx->own_stream;
    int32_t rc;
    {
        Workspace<u64> din, dout;
        if ((rc = din.alloc(ct_words * n_ct, st)) || (rc = dout.alloc(ct_words * n_ct * n_keys, st))) return rc;
        CKKS_CUDA_TRY(cudaMemcpyAsync(din.p, ct_in_host, ct_words * n_ct * 8, cudaMemcpyHostToDevice, st));
        rc = ckks_rotate_hoisted(ctx, keys, n_keys, din.p, dout.p, n_ct, st);
        if (rc == CKKS_OK)
            CKKS_CUDA_TRY(cudaMemcpyAsync(ct_out_host, dout.p, ct_words * n_ct * n_keys * 8, cudaMemcpyDeviceToHost, st));
    }
    cudaError_t e = cudaStreamSynchronize(st);
    if (rc == CKKS_OK && e != cudaSuccess) {
        ckks_set_error(std::string("ckks_rotate_hoisted_host: ") + cudaGetErrorString(e));
        return CKKS_ERR_CUDA;
    }
    return rc;
}

}  // extern "C"
