// capi_mul.cu -- C ABI: tensor, relinearization, plaintext products and the
// multiply -> relinearize -> rescale chain.
#include <cmath>

#include "keyswitch.cuh"

namespace {

int32_t check_relin_key(ckks_ctx* ctx, const ckks_ksk* key, const char* who) {
    if (int32_t rc = ckks_require_device(ctx, who)) return rc;
    CKKS_CHECK_ARG(key != nullptr, std::string(who) + ": null key");
    if (key->ctx != ctx || (key->kind != CKKS_KSK_RELIN_BOUNDED && key->kind != CKKS_KSK_RELIN_RNS_BLOCK)) {
        ckks_set_error(std::string(who) + ": key is not a relinearization key of this context");
        return CKKS_ERR_BASIS_MISMATCH;
    }
    return CKKS_OK;
}

bool overlaps(const void* a, size_t a_bytes, const void* b, size_t b_bytes) {
    const char *x = (const char*)a, *y = (const char*)b;
    return x < y + b_bytes && y < x + a_bytes;
}

}  // namespace

extern "C" {

int32_t ckks_tensor(ckks_ctx* ctx, const uint64_t* lhs, const uint64_t* rhs, uint64_t* out, uint32_t n_ct,
                    uint32_t q_limbs, void* stream) {
    if (int32_t rc = ckks_require_device(ctx, "ckks_tensor")) return rc;
    CKKS_CHECK_ARG(lhs && rhs && out, "ckks_tensor: null buffer");
    if (q_limbs < 1 || q_limbs > ctx->L) {
        ckks_set_error("ckks_tensor: q_limbs outside the context Q basis");
        return CKKS_ERR_BASIS_MISMATCH;
    }
    const size_t ct = (size_t)2 * q_limbs * ctx->n * 8 * n_ct, o = ct / 2 * 3;
    CKKS_CHECK_ARG(!overlaps(out, o, lhs, ct) && !overlaps(out, o, rhs, ct), "ckks_tensor: out overlaps an input");
    if (!n_ct) return CKKS_OK;
    return tensor_launch(ctx, lhs, rhs, out, n_ct, q_limbs, ckks_stream(ctx, stream));
}

int32_t ckks_relinearize(ckks_ctx* ctx, const ckks_ksk* key, const uint64_t* quad, uint64_t* out, uint32_t n_ct,
                         void* stream) {
    if (int32_t rc = check_relin_key(ctx, key, "ckks_relinearize")) return rc;
    CKKS_CHECK_ARG(quad && out, "ckks_relinearize: null buffer");
    const size_t poly = (size_t)key->q_limbs * ctx->n * 8 * n_ct;
    CKKS_CHECK_ARG(!overlaps(out, 2 * poly, quad, 3 * poly), "ckks_relinearize: out overlaps the input");
    if (!n_ct) return CKKS_OK;
    return relinearize_launch(ctx, key, quad, out, n_ct, ckks_stream(ctx, stream));
}

int32_t ckks_multiply_relin_rescale(ckks_ctx* ctx, const ckks_ksk* key, const uint64_t* lhs, const uint64_t* rhs,
                                    uint64_t* out, uint32_t n_ct, void* stream) {
    if (int32_t rc = check_relin_key(ctx, key, "ckks_multiply_relin_rescale")) return rc;
    CKKS_CHECK_ARG(lhs && rhs && out, "ckks_multiply_relin_rescale: null buffer");
    CKKS_CHECK_ARG(key->q_limbs >= 2, "ckks_multiply_relin_rescale: no next level to rescale to");
    const size_t in = (size_t)2 * key->q_limbs * ctx->n * 8 * n_ct, o = (size_t)2 * (key->q_limbs - 1) * ctx->n * 8 * n_ct;
    CKKS_CHECK_ARG(!overlaps(out, o, lhs, in) && !overlaps(out, o, rhs, in),
                   "ckks_multiply_relin_rescale: out overlaps an input");
    if (!n_ct) return CKKS_OK;
    return multiply_relin_rescale_launch(ctx, key, lhs, rhs, out, n_ct, ckks_stream(ctx, stream));
}

int32_t ckks_multiply_relin_rescale_host(ckks_ctx* ctx, const ckks_ksk* key, const uint64_t* lhs_host,
                                         const uint64_t* rhs_host, uint64_t* out_host, uint32_t n_ct) {
    if (int32_t rc = check_relin_key(ctx, key, "ckks_multiply_relin_rescale_host")) return rc;
    CKKS_CHECK_ARG(lhs_host && rhs_host && out_host && key->q_limbs >= 2,
                   "ckks_multiply_relin_rescale_host: bad arguments");
    if (!n_ct) return CKKS_OK;
    const size_t in = (size_t)2 * key->q_limbs * ctx->n * n_ct, o = (size_t)2 * (key->q_limbs - 1) * ctx->n * n_ct;
    cudaStream_t st = ctx->own_stream;
    int32_t rc;
    {
        Workspace<u64> d;
        if ((rc = d.alloc(2 * in + o, st))) return rc;
        CKKS_CUDA_TRY(cudaMemcpyAsync(d.p, lhs_host, in * 8, cudaMemcpyHostToDevice, st));
        CKKS_CUDA_TRY(cudaMemcpyAsync(d.p + in, rhs_host, in * 8, cudaMemcpyHostToDevice, st));
        rc = multiply_relin_rescale_launch(ctx, key, d.p, d.p + in, d.p + 2 * in, n_ct, st);
        if (rc == CKKS_OK) CKKS_CUDA_TRY(cudaMemcpyAsync(out_host, d.p + 2 * in, o * 8, cudaMemcpyDeviceToHost, st));
    }
    cudaError_t e = cudaStreamSynchronize(st);
    if (rc == CKKS_OK && e != cudaSuccess) {
        ckks_set_error(std::string("ckks_multiply_relin_rescale_host: ") + cudaGetErrorString(e));
        return CKKS_ERR_CUDA;
    }
    return rc;
}

int32_t ckks_mul_plain(ckks_ctx* ctx, const uint64_t* ct, const uint64_t* plain_ntt, uint64_t* out, uint32_t n_ct,
                       uint32_t q_limbs, uint32_t n_plain, void* stream) {
    if (int32_t rc = ckks_require_device(ctx, "ckks_mul_plain")) return rc;
    CKKS_CHECK_ARG(ct && plain_ntt && out, "ckks_mul_plain: null buffer");
    if (q_limbs < 1 || q_limbs > ctx->L) {
        ckks_set_error("ckks_mul_plain: q_limbs outside the context Q basis");
        return CKKS_ERR_BASIS_MISMATCH;
    }
    CKKS_CHECK_ARG(n_plain == 1 || n_plain == n_ct, "ckks_mul_plain: n_plain must be 1 or n_ct");
    if (!n_ct) return CKKS_OK;
    return mul_plain_launch(ctx, ct, plain_ntt, out, n_ct, q_limbs, n_plain > 1, ckks_stream(ctx, stream));
}

namespace {
int32_t diag_stage(ckks_ctx* ctx, const ckks_ksk* const* keys, uint32_t n_rot, int32_t identity,
                   const uint64_t* diag_ntt, const uint64_t* ct_in, uint64_t* ct_out, uint32_t n_ct, uint32_t q_limbs,
                   bool rescale, void* stream, const char* who) {
    if (int32_t rc = ckks_require_device(ctx, who)) return rc;
    CKKS_CHECK_ARG(diag_ntt && ct_in && ct_out && (n_rot == 0 || keys) && (n_rot || identity),
                   std::string(who) + ": bad arguments");
    CKKS_CHECK_ARG(q_limbs >= (rescale ? 2u : 1u) && q_limbs <= ctx->L,
                   std::string(who) + ": need 2..L limbs to rescale, 1..L otherwise");
    for (u32 g = 0; g < n_rot; ++g) {
        const ckks_ksk* k = keys[g];
        if (!k || k->ctx != ctx || !k->with_p || k->kind != keys[0]->kind || k->q_limbs != q_limbs ||
            k->base_log != keys[0]->base_log || k->D != keys[0]->D || k->blocks != keys[0]->blocks) {
            ckks_set_error(std::string(who) + ": keys must be hybrid Galois keys of one kind and gadget at level q_limbs");
            return CKKS_ERR_BASIS_MISMATCH;
        }
    }
    const size_t in = (size_t)2 * q_limbs * ctx->n * 8 * n_ct,
                 o = (size_t)2 * (rescale ? q_limbs - 1 : q_limbs) * ctx->n * 8 * n_ct;
    CKKS_CHECK_ARG(!overlaps(ct_out, o, ct_in, in), std::string(who) + ": out overlaps the input");
    if (!n_ct) return CKKS_OK;
    return fft_stage_launch(ctx, keys, n_rot, identity != 0, diag_ntt, ct_in, ct_out, n_ct, q_limbs,
                            ckks_stream(ctx, stream), rescale);
}
}  // namespace

int32_t ckks_fft_stage(ckks_ctx* ctx, const ckks_ksk* const* keys, uint32_t n_rot, int32_t identity,
                       const uint64_t* diag_ntt, const uint64_t* ct_in, uint64_t* ct_out, uint32_t n_ct,
                       uint32_t q_limbs, void* stream) {
    return diag_stage(ctx, keys, n_rot, identity, diag_ntt, ct_in, ct_out, n_ct, q_limbs, true, stream,
                      "ckks_fft_stage");
}

int32_t ckks_diag_stage(ckks_ctx* ctx, const ckks_ksk* const* keys, uint32_t n_rot, int32_t identity,
                        const uint64_t* diag_ntt, const uint64_t* ct_in, uint64_t* ct_out, uint32_t n_ct,
                        uint32_t q_limbs, int32_t rescale, void* stream) {
    return diag_stage(ctx, keys, n_rot, identity, diag_ntt, ct_in, ct_out, n_ct, q_limbs, rescale != 0, stream,
                      "ckks_diag_stage");
}

int32_t ckks_ccmm_structured(ckks_ctx* ctx, const ckks_ksk* key, const uint64_t* A, const uint64_t* B, uint64_t* C,
                             uint32_t m, uint32_t k, uint32_t n, void* stream) {
    if (int32_t rc = check_relin_key(ctx, key, "ckks_ccmm_structured")) return rc;
    CKKS_CHECK_ARG(A && B && C && m && k && n, "ckks_ccmm_structured: bad arguments");
    CKKS_CHECK_ARG(key->q_limbs >= 2, "ckks_ccmm_structured: no next level to rescale to");
    CKKS_CHECK_ARG((size_t)m * k <= 12288 && (size_t)k * n <= (size_t(1) << 24),
                   "ckks_ccmm_structured: matrix too large for the slot blocks");
    for (u32 l = 0; l < key->q_limbs; ++l)
        CKKS_CHECK_ARG(ctx->moduli[l] < (1ull << 60), "ckks_ccmm_structured: Q moduli must be below 2^60");
    const size_t ctb = (size_t)2 * key->q_limbs * ctx->n * 8, cto = (size_t)2 * (key->q_limbs - 1) * ctx->n * 8;
    CKKS_CHECK_ARG(!overlaps(C, cto * m * n, A, ctb * m * k) && !overlaps(C, cto * m * n, B, ctb * k * n),
                   "ckks_ccmm_structured: C overlaps an input");
    return ccmm_structured_launch(ctx, key, A, B, C, m, k, n, ckks_stream(ctx, stream));
}

int32_t ckks_fft_stage_multi(ckks_ctx* ctx, const ckks_ksk* const* keys, uint32_t n_rot, const uint32_t* terms_host,
                             uint32_t n_terms, const uint64_t* diag_ntt, const uint64_t* ct_in, uint32_t n_in,
                             uint64_t* ct_out, uint32_t n_out, uint32_t q_limbs, void* stream) {
    if (int32_t rc = ckks_require_device(ctx, "ckks_fft_stage_multi")) return rc;
    CKKS_CHECK_ARG(terms_host && diag_ntt && ct_in && ct_out && n_terms && n_in && n_out && (n_rot == 0 || keys),
                   "ckks_fft_stage_multi: bad arguments");
    CKKS_CHECK_ARG(q_limbs >= 2 && q_limbs <= ctx->L, "ckks_fft_stage_multi: need 2..L limbs (the stage rescales)");
    CKKS_CHECK_ARG(n_out <= 65535 && (size_t)2 * n_in * (n_rot + 1) <= 65535, "ckks_fft_stage_multi: batch too large");
    for (u32 t = 0; t < n_terms; ++t)
        CKKS_CHECK_ARG(terms_host[3 * t] < n_out && terms_host[3 * t + 1] < n_in && terms_host[3 * t + 2] <= n_rot,
                       "ckks_fft_stage_multi: term index out of range");
    for (u32 g = 0; g < n_rot; ++g) {
        const ckks_ksk* k = keys[g];
        if (!k || k->ctx != ctx || !k->with_p || k->kind != keys[0]->kind ||
            k->q_limbs != q_limbs || k->base_log != keys[0]->base_log || k->D != keys[0]->D ||
            k->blocks != keys[0]->blocks) {
            ckks_set_error("ckks_fft_stage_multi: keys must be hybrid Galois keys of one kind and gadget at level q_limbs");
            return CKKS_ERR_BASIS_MISMATCH;
        }
    }
    const size_t in = (size_t)2 * q_limbs * ctx->n * 8 * n_in, o = (size_t)2 * (q_limbs - 1) * ctx->n * 8 * n_out;
    CKKS_CHECK_ARG(!overlaps(ct_out, o, ct_in, in), "ckks_fft_stage_multi: out overlaps the input");
    return fft_stage_multi_launch(ctx, keys, n_rot, terms_host, n_terms, diag_ntt, ct_in, n_in, ct_out, n_out,
                                  q_limbs, ckks_stream(ctx, stream));
}

int32_t ckks_encode(ckks_ctx* ctx, const double* slots, uint64_t* out, uint32_t n_msg, uint32_t q_limbs, double scale,
                    void* stream) {
    if (int32_t rc = ckks_require_device(ctx, "ckks_encode")) return rc;
    CKKS_CHECK_ARG(slots && out, "ckks_encode: null buffer");
    CKKS_CHECK_ARG(q_limbs >= 1 && q_limbs <= ctx->L, "ckks_encode: q_limbs outside the context Q basis");
    CKKS_CHECK_ARG(std::isfinite(scale) && scale > 0, "ckks_encode: scale must be finite and positive");
    if (!n_msg) return CKKS_OK;
    CKKS_CHECK_ARG(n_msg <= 65535, "ckks_encode: at most 65535 messages per call");
    return encode_launch(ctx, slots, out, n_msg, q_limbs, scale, ckks_stream(ctx, stream));
}

int32_t ckks_decode(ckks_ctx* ctx, const uint64_t* poly, double* slots, uint32_t n_msg, uint32_t q_limbs,
                    double scale, void* stream) {
    if (int32_t rc = ckks_require_device(ctx, "ckks_decode")) return rc;
    CKKS_CHECK_ARG(poly && slots, "ckks_decode: null buffer");
    CKKS_CHECK_ARG(q_limbs >= 1 && q_limbs <= ctx->L, "ckks_decode: q_limbs outside the context Q basis");
    CKKS_CHECK_ARG(std::isfinite(scale) && scale > 0, "ckks_decode: scale must be finite and positive");
    if (!n_msg) return CKKS_OK;
    CKKS_CHECK_ARG(n_msg <= 65535, "ckks_decode: at most 65535 messages per call");
    return decode_launch(ctx, poly, slots, n_msg, q_limbs, scale, ckks_stream(ctx, stream));
}

}  // extern "C"
