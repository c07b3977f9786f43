// capi_ntt.cu -- C ABI entry points for the negacyclic NTT.
#include "context.cuh"

namespace {

int32_t check_range(ckks_ctx* ctx, uint32_t limb_begin, uint32_t limb_count, const char* who) {
    if (int32_t rc = ckks_require_device(ctx, who)) return rc;
    if ((size_t)limb_begin + limb_count > ctx->moduli.size()) {
        ckks_set_error(std::string(who) + ": limb range outside the context basis");
        return CKKS_ERR_BASIS_MISMATCH;
    }
    return CKKS_OK;
}

typedef int32_t (*ntt_fn)(ckks_ctx*, const u64*, u64*, u32, u32, u32, cudaStream_t);

int32_t host_transform(ckks_ctx* ctx, const uint64_t* in_host, uint64_t* out_host, uint32_t n_polys,
                       uint32_t limb_begin, uint32_t limb_count, ntt_fn fn, const char* who) {
    if (int32_t rc = check_range(ctx, limb_begin, limb_count, who)) return rc;
    CKKS_CHECK_ARG(in_host && out_host, std::string(who) + ": null buffer");
    size_t bytes = (size_t)n_polys * limb_count * ctx->n * sizeof(u64);
    if (!bytes) return CKKS_OK;
    cudaStream_t st = ctx->own_stream;
    u64* d = nullptr;
    if (cudaMallocAsync(&d, bytes, st) != cudaSuccess) {
        cudaGetLastError();
        ckks_set_error(std::string(who) + ": out of device memory");
        return CKKS_ERR_OOM;
    }
    int32_t rc = CKKS_OK;
    cudaError_t e = cudaMemcpyAsync(d, in_host, bytes, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) rc = fn(ctx, d, d, n_polys, limb_begin, limb_count, st);
    if (e == cudaSuccess && rc == CKKS_OK) e = cudaMemcpyAsync(out_host, d, bytes, cudaMemcpyDeviceToHost, st);
    cudaFreeAsync(d, st);
    cudaError_t s = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = s;
    if (rc != CKKS_OK) return rc;
    if (e != cudaSuccess) {
        ckks_set_error(std::string(who) + ": " + cudaGetErrorString(e));
        return CKKS_ERR_CUDA;
    }
    return CKKS_OK;
}

}  // namespace

extern "C" {

int32_t ckks_ntt_forward(ckks_ctx* ctx, const uint64_t* in, uint64_t* out, uint32_t n_polys, uint32_t limb_begin,
                         uint32_t limb_count, void* stream) {
    if (int32_t rc = check_range(ctx, limb_begin, limb_count, "ckks_ntt_forward")) return rc;
    CKKS_CHECK_ARG(in && out, "ckks_ntt_forward: null buffer");
    return ntt_forward_launch(ctx, in, out, n_polys, limb_begin, limb_count, ckks_stream(ctx, stream));
}

int32_t ckks_ntt_inverse(ckks_ctx* ctx, const uint64_t* in, uint64_t* out, uint32_t n_polys, uint32_t limb_begin,
                         uint32_t limb_count, void* stream) {
    if (int32_t rc = check_range(ctx, limb_begin, limb_count, "ckks_ntt_inverse")) return rc;
    CKKS_CHECK_ARG(in && out, "ckks_ntt_inverse: null buffer");
    return ntt_inverse_launch(ctx, in, out, n_polys, limb_begin, limb_count, ckks_stream(ctx, stream));
}

int32_t ckks_ntt_forward_host(ckks_ctx* ctx, const uint64_t* in_host, uint64_t* out_host, uint32_t n_polys,
                              uint32_t limb_begin, uint32_t limb_count) {
    return host_transform(ctx, in_host, out_host, n_polys, limb_begin, limb_count, ntt_forward_launch,
                          "ckks_ntt_forward_host");
}

int32_t ckks_ntt_inverse_host(ckks_ctx* ctx, const uint64_t* in_host, uint64_t* out_host, uint32_t n_polys,
                              uint32_t limb_begin, uint32_t limb_count) {
    return host_transform(ctx, in_host, out_host, n_polys, limb_begin, limb_count, ntt_inverse_launch,
                          "ckks_ntt_inverse_host");
}

}  // extern "C"
