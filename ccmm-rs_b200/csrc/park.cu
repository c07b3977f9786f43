// park.cu -- Park et al. modular plaintext matrix product (Mod-PP-MM) on the GPU.
//
// park_mod_pp_mm (ccmm/park.rs:1634-1647) multiplies two u64 matrices modulo an
// arbitrary modulus q > 1: out = (lhs x rhs) mod q, lhs rows x inner, rhs
// inner x cols, row-major. Every backend of the reference
// (park_matrix_mul_{reference,transposed_rhs,wide_accumulator,parallel_wide},
// :1405-1620) returns the canonical residue of the exact integer dot product;
// here each dot product is summed exactly in 192 bits (a 64 x 64 -> 128-bit
// product per term, so any u64 inputs and up to 2^64 terms are exact) and
// reduced once.
//
// Tiling: a CTA computes a 64 x 64 block of outputs with 256 threads (4 x 4
// outputs each, strided by 16 so a warp's loads of a staged tile row are
// consecutive), staging 16-deep slices of both operands in shared memory.
#include "context.cuh"

namespace {

constexpr int kTile = 64, kDepth = 16, kThreads = 256;

typedef unsigned __int128 u128;

struct Acc192 {
    u64 lo, mid, hi;
    __device__ __forceinline__ void add(u64 a, u64 b) {
        const u64 pl = a * b, ph = __umul64hi(a, b);
        asm("add.cc.u64 %0, %0, %3;\n\taddc.cc.u64 %1, %1, %4;\n\taddc.u64 %2, %2, 0;"
            : "+l"(lo), "+l"(mid), "+l"(hi)
            : "l"(pl), "l"(ph));
    }
};

// (hi 2^128 + mid 2^64 + lo) mod q with r64 = 2^64 mod q, r128 = 2^128 mod q
__device__ __forceinline__ u64 reduce192(const Acc192& a, u64 q, u64 r64, u64 r128) {
    const u128 Q = q;
    u128 t = (u128)(a.hi % q) * r128 % Q;
    t = (t + (u128)(a.mid % q) * r64 % Q) % Q;
    t = (t + a.lo % q) % Q;
    return (u64)t;
}

__global__ void __launch_bounds__(kThreads) k_park_mm(const u64* __restrict__ A, const u64* __restrict__ B,
                                                      u64* __restrict__ C, int rows, int inner, int cols, u64 q,
                                                      u64 r64, u64 r128) {
    __shared__ u64 sa[kDepth][kTile + 1];  // sa[k][r]: lhs[row0 + r][k0 + k]
    __shared__ u64 sb[kDepth][kTile];      // sb[k][c]: rhs[k0 + k][col0 + c]
    const int tid = threadIdx.x;
    const int tr = tid >> 4, tc = tid & 15;  // outputs (tr + 16 i, tc + 16 j)
    const int row0 = blockIdx.y * kTile, col0 = blockIdx.x * kTile;
    Acc192 acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = Acc192{0, 0, 0};
    for (int k0 = 0; k0 < inner; k0 += kDepth) {
        // stage lhs [64 x 16] (transposed) and rhs [16 x 64]; zeros outside the matrices
        for (int w = tid; w < kTile * kDepth; w += kThreads) {
            const int r = w / kDepth, k = w % kDepth;
            const int gr = row0 + r, gk = k0 + k;
            sa[k][r] = (gr < rows && gk < inner) ? A[(size_t)gr * inner + gk] : 0;
            const int kk = w / kTile, c = w % kTile;
            const int gk2 = k0 + kk, gc = col0 + c;
            sb[kk][c] = (gk2 < inner && gc < cols) ? B[(size_t)gk2 * cols + gc] : 0;
        }
        __syncthreads();
#pragma unroll 4
        for (int k = 0; k < kDepth; ++k) {
            u64 a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = sa[k][tr + 16 * i];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = sb[k][tc + 16 * j];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j].add(a[i], b[j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int gr = row0 + tr + 16 * i;
        if (gr >= rows) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int gc = col0 + tc + 16 * j;
            if (gc < cols) C[(size_t)gr * cols + gc] = reduce192(acc[i][j], q, r64, r128);
        }
    }
}

int32_t check_dims(uint32_t rows, uint32_t inner, uint32_t cols, uint64_t q, const char* who) {
    // the reference asserts non-empty operands and a modulus above one (ccmm/park.rs:1489-1505)
    if (rows == 0 || inner == 0 || cols == 0 || q < 2 || rows > 0x7FFFFFFFu || cols > 0x7FFFFFFFu ||
        inner > 0x7FFFFFFFu || (u64)((rows + kTile - 1) / kTile) > 65535u) {
        ckks_set_error(std::string(who) + ": empty operand, modulus below 2 or matrix too large");
        return CKKS_ERR_BAD_ARG;
    }
    return CKKS_OK;
}

}  // namespace

extern "C" {

int32_t ckks_park_mod_pp_mm(const uint64_t* lhs, const uint64_t* rhs, uint64_t* out, uint32_t rows, uint32_t inner,
                            uint32_t cols, uint64_t modulus, void* stream) {
    if (int32_t rc = check_dims(rows, inner, cols, modulus, "ckks_park_mod_pp_mm")) return rc;
    CKKS_CHECK_ARG(lhs && rhs && out, "ckks_park_mod_pp_mm: null matrix");
    const u64 r64 = (u64)(((u128)1 << 64) % modulus);
    const u64 r128 = (u64)((u128)r64 * r64 % modulus);
    dim3 grid((cols + kTile - 1) / kTile, (rows + kTile - 1) / kTile);
    k_park_mm<<<grid, kThreads, 0, (cudaStream_t)stream>>>(lhs, rhs, out, (int)rows, (int)inner, (int)cols, modulus,
                                                           r64, r128);
    CKKS_CUDA_TRY(cudaGetLastError());
    return CKKS_OK;
}

int32_t ckks_park_mod_pp_mm_host(const uint64_t* lhs, const uint64_t* rhs, uint64_t* out, uint32_t rows,
                                 uint32_t inner, uint32_t cols, uint64_t modulus) {
    if (int32_t rc = check_dims(rows, inner, cols, modulus, "ckks_park_mod_pp_mm_host")) return rc;
    CKKS_CHECK_ARG(lhs && rhs && out, "ckks_park_mod_pp_mm_host: null matrix");
    const size_t na = (size_t)rows * inner, nb = (size_t)inner * cols, nc = (size_t)rows * cols;
    u64 *dA = nullptr, *dB = nullptr, *dC = nullptr;
    int32_t rc = CKKS_OK;
    if (cudaMalloc(&dA, na * 8) != cudaSuccess || cudaMalloc(&dB, nb * 8) != cudaSuccess ||
        cudaMalloc(&dC, nc * 8) != cudaSuccess) {
        cudaGetLastError();
        ckks_set_error("ckks_park_mod_pp_mm_host: out of device memory");
        rc = CKKS_ERR_OOM;
    }
    if (rc == CKKS_OK && (cudaMemcpy(dA, lhs, na * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
                          cudaMemcpy(dB, rhs, nb * 8, cudaMemcpyHostToDevice) != cudaSuccess)) {
        ckks_set_error("ckks_park_mod_pp_mm_host: copy to the device failed");
        rc = CKKS_ERR_CUDA;
    }
    if (rc == CKKS_OK) rc = ckks_park_mod_pp_mm(dA, dB, dC, rows, inner, cols, modulus, nullptr);
    if (rc == CKKS_OK && cudaMemcpy(out, dC, nc * 8, cudaMemcpyDeviceToHost) != cudaSuccess) {
        ckks_set_error(std::string("ckks_park_mod_pp_mm_host: ") + cudaGetErrorString(cudaGetLastError()));
        rc = CKKS_ERR_CUDA;
    }
    cudaFree(dA);
    cudaFree(dB);
    cudaFree(dC);
    return rc;
}

}  // extern "C"
