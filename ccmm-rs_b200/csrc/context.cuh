// context.cuh -- the device context behind the C ABI: ring degree, the
// modulus basis (Q limbs then P limbs), per-modulus NTT tables in HBM,
// error reporting and stream handling.
#pragma once
#include <cuda_runtime.h>

#include <mutex>
#include <string>
#include <vector>

#include "modarith.cuh"
#include "../../include/ckks_b200.h"

// Per-modulus NTT tables (device pointers). N = N1 * N2 with N2 = 2^floor(logN/2).
// The forward transform is the two-pass decomposition
//   A[k2 + N2 k1] = sum_j1 w1^(j1 k1) psi^((2k2+1) j1) sum_j2 a[j1 + N1 j2] psi2^((2k2+1) j2)
// with psi2 = psi^N1 (order 2 N2) and w1 = psi^(2 N2) (order N1), which equals
// the reference definition A[k] = a(psi^(2k+1)) (ring/ntt.rs:101-127).
struct NttTab {
    u64 q;
    u64 mu_hi, mu_lo;                       // Barrett floor(2^128/q)
    const u64 *psi_rev, *psi_rev_q;         // [N2] psi2^bitrev(i)     (forward pass 1)
    const u64 *psi_inv_rev, *psi_inv_rev_q; // [N2] psi2^-bitrev(i)    (inverse pass B)
    const u64 *w, *w_q;                     // [N1/2] w1^i             (forward pass 2)
    const u64 *w_inv, *w_inv_q;             // [N1/2] w1^-i            (inverse pass A)
    const u64 *mid, *mid_q;                 // [N1][N2] psi^((2k2+1) j1)
    const u64 *imid, *imid_q;               // [N2][N1] N^-1 psi^-((2k2+1) j1)
};

struct ckks_ctx {
    int device = 0;
    u32 log_n = 0, n = 0, log_n1 = 0, log_n2 = 0;
    u32 L = 0, K = 0;
    std::vector<u64> moduli;  // Q limbs then P limbs
    std::vector<u64> psi;     // primitive 2N-th roots (reference search rule)
    u64* d_table_mem = nullptr;
    NttTab* d_tabs = nullptr;  // [L+K]
    std::vector<NttTab> h_tabs;
    cudaStream_t own_stream = nullptr;
    // scratch for in-place transforms, grown on demand
    std::mutex scratch_mutex;
    u64* scratch = nullptr;
    size_t scratch_words = 0;
};

// ---------------------------------------------------------------- errors
void ckks_set_error(const std::string& msg);

#define CKKS_CUDA_TRY(expr)                                                       \
    do {                                                                          \
        cudaError_t _e = (expr);                                                  \
        if (_e != cudaSuccess) {                                                  \
            ckks_set_error(std::string(#expr) + ": " + cudaGetErrorString(_e));   \
            return CKKS_ERR_CUDA;                                                 \
        }                                                                         \
    } while (0)

#define CKKS_CHECK_ARG(cond, msg)          \
    do {                                   \
        if (!(cond)) {                     \
            ckks_set_error(msg);           \
            return CKKS_ERR_BAD_ARG;       \
        }                                  \
    } while (0)

inline cudaStream_t ckks_stream(ckks_ctx* ctx, void* s) {
    return s ? (cudaStream_t)s : ctx->own_stream;
}

// ------------------------------------------------------------- launchers
// data layout [n_polys][limb_count][N]; table index = limb_begin + limb.
int32_t ntt_forward_launch(ckks_ctx* ctx, const u64* in, u64* out, u32 n_polys, u32 limb_begin,
                           u32 limb_count, cudaStream_t st);
int32_t ntt_inverse_launch(ckks_ctx* ctx, const u64* in, u64* out, u32 n_polys, u32 limb_begin,
                           u32 limb_count, cudaStream_t st);
// Scratch of at least `words` u64 (grown on demand; serialises growth).
int32_t ctx_scratch(ckks_ctx* ctx, size_t words, u64** out);
