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


// Per-modulus NTT tables (device pointers) of the twisted four-step
// transform N = A * B: psi_A^bitrev and psi_A^-bitrev (A entries, psi_A =
// psi^B), psi_2B^bitrev and psi_2B^-bitrev (B entries, psi_2B = psi^A), the
// twist mid[j_lo][k_a] = psi^((2k_a+1-A) j_lo) and the inverse twist
// midi[k_a][j_lo] = N^-1 psi^-((2k_a+1-A) j_lo), each with Shoup companions.
struct NttTab {
    u64 q;
    u64 mu_hi, mu_lo;  // Barrett floor(2^128/q)
    const u64 *psiA, *psiA_q, *psiA_inv, *psiA_inv_q;
    const u64 *psiB, *psiB_q, *psiB_inv, *psiB_inv_q;
    const u64 *mid, *mid_q, *midi, *midi_q;
    // FP64 networks (primes below 2^50 and transform halves of up to 2^8
    // points): the same tables as (W, fl(W / q)) pairs, q and fl(1 / q)
    int f64;
    double qd, qinv;
    const double2 *fA, *fA_inv, *fB, *fB_inv, *fmid, *fmidi;
};

constexpr int kMaxAux = 8;  // auxiliary (P) limbs
constexpr int kMaxQ = 64;   // Q limbs

// Exact ModDown constants (ring/auxiliary_modulus.rs:89-171).
struct ModDownConst {
    int K;
    u64 p[kMaxAux];
    u64 pp[kMaxAux][kMaxAux], pp_q[kMaxAux][kMaxAux];  // (p_0..p_{j-1}) mod p_i
    u64 pinv[kMaxAux], pinv_q[kMaxAux];                // ((p_0..p_{i-1}) mod p_i)^-1
    u64 half[kMaxAux];                                 // mixed-radix digits of floor(P/2)
    const u64* q;                                      // [L]
    const u64 *pre, *pre_q;                            // [L][kMaxAux]: (p_0..p_{j-1}) mod q_i
    const u64* p_mod_q;                                // [L]
    const u64 *pinv_mod_q, *pinv_mod_q_q;              // [L]: (P mod q_i)^-1
    // FP64 ModDown (K <= 3, Q primes below 2^50): P as three words, and per Q
    // limb [L][12] doubles: q, 1/q, then (c, c/q) for c = P^-1 and
    // c = 2^(47 k) P^-1 mod q (k = 0..3)
    u64 P3[3];
    const double* f64c;
};

// Garner constants of the Q basis prefix (shared by every prefix length).
struct GarnerQ {
    const u64 *gq, *gq_q;    // [L][L]: (q_0..q_{j-1}) mod q_i
    const u64 *ginv, *ginv_q;  // [L]: ((q_0..q_{i-1}) mod q_i)^-1
};

struct ckks_ctx {
    int device = 0;
    u32 log_n = 0, n = 0, log_n1 = 0, log_n2 = 0;
    u32 L = 0, K = 0;
    std::vector<u64> moduli;  // Q limbs then P limbs
    std::vector<u64> psi;     // primitive 2N-th roots (reference search rule)
    u64* d_table_mem = nullptr;
    double2* d_ftable_mem = nullptr;  // (W, W/q) tables of the FP64 moduli
    NttTab* d_tabs = nullptr;  // [L+K]
    std::vector<NttTab> h_tabs;
    cudaStream_t own_stream = nullptr;
    // (P mod q_l, Shoup) for l < L at [0, 2L)
    u64* d_pmodq = nullptr;
    // rescale: for drop index d, [2][L] = ((q_d mod q_i)^-1, Shoup) at d*2L
    u64* d_rescale_inv = nullptr;
    // exact ModDown and Q-prefix Garner constants (see kernels.cuh)
    u64* d_const_mem = nullptr;
    ModDownConst mod_down{};
    GarnerQ garner{};
    // key-switch MAC of bounded hoisted rotations: tcgen05 INT8 tensor cores
    // (when the device has them) or the CUDA-core split-accumulator form
    bool tensor_cores = true;
    // MAC of the most recent hoisted rotation on this context: 1 tensor cores,
    // 0 CUDA cores, -1 none yet (diagnostic; read by ckks_ctx_last_mac_path)
    int last_mac_path = -1;
    // NTT columns per CTA (log2) per pass: forward 1, forward 1 of digits,
    // forward 2, inverse 1, inverse 2; -1 = built-in choice; set by the autotuner
    int ntt_log_c[5] = {-1, -1, -1, -1, -1};
    std::string tuning_report;
    // pinned host buffers for asynchronous status read-backs (counts, error
    // flags), reused across calls; a call takes one and gives it back
    std::mutex pinned_mu;
    std::vector<std::pair<void*, size_t>> pinned_free;
};

// A pinned host buffer of at least `bytes` from the context's free list (null
// if pinned memory cannot be had), and its return.
void* pinned_take(ckks_ctx* ctx, size_t bytes, size_t* got);
void pinned_give(ckks_ctx* ctx, void* p, size_t bytes);

// ---------------------------------------------------------------- errors
void ckks_set_error(const std::string& msg);

// Entry points that touch device memory require the calling thread's current
// CUDA device to be the context's device (its tables, keys and constants live
// there): a mismatch returns CKKS_ERR_BAD_ARG instead of mixing two GPUs'
// memory in one launch.
int32_t ckks_require_device(const ckks_ctx* ctx, const char* who);

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

// NULL selects the CUDA default (legacy) stream, so calls order with the
// caller's default-stream work; the context's own stream serves the
// host-buffer entry points only.
inline cudaStream_t ckks_stream(ckks_ctx*, void* s) {
    return (cudaStream_t)s;
}

// Local limb index -> table index: limbs [0, split) map to b0 + limb, the rest
// to b1 + (limb - split). Covers a contiguous range and "Q prefix + P".
struct LimbMap {
    int b0, split, b1;
    CKKS_HD int operator()(int limb) const { return limb < split ? b0 + limb : b1 + (limb - split); }
    static LimbMap range(u32 begin, u32 count) { return LimbMap{(int)begin, (int)count, 0}; }
    // Q limbs 0..q_limbs-1 followed by the context's K auxiliary limbs
    static LimbMap qp(const ckks_ctx* c, u32 q_limbs);
};

// ------------------------------------------------------------- launchers
// data layout [n_polys][limb_count][N]; table index = limb_begin + limb.
int32_t ntt_forward_launch(ckks_ctx* ctx, const u64* in, u64* out, u32 n_polys, u32 limb_begin,
                           u32 limb_count, cudaStream_t st);
int32_t ntt_inverse_launch(ckks_ctx* ctx, const u64* in, u64* out, u32 n_polys, u32 limb_begin,
                           u32 limb_count, cudaStream_t st);
int32_t ntt_forward_launch_map(ckks_ctx* ctx, const u64* in, u64* out, u32 n_polys, LimbMap lm, u32 limb_count,
                               cudaStream_t st);
int32_t ntt_inverse_launch_map(ckks_ctx* ctx, const u64* in, u64* out, u32 n_polys, LimbMap lm, u32 limb_count,
                               cudaStream_t st);
// Optional epilogue of the inverse transform for key-switch accumulators
// [n_ct][n_keys][2][limbs][N]: the b component (even poly p) of ciphertext
// c = p / (2 n_keys) gets P b_c added on its first q_limbs limbs, with
// b_c = b + c * b_stride ([q_limbs][N], coefficient domain) and (P mod q_l,
// Shoup) = (pf[l], pf_q[l]). ModDown then yields ModDown(x) + b_c exactly.
struct InvBase {
    const u64* b = nullptr;
    size_t b_stride = 0;
    u32 n_keys = 1, q_limbs = 0;
    const u64 *pf = nullptr, *pf_q = nullptr;
};
// Optional Galois automorphism folded into the inverse transform of key-switch
// accumulators [n_ct][n_keys][2][limbs][N]: polynomial p leaves as
// sigma_k(INTT(p)) with k = exps[(p / 2) % n_keys] (X^j -> X^(j k), a sign
// flip past N) and exps_inv[g] = k^-1 mod 2N. Pass 1 stores each row with its
// columns permuted (j_lo -> j_lo k mod B); pass 2 reads consecutive permuted
// columns and writes every element to its image row through shared memory.
struct GaloisOut {
    const u64* exps = nullptr;
    const u64* exps_inv = nullptr;
    u32 n_keys = 1;
};
int32_t ntt_inverse_base_launch(ckks_ctx* ctx, const u64* in, u64* out, u32 n_polys, LimbMap lm, u32 limb_count,
                                const InvBase& ib, cudaStream_t st, const GaloisOut& go = GaloisOut{});
// Inverse NTT of key-switch accumulators [polys][q_limbs + K][N] with sigma
// folded (go), fused with the FP64 ModDown into out [polys][q_limbs][N]
// (ntt.cu). Supported when K <= 3, every Q prime is below 2^50 and the
// transform halves have at most 2^8 points.
bool ntt_inverse_moddown_supported(const ckks_ctx* ctx, u32 q_limbs);
int32_t ntt_inverse_moddown_launch(ckks_ctx* ctx, const u64* in, u64* mid, double* words, u64* zp, u64* out,
                                   u32 polys, u32 q_limbs, const GaloisOut& go, cudaStream_t st);
// Times every admissible columns-per-CTA choice of the five NTT passes on a
// scratch batch (limbs x polys) and keeps the fastest in ctx (ntt.cu).
int32_t ntt_autotune(ckks_ctx* ctx, u32 limbs, u32 polys, cudaStream_t st);
inline LimbMap LimbMap::qp(const ckks_ctx* c, u32 q_limbs) { return LimbMap{0, (int)q_limbs, (int)c->L}; }
// Stream-ordered workspace (cudaMallocAsync / cudaFreeAsync on `st`).
template <typename T>
struct Workspace {
    T* p = nullptr;
    cudaStream_t st = nullptr;
    int32_t alloc(size_t count, cudaStream_t s) {
        st = s;
        if (cudaMallocAsync((void**)&p, count * sizeof(T) + 16, s) != cudaSuccess) {
            cudaGetLastError();
            p = nullptr;
            ckks_set_error("out of device memory for a workspace");
            return CKKS_ERR_OOM;
        }
        return CKKS_OK;
    }
    void release() {
        if (p) cudaFreeAsync(p, st);
        p = nullptr;
    }
    ~Workspace() { release(); }
};
