// kernels.cuh -- shared device helpers, constant blocks and launcher
// declarations of the elementwise, gadget and key-switching kernels.
#pragma once
#include "context.cuh"

// ring/ntt_galois_permutation.rs:5-19 source index of output i under X -> X^k
CKKS_HD u32 galois_src(u32 i, u64 k, int log_n) {
    u64 mask = (2ull << log_n) - 1;
    u64 rot = (k * (2ull * i + 1)) & mask;
    return (u32)((rot - 1) >> 1);
}

int32_t automorphism_coef_launch(ckks_ctx* ctx, const u64* in, u64* out, u32 n_polys, LimbMap lm, u32 limbs, u64 k,
                                 cudaStream_t st);
int32_t automorphism_ntt_launch(ckks_ctx* ctx, const u64* in, u64* out, u32 n_polys, u32 limbs, u64 k,
                                cudaStream_t st);
int32_t pointwise_launch(ckks_ctx* ctx, const u64* a, const u64* b, u64* out, u32 n_polys, LimbMap lm, u32 limbs,
                         int op, cudaStream_t st);
int32_t rescale_launch(ckks_ctx* ctx, const u64* in, u64* out, u32 n_polys, u32 limbs_in, cudaStream_t st);
int32_t mod_down_launch(ckks_ctx* ctx, const u64* in, u64* out, u32 n_polys, u32 q_limbs, cudaStream_t st);
// ModDown of n_polys polynomials; poly p is then mapped by X -> X^k where
// d_exps_inv[(p / 2) % n_keys] = k^-1 mod 2N (device array; null: no automorphism).
int32_t mod_down_sigma_multi(ckks_ctx* ctx, const u64* in, u64* out, u32 n_polys, u32 q_limbs,
                             const u64* d_exps_inv, u32 n_keys, cudaStream_t st);

// Bounded (balanced base-2^base_log) gadget, grafting/bounded_gadget.rs.
int32_t bounded_digit_count(ckks_ctx* ctx, u32 q_limbs, u32 base_log, u32* out);
// poly_stride: words between consecutive input polynomials (0: q_limbs N, contiguous)
int32_t bounded_decompose_launch(ckks_ctx* ctx, const u64* poly, u32 n_polys, u32 q_limbs, u32 base_log, i64* digits,
                                 u32* flags, cudaStream_t st, size_t poly_stride = 0);
int32_t digits_automorphism_launch(ckks_ctx* ctx, const i64* in, i64* out, u32 n_polys, u32 D, u32 base_log, u64 k,
                                   cudaStream_t st);
// Forward NTT of signed digits lifted to every limb of `lm` ([D][limbs][N] out).
// Bounded relinearization key sum from signed digits [n_ct][D][N] with the
// digit transforms' second pass fused into the key MAC (FP64 networks: every
// limb's prime below 2^50, transform halves of up to 2^8 points).
// mid: workspace [n_ct][D][L][N]; key [D][2][L][N]; base, acc [n_ct][2][L][N].
bool ntt_relin_fused_supported(const ckks_ctx* ctx, u32 L);
int32_t ntt_relin_fused_launch(ckks_ctx* ctx, const i64* digits, u64* mid, const u64* key, const u64* base, u64* acc,
                               u32 n_ct, u32 L, u32 D, cudaStream_t st);
int32_t ntt_forward_digits_launch(ckks_ctx* ctx, const i64* digits, u64* out, u32 D, LimbMap lm, u32 limbs,
                                  cudaStream_t st);

// Exact centred CRT of [n][q_limbs][N] residues to nearest doubles divided by scale ([n][N]).
int32_t crt_to_double_launch(ckks_ctx* ctx, const u64* poly, u32 n_polys, u32 q_limbs, double scale, double* out,
                             cudaStream_t st);

// FP64 canonical embedding (embed.cu).
int32_t encode_launch(ckks_ctx* ctx, const double* slots, u64* out, u32 n_msg, u32 q_limbs, double scale,
                      cudaStream_t st);
int32_t decode_launch(ckks_ctx* ctx, const u64* poly, double* slots, u32 n_msg, u32 q_limbs, double scale,
                      cudaStream_t st);

// Per-context caches of gadget.cu and embed.cu, released by ckks_ctx_destroy.
void gadget_release_ctx(const ckks_ctx* ctx);
void embed_release_ctx(const ckks_ctx* ctx);
// Packed Galois-key sets of the tensor-core MAC (hoisted.cu): all of a context,
// or every set that contains a key (called when the key is destroyed).
struct ckks_ksk;
void keyset_release_ctx(const ckks_ctx* ctx);
void keyset_forget_key(const ckks_ksk* key);
// true on compute capability 10.0 devices (the tcgen05 INT8 key-switch MAC)
bool tc_enabled();
