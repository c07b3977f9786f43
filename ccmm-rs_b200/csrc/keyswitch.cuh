// keyswitch.cuh -- key-switching key objects and pipeline entry points.
#pragma once
#include <vector>

#include "kernels.cuh"

// A key-switching key resident in HBM.
//   HYBRID_BOUNDED : entries [D][q_limbs+K][2][N], NTT domain, encrypting
//                    P * B^j * sigma(s) over QP (hybrid_rns_galois_key.rs:61-170)
//   HYBRID_RNS_BLOCK: entries [dnum][q_limbs+K][2][N], encrypting P * E_i * sigma(s)
//   RELIN_BOUNDED  : entries [D][2][q_limbs][N], NTT domain, encrypting B^j * s^2
//                    over Q (bounded_key_switch.rs:22-120)
//   RNS_BLOCK      : entries [dnum][q_limbs][2][N], NTT domain, encrypting
//                    E_i * sigma(s) over Q, no auxiliary limbs (the ordinary RNS
//                    key switch, grafting/rns_key_switch.rs:1155-1258)
//   RELIN_RNS_BLOCK: entries [dnum][2][q_limbs][N], NTT domain, encrypting
//                    E_i * s^2 over Q (RnsMultiplicationKey)
// Galois keys are stored permuted by their own automorphism: slot pi_g(k)
// (ring/ntt_galois_permutation.rs:5-19 source index) holds the reference
// entry of slot k, so the key-switch MAC runs contiguously in the permuted
// index and sigma_g is applied as the final coefficient scatter. Upload and
// download convert from and to the reference layout.
struct ckks_ksk {
    ckks_ctx* ctx = nullptr;
    int kind = 0;
    bool with_p = true;
    u32 q_limbs = 0, base_log = 0, D = 0;
    u64 exponent = 1;
    std::vector<u32> blocks;    // RNS-block sizes
    u64* d_entries = nullptr;
    size_t words = 0;
    u64* d_block_const = nullptr;  // RNS-block ModUp constants
};

u32 ksk_limbs(const ckks_ksk* k);
// A key of the given kind and shape with its entries allocated, not filled
// (bounded kinds; capi_ks.cu).
int32_t ksk_new(ckks_ctx* ctx, int kind, u32 q_limbs, u32 base_log, u64 exponent, ckks_ksk** out, const char* who);
int32_t ksk_alloc(ckks_ctx* ctx, ckks_ksk* key);
// Host-sampled randomness of a key (the reference's ChaCha20 stream, rng.cu):
// e [D][N] one logical error polynomial per entry, a [D][LK][N] uniform
// residues in the coefficient domain (transformed here). Null members: the
// counter-based stream of (seed, tags) is sampled on the GPU instead.
struct KeySamples {
    const i64* e = nullptr;
    const u64* a = nullptr;
};
int32_t ksk_generate(ckks_ctx* ctx, ckks_ksk* key, const int8_t* secret, u64 seed, double sigma,
                     const std::vector<u64>& factors, const std::vector<int8_t>& s_target, bool comp_major, u64 tag_a,
                     u64 tag_e, cudaStream_t st, const u64* d_target_limbs = nullptr,
                     const KeySamples& smp = KeySamples{});
int32_t relin_generate(ckks_ctx* ctx, ckks_ksk* key, const int8_t* secret, u64 seed, double sigma, cudaStream_t st,
                       const KeySamples& smp = KeySamples{});
// Block factors E_i mod q_l = [l in block i] without the auxiliary P (RNS_BLOCK, RELIN_RNS_BLOCK).
std::vector<u64> rns_factors(ckks_ctx* ctx, const ckks_ksk* key);
// Ordinary RNS key-switched Galois automorphism with an RNS_BLOCK key in the
// reference's order: sigma on (b, a), block digits of sigma(a) lifted to every
// Q limb, NTT, MAC with the key plus NTT(sigma(b)), inverse NTT (no ModDown).
// Output c goes to ct_out + c * out_stride words.
int32_t rotate_rns(ckks_ctx* ctx, const ckks_ksk* key, const u64* ct_in, u64* ct_out, u32 n_ct, size_t out_stride,
                   cudaStream_t st);
std::vector<u64> hybrid_factors(ckks_ctx* ctx, const ckks_ksk* key);
std::vector<u64> rnsblock_factors(ckks_ctx* ctx, const ckks_ksk* key);
std::vector<u64> relin_factors(ckks_ctx* ctx, const ckks_ksk* key);
std::vector<int8_t> host_secret_automorphism(const int8_t* s, u32 n, u64 k);
int32_t rnsblock_prepare(ckks_ctx* ctx, ckks_ksk* key);
int32_t rnsblock_modup_launch(ckks_ctx* ctx, const ckks_ksk* key, const u64* a, u64* Y, cudaStream_t st);

// n_ct ciphertexts: Y [n_ct][D][LK][N], base b_stride words apart, acc [n_ct][2][LK][N]
int32_t ks_mac_launch(ckks_ctx* ctx, const u64* Y, const u64* key, const u64* base, u64* acc, u32 q_limbs, u32 D,
                      bool with_p, u64 perm_y, u64 perm_b, cudaStream_t st, u64 perm_key = 0, u32 n_ct = 1,
                      size_t b_stride = 0);
// Galois key entries [D][LK][2][N]: reference layout <-> permuted storage.
int32_t ksk_permute_entries(ckks_ctx* ctx, const u64* src, u64* dst, size_t polys, u64 exponent, bool to_storage,
                            cudaStream_t st);

int32_t rotate_hybrid(ckks_ctx* ctx, const ckks_ksk* key, const u64* ct_in, u64* ct_out, u32 n_ct, cudaStream_t st);
// phase_ms (optional, [8], accumulated): 0 decomposition and digit/base
// transforms, 2 correction lists, 3 key-switch MAC, 4 inverse NTT, 5 ModDown+sigma.
int32_t rotate_hoisted_ntt(ckks_ctx* ctx, const ckks_ksk* const* keys, u32 n_keys, const u64* ct_in, u64* ct_out,
                           u32 n_ct, cudaStream_t st, double* phase_ms = nullptr);
int32_t rotate_hybrid_hoisted(ckks_ctx* ctx, const ckks_ksk* const* keys, u32 n_keys, const u64* ct_in, u64* ct_out,
                              u32 n_ct, cudaStream_t st);

// Ciphertext products (multiply.cu). Layouts: ciphertexts [n][2][L][N],
// quadratic ciphertexts [n][3][L][N], coefficient domain; prepared plaintexts
// [n_plain][L][N], NTT domain.
int32_t tensor_launch(ckks_ctx* ctx, const u64* lhs, const u64* rhs, u64* out, u32 n_ct, u32 L, cudaStream_t st);
int32_t relinearize_launch(ckks_ctx* ctx, const ckks_ksk* key, const u64* quad, u64* out, u32 n_ct, cudaStream_t st);
int32_t multiply_relin_rescale_launch(ckks_ctx* ctx, const ckks_ksk* key, const u64* lhs, const u64* rhs, u64* out,
                                      u32 n_ct, cudaStream_t st);
// Bounded relinearization key sum: c2 [n][L][N] coefficient domain; acc01
// [n][2][L][N] holds the NTT-domain c0, c1 on entry and the NTT-domain
// relinearized (b, a) on return.
// relin_fused: bounded keys over FP64-network limbs take the fused digit-transform
// + key MAC kernel (false: separate transform and MAC launches, the same words).
int32_t relin_core_launch(ckks_ctx* ctx, const ckks_ksk* key, const u64* c2, u64* acc01, u32 n, cudaStream_t st,
                          bool relin_fused = true);
int32_t mul_plain_launch(ckks_ctx* ctx, const u64* ct_in, const u64* plain_ntt, u64* out, u32 n_ct, u32 L,
                         bool plain_per_ct, cudaStream_t st);

// One diagonal-rotation FFT stage (fft.cu): diag_ntt [n_rot + identity][L][N].
// rescale false: the sum stays at level L (scale * plaintext scale).
int32_t fft_stage_launch(ckks_ctx* ctx, const ckks_ksk* const* keys, u32 n_rot, bool identity, const u64* diag_ntt,
                         const u64* ct_in, u64* ct_out, u32 n_ct, u32 L, cudaStream_t st, bool rescale = true);

// Structured CCMM (ccmm.cu): A [k][m], B [n][k], C [n][m] column-major
// ciphertexts [2][L][N] at the key's level L; C one level down.
int32_t ccmm_structured_launch(ckks_ctx* ctx, const ckks_ksk* key, const u64* A, const u64* B, u64* C, u32 m, u32 kd,
                               u32 nd, cudaStream_t st);
// Per-(limb, slot) products of the structured CCMM on the INT8 tensor cores
// (ccmm_tc.cu): At, Bt slot-major canonical residues, m, kd <= 64.
bool ccmm_tc_supported(const ckks_ctx* ctx, u32 m, u32 kd);
int32_t ccmm_slot_tc_launch(ckks_ctx* ctx, const u64* At, const u64* Bt, u64* Ct, u32 L, u32 m, u32 kd, u32 nd,
                            u32 c_begin, u32 nc, int* err, cudaStream_t st);

// Multi-ciphertext diagonal stage: terms_host [n_terms][3] = (output, source, key or n_rot
// for the unrotated source); diag_ntt [n_terms][L][N] in the caller's term order.
int32_t fft_stage_multi_launch(ckks_ctx* ctx, const ckks_ksk* const* keys, u32 n_rot, const u32* terms_host,
                               u32 n_terms, const u64* diag_ntt, const u64* ct_in, u32 n_in, u64* ct_out, u32 n_out,
                               u32 L, cudaStream_t st);

// sampling stream tags (shared with the oracle's restatement)
constexpr u64 TAG_KEY_A = 1ull << 56, TAG_KEY_E = 2ull << 56, TAG_ENC_A = 3ull << 56, TAG_ENC_E = 4ull << 56,
              TAG_RLK_A = 5ull << 56, TAG_RLK_E = 6ull << 56;
