/*
 * ckks_b200.h -- C ABI of libckks_b200.so, the B200 (sm_100a) implementation
 * of the leveled RNS-CKKS evaluation hot path of ccmm-rs ("FHE-rs").
 *
 * Each entry point names the reference function it replaces (paths are
 * relative to the reference project root). The reference reports errors by
 * panicking (assert!); this library returns a negative status instead and
 * never aborts; ckks_last_error_string() describes the last failure on the
 * calling thread.
 *
 * Data conventions (all device pointers unless a name ends in _host):
 *   - residues: canonical uint64_t in [0, q);
 *   - RNS polynomial batch: [n_polys][limbs][N], limb-major, N contiguous;
 *   - ciphertext: [2][limbs][N] -- component b, then component a; a
 *     ciphertext decrypts as b + a*s (grafting/rns_key_switch.rs:380);
 *   - NTT domain values are in natural order, entry k = poly(psi^(2k+1))
 *     (ring/ntt.rs:101-127), psi found by the reference rule
 *     (ring/ntt_params.rs:16-50);
 *   - a context holds the full basis: Q limbs q_0..q_{L-1} (chain order, the
 *     trailing limb is dropped first by rescale, ring/modulus_chain.rs:19-27)
 *     followed by auxiliary limbs p_0..p_{K-1}. Limb indices in the calls
 *     below index that combined list.
 *   - stream: a cudaStream_t passed as void*; NULL selects the CUDA default
 *     stream. Work is stream-ordered; workspaces come from the stream-ordered
 *     allocator (cudaMallocAsync). Calls on one context are thread-safe when
 *     given distinct streams.
 *   - device: a context belongs to the CUDA device that was current when it
 *     was created; every call that touches device memory must be made with
 *     that device current and returns CKKS_ERR_BAD_ARG otherwise.
 */
#ifndef CKKS_B200_H
#define CKKS_B200_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    CKKS_OK = 0,
    CKKS_ERR_BAD_ARG = -1,
    CKKS_ERR_BASIS_MISMATCH = -2,
    CKKS_ERR_EXPONENT_MISMATCH = -3,
    CKKS_ERR_OOM = -4,
    CKKS_ERR_CUDA = -5,
    CKKS_ERR_TIMEOUT = -6,
    CKKS_ERR_GADGET_CAPACITY = -7
};

typedef struct ckks_ctx ckks_ctx;

/* Last error message of the calling thread ("" when none). */
const char* ckks_last_error_string(void);

/* Library version string. */
const char* ckks_version(void);

/* Parameter search on the host.
 * ckks_primes_below_bits: the first `count` primes q = 1 mod 2*degree below
 * 2^bits in descending order (ring/ntt_prime.rs:65-94 generalised as in
 * security/p6a/generate_candidates.py:53-73, deterministic Miller-Rabin with
 * the witnesses of ring/ntt_prime.rs:28). bits <= 62.
 * ckks_find_negacyclic_root: smallest-generator primitive 2N-th root
 * (ring/ntt_params.rs:16-50); 0 when q is not 1 mod 2N. */
int32_t ckks_primes_below_bits(uint32_t bits, uint32_t degree, uint32_t count, uint64_t* out_host);
uint64_t ckks_find_negacyclic_root(uint64_t q, uint32_t degree);
int32_t ckks_is_prime(uint64_t value);

/* Creates a context for ring degree N = 2^log_n (2 <= log_n <= 17) over the
 * basis q[0..L) followed by p[0..K). Every modulus must be an odd prime below
 * 2^62 with q = 1 mod 2N; they must be pairwise distinct. Precomputes psi by
 * the reference's search (ring/ntt_params.rs:16-50) and the NTT tables
 * (replaces RnsNttPlan::new / PreparedRnsNttPlan::new,
 * ring/rns_ntt.rs:12-35, ring/prepared_rns_ntt.rs:8-84). */
int32_t ckks_ctx_create(uint32_t log_n, const uint64_t* q, uint32_t L, const uint64_t* p, uint32_t K,
                        ckks_ctx** out);
int32_t ckks_ctx_destroy(ckks_ctx* ctx);
/* Selects the key-switch MAC of bounded hoisted rotations and the per-slot
 * products of ckks_ccmm_structured (rows and inner dimension <= 64): enable != 0
 * (the default) runs them on the tcgen05 INT8 tensor cores when the device has
 * them, 0 on CUDA cores (split-operand 64-bit accumulators). Both are
 * bit-exact; the switch exists to compare them. No counterpart in the reference
 * (its MAC is the serial loop of ring/ntt_polynomial.rs:211-236, its CCMM the
 * per-product loop of matrix/rns_ckks_ciphertext.rs:220-318). */
int32_t ckks_ctx_set_tensor_cores(ckks_ctx* ctx, int32_t enable);
/* 1 when bounded hoisted rotations and CCMM products of this context use the
 * tensor cores. */
int32_t ckks_ctx_tensor_cores(const ckks_ctx* ctx);
/* Which path the most recent hoisted rotation MAC (ckks_rotate_hoisted and the
 * calls built on it) or structured CCMM slot product on this context ran: 1 the
 * tcgen05 INT8 tensor cores, 0 the CUDA cores (tensor cores switched off,
 * RNS-block keys, rings below the tensor-core tile, too little free device
 * memory for the packed key set, or CCMM blocks beyond 64 rows or inner
 * entries), -1 neither yet. Diagnostic only; no counterpart in the reference. */
int32_t ckks_ctx_last_mac_path(const ckks_ctx* ctx);
/* Autotuner (no counterpart in the reference, whose NTT has no launch shape):
 * times every admissible columns-per-CTA choice of the five NTT passes
 * (forward 1, forward 1 of signed digits, forward 2, inverse 1, inverse 2) on
 * a scratch batch of `polys` polynomials x `limbs` limbs and keeps the fastest
 * for every later transform of the context. Synchronous. */
int32_t ckks_ctx_autotune(ckks_ctx* ctx, uint32_t limbs, uint32_t polys, void* stream);
/* The autotuner's record (candidates, times, choices) as text, NUL-terminated,
 * truncated to len - 1 characters. */
int32_t ckks_ctx_tuning_report(const ckks_ctx* ctx, char* buf, uint64_t len);
/* Writes the L+K roots psi (host array). */
int32_t ckks_ctx_psi(const ckks_ctx* ctx, uint64_t* psi_host);

/* Forward negacyclic NTT, natural order, of n_polys polynomials over the
 * limbs [limb_begin, limb_begin+limb_count) of the context basis; data
 * layout [n_polys][limb_count][N]. `in` may equal `out`.
 * Replaces PreparedNttPlan::forward/forward_batch (ring/prepared_ntt.rs:156-321)
 * and PreparedRnsNttPlan::forward (ring/prepared_rns_ntt.rs:39-60). */
int32_t ckks_ntt_forward(ckks_ctx* ctx, const uint64_t* in, uint64_t* out, uint32_t n_polys,
                         uint32_t limb_begin, uint32_t limb_count, void* stream);
/* Inverse transform. Replaces PreparedNttPlan::inverse / inverse_prepared_mul
 * (ring/prepared_ntt.rs:327-398), PreparedRnsNttPlan::inverse (:62-83). */
int32_t ckks_ntt_inverse(ckks_ctx* ctx, const uint64_t* in, uint64_t* out, uint32_t n_polys,
                         uint32_t limb_begin, uint32_t limb_count, void* stream);
/* In-place forward NTT that allocates no device memory (no counterpart in
 * the reference). For callers that cannot let a library allocate device
 * memory -- their device memory is reserved up front by their own arena or a
 * serving framework, or their deployment forbids device allocation after
 * start-up. The pass-1 intermediate lives in a fixed 16 MiB device array
 * compiled into the library (resident on every device that loads it until the
 * process exits); batches with n_polys * limb_count * N > 2^21 words are
 * rejected with CKKS_ERR_BAD_ARG. The first call on a device looks up the
 * array's device address (cudaGetSymbolAddress) and keeps it for the process;
 * make that first call before any stream capture, and do not use this entry
 * point on a device after a cudaDeviceReset (the reset reloads the module, so
 * the kept address no longer names the array). All calls share the array:
 * calls whose work overlaps on the GPU race. Output equals ckks_ntt_forward
 * word for word. */
int32_t ckks_ntt_forward_inplace_static(ckks_ctx* ctx, uint64_t* data, uint32_t n_polys, uint32_t limb_begin,
                                        uint32_t limb_count, void* stream);
/* Host-buffer forms: copy in, transform, copy out (synchronous). */
int32_t ckks_ntt_forward_host(ckks_ctx* ctx, const uint64_t* in_host, uint64_t* out_host, uint32_t n_polys,
                              uint32_t limb_begin, uint32_t limb_count);
int32_t ckks_ntt_inverse_host(ckks_ctx* ctx, const uint64_t* in_host, uint64_t* out_host, uint32_t n_polys,
                              uint32_t limb_begin, uint32_t limb_count);


/* ------------------------------------------------------------ ring ops ----
 * Polynomial batches [n_polys][limbs][N] over the context limbs
 * [limb_begin, limb_begin + limbs). */

/* Coefficient-domain Galois automorphism X -> X^k, k odd mod 2N
 * (ckks/automorphism.rs:8-48, ckks/rns_automorphism.rs:12-28). in != out. */
int32_t ckks_automorphism_coef(ckks_ctx* ctx, const uint64_t* in, uint64_t* out, uint32_t n_polys,
                               uint32_t limb_begin, uint32_t limbs, uint64_t exponent, void* stream);
/* NTT-domain automorphism as an index permutation
 * (ring/ntt_galois_permutation.rs:5-19). in != out. */
int32_t ckks_automorphism_ntt(ckks_ctx* ctx, const uint64_t* in, uint64_t* out, uint32_t n_polys,
                              uint32_t limb_begin, uint32_t limbs, uint64_t exponent, void* stream);
/* Galois exponents for slot rotations and conjugation (ckks/automorphism.rs:179-240). */
uint64_t ckks_rotation_exponent_left(uint32_t degree, uint64_t steps);
uint64_t ckks_rotation_exponent_right(uint32_t degree, uint64_t steps);
uint64_t ckks_conjugation_exponent(uint32_t degree);

/* Element-wise out = a op b (op 0: product, NTT domain, ring/ntt_polynomial.rs:186;
 * 1: sum; 2: difference). out may alias a or b. */
int32_t ckks_pointwise(ckks_ctx* ctx, const uint64_t* a, const uint64_t* b, uint64_t* out, uint32_t n_polys,
                       uint32_t limb_begin, uint32_t limbs, int32_t op, void* stream);

/* CKKS rescale: drop the trailing limb of the Q prefix q_0..q_{limbs_in-1}:
 * out_i = ((x_i - centered(x mod q_d)) * q_d^-1) mod q_i, coefficient domain
 * (ckks/rns_rescale.rs:107-167). in [n][limbs_in][N] -> out [n][limbs_in-1][N]. */
int32_t ckks_rescale(ckks_ctx* ctx, const uint64_t* in, uint64_t* out, uint32_t n_polys, uint32_t limbs_in,
                     void* stream);

/* Modulus switch without rescaling: ciphertexts [n_ct][2][limbs_in][N] ->
 * [n_ct][2][limbs_out][N] keeping the leading limbs_out limbs (the lower
 * chain level), scale unchanged. Replaces mod_switch_rns_ckks_to_next
 * (ckks/rns_mod_switch.rs:14-58) for limbs_out = limbs_in - 1 and chains of
 * such switches otherwise. out must not overlap in. */
int32_t ckks_mod_switch(ckks_ctx* ctx, const uint64_t* in, uint64_t* out, uint32_t n_ct, uint32_t limbs_in,
                        uint32_t limbs_out, void* stream);

/* Exact ModDown by P: in [n][q_limbs + K][N] (Q prefix then all K auxiliary
 * limbs, coefficient domain) -> out [n][q_limbs][N]
 * (ring/auxiliary_modulus.rs:89-171 auxiliary_mod_down_rns_candidate). */
int32_t ckks_mod_down(ckks_ctx* ctx, const uint64_t* in, uint64_t* out, uint32_t n_polys, uint32_t q_limbs,
                      void* stream);

/* ------------------------------------------------------------- gadgets ----
 * Balanced base-2^base_log digits (grafting/bounded_gadget.rs): count
 * ceil((bits(Q)+1)/base_log) (:17-37); decomposition of the centred exact CRT
 * value (:59-118) of n_polys polynomials over the Q prefix of q_limbs limbs,
 * digits [n][D][N] as int64; base_log in [1, 62] (the reference allows 63). */
int32_t ckks_bounded_digit_count(ckks_ctx* ctx, uint32_t q_limbs, uint32_t base_log, uint32_t* out);
int32_t ckks_bounded_decompose(ckks_ctx* ctx, const uint64_t* poly, uint32_t n_polys, uint32_t q_limbs,
                               uint32_t base_log, int64_t* digits, void* stream);
/* BoundedGadgetDecomposition::automorphism_hoisted (bounded_gadget.rs:273-312):
 * digits [n][D][N] -> digits of sigma_k of the decomposed value. */
int32_t ckks_bounded_digits_automorphism(ckks_ctx* ctx, const int64_t* in, int64_t* out, uint32_t n_polys,
                                         uint32_t digit_count, uint32_t base_log, uint64_t exponent, void* stream);

/* ------------------------------------------------ key-switching keys -----
 * Key kinds:
 *   CKKS_KSK_HYBRID_BOUNDED : hybrid-QP Galois key, entries [D][q_limbs+K][2][N]
 *     (b_ntt, a_ntt) encrypting P * B^j * sigma(s) -- the reference's
 *     PreparedHybridRnsGaloisKey (ckks/hybrid_rns_galois_key.rs:20-170).
 *   CKKS_KSK_HYBRID_RNS_BLOCK : hybrid Galois key over RNS blocks ("dnum"),
 *     entries [dnum][q_limbs+K][2][N] encrypting P * E_i * sigma(s) with E_i the
 *     CRT idempotent of block i (grafting/rns_gadget.rs:92-135).
 *   CKKS_KSK_RELIN_BOUNDED : bounded relinearization key over Q only,
 *     BoundedRnsMultiplicationKey (grafting/bounded_key_switch.rs:22-120);
 *     uploaded in the reference's coefficient-domain layout [D][2][q_limbs][N],
 *     stored NTT-domain.
 *   CKKS_KSK_RNS_BLOCK : the ordinary RNS Galois key without auxiliary limbs,
 *     PreparedRnsGaloisKey / PreparedRnsKeySwitchKey
 *     (grafting/rns_key_switch.rs:1155-1258, ckks/rns_galois_key.rs): block i
 *     of consecutive Q limbs, entries [dnum][q_limbs][2][N] (b_ntt, a_ntt)
 *     encrypting E_i * sigma(s) over Q (E_i mod q_l = [l in block i]).
 *   CKKS_KSK_RELIN_RNS_BLOCK : the RNS-block relinearization key without
 *     auxiliary limbs, RnsMultiplicationKey (target s^2): uploaded
 *     coefficient-domain [dnum][2][q_limbs][N], stored NTT-domain.
 * Generation samples a counter-based stream (seed) on the GPU: uniform a in
 * the NTT domain, discrete Gaussian e of width sigma shared across limbs;
 * secret_host is the ternary secret (int8 in {-1,0,1}, N entries). */
enum {
    CKKS_KSK_HYBRID_BOUNDED = 0,
    CKKS_KSK_HYBRID_RNS_BLOCK = 1,
    CKKS_KSK_RELIN_BOUNDED = 2,
    CKKS_KSK_RNS_BLOCK = 3,
    CKKS_KSK_RELIN_RNS_BLOCK = 4
};
typedef struct ckks_ksk ckks_ksk;

int32_t ckks_hybrid_key_generate(ckks_ctx* ctx, uint32_t q_limbs, uint32_t base_log, uint64_t exponent,
                                 const int8_t* secret_host, uint64_t seed, double sigma, ckks_ksk** out);
int32_t ckks_hybrid_key_upload(ckks_ctx* ctx, uint32_t q_limbs, uint32_t base_log, uint64_t exponent,
                               const uint64_t* entries_host, ckks_ksk** out);
int32_t ckks_rnsblock_key_generate(ckks_ctx* ctx, uint32_t q_limbs, const uint32_t* block_sizes, uint32_t n_blocks,
                                   uint64_t exponent, const int8_t* secret_host, uint64_t seed, double sigma,
                                   ckks_ksk** out);
int32_t ckks_rnsblock_key_upload(ckks_ctx* ctx, uint32_t q_limbs, const uint32_t* block_sizes, uint32_t n_blocks,
                                 uint64_t exponent, const uint64_t* entries_host, ckks_ksk** out);
/* Ordinary RNS Galois key (no auxiliary limbs) over the Q prefix of q_limbs
 * limbs split into consecutive blocks of block_sizes (1..16 limbs each):
 * replaces PreparedRnsGaloisKey generation (ckks/rns_galois_key.rs with
 * grafting/rns_key_switch.rs:1155-1258); upload takes the reference's
 * NTT-domain entries [dnum][q_limbs][2][N]. */
int32_t ckks_rns_key_generate(ckks_ctx* ctx, uint32_t q_limbs, const uint32_t* block_sizes, uint32_t n_blocks,
                              uint64_t exponent, const int8_t* secret_host, uint64_t seed, double sigma,
                              ckks_ksk** out);
int32_t ckks_rns_key_upload(ckks_ctx* ctx, uint32_t q_limbs, const uint32_t* block_sizes, uint32_t n_blocks,
                            uint64_t exponent, const uint64_t* entries_host, ckks_ksk** out);
/* RNS-block relinearization key without auxiliary limbs (RnsMultiplicationKey,
 * target s^2); upload takes coefficient-domain entries [dnum][2][q_limbs][N]. */
int32_t ckks_rns_relin_key_generate(ckks_ctx* ctx, uint32_t q_limbs, const uint32_t* block_sizes, uint32_t n_blocks,
                                    const int8_t* secret_host, uint64_t seed, double sigma, ckks_ksk** out);
int32_t ckks_rns_relin_key_upload(ckks_ctx* ctx, uint32_t q_limbs, const uint32_t* block_sizes, uint32_t n_blocks,
                                  const uint64_t* entries_host, ckks_ksk** out);
int32_t ckks_relin_key_generate(ckks_ctx* ctx, uint32_t q_limbs, uint32_t base_log, const int8_t* secret_host,
                                uint64_t seed, double sigma, ckks_ksk** out);
int32_t ckks_relin_key_upload(ckks_ctx* ctx, uint32_t q_limbs, uint32_t base_log, const uint64_t* entries_host,
                              ckks_ksk** out);
/* digits/blocks, words of HBM payload, stored entries (NTT domain) to host */
int32_t ckks_ksk_info(const ckks_ksk* key, uint32_t* digits, uint64_t* words);
int32_t ckks_ksk_download(const ckks_ksk* key, uint64_t* entries_host);
int32_t ckks_ksk_destroy(ckks_ksk* key);

/* --------------------------------------------------- Park Mod-PP-MM -----
 * park_mod_pp_mm (ccmm/park.rs:1634-1647, backends :1405-1620): the modular
 * plaintext matrix product out = (lhs x rhs) mod modulus of row-major u64
 * matrices (lhs rows x inner, rhs inner x cols), for any modulus > 1 and any
 * u64 entries: the canonical residue of each exact integer dot product (the
 * reference's Reference backend; the others agree on canonical inputs).
 * Device pointers on the current device (see the backends below); _host: host buffers,
 * synchronous. Empty operands or a modulus below 2 return CKKS_ERR_BAD_ARG. */
int32_t ckks_park_mod_pp_mm(const uint64_t* lhs, const uint64_t* rhs, uint64_t* out, uint32_t rows, uint32_t inner,
                            uint32_t cols, uint64_t modulus, void* stream);
/* park_matrix_mul_with_backend (ccmm/park.rs:1643-1655) for the device
 * backends: AUTO takes the tensor cores (unsigned 8-bit products of the
 * residues' bytes against byte-split weights 2^(8i) rhs mod q, summed exactly
 * in 32 bits; the call waits for its status word, so it returns with the
 * stream drained) and otherwise the CUDA cores (exact 192-bit sums, stream-
 * ordered). Both return the same words. A backend that cannot run returns
 * CKKS_ERR_BAD_ARG; a tensor-core pipeline wait that timed out returns
 * CKKS_ERR_TIMEOUT. The tensor cores take stream-ordered workspace for the
 * packed operands, about nb * rows * inner + nb^2 * inner * cols bytes (nb =
 * bytes of modulus - 1, rows, inner and cols rounded up to their tiles); when
 * it does not fit the call returns CKKS_ERR_OOM and leaves the choice of the
 * CUDA-core backend to the caller. */
enum { CKKS_PARK_AUTO = 0, CKKS_PARK_TENSOR_CORES = 1, CKKS_PARK_CUDA_CORES = 2 };
int32_t ckks_park_mod_pp_mm_with_backend(const uint64_t* lhs, const uint64_t* rhs, uint64_t* out, uint32_t rows,
                                         uint32_t inner, uint32_t cols, uint64_t modulus, int32_t backend,
                                         void* stream);
/* CUDA-event times (ms) of the byte packing and of the GEMM launches of this
 * thread's last tensor-core Park call; CKKS_ERR_BAD_ARG before the first. */
int32_t ckks_park_last_timing(float* pack_ms, float* gemm_ms);
int32_t ckks_park_mod_pp_mm_host(const uint64_t* lhs, const uint64_t* rhs, uint64_t* out, uint32_t rows,
                                 uint32_t inner, uint32_t cols, uint64_t modulus);

/* --------------------------------------------- seeded sampling stream -----
 * The reference draws every secret, error and uniform mask from
 * rand_chacha 0.3.1's ChaCha20Rng (ChaCha20, 64-bit block counter, stream 0)
 * seeded by rand_core 0.6.4's seed_from_u64, through rand 0.8's gen_range.
 * A ckks_rng is that generator, restated on the host: the same seed gives the
 * same keystream words, and the samplers and key generation / encryption
 * below consume them in the reference's order, so keys and ciphertexts made
 * from one seed are the reference's (the sampling is sequential and runs on
 * the host; the arithmetic runs on the GPU). Handles are not thread-safe. */
typedef struct ckks_rng ckks_rng;
enum { CKKS_DIST_BOUNDED_UNIFORM = 0, CKKS_DIST_GAUSSIAN = 1 };
/* ChaCha20Rng::seed_from_u64 / ChaCha20Rng::from_seed (32 bytes). */
int32_t ckks_rng_create(uint64_t seed, ckks_rng** out);
int32_t ckks_rng_create_from_seed(const uint8_t* seed32, ckks_rng** out);
int32_t ckks_rng_destroy(ckks_rng* rng);
/* RngCore::next_u32 / next_u64 (two words, low first); fill: n next words. */
int32_t ckks_rng_next_u32(ckks_rng* rng, uint32_t* out);
int32_t ckks_rng_next_u64(ckks_rng* rng, uint64_t* out);
int32_t ckks_rng_fill_u32(ckks_rng* rng, uint32_t* out, uint64_t n);
/* keystream words consumed so far */
int32_t ckks_rng_word_position(const ckks_rng* rng, uint64_t* out);
/* SecretKey::generate_with_rng (rlwe/secret_key.rs:25-40): gen_range(0u8..3)
 * per coefficient (0, 1, -1), redrawn while all are zero. */
int32_t ckks_rng_ternary_secret(ckks_rng* rng, uint32_t n, int8_t* out);
/* sample_error_coefficients (rlwe/error.rs:33-57): kind BOUNDED_UNIFORM
 * (param = integer bound, gen_range(-bound..=bound)) or GAUSSIAN (param =
 * sigma, the 16-sigma table of :64-113). */
int32_t ckks_rng_error(ckks_rng* rng, uint32_t n, int32_t kind, double param, int64_t* out);
/* sample_uniform_residues (rlwe/uniform.rs:12-30): rejection below 2^64 mod q. */
int32_t ckks_rng_uniform_residues(ckks_rng* rng, uint32_t n, uint64_t modulus, uint64_t* out);
/* PreparedHybridRnsGaloisKey::generate_with_distribution_ntt_rng
 * (ckks/hybrid_rns_galois_key.rs:61-170): per digit one error polynomial,
 * then one uniform a per QP limb, entry = (NTT(target + e) - NTT(a) NTT(s),
 * NTT(a)). */
int32_t ckks_hybrid_key_generate_rng(ckks_ctx* ctx, uint32_t q_limbs, uint32_t base_log, uint64_t exponent,
                                     const int8_t* secret_host, int32_t dist_kind, double dist_param, ckks_rng* rng,
                                     ckks_ksk** out);
/* BoundedRnsMultiplicationKey::generate_with_distribution_ntt_rng
 * (grafting/bounded_key_switch.rs:28-106): entry j encrypts B^j s^2 over Q. */
int32_t ckks_relin_key_generate_rng(ckks_ctx* ctx, uint32_t q_limbs, uint32_t base_log, const int8_t* secret_host,
                                    int32_t dist_kind, double dist_param, ckks_rng* rng, ckks_ksk** out);
/* encrypt_rns_raw_with_distribution_ntt_rng (grafting/rns_key_switch.rs:245-387):
 * message [q_limbs][N] (coefficients) -> ciphertext [2][q_limbs][N] (b, a),
 * b = m + e - a s. Host buffers, synchronous. */
int32_t ckks_encrypt_rng_host(ckks_ctx* ctx, uint32_t q_limbs, const uint64_t* message_host,
                              const int8_t* secret_host, int32_t dist_kind, double dist_param, ckks_rng* rng,
                              uint64_t* ct_host);

/* ---------------------------------------------------------- rotations ----
 * Key-switched Galois automorphism of n_ct ciphertexts [n_ct][2][q_limbs][N]
 * (coefficient domain) with one key; the output stays at the same level.
 * Replaces apply_hybrid_rns_galois_automorphism_{with_prepared_ntt,
 * prepared_qp} and rotate_{left,right}_hybrid_rns_ckks_with_prepared_ntt
 * (ckks/hybrid_rns_galois_key.rs:202-273, 293-521). With a CKKS_KSK_RNS_BLOCK
 * key it is the ordinary RNS key switch in the reference's order: sigma on
 * (b, a), block digits of sigma(a), NTT-domain MAC plus NTT(sigma(b)), inverse
 * NTT, no ModDown (apply_rns_galois_automorphism_with_prepared_ntt,
 * ckks/rns_galois_key.rs:439-469, rns_key_switch_with_prepared_ntt,
 * grafting/rns_key_switch.rs:2438-2524). in != out. */
int32_t ckks_rotate(ckks_ctx* ctx, const ckks_ksk* key, const uint64_t* ct_in, uint64_t* ct_out, uint32_t n_ct,
                    void* stream);
/* Hoisted rotations: one decomposition per ciphertext shared by n_keys Galois
 * keys (all of one kind, level and gadget). out [n_ct][n_keys][2][q_limbs][N].
 * Bounded keys: digits re-normalised per key exactly as
 * BoundedGadgetDecomposition::automorphism_hoisted (bounded_gadget.rs:273-312),
 * so every word equals the non-hoisted rotation. The host waits inside the call
 * only for each group's carry-correction counts and MAC status (to schedule the
 * exact recomputation of any pair whose correction list overflowed); the
 * inverse transforms and ModDown of the last group are still in flight on
 * `stream` when it returns. */
int32_t ckks_rotate_hoisted(ckks_ctx* ctx, const ckks_ksk* const* keys, uint32_t n_keys, const uint64_t* ct_in,
                            uint64_t* ct_out, uint32_t n_ct, void* stream);
/* ckks_rotate_hoisted with per-phase device time in milliseconds (CUDA
 * events on `stream`, summed over ciphertext groups; waits for completion):
 * phase_ms[0] decomposition and the digit/base transforms, [2] carry-correction
 * lists, [3] key-switch MAC, [4] inverse NTT, [5] ModDown and sigma; others 0.
 * The analogue of HybridRotationTiming (ckks/hybrid_rns_galois_key.rs:323-336). */
int32_t ckks_rotate_hoisted_timed(ckks_ctx* ctx, const ckks_ksk* const* keys, uint32_t n_keys, const uint64_t* ct_in,
                                  uint64_t* ct_out, uint32_t n_ct, void* stream, double* phase_ms);
/* Host-buffer form of ckks_rotate_hoisted (copies in, rotates, copies out). */
int32_t ckks_rotate_hoisted_host(ckks_ctx* ctx, const ckks_ksk* const* keys, uint32_t n_keys,
                                 const uint64_t* ct_in_host, uint64_t* ct_out_host, uint32_t n_ct);


/* ------------------------------------------------- ciphertext products ----
 * Layouts: ciphertexts [n_ct][2][q_limbs][N] (b, a), quadratic ciphertexts
 * [n_ct][3][q_limbs][N] (c0, c1, c2), coefficient domain, canonical residues
 * over the Q prefix q_0..q_{q_limbs-1}. Every output word equals the
 * reference's (exact modular arithmetic). */

/* Tensor product of ciphertext pairs: c0 = b1 b2, c1 = b1 a2 + a1 b2,
 * c2 = a1 a2 (negacyclic products per limb). Replaces rns_tensor_with_ntt
 * (grafting/rns_key_switch.rs:1675-1722) and tensor (rlwe/quadratic.rs:70-140).
 * out [n_ct][3][q_limbs][N] must not overlap the inputs. */
int32_t ckks_tensor(ckks_ctx* ctx, const uint64_t* lhs, const uint64_t* rhs, uint64_t* out, uint32_t n_ct,
                    uint32_t q_limbs, void* stream);
/* Bounded relinearization with a CKKS_KSK_RELIN_BOUNDED key of the same
 * level: b = c0 + sum_j d_j k_b[j], a = c1 + sum_j d_j k_a[j] with d_j the
 * balanced base-2^base_log digits of c2. Replaces
 * bounded_rns_relinearize_with_ntt(_observed) (grafting/bounded_key_switch.rs:139-223).
 * With a CKKS_KSK_RELIN_RNS_BLOCK key the digits are the block residues of c2
 * (canonical mod Q_i): rns_relinearize_with_ntt (grafting/rns_key_switch.rs:1842-1905).
 * quad [n_ct][3][L][N] -> out [n_ct][2][L][N] (no overlap). */
int32_t ckks_relinearize(ckks_ctx* ctx, const ckks_ksk* key, const uint64_t* quad, uint64_t* out, uint32_t n_ct,
                         void* stream);
/* Multiply, relinearize, rescale: lhs, rhs [n_ct][2][L][N] at the key's level
 * L >= 2 -> out [n_ct][2][L-1][N]. Replaces
 * multiply_relinearize_rescale_rns_ckks_bounded_with_ntt (ckks/rns_multiply.rs:262-300);
 * the CKKS scale bookkeeping (scale_l * scale_r / q_{L-1}) stays with the caller. */
int32_t ckks_multiply_relin_rescale(ckks_ctx* ctx, const ckks_ksk* key, const uint64_t* lhs, const uint64_t* rhs,
                                    uint64_t* out, uint32_t n_ct, void* stream);
/* Host-buffer form of ckks_multiply_relin_rescale (copies in, runs, copies out). */
int32_t ckks_multiply_relin_rescale_host(ckks_ctx* ctx, const ckks_ksk* key, const uint64_t* lhs_host,
                                         const uint64_t* rhs_host, uint64_t* out_host, uint32_t n_ct);
/* Plaintext multiply: out = INTT(NTT(ct) * plain_ntt) per component and limb.
 * plain_ntt is the NTT-domain plaintext ([n_plain][q_limbs][N], n_plain 1 =
 * one plaintext for every ciphertext, or n_ct), the reference's
 * PreparedRnsPlaintextNtt. Replaces multiply_plain_rns_ckks_with_prepared_ntt
 * (ckks/rns_plain_multiply.rs:193-260); the result scale is scale * plaintext_scale.
 * out may equal ct. */
int32_t ckks_mul_plain(ckks_ctx* ctx, const uint64_t* ct, const uint64_t* plain_ntt, uint64_t* out, uint32_t n_ct,
                       uint32_t q_limbs, uint32_t n_plain, void* stream);


/* One diagonal-rotation stage of the encrypted radix-4 FFT:
 *   out = Rescale( sum_t multiply_plain(rotate(ct, offset_t), diag_t) ).
 * keys: n_rot Galois keys, one per nonzero offset (one kind, level q_limbs
 * and gadget); diag_ntt [n_rot + (identity ? 1 : 0)][q_limbs][N]: the
 * NTT-prepared diagonals in the order of `keys`, then the offset-0 diagonal
 * (applied to the unrotated input) when identity != 0. ct_in
 * [n_ct][2][q_limbs][N] -> ct_out [n_ct][2][q_limbs-1][N]. The rotations of a
 * ciphertext share one hoisted decomposition. Replaces apply_stage /
 * apply_stage_canonical (eblas/prepared_radix4_fft256.rs:744-822); the scale
 * becomes scale * plain_scale / q_{q_limbs-1} with the caller. */
int32_t ckks_fft_stage(ckks_ctx* ctx, const ckks_ksk* const* keys, uint32_t n_rot, int32_t identity,
                       const uint64_t* diag_ntt, const uint64_t* ct_in, uint64_t* ct_out, uint32_t n_ct,
                       uint32_t q_limbs, void* stream);


/* ckks_fft_stage with the rescale optional: rescale == 0 leaves the sum at
 * level q_limbs (ct_out [n_ct][2][q_limbs][N], scale * plaintext scale).
 * With two keys rotating left and right by the same span and the identity
 * term it is the packed radix-2 DIF FFT2 stage
 * (execute_repeated_packed_fft2_dif_stage_cp_hybrid_prepared,
 * eblas/fft.rs:3378-3470: direct, left and right complex-slot diagonals,
 * summed) and, with rescale, its fused-rescale form (:3906-4000). */
int32_t ckks_diag_stage(ckks_ctx* ctx, const ckks_ksk* const* keys, uint32_t n_rot, int32_t identity,
                        const uint64_t* diag_ntt, const uint64_t* ct_in, uint64_t* ct_out, uint32_t n_ct,
                        uint32_t q_limbs, int32_t rescale, void* stream);


/* Structured encrypted matrix product (one ciphertext per entry):
 *   C[r][c] = Rescale( Relinearize( sum_k tensor(A[r][k], B[k][c]) ) )
 * with the bounded relinearization key at the entries' level L = key q_limbs
 * (>= 2). Matrices are column-major arrays of ciphertexts [2][L][N] (entry
 * row + col * rows): A m x k, B k x n, C m x n at level L-1. Requires every Q
 * modulus below 2^60 and 2 * 8 * (m * k + k) bytes of shared memory per slot
 * block (m * k <= 12288). Replaces matmul_structured_bounded_with_ntt(_observed)
 * (matrix/rns_ckks_ciphertext.rs:204-318); results equal it word for word. */
int32_t ckks_ccmm_structured(ckks_ctx* ctx, const ckks_ksk* key, const uint64_t* A, const uint64_t* B, uint64_t* C,
                             uint32_t m, uint32_t k, uint32_t n, void* stream);


/* ------------------------------------------------------ encode / decode ----
 * FP64 canonical embedding on the GPU with the reference's rounding (every
 * double equals the reference operation sequence bit for bit).
 * Encode: n_msg messages of N/2 complex slots (device, interleaved re, im
 * doubles) -> plaintexts [n_msg][q_limbs][N] (device, coefficient domain),
 * round(coefficient * scale) (half away from zero) mod q_l. Replaces
 * encode_rns (application_support/ckks.rs:39-62) with
 * CkksCanonicalEmbedding::slots_to_coefficients (ckks/embedding.rs:261-349). */
int32_t ckks_encode(ckks_ctx* ctx, const double* slots, uint64_t* out, uint32_t n_msg, uint32_t q_limbs, double scale,
                    void* stream);
/* Decode: plaintexts [n_msg][q_limbs][N] -> slots [n_msg][N/2][2] (device):
 * exact CRT, centred, rounded to the nearest double (ties to even), divided by
 * scale, then coefficients_to_slots (ckks/embedding.rs:174-258). Replaces the
 * decode of application_support/ckks.rs:106-130. */
int32_t ckks_decode(ckks_ctx* ctx, const uint64_t* poly, double* slots, uint32_t n_msg, uint32_t q_limbs,
                    double scale, void* stream);


/* Diagonal-rotation stage over several ciphertexts (a stage of a transform
 * whose vectors span n_in ciphertexts, e.g. the last column stage of a 2-D
 * FFT over two ciphertexts):
 *   out[a] = Rescale( sum_{t: terms[t][0] = a} diag_t * rot_{terms[t][2]}(in[terms[t][1]]) )
 * terms_host [n_terms][3] = (output index, input index, key index, or n_rot
 * for the unrotated input); diag_ntt [n_terms][q_limbs][N] NTT-prepared, in
 * term order. Every input is rotated by every key with one hoisted
 * decomposition. ct_in [n_in][2][q_limbs][N] -> ct_out [n_out][2][q_limbs-1][N].
 * With n_in = n_out = 1 it is ckks_fft_stage (eblas/prepared_radix4_fft256.rs:744-822). */
int32_t ckks_fft_stage_multi(ckks_ctx* ctx, const ckks_ksk* const* keys, uint32_t n_rot, const uint32_t* terms_host,
                             uint32_t n_terms, const uint64_t* diag_ntt, const uint64_t* ct_in, uint32_t n_in,
                             uint64_t* ct_out, uint32_t n_out, uint32_t q_limbs, void* stream);

#ifdef __cplusplus
}
#endif
#endif
