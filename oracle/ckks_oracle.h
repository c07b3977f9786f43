/*
 * ckks_oracle.h -- TEST INFRASTRUCTURE, NOT PRODUCT CODE.
 *
 * CPU restatement of the ccmm-rs ("FHE-rs") reference algorithms on the
 * leveled RNS-CKKS evaluation path. Only the tests, the smoke check and the
 * CPU-baseline leg of bench.py may load this library; the product
 * (libckks_b200.so) never links or calls it.
 *
 * The reference is safe Rust built with cargo, which is absent here, so
 * parity is pinned against the reference's own published constants (prime
 * pools, psi values), its Python oracles (tools/, security/p6a/) and exact
 * big-integer definitions (Python int) in tests/golden.
 *
 * Conventions shared with the product ABI (include/ckks_b200.h):
 *   - residues are canonical u64 in [0, q);
 *   - an RNS polynomial batch is [n_polys][limbs][N] (limb-major);
 *   - a ciphertext is [2][limbs][N]: component b, then component a,
 *     decrypting as b + a*s (grafting/rns_key_switch.rs:380);
 *   - NTT outputs are in natural order: entry k = poly(psi^(2k+1))
 *     (ring/ntt.rs:101-127).
 */
#ifndef CKKS_ORACLE_H
#define CKKS_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ring/ntt_prime.rs, ring/ntt_params.rs, security/p6a/generate_candidates.py */
int32_t  oracle_is_prime(uint64_t value);
uint64_t oracle_find_ntt_prime_below_bits(uint32_t bits, uint32_t degree);
int32_t  oracle_primes_below_bits(uint32_t bits, uint32_t degree, uint32_t count, uint64_t* out);
uint64_t oracle_find_negacyclic_root(uint64_t q, uint32_t degree);
uint64_t oracle_pow_mod(uint64_t base, uint64_t exponent, uint64_t q);
uint64_t oracle_shoup_quotient(uint64_t operand, uint64_t q);
uint64_t oracle_shoup_mul(uint64_t value, uint64_t operand, uint64_t quotient, uint64_t q);
uint64_t oracle_barrett_mul(uint64_t a, uint64_t b, uint64_t q);

/* ring/ntt.rs (O(N^2) definition) and ring/ntt_radix2.rs / ring/prepared_ntt.rs */
void oracle_ntt_forward_reference(uint64_t q, uint32_t degree, const uint64_t* in, uint64_t* out);
void oracle_ntt_inverse_reference(uint64_t q, uint32_t degree, const uint64_t* in, uint64_t* out);
void oracle_ntt_forward(const uint64_t* moduli, uint32_t limbs, uint32_t degree, uint64_t* data, uint32_t n_polys);
void oracle_ntt_inverse(const uint64_t* moduli, uint32_t limbs, uint32_t degree, uint64_t* data, uint32_t n_polys);
void oracle_negacyclic_mul(const uint64_t* moduli, uint32_t limbs, uint32_t degree,
                           const uint64_t* lhs, const uint64_t* rhs, uint64_t* out);
void oracle_pointwise_mul(const uint64_t* moduli, uint32_t limbs, uint32_t degree,
                          const uint64_t* lhs, const uint64_t* rhs, uint64_t* out, uint32_t n_polys);

/* ckks/automorphism.rs, ckks/rns_automorphism.rs, ring/ntt_galois_permutation.rs */
uint64_t oracle_rotation_exponent_left(uint32_t degree, uint64_t steps);
uint64_t oracle_rotation_exponent_right(uint32_t degree, uint64_t steps);
void oracle_automorphism_coef(const uint64_t* moduli, uint32_t limbs, uint32_t degree, uint64_t exponent,
                              const uint64_t* in, uint64_t* out, uint32_t n_polys);
void oracle_automorphism_ntt(uint32_t limbs, uint32_t degree, uint64_t exponent,
                             const uint64_t* in, uint64_t* out, uint32_t n_polys);

/* ckks/rns_rescale.rs:107-167 -- in [n][L][N] -> out [n][L-1][N] */
void oracle_rescale(const uint64_t* moduli, uint32_t limbs, uint32_t degree,
                    const uint64_t* in, uint64_t* out, uint32_t n_polys);

/* ring/auxiliary_modulus.rs:89-171 -- in [n][L+K][N] (Q then P) -> out [n][L][N] */
void oracle_mod_down(const uint64_t* q, uint32_t L, const uint64_t* p, uint32_t K, uint32_t degree,
                     const uint64_t* in, uint64_t* out, uint32_t n_polys);

/* ring/wide_crt.rs:56-111 -- canonical CRT value, little-endian words [N][words] */
uint32_t oracle_crt_words(const uint64_t* moduli, uint32_t limbs);
void oracle_crt_reconstruct(const uint64_t* moduli, uint32_t limbs, uint32_t degree,
                            const uint64_t* poly, uint64_t* words_out);

/* grafting/bounded_gadget.rs:17-118, 273-312 -- digits [D][N] as int64 */
uint32_t oracle_bounded_digit_count(const uint64_t* moduli, uint32_t limbs, uint32_t base_log);
void oracle_bounded_decompose(const uint64_t* moduli, uint32_t limbs, uint32_t degree, uint32_t base_log,
                              const uint64_t* poly, int64_t* digits);
void oracle_bounded_automorphism_hoisted(uint32_t digit_count, uint32_t degree, uint32_t base_log,
                                         uint64_t exponent, const int64_t* in, int64_t* out);

/* grafting/rns_gadget.rs:231-273 -- block digits x mod Q_block, words [blocks][N][words] */
uint32_t oracle_rns_block_words(const uint64_t* moduli, const uint32_t* block_sizes, uint32_t n_blocks);
void oracle_rns_block_decompose(const uint64_t* moduli, uint32_t limbs, const uint32_t* block_sizes,
                                uint32_t n_blocks, uint32_t degree, const uint64_t* poly, uint64_t* words_out);

/* Sampling shared with the product's key generation (counter-based, see oracle source). */
uint64_t oracle_rng_word(uint64_t seed, uint64_t stream, uint64_t index);
int64_t  oracle_gaussian(double sigma, uint64_t seed, uint64_t stream, uint64_t index);
uint64_t oracle_uniform_mod(uint64_t q, uint64_t seed, uint64_t stream, uint64_t index);

/* grafting/rns_key_switch.rs:278-387 (encryption), :906-948 (decryption) */
void oracle_encrypt(const uint64_t* moduli, uint32_t limbs, uint32_t degree, const int8_t* secret,
                    uint64_t seed, double sigma, const uint64_t* message, uint64_t* ct);
void oracle_decrypt(const uint64_t* moduli, uint32_t limbs, uint32_t degree, const int8_t* secret,
                    const uint64_t* ct, uint64_t* message);

/* ckks/hybrid_rns_galois_key.rs:61-170 keygen; :550-780 rotation core.
 * key layout [D][L+K][2][N] (b_ntt, a_ntt), the reference's entries[digit][limb]. */
void oracle_hybrid_key_generate(const uint64_t* q, uint32_t L, const uint64_t* p, uint32_t K, uint32_t degree,
                                uint32_t base_log, const int8_t* secret, uint64_t exponent, uint64_t seed,
                                double sigma, uint64_t* key);
void oracle_hybrid_rotate(const uint64_t* q, uint32_t L, const uint64_t* p, uint32_t K, uint32_t degree,
                          uint32_t base_log, uint64_t exponent, const uint64_t* key,
                          const uint64_t* ct_in, uint64_t* ct_out);
/* Hoisted form: one decomposition, many Galois elements (bounded_gadget.rs:273-312).
 * keys: n_keys pointers; out [n_keys][2][L][N]. */
void oracle_hybrid_rotate_hoisted(const uint64_t* q, uint32_t L, const uint64_t* p, uint32_t K, uint32_t degree,
                                  uint32_t base_log, uint32_t n_keys, const uint64_t* exponents,
                                  const uint64_t* const* keys, const uint64_t* ct_in, uint64_t* ct_out);
/* Timed CPU baseline: n_ct ciphertexts x n_keys Galois elements, threads over ciphertexts. */
void oracle_hybrid_rotate_hoisted_batch(const uint64_t* q, uint32_t L, const uint64_t* p, uint32_t K,
                                        uint32_t degree, uint32_t base_log, uint32_t n_keys,
                                        const uint64_t* exponents, const uint64_t* const* keys,
                                        uint32_t n_ct, const uint64_t* ct_in, uint64_t* ct_out, uint32_t threads);

/* RNS-block ("dnum") hybrid key switching with auxiliary P: composition of
 * grafting/rns_gadget.rs block digits, P-scaled keys (hybrid_rns_galois_key.rs:94-101)
 * and ModDown (auxiliary_modulus.rs:89-171). key layout [dnum][L+K][2][N]. */
void oracle_rnsblock_key_generate(const uint64_t* q, uint32_t L, const uint64_t* p, uint32_t K, uint32_t degree,
                                  const uint32_t* block_sizes, uint32_t n_blocks, const int8_t* secret,
                                  uint64_t exponent, uint64_t seed, double sigma, uint64_t* key);
void oracle_rnsblock_rotate(const uint64_t* q, uint32_t L, const uint64_t* p, uint32_t K, uint32_t degree,
                            const uint32_t* block_sizes, uint32_t n_blocks, uint64_t exponent,
                            const uint64_t* key, const uint64_t* ct_in, uint64_t* ct_out);
// Ordinary RNS key switch without auxiliary limbs (rns_galois_key.rs:439-469,
// rns_key_switch.rs:2438-2524, 1842-1905); the Galois key is
// oracle_rnsblock_key_generate with K = 0.
void oracle_rns_rotate(const uint64_t* q, uint32_t L, uint32_t degree, const uint32_t* block_sizes,
                       uint32_t n_blocks, uint64_t exponent, const uint64_t* key, const uint64_t* ct_in,
                       uint64_t* ct_out);
void oracle_rns_relin_key_generate(const uint64_t* q, uint32_t L, uint32_t degree, const uint32_t* block_sizes,
                                   uint32_t n_blocks, const int8_t* secret, uint64_t seed, double sigma,
                                   uint64_t* key);
void oracle_rns_relinearize(const uint64_t* q, uint32_t L, uint32_t degree, const uint32_t* block_sizes,
                            uint32_t n_blocks, const uint64_t* quad, const uint64_t* key, uint64_t* out);

/* rlwe/quadratic.rs:99-140 -- out [3][L][N] */
void oracle_tensor(const uint64_t* moduli, uint32_t limbs, uint32_t degree,
                   const uint64_t* lhs, const uint64_t* rhs, uint64_t* out);
/* grafting/bounded_key_switch.rs:22-120 keygen (coefficient domain, [D][2][L][N]); :139-223 relinearize */
void oracle_bounded_relin_key_generate(const uint64_t* moduli, uint32_t limbs, uint32_t degree, uint32_t base_log,
                                       const int8_t* secret, uint64_t seed, double sigma, uint64_t* key);
void oracle_bounded_relinearize(const uint64_t* moduli, uint32_t limbs, uint32_t degree, uint32_t base_log,
                                const uint64_t* quadratic, const uint64_t* key, uint64_t* out);
/* ckks/rns_plain_multiply.rs:193-260 -- plaintext in coefficient domain */
void oracle_mul_plain(const uint64_t* moduli, uint32_t limbs, uint32_t degree,
                      const uint64_t* ct, const uint64_t* plain, uint64_t* out);

/* ckks/embedding.rs:57-349 + application_support/ckks.rs:39-62 (encode), :106-130 (decode).
 * slots are interleaved (re, im) doubles, N/2 of them. */
void oracle_slots_to_coefficients(uint32_t degree, const double* slots, double* coefficients);
void oracle_coefficients_to_slots(uint32_t degree, const double* coefficients, double* slots);
void oracle_encode(uint32_t degree, const double* slots, const uint64_t* moduli, uint32_t limbs,
                   double scale, uint64_t* out);
void oracle_decode(uint32_t degree, const uint64_t* moduli, uint32_t limbs, const uint64_t* poly,
                   double scale, double* slots);

/* Seeded ChaCha20 stream of the reference (rand_chacha 0.3.1 ChaCha20Rng,
 * rand_core 0.6.4 seed_from_u64, rand 0.8 gen_range) and the samplers and
 * key generation / encryption that consume it in the reference's order
 * (rlwe/secret_key.rs:25-40, rlwe/error.rs:33-156, rlwe/uniform.rs:12-30,
 * ckks/hybrid_rns_galois_key.rs:61-170, grafting/bounded_key_switch.rs:28-104,
 * grafting/rns_key_switch.rs:278-387). error kind 0 bounded uniform, 1 Gaussian. */
void* oracle_chacha_new(uint64_t seed);
void* oracle_chacha_new_from_seed(const uint8_t* seed32);
void oracle_chacha_free(void* rng);
void oracle_chacha_words(void* rng, uint32_t* out, uint64_t n);
uint64_t oracle_chacha_next_u64(void* rng);
void oracle_chacha_ternary(void* rng, uint32_t n, int8_t* out);
void oracle_chacha_error(void* rng, uint32_t n, int kind, double param, int64_t* out);
void oracle_chacha_uniform(void* rng, uint32_t n, uint64_t q, uint64_t* out);
void oracle_hybrid_key_generate_chacha(const uint64_t* q, uint32_t L, const uint64_t* p, uint32_t K, uint32_t degree,
                                       uint32_t base_log, const int8_t* secret, uint64_t exponent, int kind,
                                       double param, void* rng, uint64_t* key);
void oracle_bounded_relin_key_generate_chacha(const uint64_t* q, uint32_t L, uint32_t degree, uint32_t base_log,
                                              const int8_t* secret, int kind, double param, void* rng,
                                              uint64_t* key);
void oracle_encrypt_chacha(const uint64_t* q, uint32_t L, uint32_t degree, const int8_t* secret, int kind,
                           double param, void* rng, const uint64_t* message, uint64_t* ct);

/* ccmm/park.rs:1405-1434 Mod-PP-MM, Reference backend (row-major). */
void oracle_park_mod_pp_mm(const uint64_t* lhs, const uint64_t* rhs, uint32_t rows, uint32_t inner, uint32_t cols,
                           uint64_t q, uint64_t* out);

#ifdef __cplusplus
}
#endif
#endif
