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
 *   - stream: a cudaStream_t passed as void*; NULL selects the context's own
 *     stream. Calls on one context are thread-safe when given distinct
 *     streams, except where noted.
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
/* Host-buffer forms: copy in, transform, copy out (synchronous). */
int32_t ckks_ntt_forward_host(ckks_ctx* ctx, const uint64_t* in_host, uint64_t* out_host, uint32_t n_polys,
                              uint32_t limb_begin, uint32_t limb_count);
int32_t ckks_ntt_inverse_host(ckks_ctx* ctx, const uint64_t* in_host, uint64_t* out_host, uint32_t n_polys,
                              uint32_t limb_begin, uint32_t limb_count);

#ifdef __cplusplus
}
#endif
#endif
