/*
 * ckks_oracle.cpp -- TEST INFRASTRUCTURE, NOT PRODUCT CODE.
 *
 * CPU restatement of the ccmm-rs reference algorithms on the leveled
 * RNS-CKKS evaluation path, used as the bit-exact checker for the CUDA
 * library and as the timed CPU baseline. Every function cites the reference
 * file:line it restates (paths relative to the reference project root).
 * Exact big-integer steps (CRT, balanced digits, ModDown) use fixed-width
 * little-endian u64 words instead of num-bigint; the integer results are
 * the same by definition.
 *
 * Build: see oracle/Makefile (g++ -O2 -ffp-contract=off, no FMA contraction
 * so the FP64 embedding follows the reference's operation order).
 */
#include "ckks_oracle.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <complex>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <thread>
#include <vector>

typedef uint64_t u64;
typedef int64_t i64;
typedef unsigned __int128 u128;
typedef __int128 i128;

namespace {

// ---------------------------------------------------------------- modulus.rs
inline u64 mul_mod(u64 a, u64 b, u64 q) { return (u64)((u128)a * b % q); }          // modulus.rs:210-214
inline u64 add_mod(u64 a, u64 b, u64 q) { u64 s = a + b; return s >= q ? s - q : s; }  // modulus.rs:150-170 (q < 2^63)
inline u64 sub_mod(u64 a, u64 b, u64 q) { return a >= b ? a - b : q - (b - a); }        // modulus.rs:172-185
inline u64 neg_mod(u64 a, u64 q) { return a == 0 ? 0 : q - a; }                        // modulus.rs:187-196

u64 pow_mod(u64 base, u64 e, u64 q) {  // modulus.rs:233-248
    u64 r = 1 % q;
    base %= q;
    while (e) {
        if (e & 1) r = mul_mod(r, base, q);
        base = mul_mod(base, base, q);
        e >>= 1;
    }
    return r;
}
u64 inv_mod(u64 a, u64 q) { return pow_mod(a % q, q - 2, q); }  // modulus.rs:260-265 (Fermat)

inline u64 shoup_quotient(u64 w, u64 q) { return (u64)(((u128)w << 64) / q); }  // modulus.rs:97-104
inline u64 shoup_mul(u64 x, u64 w, u64 wq, u64 q) {                              // modulus.rs:107-124
    u64 est = (u64)(((u128)x * wq) >> 64);
    u64 r = x * w - est * q;
    return r >= q ? r - q : r;
}

// Signed integer reduced to [0, q) (hybrid_rns_galois_key.rs:55-57 signed_mod = rem_euclid).
inline u64 signed_mod(i64 v, u64 q) {
    i128 r = (i128)v % (i128)q;
    if (r < 0) r += q;
    return (u64)r;
}

// -------------------------------------------------------------- ntt_prime.rs
bool mr_round(u64 n, u64 d, int s, u64 a) {  // ntt_prime.rs miller_rabin_round
    a %= n;
    if (a == 0) return true;
    u64 x = pow_mod(a, d, n);
    if (x == 1 || x == n - 1) return true;
    for (int i = 1; i < s; ++i) {
        x = mul_mod(x, x, n);
        if (x == n - 1) return true;
        if (x == 1) return false;
    }
    return false;
}

bool is_prime_u64(u64 n) {  // ntt_prime.rs:8-47 (u64 branch), generate_candidates.py:16-48
    static const u64 small[] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};
    static const u64 wit[] = {2, 325, 9375, 28178, 450775, 9780504, 1795265022};
    if (n < 2) return false;
    for (u64 p : small) {
        if (n == p) return true;
        if (n % p == 0) return false;
    }
    u64 d = n - 1;
    int s = 0;
    while (!(d & 1)) { d >>= 1; ++s; }
    for (u64 w : wit)
        if (!mr_round(n, d, s, w)) return false;
    return true;
}

// ------------------------------------------------------------- NTT tables
// Restates ring/prepared_ntt.rs:34-110: forward twists psi^j, stage twiddles
// of omega = psi^2 (stage_twiddles :413-434), Shoup companions, inverse
// twiddles of omega^-1 and the untwist n^-1 psi^-j.
struct NttTables {
    u64 q = 0;
    uint32_t n = 0;
    u64 psi = 0, psi_inv = 0, n_inv = 0;
    std::vector<u64> twist, twist_q;          // psi^j
    std::vector<u64> untwist, untwist_q;      // n^-1 psi^-j
    std::vector<std::vector<u64>> fwd_stage, fwd_stage_q, inv_stage, inv_stage_q;
};

u64 find_root(u64 q, uint32_t n) {  // ring/ntt_params.rs:16-50
    if (n == 0 || (n & (n - 1)) || (q - 1) % (2ull * n) != 0) return 0;
    u64 e = (q - 1) / (2ull * n);
    for (u64 g = 2; g < q; ++g) {
        u64 psi = pow_mod(g, e, q);
        if (pow_mod(psi, n, q) == q - 1 && pow_mod(psi, 2ull * n, q) == 1) return psi;
    }
    return 0;
}

std::vector<std::vector<u64>> stage_twiddles(u64 q, uint32_t n, u64 root) {  // prepared_ntt.rs:413-434
    std::vector<std::vector<u64>> st;
    for (uint32_t len = 2; len <= n; len *= 2) {
        u64 step = pow_mod(root, n / len, q), t = 1;
        std::vector<u64> v(len / 2);
        for (uint32_t i = 0; i < len / 2; ++i) { v[i] = t; t = mul_mod(t, step, q); }
        st.push_back(std::move(v));
    }
    return st;
}

std::mutex g_tables_mutex;
std::map<std::pair<u64, uint32_t>, std::shared_ptr<NttTables>> g_tables;

std::shared_ptr<NttTables> tables(u64 q, uint32_t n) {
    std::lock_guard<std::mutex> lock(g_tables_mutex);
    auto key = std::make_pair(q, n);
    auto it = g_tables.find(key);
    if (it != g_tables.end()) return it->second;
    auto t = std::make_shared<NttTables>();
    t->q = q;
    t->n = n;
    t->psi = find_root(q, n);
    if (!t->psi) throw std::runtime_error("modulus is not NTT friendly for this degree");
    t->psi_inv = inv_mod(t->psi, q);
    t->n_inv = inv_mod(n % q, q);
    t->twist.resize(n); t->twist_q.resize(n); t->untwist.resize(n); t->untwist_q.resize(n);
    u64 a = 1, b = t->n_inv;
    for (uint32_t j = 0; j < n; ++j) {
        t->twist[j] = a; t->twist_q[j] = shoup_quotient(a, q);
        t->untwist[j] = b; t->untwist_q[j] = shoup_quotient(b, q);
        a = mul_mod(a, t->psi, q);
        b = mul_mod(b, t->psi_inv, q);
    }
    u64 omega = mul_mod(t->psi, t->psi, q), omega_inv = mul_mod(t->psi_inv, t->psi_inv, q);
    t->fwd_stage = stage_twiddles(q, n, omega);
    t->inv_stage = stage_twiddles(q, n, omega_inv);
    for (auto* pair : {&t->fwd_stage, &t->inv_stage}) {
        auto& dst = (pair == &t->fwd_stage) ? t->fwd_stage_q : t->inv_stage_q;
        for (auto& v : *pair) {
            std::vector<u64> qv(v.size());
            for (size_t i = 0; i < v.size(); ++i) qv[i] = shoup_quotient(v[i], q);
            dst.push_back(std::move(qv));
        }
    }
    g_tables[key] = t;
    return t;
}

void bit_reverse_permute(u64* v, uint32_t n) {  // ntt_radix2.rs bit_reverse_permute
    uint32_t j = 0;
    for (uint32_t i = 1; i < n; ++i) {
        uint32_t bit = n >> 1;
        while (j & bit) { j ^= bit; bit >>= 1; }
        j ^= bit;
        if (i < j) std::swap(v[i], v[j]);
    }
}

// prepared_ntt.rs:531-606 cyclic_ntt_shoup (radix-2 DIT after bit reversal)
void cyclic_ntt(u64* v, uint32_t n, u64 q, const std::vector<std::vector<u64>>& tw,
                const std::vector<std::vector<u64>>& twq) {
    bit_reverse_permute(v, n);
    size_t stage = 0;
    for (uint32_t len = 2; len <= n; len *= 2, ++stage) {
        uint32_t half = len / 2;
        const u64* w = tw[stage].data();
        const u64* wq = twq[stage].data();
        for (uint32_t s = 0; s < n; s += len)
            for (uint32_t o = 0; o < half; ++o) {
                u64 e = v[s + o];
                u64 od = shoup_mul(v[s + o + half], w[o], wq[o], q);
                v[s + o] = add_mod(e, od, q);
                v[s + o + half] = sub_mod(e, od, q);
            }
    }
}

void ntt_forward_1(const NttTables& t, u64* v) {  // prepared_ntt.rs:200-231
    for (uint32_t j = 0; j < t.n; ++j) v[j] = shoup_mul(v[j], t.twist[j], t.twist_q[j], t.q);
    cyclic_ntt(v, t.n, t.q, t.fwd_stage, t.fwd_stage_q);
}

void ntt_inverse_1(const NttTables& t, u64* v) {  // prepared_ntt.rs:327-368 inverse_prepared_mul
    cyclic_ntt(v, t.n, t.q, t.inv_stage, t.inv_stage_q);
    for (uint32_t j = 0; j < t.n; ++j) v[j] = shoup_mul(v[j], t.untwist[j], t.untwist_q[j], t.q);
}

void ntt_forward_poly(u64 q, uint32_t n, u64* v) { ntt_forward_1(*tables(q, n), v); }
void ntt_inverse_poly(u64 q, uint32_t n, u64* v) { ntt_inverse_1(*tables(q, n), v); }

// ------------------------------------------------------- galois / automorphism
u64 automorphism_target(u64 src, u64 k, uint32_t n, bool* negate) {  // ckks/automorphism.rs:29-38
    u64 mapped = (src * k) % (2ull * n);
    *negate = mapped >= n;
    return *negate ? mapped - n : mapped;
}

void automorphism_coef_1(const u64* in, u64* out, uint32_t n, u64 k, u64 q) {  // automorphism.rs:8-48
    for (uint32_t s = 0; s < n; ++s) {
        bool neg;
        u64 t = automorphism_target(s, k, n, &neg);
        out[t] = neg ? neg_mod(in[s], q) : in[s];
    }
}

void automorphism_ntt_1(const u64* in, u64* out, uint32_t n, u64 k) {  // ntt_galois_permutation.rs:5-19
    u64 two_n = 2ull * n;
    k %= two_n;
    for (uint32_t i = 0; i < n; ++i) {
        u64 rotated = (k * (2ull * i + 1)) % two_n;
        out[i] = in[(rotated - 1) / 2];
    }
}

// ------------------------------------------------------------ wide integers
// Little-endian u64 words; fixed capacity per value.
struct Wide {
    std::vector<u64> w;
    explicit Wide(size_t words = 0) : w(words, 0) {}
};

void wide_mul_small_add(u64* x, size_t words, u64 m, u64 a) {  // x = x*m + a
    u128 carry = a;
    for (size_t i = 0; i < words; ++i) {
        u128 t = (u128)x[i] * m + carry;
        x[i] = (u64)t;
        carry = t >> 64;
    }
}

int wide_cmp(const u64* a, const u64* b, size_t words) {
    for (size_t i = words; i-- > 0;) {
        if (a[i] != b[i]) return a[i] < b[i] ? -1 : 1;
    }
    return 0;
}

void wide_sub(u64* a, const u64* b, size_t words) {  // a -= b (a >= b)
    u64 borrow = 0;
    for (size_t i = 0; i < words; ++i) {
        u64 bi = b[i] + borrow;
        u64 nb = (bi < borrow) || (a[i] < bi);
        a[i] = a[i] - bi;
        borrow = nb;
    }
}

void wide_negate(u64* a, size_t words) {  // two's complement
    u64 carry = 1;
    for (size_t i = 0; i < words; ++i) {
        u64 v = ~a[i] + carry;
        carry = (carry && v == 0) ? 1 : 0;
        a[i] = v;
    }
}

u64 wide_mod_small(const u64* x, size_t words, u64 m) {
    u128 r = 0;
    for (size_t i = words; i-- > 0;) r = ((r << 64) | x[i]) % m;
    return (u64)r;
}

// Composite modulus of a basis as words.
std::vector<u64> composite(const u64* moduli, uint32_t count, size_t words) {
    std::vector<u64> Q(words, 0);
    Q[0] = 1;
    for (uint32_t i = 0; i < count; ++i) wide_mul_small_add(Q.data(), words, moduli[i], 0);
    return Q;
}

size_t words_for(const u64* moduli, uint32_t count) {
    double bits = 0;
    for (uint32_t i = 0; i < count; ++i) bits += std::log2((double)moduli[i]);
    return (size_t)(bits / 64.0) + 2;  // headroom for sign and rounding
}

// Exact CRT to the canonical value in [0, Q) (wide_crt.rs:56-92). The
// reference uses an incremental Garner update over BigUint; this restatement
// uses the equivalent mixed-radix Garner form (same unique integer).
struct Garner {
    std::vector<u64> q;
    std::vector<std::vector<u64>> prefix_mod;  // prefix_mod[i][j] = (q_0..q_{j-1}) mod q_i
    std::vector<u64> prefix_inv;               // (q_0..q_{i-1})^-1 mod q_i
    size_t words;
    Garner(const u64* moduli, uint32_t count) : q(moduli, moduli + count) {
        words = words_for(moduli, count);
        prefix_mod.assign(count, std::vector<u64>(count, 0));
        prefix_inv.assign(count, 1);
        for (uint32_t i = 0; i < count; ++i) {
            u64 pm = 1 % q[i];
            for (uint32_t j = 0; j < count; ++j) {
                prefix_mod[i][j] = pm;
                if (j < i) pm = mul_mod(pm, q[j] % q[i], q[i]);
            }
            prefix_inv[i] = inv_mod(prefix_mod[i][i], q[i]);
        }
    }
    // residues r[i] (stride) -> words x (size `words`)
    void reconstruct(const u64* r, size_t stride, u64* x) const {
        uint32_t L = (uint32_t)q.size();
        u64 v[64];
        for (uint32_t i = 0; i < L; ++i) {
            u64 acc = 0;
            for (uint32_t j = 0; j < i; ++j) acc = add_mod(acc, mul_mod(v[j], prefix_mod[i][j], q[i]), q[i]);
            u64 d = sub_mod(r[i * stride] % q[i], acc, q[i]);
            v[i] = mul_mod(d, prefix_inv[i], q[i]);
        }
        // mixed radix -> binary: x = v_{L-1}; x = x*q_i + v_i for i = L-2..0
        std::fill(x, x + words, 0);
        x[0] = v[L - 1];
        for (uint32_t i = L - 1; i-- > 0;) wide_mul_small_add(x, words, q[i], v[i]);
    }
};

// Centered representative in two's complement (wide_crt.rs:96-111: value > Q/2 -> value - Q).
void center(u64* x, const std::vector<u64>& Q, const std::vector<u64>& half, size_t words) {
    if (wide_cmp(x, half.data(), words) > 0) {
        std::vector<u64> t(Q);
        wide_sub(t.data(), x, words);  // Q - x
        std::memcpy(x, t.data(), words * 8);
        wide_negate(x, words);
    }
}

std::vector<u64> half_of(const std::vector<u64>& Q) {
    std::vector<u64> h(Q.size());
    for (size_t i = 0; i < Q.size(); ++i) h[i] = (Q[i] >> 1) | (i + 1 < Q.size() ? (Q[i + 1] << 63) : 0);
    return h;
}

// bits [start, start+len) of a two's complement value (sign extended), len <= 63
u64 wide_bits(const u64* x, size_t words, uint32_t start, uint32_t len) {
    auto word = [&](size_t i) -> u64 { return i < words ? x[i] : ((x[words - 1] >> 63) ? ~0ull : 0ull); };
    size_t wi = start / 64;
    uint32_t off = start % 64;
    u64 lo = word(wi) >> off;
    if (off && off + len > 64) lo |= word(wi + 1) << (64 - off);
    return len == 64 ? lo : (lo & ((1ull << len) - 1));
}

// ---------------------------------------------------- bounded_gadget.rs
uint32_t bit_length(const std::vector<u64>& Q) {
    for (size_t i = Q.size(); i-- > 0;)
        if (Q[i]) return (uint32_t)(i * 64 + 64 - __builtin_clzll(Q[i]));
    return 0;
}

uint32_t digit_count(const u64* q, uint32_t L, uint32_t base_log) {  // bounded_gadget.rs:17-37
    size_t words = words_for(q, L);
    auto Q = composite(q, L, words);
    uint32_t bits = bit_length(Q);
    return (bits + 1 + base_log - 1) / base_log;
}

// decompose_canonical (bounded_gadget.rs:75-118): centered value, balanced
// digits in [-B/2, B/2), value = (value - digit) / B. On the two's
// complement words this is: chunk_j + carry, subtract B when >= B/2.
void decompose_coefficient(const u64* x, size_t words, uint32_t base_log, uint32_t D, i64* out, size_t stride) {
    i64 B = (i64)1 << base_log, half = B / 2;
    i64 carry = 0;
    for (uint32_t j = 0; j < D; ++j) {
        i64 d = (i64)wide_bits(x, words, j * base_log, base_log) + carry;
        if (d >= half) { d -= B; carry = 1; } else { carry = 0; }
        out[j * stride] = d;
    }
    // remaining value must vanish (bounded_gadget.rs:111-114)
    i64 rem = (i64)wide_bits(x, words, D * base_log, 63);
    if (rem & ((u64)1 << 62)) rem |= (i64)((u64)1 << 63);  // sign-extend 63-bit field
    if (rem + carry != 0) throw std::runtime_error("bounded gadget digit count is insufficient");
}

void bounded_decompose(const u64* q, uint32_t L, uint32_t n, uint32_t base_log, const u64* poly, i64* digits) {
    Garner g(q, L);
    auto Q = composite(q, L, g.words);
    auto half = half_of(Q);
    uint32_t D = digit_count(q, L, base_log);
    std::vector<u64> x(g.words);
    for (uint32_t c = 0; c < n; ++c) {
        g.reconstruct(poly + c, n, x.data());
        center(x.data(), Q, half, g.words);
        decompose_coefficient(x.data(), g.words, base_log, D, digits + c, n);
    }
}

// automorphism_hoisted (bounded_gadget.rs:273-312)
void automorphism_hoisted(uint32_t D, uint32_t n, uint32_t base_log, u64 k, const i64* in, i64* out) {
    i128 base = (i128)1 << base_log, half = base / 2;
    k %= 2ull * n;
    for (uint32_t s = 0; s < n; ++s) {
        bool neg;
        u64 t = automorphism_target(s, k, n, &neg);
        if (!neg) {
            for (uint32_t j = 0; j < D; ++j) out[(size_t)j * n + t] = in[(size_t)j * n + s];
            continue;
        }
        i128 carry = 0;
        for (uint32_t j = 0; j < D; ++j) {
            i128 value = -(i128)in[(size_t)j * n + s] + carry;
            i128 m = (value + half) % base;
            if (m < 0) m += base;
            i128 normalized = m - half;
            out[(size_t)j * n + t] = (i64)normalized;
            carry = (value - normalized) / base;
        }
        if (carry != 0) throw std::runtime_error("hoisted digit negation exceeded gadget capacity");
    }
}

// ------------------------------------------------------ rns_gadget.rs
struct BlockLayout {
    std::vector<uint32_t> start, size;
    size_t words = 0;
};

BlockLayout block_layout(const u64* q, const uint32_t* sizes, uint32_t nb) {
    BlockLayout b;
    uint32_t s = 0;
    for (uint32_t i = 0; i < nb; ++i) {
        b.start.push_back(s);
        b.size.push_back(sizes[i]);
        b.words = std::max(b.words, words_for(q + s, sizes[i]));
        s += sizes[i];
    }
    return b;
}

// ------------------------------------------------------------ sampling
// Counter-based generator shared (restated) with the product's key
// generation kernels: splitmix64 finaliser over (seed, stream, index).
inline u64 mix64(u64 z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
inline u64 rng_word(u64 seed, u64 stream, u64 index) {
    return mix64(mix64(seed ^ mix64(stream + 0x9E3779B97F4A7C15ull)) + index * 0x9E3779B97F4A7C15ull);
}
inline u64 uniform_mod(u64 q, u64 seed, u64 stream, u64 index) {
    u128 v = ((u128)rng_word(seed, stream, 2 * index) << 64) | rng_word(seed, stream, 2 * index + 1);
    return (u64)(v % q);
}

// Cumulative distribution table of |e| for a discrete Gaussian of width
// sigma, tail cut at ceil(12 sigma), in 63-bit fixed point.
std::vector<u64> cdt_table(double sigma) {
    int T = (int)std::ceil(12.0 * sigma);
    std::vector<double> rho(T + 1);
    double S = 0;
    for (int k = 0; k <= T; ++k) {
        rho[k] = std::exp(-(double)k * k / (2.0 * sigma * sigma));
        S += k ? 2.0 * rho[k] : rho[k];
    }
    std::vector<u64> cdt(T + 1);
    double c = 0;
    for (int k = 0; k <= T; ++k) {
        c += (k ? 2.0 * rho[k] : rho[k]) / S;
        double v = std::ldexp(c, 63);
        cdt[k] = v >= 9223372036854775807.0 ? (1ull << 63) : (u64)v;
    }
    cdt[T] = 1ull << 63;
    return cdt;
}
inline i64 gaussian_from(const std::vector<u64>& cdt, u64 word) {
    u64 v = word >> 1;
    i64 k = 0;
    while ((size_t)k + 1 < cdt.size() && v >= cdt[k]) ++k;
    return (word & 1) ? -k : k;
}

// Stream tags (high bits) for independent sampling domains.
constexpr u64 TAG_KEY_A = 1ull << 56, TAG_KEY_E = 2ull << 56, TAG_ENC_A = 3ull << 56, TAG_ENC_E = 4ull << 56,
              TAG_RLK_A = 5ull << 56, TAG_RLK_E = 6ull << 56;

// ------------------------------------------------------------ helpers
std::vector<u64> secret_ntt(const u64* q, uint32_t L, uint32_t n, const int8_t* s) {
    std::vector<u64> out((size_t)L * n);
    for (uint32_t l = 0; l < L; ++l) {
        for (uint32_t c = 0; c < n; ++c) out[(size_t)l * n + c] = signed_mod(s[c], q[l]);
        ntt_forward_poly(q[l], n, &out[(size_t)l * n]);
    }
    return out;
}

// ternary secret automorphism (hybrid_rns_galois_key.rs:29-53)
std::vector<int8_t> secret_automorphism(const int8_t* s, uint32_t n, u64 k) {
    std::vector<int8_t> o(n, 0);
    for (uint32_t i = 0; i < n; ++i) {
        bool neg;
        u64 t = automorphism_target(i, k, n, &neg);
        o[t] = neg ? (int8_t)-s[i] : s[i];
    }
    return o;
}

// One RLWE encryption in the NTT domain of `target` (coefficient domain, per
// limb) under secret_ntt: a uniform (sampled in the NTT domain), e Gaussian
// shared across limbs; b = target + e - a*s. Output NTT-domain (b, a) pairs.
void rlwe_encrypt_ntt(const u64* q, uint32_t L, uint32_t n, const std::vector<u64>& s_ntt, const u64* target,
                      u64 seed, u64 tag_a, u64 tag_e, u64 entry, const std::vector<u64>& cdt, u64* b_out,
                      size_t b_stride, u64* a_out, size_t a_stride) {
    std::vector<i64> e(n);
    for (uint32_t c = 0; c < n; ++c) e[c] = gaussian_from(cdt, rng_word(seed, tag_e | entry, c));
    std::vector<u64> t(n);
    for (uint32_t l = 0; l < L; ++l) {
        u64 m = q[l];
        for (uint32_t c = 0; c < n; ++c) t[c] = add_mod(target[(size_t)l * n + c], signed_mod(e[c], m), m);
        ntt_forward_poly(m, n, t.data());
        u64* bo = b_out + l * b_stride;
        u64* ao = a_out + l * a_stride;
        u64 stream = tag_a | (entry << 16) | l;
        for (uint32_t c = 0; c < n; ++c) {
            u64 a = uniform_mod(m, seed, stream, c);
            ao[c] = a;
            bo[c] = sub_mod(t[c], mul_mod(a, s_ntt[(size_t)l * n + c], m), m);
        }
    }
}

// Exact ModDown (auxiliary_modulus.rs:89-171) of one QP polynomial.
struct ModDown {
    std::vector<u64> q, p;
    Garner gp;
    std::vector<u64> P, Phalf, p_mod_q, p_inv_q;
    ModDown(const u64* q_, uint32_t L, const u64* p_, uint32_t K) : q(q_, q_ + L), p(p_, p_ + K), gp(p_, K) {
        P = composite(p_, K, gp.words);
        Phalf = half_of(P);
        for (uint32_t i = 0; i < L; ++i) {
            p_mod_q.push_back(wide_mod_small(P.data(), P.size(), q[i]));
            p_inv_q.push_back(inv_mod(p_mod_q.back(), q[i]));
        }
    }
    void apply(const u64* in, u64* out, uint32_t n) const {
        uint32_t L = (uint32_t)q.size();
        std::vector<u64> x(gp.words);
        for (uint32_t c = 0; c < n; ++c) {
            gp.reconstruct(in + (size_t)L * n + c, n, x.data());
            bool neg = wide_cmp(x.data(), Phalf.data(), gp.words) > 0;
            std::vector<u64> mag(x);
            if (neg) {
                mag = P;
                wide_sub(mag.data(), x.data(), gp.words);  // P - x = |x - P|
            }
            for (uint32_t i = 0; i < L; ++i) {
                u64 r = wide_mod_small(mag.data(), gp.words, q[i]);
                if (neg) r = neg_mod(r, q[i]);
                u64 diff = sub_mod(in[(size_t)i * n + c], r, q[i]);
                out[(size_t)i * n + c] = mul_mod(diff, p_inv_q[i], q[i]);
            }
        }
    }
};

std::vector<u64> qp_moduli(const u64* q, uint32_t L, const u64* p, uint32_t K) {
    std::vector<u64> m(q, q + L);
    m.insert(m.end(), p, p + K);
    return m;
}

// Hybrid-QP key switch after decomposition: base term P*sigma(b) on the Q limbs,
// per QP limb: NTT(base) + sum_j NTT(signed_mod(d_j)) * key[j][limb], INTT,
// ModDown (hybrid_rns_galois_key.rs:620-780).
void hybrid_switch(const u64* q, uint32_t L, const u64* p, uint32_t K, uint32_t n, uint32_t D,
                   const i64* digits, const u64* key, const u64* sb, u64* out) {
    auto m = qp_moduli(q, L, p, K);
    uint32_t LK = L + K;
    std::vector<u64> acc_b((size_t)LK * n), acc_a((size_t)LK * n), dig(n);
    for (uint32_t l = 0; l < LK; ++l) {
        u64 mod = m[l];
        u64* bb = &acc_b[(size_t)l * n];
        u64* aa = &acc_a[(size_t)l * n];
        if (l < L) {
            u64 pf = 1;
            for (uint32_t k = 0; k < K; ++k) pf = mul_mod(pf, p[k] % mod, mod);
            for (uint32_t c = 0; c < n; ++c) bb[c] = mul_mod(sb[(size_t)l * n + c], pf, mod);
            ntt_forward_poly(mod, n, bb);
        } else {
            std::fill(bb, bb + n, 0);
        }
        std::fill(aa, aa + n, 0);
        for (uint32_t j = 0; j < D; ++j) {
            for (uint32_t c = 0; c < n; ++c) dig[c] = signed_mod(digits[(size_t)j * n + c], mod);
            ntt_forward_poly(mod, n, dig.data());
            const u64* kb = key + (((size_t)j * LK + l) * 2 + 0) * n;
            const u64* ka = key + (((size_t)j * LK + l) * 2 + 1) * n;
            for (uint32_t c = 0; c < n; ++c) {  // ntt_polynomial.rs:222-236
                bb[c] = add_mod(bb[c], mul_mod(dig[c], kb[c], mod), mod);
                aa[c] = add_mod(aa[c], mul_mod(dig[c], ka[c], mod), mod);
            }
        }
        ntt_inverse_poly(mod, n, bb);
        ntt_inverse_poly(mod, n, aa);
    }
    ModDown md(q, L, p, K);
    md.apply(acc_b.data(), out, n);
    md.apply(acc_a.data(), out + (size_t)L * n, n);
}

// ------------------------------------------------------------ embedding.rs
typedef std::complex<double> cplx;
inline cplx cmul(cplx a, cplx b) {  // num-complex Mul: (ac - bd) + (ad + bc)i
    return cplx(a.real() * b.real() - a.imag() * b.imag(), a.real() * b.imag() + a.imag() * b.real());
}
inline cplx from_polar1(double angle) { return cplx(1.0 * std::cos(angle), 1.0 * std::sin(angle)); }

void radix2_dft_in_place(std::vector<cplx>& v, double sign) {  // embedding.rs:57-117
    size_t n = v.size();
    size_t j = 0;
    for (size_t i = 1; i < n; ++i) {
        size_t bit = n >> 1;
        while (j & bit) { j ^= bit; bit >>= 1; }
        j ^= bit;
        if (i < j) std::swap(v[i], v[j]);
    }
    for (size_t len = 2; len <= n; len *= 2) {
        double angle = sign * 2.0 * M_PI / (double)len;
        cplx root = from_polar1(angle);
        size_t half = len / 2;
        for (size_t s = 0; s < n; s += len) {
            cplx tw(1.0, 0.0);
            for (size_t o = 0; o < half; ++o) {
                cplx even = v[s + o];
                cplx odd = cmul(v[s + o + half], tw);
                v[s + o] = cplx(even.real() + odd.real(), even.imag() + odd.imag());
                v[s + o + half] = cplx(even.real() - odd.real(), even.imag() - odd.imag());
                tw = cmul(tw, root);
            }
        }
    }
}

std::vector<size_t> slot_root_indices(uint32_t n) {  // embedding.rs:119-158
    std::vector<size_t> r;
    u64 e = 1, two_n = 2ull * n;
    for (uint32_t i = 0; i < n / 2; ++i) {
        r.push_back((e - 1) / 2);
        e = (e * 5) % two_n;
    }
    return r;
}

void slots_to_coeffs(uint32_t n, const double* slots, double* coeffs) {  // embedding.rs:261-349
    auto idx = slot_root_indices(n);
    std::vector<cplx> ev(n, cplx(0.0, 0.0));
    for (uint32_t i = 0; i < n / 2; ++i) {
        cplx s(slots[2 * i], slots[2 * i + 1]);
        ev[idx[i]] = s;
        ev[n - 1 - idx[i]] = std::conj(s);
    }
    radix2_dft_in_place(ev, -1.0);
    double norm = 1.0 / (double)n;
    cplx izeta = from_polar1(-M_PI / (double)n);
    cplx tw(1.0, 0.0);
    for (uint32_t c = 0; c < n; ++c) {
        cplx t(ev[c].real() * norm, ev[c].imag() * norm);
        cplx co = cmul(t, tw);
        tw = cmul(tw, izeta);
        coeffs[c] = co.real();
    }
}

void coeffs_to_slots(uint32_t n, const double* coeffs, double* slots) {  // embedding.rs:174-258
    cplx zeta = from_polar1(M_PI / (double)n);
    cplx tw(1.0, 0.0);
    std::vector<cplx> ev(n);
    for (uint32_t c = 0; c < n; ++c) {
        ev[c] = cmul(cplx(coeffs[c], 0.0), tw);
        tw = cmul(tw, zeta);
    }
    radix2_dft_in_place(ev, 1.0);
    auto idx = slot_root_indices(n);
    for (uint32_t i = 0; i < n / 2; ++i) {
        slots[2 * i] = ev[idx[i]].real();
        slots[2 * i + 1] = ev[idx[i]].imag();
    }
}

// Correctly rounded conversion of a two's complement wide integer to double
// (the reference's num-bigint to_f64 is unpinned; round-half-even is used).
double wide_to_double(const u64* x, size_t words) {
    bool neg = (x[words - 1] >> 63) != 0;
    std::vector<u64> m(x, x + words);
    if (neg) wide_negate(m.data(), words);
    int top = -1;
    for (size_t i = words; i-- > 0;)
        if (m[i]) { top = (int)(i * 64 + 63 - __builtin_clzll(m[i])); break; }
    if (top < 0) return 0.0;
    double r;
    if (top < 64) {
        r = (double)m[0];  // hardware conversion rounds to nearest even
    } else {
        // leading 64 bits with a sticky bit for everything below: the
        // conversion then rounds exactly as the full value would.
        uint32_t shift = (uint32_t)top - 63;
        u64 lead = wide_bits(m.data(), words, shift, 64);
        bool sticky = false;
        for (uint32_t b = 0; b < shift && !sticky; b += 64) {
            uint32_t len = std::min<uint32_t>(64, shift - b);
            if (wide_bits(m.data(), words, b, len)) sticky = true;
        }
        if (sticky) lead |= 1;
        r = std::ldexp((double)lead, (int)shift);
    }
    return neg ? -r : r;
}

}  // namespace

// =================================================================== C ABI
extern "C" {

int32_t oracle_is_prime(uint64_t v) { return is_prime_u64(v) ? 1 : 0; }

uint64_t oracle_find_ntt_prime_below_bits(uint32_t bits, uint32_t degree) {  // ntt_prime.rs:65-94
    if (bits < 2 || bits > 64 || degree < 2 || (degree & (degree - 1))) return 0;
    u64 two_n = 2ull * degree;
    u64 cand = bits == 64 ? ~0ull : ((1ull << bits) - 1);
    cand -= (cand - 1) % two_n;
    for (;;) {
        if (cand > 2 && (cand - 1) % two_n == 0 && is_prime_u64(cand)) return cand;
        if (cand <= two_n + 1) return 0;
        cand -= two_n;
    }
}

int32_t oracle_primes_below_bits(uint32_t bits, uint32_t degree, uint32_t count, uint64_t* out) {
    // security/p6a/generate_candidates.py:53-73
    if (bits < 2 || bits > 63 || degree < 2) return -1;
    u64 two_n = 2ull * degree;
    u64 cand = (1ull << bits) - 1;
    cand -= (cand - 1) % two_n;
    uint32_t found = 0;
    while (cand > two_n + 1 && found < count) {
        if (is_prime_u64(cand)) out[found++] = cand;
        cand -= two_n;
    }
    return found == count ? 0 : -1;
}

uint64_t oracle_find_negacyclic_root(uint64_t q, uint32_t degree) { return find_root(q, degree); }
uint64_t oracle_pow_mod(uint64_t b, uint64_t e, uint64_t q) { return pow_mod(b, e, q); }
uint64_t oracle_shoup_quotient(uint64_t w, uint64_t q) { return shoup_quotient(w, q); }
uint64_t oracle_shoup_mul(uint64_t x, uint64_t w, uint64_t wq, uint64_t q) { return shoup_mul(x, w, wq, q); }

uint64_t oracle_barrett_mul(uint64_t a, uint64_t b, uint64_t q) {  // modulus.rs:9-88 PreparedModulus
    u128 qq = q;
    u128 recip = (~(u128)0) / qq;
    if ((~(u128)0) % qq == qq - 1) recip += 1;
    u128 x = (u128)a * b;
    u128 x_hi = x >> 64, x_lo = (u64)x;
    u128 r_hi = recip >> 64, r_lo = (u64)recip;
    u128 p0 = x_lo * r_lo, p1 = x_lo * r_hi, p2 = x_hi * r_lo, p3 = x_hi * r_hi;
    u128 mask = ((u128)1 << 64) - 1;
    u128 carry = ((p0 >> 64) + (p1 & mask) + (p2 & mask)) >> 64;
    u128 quot = p3 + (p1 >> 64) + (p2 >> 64) + carry;
    u128 red = x - quot * qq;
    while (red >= qq) red -= qq;
    return (u64)red;
}

void oracle_ntt_forward_reference(uint64_t q, uint32_t n, const uint64_t* in, uint64_t* out) {  // ntt.rs:106-127
    u64 psi = find_root(q, n);
    for (uint32_t k = 0; k < n; ++k) {
        u64 point = pow_mod(psi, 2ull * k + 1, q), power = 1, sum = 0;
        for (uint32_t j = 0; j < n; ++j) {
            sum = add_mod(sum, mul_mod(in[j] % q, power, q), q);
            power = mul_mod(power, point, q);
        }
        out[k] = sum;
    }
}

void oracle_ntt_inverse_reference(uint64_t q, uint32_t n, const uint64_t* in, uint64_t* out) {  // ntt.rs:133-159
    u64 psi_inv = inv_mod(find_root(q, n), q), n_inv = inv_mod(n % q, q);
    for (uint32_t j = 0; j < n; ++j) {
        u64 sum = 0;
        for (uint32_t k = 0; k < n; ++k)
            sum = add_mod(sum, mul_mod(in[k] % q, pow_mod(psi_inv, (u64)(2ull * k + 1) * j % (2ull * n), q), q), q);
        out[j] = mul_mod(sum, n_inv, q);
    }
}

void oracle_ntt_forward(const uint64_t* q, uint32_t L, uint32_t n, uint64_t* data, uint32_t n_polys) {
    for (uint32_t p = 0; p < n_polys; ++p)
        for (uint32_t l = 0; l < L; ++l) ntt_forward_poly(q[l], n, data + ((size_t)p * L + l) * n);
}

void oracle_ntt_inverse(const uint64_t* q, uint32_t L, uint32_t n, uint64_t* data, uint32_t n_polys) {
    for (uint32_t p = 0; p < n_polys; ++p)
        for (uint32_t l = 0; l < L; ++l) ntt_inverse_poly(q[l], n, data + ((size_t)p * L + l) * n);
}

void oracle_negacyclic_mul(const uint64_t* q, uint32_t L, uint32_t n, const uint64_t* lhs, const uint64_t* rhs,
                           uint64_t* out) {  // ntt_radix2.rs negacyclic_mul
    std::vector<u64> a(n), b(n);
    for (uint32_t l = 0; l < L; ++l) {
        std::copy(lhs + (size_t)l * n, lhs + (size_t)(l + 1) * n, a.begin());
        std::copy(rhs + (size_t)l * n, rhs + (size_t)(l + 1) * n, b.begin());
        ntt_forward_poly(q[l], n, a.data());
        ntt_forward_poly(q[l], n, b.data());
        for (uint32_t c = 0; c < n; ++c) a[c] = mul_mod(a[c], b[c], q[l]);
        ntt_inverse_poly(q[l], n, a.data());
        std::copy(a.begin(), a.end(), out + (size_t)l * n);
    }
}

void oracle_pointwise_mul(const uint64_t* q, uint32_t L, uint32_t n, const uint64_t* lhs, const uint64_t* rhs,
                          uint64_t* out, uint32_t n_polys) {
    for (uint32_t p = 0; p < n_polys; ++p)
        for (uint32_t l = 0; l < L; ++l)
            for (uint32_t c = 0; c < n; ++c) {
                size_t i = ((size_t)p * L + l) * n + c;
                out[i] = mul_mod(lhs[i], rhs[i], q[l]);
            }
}

uint64_t oracle_rotation_exponent_left(uint32_t n, uint64_t steps) {  // automorphism.rs:179-192
    u64 slots = n / 2;
    steps %= slots;
    u64 r = 1, b = 5 % (2ull * n);
    while (steps) {
        if (steps & 1) r = r * b % (2ull * n);
        b = b * b % (2ull * n);
        steps >>= 1;
    }
    return r;
}

uint64_t oracle_rotation_exponent_right(uint32_t n, uint64_t steps) {  // automorphism.rs:195-207
    u64 slots = n / 2;
    steps %= slots;
    return oracle_rotation_exponent_left(n, (slots - steps) % slots);
}

void oracle_automorphism_coef(const uint64_t* q, uint32_t L, uint32_t n, uint64_t k, const uint64_t* in,
                              uint64_t* out, uint32_t n_polys) {
    for (uint32_t p = 0; p < n_polys; ++p)
        for (uint32_t l = 0; l < L; ++l)
            automorphism_coef_1(in + ((size_t)p * L + l) * n, out + ((size_t)p * L + l) * n, n, k, q[l]);
}

void oracle_automorphism_ntt(uint32_t L, uint32_t n, uint64_t k, const uint64_t* in, uint64_t* out,
                             uint32_t n_polys) {
    for (uint32_t p = 0; p < n_polys; ++p)
        for (uint32_t l = 0; l < L; ++l)
            automorphism_ntt_1(in + ((size_t)p * L + l) * n, out + ((size_t)p * L + l) * n, n, k);
}

void oracle_rescale(const uint64_t* q, uint32_t L, uint32_t n, const uint64_t* in, uint64_t* out,
                    uint32_t n_polys) {  // rns_rescale.rs:107-167
    u64 qd = q[L - 1];
    for (uint32_t p = 0; p < n_polys; ++p) {
        const u64* src = in + (size_t)p * L * n;
        u64* dst = out + (size_t)p * (L - 1) * n;
        const u64* dropped = src + (size_t)(L - 1) * n;
        for (uint32_t i = 0; i + 1 < L; ++i) {
            u64 qi = q[i], inv = inv_mod(qd % qi, qi);
            for (uint32_t c = 0; c < n; ++c) {
                u64 r = dropped[c];
                i128 centered = r > qd / 2 ? (i128)r - (i128)qd : (i128)r;
                u64 rq;
                if (centered >= 0) rq = (u64)((u128)centered % qi);
                else {
                    u64 mag = (u64)((u128)(-centered) % qi);
                    rq = mag == 0 ? 0 : qi - mag;
                }
                dst[(size_t)i * n + c] = mul_mod(sub_mod(src[(size_t)i * n + c], rq, qi), inv, qi);
            }
        }
    }
}

void oracle_mod_down(const uint64_t* q, uint32_t L, const uint64_t* p, uint32_t K, uint32_t n, const uint64_t* in,
                     uint64_t* out, uint32_t n_polys) {
    ModDown md(q, L, p, K);
    for (uint32_t i = 0; i < n_polys; ++i) md.apply(in + (size_t)i * (L + K) * n, out + (size_t)i * L * n, n);
}

uint32_t oracle_crt_words(const uint64_t* q, uint32_t L) { return (uint32_t)words_for(q, L); }

void oracle_crt_reconstruct(const uint64_t* q, uint32_t L, uint32_t n, const uint64_t* poly, uint64_t* words_out) {
    Garner g(q, L);
    for (uint32_t c = 0; c < n; ++c) g.reconstruct(poly + c, n, words_out + (size_t)c * g.words);
}

uint32_t oracle_bounded_digit_count(const uint64_t* q, uint32_t L, uint32_t base_log) {
    return digit_count(q, L, base_log);
}

void oracle_bounded_decompose(const uint64_t* q, uint32_t L, uint32_t n, uint32_t base_log, const uint64_t* poly,
                              int64_t* digits) {
    bounded_decompose(q, L, n, base_log, poly, digits);
}

void oracle_bounded_automorphism_hoisted(uint32_t D, uint32_t n, uint32_t base_log, uint64_t k, const int64_t* in,
                                         int64_t* out) {
    automorphism_hoisted(D, n, base_log, k, in, out);
}

uint32_t oracle_rns_block_words(const uint64_t* q, const uint32_t* sizes, uint32_t nb) {
    return (uint32_t)block_layout(q, sizes, nb).words;
}

void oracle_rns_block_decompose(const uint64_t* q, uint32_t L, const uint32_t* sizes, uint32_t nb, uint32_t n,
                                const uint64_t* poly, uint64_t* words_out) {  // rns_gadget.rs:143-228
    (void)L;
    BlockLayout b = block_layout(q, sizes, nb);
    for (uint32_t i = 0; i < nb; ++i) {
        Garner g(q + b.start[i], b.size[i]);
        std::vector<u64> x(g.words);
        for (uint32_t c = 0; c < n; ++c) {
            g.reconstruct(poly + (size_t)b.start[i] * n + c, n, x.data());
            u64* dst = words_out + ((size_t)i * n + c) * b.words;
            std::fill(dst, dst + b.words, 0);
            std::copy(x.begin(), x.begin() + std::min(g.words, b.words), dst);
        }
    }
}

uint64_t oracle_rng_word(uint64_t seed, uint64_t stream, uint64_t index) { return rng_word(seed, stream, index); }
int64_t oracle_gaussian(double sigma, uint64_t seed, uint64_t stream, uint64_t index) {
    static std::mutex m;
    static std::map<double, std::vector<u64>> cache;
    std::lock_guard<std::mutex> lock(m);
    auto it = cache.find(sigma);
    if (it == cache.end()) it = cache.emplace(sigma, cdt_table(sigma)).first;
    return gaussian_from(it->second, rng_word(seed, stream, index));
}
uint64_t oracle_uniform_mod(uint64_t q, uint64_t seed, uint64_t stream, uint64_t index) {
    return uniform_mod(q, seed, stream, index);
}

void oracle_encrypt(const uint64_t* q, uint32_t L, uint32_t n, const int8_t* secret, uint64_t seed, double sigma,
                    const uint64_t* message, uint64_t* ct) {
    // rns_key_switch.rs:278-387: b = m + e - a*s (a sampled in the NTT domain here)
    auto cdt = cdt_table(sigma);
    auto s = secret_ntt(q, L, n, secret);
    rlwe_encrypt_ntt(q, L, n, s, message, seed, TAG_ENC_A, TAG_ENC_E, 0, cdt, ct, n, ct + (size_t)L * n, n);
    for (uint32_t l = 0; l < L; ++l) {
        ntt_inverse_poly(q[l], n, ct + (size_t)l * n);
        ntt_inverse_poly(q[l], n, ct + (size_t)(L + l) * n);
    }
}

void oracle_decrypt(const uint64_t* q, uint32_t L, uint32_t n, const int8_t* secret, const uint64_t* ct,
                    uint64_t* message) {  // rns_key_switch.rs:906-948: m = b + a*s
    auto s = secret_ntt(q, L, n, secret);
    std::vector<u64> a(n);
    for (uint32_t l = 0; l < L; ++l) {
        std::copy(ct + (size_t)(L + l) * n, ct + (size_t)(L + l + 1) * n, a.begin());
        ntt_forward_poly(q[l], n, a.data());
        for (uint32_t c = 0; c < n; ++c) a[c] = mul_mod(a[c], s[(size_t)l * n + c], q[l]);
        ntt_inverse_poly(q[l], n, a.data());
        for (uint32_t c = 0; c < n; ++c) message[(size_t)l * n + c] = add_mod(ct[(size_t)l * n + c], a[c], q[l]);
    }
}

void oracle_hybrid_key_generate(const uint64_t* q, uint32_t L, const uint64_t* p, uint32_t K, uint32_t n,
                                uint32_t base_log, const int8_t* secret, uint64_t exponent, uint64_t seed,
                                double sigma, uint64_t* key) {
    // hybrid_rns_galois_key.rs:61-170: entry j encrypts P * B^j * sigma(s) over QP
    auto m = qp_moduli(q, L, p, K);
    uint32_t LK = L + K, D = digit_count(q, L, base_log);
    exponent %= 2ull * n;
    auto cdt = cdt_table(sigma);
    auto s_ntt = secret_ntt(m.data(), LK, n, secret);
    auto ts = secret_automorphism(secret, n, exponent);
    std::vector<u64> pf(LK, 1), gf(LK, 1), target((size_t)LK * n);
    for (uint32_t l = 0; l < LK; ++l)
        for (uint32_t k = 0; k < K; ++k) pf[l] = mul_mod(pf[l], p[k] % m[l], m[l]);
    for (uint32_t j = 0; j < D; ++j) {
        for (uint32_t l = 0; l < LK; ++l) {
            u64 mult = mul_mod(pf[l], gf[l], m[l]);
            for (uint32_t c = 0; c < n; ++c) target[(size_t)l * n + c] = mul_mod(signed_mod(ts[c], m[l]), mult, m[l]);
        }
        u64* e0 = key + (size_t)j * LK * 2 * n;
        rlwe_encrypt_ntt(m.data(), LK, n, s_ntt, target.data(), seed, TAG_KEY_A, TAG_KEY_E, j, cdt, e0, 2 * n,
                         e0 + n, 2 * n);
        for (uint32_t l = 0; l < LK; ++l) {
            u64 b = ((u128)1 << base_log) % m[l];
            gf[l] = mul_mod(gf[l], b, m[l]);
        }
    }
}

void oracle_hybrid_rotate(const uint64_t* q, uint32_t L, const uint64_t* p, uint32_t K, uint32_t n,
                          uint32_t base_log, uint64_t exponent, const uint64_t* key, const uint64_t* ct_in,
                          uint64_t* ct_out) {
    // hybrid_rns_galois_key.rs:550-780 (automorphism, decompose sigma(a), base term, MAC, INTT, ModDown)
    exponent %= 2ull * n;
    std::vector<u64> sb((size_t)L * n), sa((size_t)L * n);
    oracle_automorphism_coef(q, L, n, exponent, ct_in, sb.data(), 1);
    oracle_automorphism_coef(q, L, n, exponent, ct_in + (size_t)L * n, sa.data(), 1);
    uint32_t D = digit_count(q, L, base_log);
    std::vector<i64> digits((size_t)D * n);
    bounded_decompose(q, L, n, base_log, sa.data(), digits.data());
    hybrid_switch(q, L, p, K, n, D, digits.data(), key, sb.data(), ct_out);
}

void oracle_hybrid_rotate_hoisted(const uint64_t* q, uint32_t L, const uint64_t* p, uint32_t K, uint32_t n,
                                  uint32_t base_log, uint32_t n_keys, const uint64_t* exponents,
                                  const uint64_t* const* keys, const uint64_t* ct_in, uint64_t* ct_out) {
    // One decomposition of a, then automorphism_hoisted per Galois element
    // (bounded_gadget.rs:273-312; equality with re-decomposition :446-500).
    uint32_t D = digit_count(q, L, base_log);
    std::vector<i64> base_digits((size_t)D * n), digits((size_t)D * n);
    bounded_decompose(q, L, n, base_log, ct_in + (size_t)L * n, base_digits.data());
    std::vector<u64> sb((size_t)L * n);
    for (uint32_t g = 0; g < n_keys; ++g) {
        u64 k = exponents[g] % (2ull * n);
        automorphism_hoisted(D, n, base_log, k, base_digits.data(), digits.data());
        oracle_automorphism_coef(q, L, n, k, ct_in, sb.data(), 1);
        hybrid_switch(q, L, p, K, n, D, digits.data(), keys[g], sb.data(), ct_out + (size_t)g * 2 * L * n);
    }
}

void oracle_hybrid_rotate_hoisted_batch(const uint64_t* q, uint32_t L, const uint64_t* p, uint32_t K, uint32_t n,
                                        uint32_t base_log, uint32_t n_keys, const uint64_t* exponents,
                                        const uint64_t* const* keys, uint32_t n_ct, const uint64_t* ct_in,
                                        uint64_t* ct_out, uint32_t threads) {
    // Independent ciphertexts spread over host threads, each rotation single
    // threaded (the reference's rayon granularity, prepared_radix4_fft256.rs:566-575).
    if (threads == 0) threads = 1;
    // warm the table cache before threading
    for (uint32_t l = 0; l < L; ++l) tables(q[l], n);
    for (uint32_t k = 0; k < K; ++k) tables(p[k], n);
    std::vector<std::thread> pool;
    std::atomic<uint32_t> next{0};
    for (uint32_t t = 0; t < threads; ++t)
        pool.emplace_back([&]() {
            for (;;) {
                uint32_t i = next.fetch_add(1);
                if (i >= n_ct) break;
                oracle_hybrid_rotate_hoisted(q, L, p, K, n, base_log, n_keys, exponents, keys,
                                             ct_in + (size_t)i * 2 * L * n, ct_out + (size_t)i * n_keys * 2 * L * n);
            }
        });
    for (auto& th : pool) th.join();
}

void oracle_rnsblock_key_generate(const uint64_t* q, uint32_t L, const uint64_t* p, uint32_t K, uint32_t n,
                                  const uint32_t* sizes, uint32_t nb, const int8_t* secret, uint64_t exponent,
                                  uint64_t seed, double sigma, uint64_t* key) {
    // Block i encrypts P * E_i * sigma(s); E_i mod q_j = [j in block i]
    // (rns_gadget.rs:92-135), P factor as hybrid_rns_galois_key.rs:94-101; zero on P limbs.
    auto m = qp_moduli(q, L, p, K);
    uint32_t LK = L + K;
    exponent %= 2ull * n;
    auto cdt = cdt_table(sigma);
    auto s_ntt = secret_ntt(m.data(), LK, n, secret);
    auto ts = secret_automorphism(secret, n, exponent);
    BlockLayout b = block_layout(q, sizes, nb);
    std::vector<u64> target((size_t)LK * n);
    for (uint32_t i = 0; i < nb; ++i) {
        for (uint32_t l = 0; l < LK; ++l) {
            u64 f = 0;
            if (l >= b.start[i] && l < b.start[i] + b.size[i]) {
                f = 1;
                for (uint32_t k = 0; k < K; ++k) f = mul_mod(f, p[k] % m[l], m[l]);
            }
            for (uint32_t c = 0; c < n; ++c) target[(size_t)l * n + c] = mul_mod(signed_mod(ts[c], m[l]), f, m[l]);
        }
        u64* e0 = key + (size_t)i * LK * 2 * n;
        rlwe_encrypt_ntt(m.data(), LK, n, s_ntt, target.data(), seed, TAG_KEY_A, TAG_KEY_E, i, cdt, e0, 2 * n,
                         e0 + n, 2 * n);
    }
}

void oracle_rnsblock_rotate(const uint64_t* q, uint32_t L, const uint64_t* p, uint32_t K, uint32_t n,
                            const uint32_t* sizes, uint32_t nb, uint64_t exponent, const uint64_t* key,
                            const uint64_t* ct_in, uint64_t* ct_out) {
    // Hoistable semantics: block digits d_i = a mod Q_i (canonical, rns_gadget.rs:231-273)
    // lifted to every QP limb and transformed once; the Galois element acts
    // as the NTT-domain permutation (ntt_galois_permutation.rs:5-19) on the
    // lifted digits and on NTT(b); then MAC, INTT, ModDown.
    auto m = qp_moduli(q, L, p, K);
    uint32_t LK = L + K;
    exponent %= 2ull * n;
    BlockLayout b = block_layout(q, sizes, nb);
    std::vector<u64> words((size_t)nb * n * b.words);
    oracle_rns_block_decompose(q, L, sizes, nb, n, ct_in + (size_t)L * n, words.data());
    std::vector<u64> acc_b((size_t)LK * n), acc_a((size_t)LK * n), dig(n), perm(n), tmp(n);
    for (uint32_t l = 0; l < LK; ++l) {
        u64 mod = m[l];
        u64* bb = &acc_b[(size_t)l * n];
        u64* aa = &acc_a[(size_t)l * n];
        if (l < L) {
            u64 pf = 1;
            for (uint32_t k = 0; k < K; ++k) pf = mul_mod(pf, p[k] % mod, mod);
            for (uint32_t c = 0; c < n; ++c) tmp[c] = mul_mod(ct_in[(size_t)l * n + c], pf, mod);
            ntt_forward_poly(mod, n, tmp.data());
            automorphism_ntt_1(tmp.data(), bb, n, exponent);
        } else {
            std::fill(bb, bb + n, 0);
        }
        std::fill(aa, aa + n, 0);
        for (uint32_t i = 0; i < nb; ++i) {
            for (uint32_t c = 0; c < n; ++c) dig[c] = wide_mod_small(&words[((size_t)i * n + c) * b.words], b.words, mod);
            ntt_forward_poly(mod, n, dig.data());
            automorphism_ntt_1(dig.data(), perm.data(), n, exponent);
            const u64* kb = key + (((size_t)i * LK + l) * 2 + 0) * n;
            const u64* ka = key + (((size_t)i * LK + l) * 2 + 1) * n;
            for (uint32_t c = 0; c < n; ++c) {
                bb[c] = add_mod(bb[c], mul_mod(perm[c], kb[c], mod), mod);
                aa[c] = add_mod(aa[c], mul_mod(perm[c], ka[c], mod), mod);
            }
        }
        ntt_inverse_poly(mod, n, bb);
        ntt_inverse_poly(mod, n, aa);
    }
    ModDown md(q, L, p, K);
    md.apply(acc_b.data(), ct_out, n);
    md.apply(acc_a.data(), ct_out + (size_t)L * n, n);
}

void oracle_rns_rotate(const uint64_t* q, uint32_t L, uint32_t n, const uint32_t* sizes, uint32_t nb,
                       uint64_t exponent, const uint64_t* key, const uint64_t* ct_in, uint64_t* ct_out) {
    // The ordinary RNS Galois path without auxiliary limbs, in the reference's
    // order: apply_rns_automorphism on (b, a) (rns_galois_key.rs:439-469), then
    // rns_key_switch_with_prepared_ntt (rns_key_switch.rs:2438-2524): block
    // digits of sigma(a) (canonical mod Q_i, rns_gadget.rs:143-228) reduced
    // into each limb, b' = NTT(sigma(b)) + sum_i NTT(d_i) k_b, a' = sum_i NTT(d_i) k_a,
    // inverse NTT. key: [nb][L][2][N] NTT domain (reference layout).
    exponent %= 2ull * n;
    std::vector<u64> sct((size_t)2 * L * n);
    oracle_automorphism_coef(q, L, n, exponent, ct_in, sct.data(), 2);
    BlockLayout b = block_layout(q, sizes, nb);
    std::vector<u64> words((size_t)nb * n * b.words);
    oracle_rns_block_decompose(q, L, sizes, nb, n, sct.data() + (size_t)L * n, words.data());
    std::vector<u64> dig(n);
    for (uint32_t l = 0; l < L; ++l) {
        const u64 mod = q[l];
        u64* bb = ct_out + (size_t)l * n;
        u64* aa = ct_out + (size_t)(L + l) * n;
        std::copy(sct.begin() + (size_t)l * n, sct.begin() + (size_t)(l + 1) * n, bb);
        ntt_forward_poly(mod, n, bb);
        std::fill(aa, aa + n, 0);
        for (uint32_t i = 0; i < nb; ++i) {
            for (uint32_t c = 0; c < n; ++c) dig[c] = wide_mod_small(&words[((size_t)i * n + c) * b.words], b.words, mod);
            ntt_forward_poly(mod, n, dig.data());
            const u64* kb = key + (((size_t)i * L + l) * 2 + 0) * n;
            const u64* ka = key + (((size_t)i * L + l) * 2 + 1) * n;
            for (uint32_t c = 0; c < n; ++c) {
                bb[c] = add_mod(bb[c], mul_mod(dig[c], kb[c], mod), mod);
                aa[c] = add_mod(aa[c], mul_mod(dig[c], ka[c], mod), mod);
            }
        }
        ntt_inverse_poly(mod, n, bb);
        ntt_inverse_poly(mod, n, aa);
    }
}

void oracle_rns_relin_key_generate(const uint64_t* q, uint32_t L, uint32_t n, const uint32_t* sizes, uint32_t nb,
                                   const int8_t* secret, uint64_t seed, double sigma, uint64_t* key) {
    // RnsMultiplicationKey (rns_key_switch.rs:1155-1258 with target s^2): block i
    // encrypts E_i * s^2, E_i mod q_l = [l in block i]; coefficient domain [nb][2][L][N]
    auto cdt = cdt_table(sigma);
    auto s_ntt = secret_ntt(q, L, n, secret);
    BlockLayout b = block_layout(q, sizes, nb);
    std::vector<u64> s2((size_t)L * n), target((size_t)L * n);
    for (uint32_t l = 0; l < L; ++l) {
        for (uint32_t c = 0; c < n; ++c) s2[(size_t)l * n + c] = mul_mod(s_ntt[(size_t)l * n + c], s_ntt[(size_t)l * n + c], q[l]);
        ntt_inverse_poly(q[l], n, &s2[(size_t)l * n]);
    }
    for (uint32_t i = 0; i < nb; ++i) {
        for (uint32_t l = 0; l < L; ++l) {
            const bool in_block = l >= b.start[i] && l < b.start[i] + b.size[i];
            for (uint32_t c = 0; c < n; ++c) target[(size_t)l * n + c] = in_block ? s2[(size_t)l * n + c] : 0;
        }
        u64* e0 = key + (size_t)i * 2 * L * n;
        rlwe_encrypt_ntt(q, L, n, s_ntt, target.data(), seed, TAG_RLK_A, TAG_RLK_E, i, cdt, e0, n, e0 + (size_t)L * n, n);
        for (uint32_t l = 0; l < L; ++l) {
            ntt_inverse_poly(q[l], n, e0 + (size_t)l * n);
            ntt_inverse_poly(q[l], n, e0 + (size_t)(L + l) * n);
        }
    }
}

void oracle_rns_relinearize(const uint64_t* q, uint32_t L, uint32_t n, const uint32_t* sizes, uint32_t nb,
                            const uint64_t* quad, const uint64_t* key, uint64_t* out) {
    // rns_relinearize_with_ntt (rns_key_switch.rs:1842-1905): block digits of c2;
    // per limb b = c0 + sum_i negacyclic_mul(d_i, k_b[i]), a = c1 + sum_i negacyclic_mul(d_i, k_a[i])
    BlockLayout b = block_layout(q, sizes, nb);
    std::vector<u64> words((size_t)nb * n * b.words);
    oracle_rns_block_decompose(q, L, sizes, nb, n, quad + (size_t)2 * L * n, words.data());
    std::vector<u64> d(n), kb(n), ka(n);
    for (uint32_t l = 0; l < L; ++l) {
        const u64 mod = q[l];
        u64* ob = out + (size_t)l * n;
        u64* oa = out + (size_t)(L + l) * n;
        std::copy(quad + (size_t)l * n, quad + (size_t)(l + 1) * n, ob);
        std::copy(quad + (size_t)(L + l) * n, quad + (size_t)(L + l + 1) * n, oa);
        for (uint32_t i = 0; i < nb; ++i) {
            for (uint32_t c = 0; c < n; ++c) d[c] = wide_mod_small(&words[((size_t)i * n + c) * b.words], b.words, mod);
            ntt_forward_poly(mod, n, d.data());
            const u64* e0 = key + (size_t)i * 2 * L * n;
            std::copy(e0 + (size_t)l * n, e0 + (size_t)(l + 1) * n, kb.begin());
            std::copy(e0 + (size_t)(L + l) * n, e0 + (size_t)(L + l + 1) * n, ka.begin());
            ntt_forward_poly(mod, n, kb.data());
            ntt_forward_poly(mod, n, ka.data());
            for (uint32_t c = 0; c < n; ++c) {
                kb[c] = mul_mod(d[c], kb[c], mod);
                ka[c] = mul_mod(d[c], ka[c], mod);
            }
            ntt_inverse_poly(mod, n, kb.data());
            ntt_inverse_poly(mod, n, ka.data());
            for (uint32_t c = 0; c < n; ++c) {
                ob[c] = add_mod(ob[c], kb[c], mod);
                oa[c] = add_mod(oa[c], ka[c], mod);
            }
        }
    }
}

void oracle_tensor(const uint64_t* q, uint32_t L, uint32_t n, const uint64_t* lhs, const uint64_t* rhs,
                   uint64_t* out) {  // quadratic.rs:99-140
    const u64 *b0 = lhs, *a0 = lhs + (size_t)L * n, *b1 = rhs, *a1 = rhs + (size_t)L * n;
    std::vector<u64> t((size_t)L * n), u((size_t)L * n);
    u64 *c0 = out, *c1 = out + (size_t)L * n, *c2 = out + (size_t)2 * L * n;
    oracle_negacyclic_mul(q, L, n, b0, b1, c0);
    oracle_negacyclic_mul(q, L, n, b0, a1, t.data());
    oracle_negacyclic_mul(q, L, n, a0, b1, u.data());
    for (uint32_t l = 0; l < L; ++l)
        for (uint32_t c = 0; c < n; ++c) {
            size_t i = (size_t)l * n + c;
            c1[i] = add_mod(t[i], u[i], q[l]);
        }
    oracle_negacyclic_mul(q, L, n, a0, a1, c2);
}

void oracle_bounded_relin_key_generate(const uint64_t* q, uint32_t L, uint32_t n, uint32_t base_log,
                                       const int8_t* secret, uint64_t seed, double sigma, uint64_t* key) {
    // bounded_key_switch.rs:28-104: entry j encrypts B^j * s^2 (coefficient domain)
    uint32_t D = digit_count(q, L, base_log);
    auto cdt = cdt_table(sigma);
    auto s_ntt = secret_ntt(q, L, n, secret);
    std::vector<u64> s2((size_t)L * n), target((size_t)L * n);
    for (uint32_t l = 0; l < L; ++l) {
        for (uint32_t c = 0; c < n; ++c) s2[(size_t)l * n + c] = mul_mod(s_ntt[(size_t)l * n + c], s_ntt[(size_t)l * n + c], q[l]);
        ntt_inverse_poly(q[l], n, &s2[(size_t)l * n]);
    }
    for (uint32_t j = 0; j < D; ++j) {
        for (uint32_t l = 0; l < L; ++l) {
            u64 f = 1, bm = ((u128)1 << base_log) % q[l];
            for (uint32_t t = 0; t < j; ++t) f = mul_mod(f, bm, q[l]);
            for (uint32_t c = 0; c < n; ++c) target[(size_t)l * n + c] = mul_mod(s2[(size_t)l * n + c], f, q[l]);
        }
        u64* e0 = key + (size_t)j * 2 * L * n;
        rlwe_encrypt_ntt(q, L, n, s_ntt, target.data(), seed, TAG_RLK_A, TAG_RLK_E, j, cdt, e0, n, e0 + (size_t)L * n, n);
        for (uint32_t l = 0; l < L; ++l) {
            ntt_inverse_poly(q[l], n, e0 + (size_t)l * n);
            ntt_inverse_poly(q[l], n, e0 + (size_t)(L + l) * n);
        }
    }
}

void oracle_bounded_relinearize(const uint64_t* q, uint32_t L, uint32_t n, uint32_t base_log,
                                const uint64_t* quad, const uint64_t* key, uint64_t* out) {
    // bounded_key_switch.rs:139-223: b = c0 + sum_j d_j*k_b[j], a = c1 + sum_j d_j*k_a[j]
    uint32_t D = digit_count(q, L, base_log);
    std::vector<i64> digits((size_t)D * n);
    bounded_decompose(q, L, n, base_log, quad + (size_t)2 * L * n, digits.data());
    std::vector<u64> d(n), kb(n), ka(n), db(n);
    for (uint32_t l = 0; l < L; ++l) {
        u64 mod = q[l];
        u64* ob = out + (size_t)l * n;
        u64* oa = out + (size_t)(L + l) * n;
        std::copy(quad + (size_t)l * n, quad + (size_t)(l + 1) * n, ob);
        std::copy(quad + (size_t)(L + l) * n, quad + (size_t)(L + l + 1) * n, oa);
        for (uint32_t j = 0; j < D; ++j) {
            for (uint32_t c = 0; c < n; ++c) d[c] = signed_mod(digits[(size_t)j * n + c], mod);
            ntt_forward_poly(mod, n, d.data());
            const u64* e0 = key + (size_t)j * 2 * L * n;
            std::copy(e0 + (size_t)l * n, e0 + (size_t)(l + 1) * n, kb.begin());
            std::copy(e0 + (size_t)(L + l) * n, e0 + (size_t)(L + l + 1) * n, ka.begin());
            ntt_forward_poly(mod, n, kb.data());
            ntt_forward_poly(mod, n, ka.data());
            for (uint32_t c = 0; c < n; ++c) {
                db[c] = mul_mod(d[c], kb[c], mod);
                ka[c] = mul_mod(d[c], ka[c], mod);
            }
            ntt_inverse_poly(mod, n, db.data());
            ntt_inverse_poly(mod, n, ka.data());
            for (uint32_t c = 0; c < n; ++c) {
                ob[c] = add_mod(ob[c], db[c], mod);
                oa[c] = add_mod(oa[c], ka[c], mod);
            }
        }
    }
}

void oracle_mul_plain(const uint64_t* q, uint32_t L, uint32_t n, const uint64_t* ct, const uint64_t* plain,
                      uint64_t* out) {  // rns_plain_multiply.rs:193-260
    for (int comp = 0; comp < 2; ++comp)
        oracle_negacyclic_mul(q, L, n, ct + (size_t)comp * L * n, plain, out + (size_t)comp * L * n);
}

void oracle_slots_to_coefficients(uint32_t n, const double* slots, double* coeffs) { slots_to_coeffs(n, slots, coeffs); }
void oracle_coefficients_to_slots(uint32_t n, const double* coeffs, double* slots) { coeffs_to_slots(n, coeffs, slots); }

void oracle_encode(uint32_t n, const double* slots, const uint64_t* q, uint32_t L, double scale, uint64_t* out) {
    // application_support/ckks.rs:39-62: round half away from zero, rem_euclid
    std::vector<double> co(n);
    slots_to_coeffs(n, slots, co.data());
    for (uint32_t c = 0; c < n; ++c) {
        double v = std::round(co[c] * scale);
        i128 s = (i128)v;
        for (uint32_t l = 0; l < L; ++l) {
            i128 r = s % (i128)q[l];
            if (r < 0) r += q[l];
            out[(size_t)l * n + c] = (u64)r;
        }
    }
}

void oracle_decode(uint32_t n, const uint64_t* q, uint32_t L, const uint64_t* poly, double scale, double* slots) {
    // application_support/ckks.rs:106-130: CRT, centre, to f64, / scale, coefficients_to_slots
    Garner g(q, L);
    auto Q = composite(q, L, g.words);
    auto half = half_of(Q);
    std::vector<u64> x(g.words);
    std::vector<double> co(n);
    for (uint32_t c = 0; c < n; ++c) {
        g.reconstruct(poly + c, n, x.data());
        center(x.data(), Q, half, g.words);
        co[c] = wide_to_double(x.data(), g.words) / scale;
    }
    coeffs_to_slots(n, co.data(), slots);
}


// --------------------------------------------------- seeded ChaCha20 stream
// rand_chacha 0.3.1 ChaCha20Rng as the reference consumes it: ChaCha20Core
// refills a BlockRng of 64 words (four 16-word blocks, counters c .. c+3);
// next_u32 / next_u64 follow rand_core 0.6.4 BlockRng (next_u64 joins two
// words, low first, also across a refill). seed_from_u64 is rand_core's PCG32
// fill of the 32-byte seed. gen_range is rand 0.8's UniformInt
// sample_single_inclusive (u8 through u32 with a modulus zone, i64 with the
// leading-zeros zone). Call sites: rlwe/secret_key.rs:25-40,
// rlwe/error.rs:33-156, rlwe/uniform.rs:12-30.
struct OracleChaCha {
    uint32_t key[8];
    uint64_t counter = 0;   // next block
    uint32_t results[64];
    uint32_t index = 64;

    static uint32_t rotl(uint32_t v, int c) { return (v << c) | (v >> (32 - c)); }
    void refill() {
        for (int b = 0; b < 4; ++b) {
            const uint64_t ctr = counter + (uint64_t)b;
            uint32_t st[16] = {0x61707865u, 0x3320646eu, 0x79622d32u, 0x6b206574u};
            for (int i = 0; i < 8; ++i) st[4 + i] = key[i];
            st[12] = (uint32_t)ctr;
            st[13] = (uint32_t)(ctr >> 32);
            st[14] = 0;
            st[15] = 0;
            uint32_t w[16];
            for (int i = 0; i < 16; ++i) w[i] = st[i];
            auto qr = [&](int a, int b2, int c, int d) {
                w[a] += w[b2]; w[d] = rotl(w[d] ^ w[a], 16);
                w[c] += w[d]; w[b2] = rotl(w[b2] ^ w[c], 12);
                w[a] += w[b2]; w[d] = rotl(w[d] ^ w[a], 8);
                w[c] += w[d]; w[b2] = rotl(w[b2] ^ w[c], 7);
            };
            for (int r = 0; r < 20; r += 2) {
                qr(0, 4, 8, 12); qr(1, 5, 9, 13); qr(2, 6, 10, 14); qr(3, 7, 11, 15);
                qr(0, 5, 10, 15); qr(1, 6, 11, 12); qr(2, 7, 8, 13); qr(3, 4, 9, 14);
            }
            for (int i = 0; i < 16; ++i) results[16 * b + i] = w[i] + st[i];
        }
        counter += 4;
    }
    void seed_u64(uint64_t state) {
        uint8_t seed[32];
        for (int k = 0; k < 8; ++k) {  // pcg32: advance, then XSH-RR output
            state = state * 6364136223846793005ull + 11634580027462260723ull;
            const uint32_t xs = (uint32_t)(((state >> 18) ^ state) >> 27);
            const uint32_t rot = (uint32_t)(state >> 59);
            const uint32_t x = rot ? (xs >> rot) | (xs << (32 - rot)) : xs;
            for (int i = 0; i < 4; ++i) seed[4 * k + i] = (uint8_t)(x >> (8 * i));
        }
        seed_bytes(seed);
    }
    void seed_bytes(const uint8_t* seed) {
        for (int i = 0; i < 8; ++i)
            key[i] = (uint32_t)seed[4 * i] | ((uint32_t)seed[4 * i + 1] << 8) | ((uint32_t)seed[4 * i + 2] << 16) |
                     ((uint32_t)seed[4 * i + 3] << 24);
        counter = 0;
        index = 64;
    }
    uint32_t next_u32() {
        if (index >= 64) {
            refill();
            index = 0;
        }
        return results[index++];
    }
    uint64_t next_u64() {
        if (index < 63) {
            const uint64_t v = (uint64_t)results[index] | ((uint64_t)results[index + 1] << 32);
            index += 2;
            return v;
        }
        if (index >= 64) {
            refill();
            index = 2;
            return (uint64_t)results[0] | ((uint64_t)results[1] << 32);
        }
        const uint64_t lo = results[63];
        refill();
        index = 1;
        return lo | ((uint64_t)results[0] << 32);
    }
    uint8_t gen_u8_below3() {  // gen_range(0u8..3): UniformInt<u8> via u32
        const uint32_t range = 3, umax = 0xFFFFFFFFu;
        const uint32_t zone = umax - (umax - range + 1) % range;
        for (;;) {
            const uint64_t prod = (uint64_t)next_u32() * range;
            if ((uint32_t)prod <= zone) return (uint8_t)(prod >> 32);
        }
    }
    int64_t gen_i64_inclusive(int64_t lo, int64_t hi) {
        const uint64_t range = (uint64_t)(hi - lo) + 1;
        if (range == 0) return (int64_t)next_u64();
        int lz = 0;
        while (!((range << lz) >> 63)) ++lz;
        const uint64_t zone = (range << lz) - 1;
        for (;;) {
            const u128 prod = (u128)next_u64() * range;
            if ((uint64_t)prod <= zone) return lo + (int64_t)(uint64_t)(prod >> 64);
        }
    }
};

void chacha_error(OracleChaCha& r, uint32_t n, int kind, double param, int64_t* out) {
    if (kind == 0) {  // BoundedUniform (error.rs:44-50)
        const int64_t bound = (int64_t)param;
        for (uint32_t i = 0; i < n; ++i) out[i] = bound == 0 ? 0 : r.gen_i64_inclusive(-bound, bound);
        return;
    }
    // DiscreteGaussian table (error.rs:73-113), uniform_open_unit (:141-151)
    const double sigma = param;
    const int64_t tail = (int64_t)std::ceil(16.0 * sigma);
    std::vector<std::pair<int64_t, double>> weights;
    double total = 0.0;
    for (int64_t x = -tail; x <= tail; ++x) {
        const double xf = (double)x;
        const double w = std::exp(-(xf * xf) / (2.0 * sigma * sigma));
        weights.emplace_back(x, w);
        total += w;
    }
    for (uint32_t i = 0; i < n; ++i) {
        const uint64_t v = r.next_u64() >> 11;
        const double u = ((double)v + 0.5) * (1.0 / (double)(1ull << 53));
        const double target = u * total;
        double cumulative = 0.0;
        int64_t pick = tail;
        for (auto& xw : weights) {
            cumulative += xw.second;
            if (target < cumulative) {
                pick = xw.first;
                break;
            }
        }
        out[i] = pick;
    }
}

void chacha_uniform(OracleChaCha& r, uint32_t n, uint64_t q, uint64_t* out) {  // uniform.rs:12-30
    const uint64_t threshold = (0 - q) % q;
    uint32_t k = 0;
    while (k < n) {
        const uint64_t c = r.next_u64();
        if (c >= threshold) out[k++] = c % q;
    }
}

// Reference-order RLWE encryption into NTT-domain limbs (rns_key_switch.rs:818-850):
// one logical error, then per limb a uniform a; b_ntt = NTT(t + e) - NTT(a) NTT(s).
void chacha_encrypt_ntt(OracleChaCha& r, const u64* m, uint32_t L, uint32_t n, const std::vector<u64>& s_ntt,
                        const u64* target, int kind, double param, u64* b_out, size_t b_stride, u64* a_out,
                        size_t a_stride) {
    std::vector<i64> e(n);
    chacha_error(r, n, kind, param, e.data());
    std::vector<u64> a(n), t(n);
    for (uint32_t l = 0; l < L; ++l) {
        chacha_uniform(r, n, m[l], a.data());
        ntt_forward_poly(m[l], n, a.data());
        for (uint32_t c = 0; c < n; ++c) t[c] = add_mod(target[(size_t)l * n + c], signed_mod(e[c], m[l]), m[l]);
        ntt_forward_poly(m[l], n, t.data());
        u64* bo = b_out + l * b_stride;
        u64* ao = a_out + l * a_stride;
        for (uint32_t c = 0; c < n; ++c) {
            ao[c] = a[c];
            bo[c] = sub_mod(t[c], mul_mod(a[c], s_ntt[(size_t)l * n + c], m[l]), m[l]);
        }
    }
}

void* oracle_chacha_new(uint64_t seed) {
    auto* r = new OracleChaCha();
    r->seed_u64(seed);
    return r;
}
void* oracle_chacha_new_from_seed(const uint8_t* seed32) {
    auto* r = new OracleChaCha();
    r->seed_bytes(seed32);
    return r;
}
void oracle_chacha_free(void* rng) { delete (OracleChaCha*)rng; }
void oracle_chacha_words(void* rng, uint32_t* out, uint64_t n) {
    for (uint64_t i = 0; i < n; ++i) out[i] = ((OracleChaCha*)rng)->next_u32();
}
uint64_t oracle_chacha_next_u64(void* rng) { return ((OracleChaCha*)rng)->next_u64(); }
void oracle_chacha_ternary(void* rng, uint32_t n, int8_t* out) {  // secret_key.rs:25-40
    auto& r = *(OracleChaCha*)rng;
    for (;;) {
        bool any = false;
        for (uint32_t i = 0; i < n; ++i) {
            const uint8_t v = r.gen_u8_below3();
            out[i] = v == 0 ? 0 : (v == 1 ? 1 : -1);
            any = any || v;
        }
        if (any) return;
    }
}
void oracle_chacha_error(void* rng, uint32_t n, int kind, double param, int64_t* out) {
    chacha_error(*(OracleChaCha*)rng, n, kind, param, out);
}
void oracle_chacha_uniform(void* rng, uint32_t n, uint64_t q, uint64_t* out) {
    chacha_uniform(*(OracleChaCha*)rng, n, q, out);
}

void oracle_hybrid_key_generate_chacha(const uint64_t* q, uint32_t L, const uint64_t* p, uint32_t K, uint32_t n,
                                       uint32_t base_log, const int8_t* secret, uint64_t exponent, int kind,
                                       double param, void* rng, uint64_t* key) {
    // hybrid_rns_galois_key.rs:61-170 with the stream of encrypt_rns_raw_prepared_with_cached_secret_ntt_rng
    auto m = qp_moduli(q, L, p, K);
    uint32_t LK = L + K, D = digit_count(q, L, base_log);
    exponent %= 2ull * n;
    auto s_ntt = secret_ntt(m.data(), LK, n, secret);
    auto ts = secret_automorphism(secret, n, exponent);
    std::vector<u64> pf(LK, 1), gf(LK, 1), target((size_t)LK * n);
    for (uint32_t l = 0; l < LK; ++l)
        for (uint32_t k = 0; k < K; ++k) pf[l] = mul_mod(pf[l], p[k] % m[l], m[l]);
    for (uint32_t j = 0; j < D; ++j) {
        for (uint32_t l = 0; l < LK; ++l) {
            u64 mult = mul_mod(pf[l], gf[l], m[l]);
            for (uint32_t c = 0; c < n; ++c) target[(size_t)l * n + c] = mul_mod(signed_mod(ts[c], m[l]), mult, m[l]);
        }
        u64* e0 = key + (size_t)j * LK * 2 * n;
        chacha_encrypt_ntt(*(OracleChaCha*)rng, m.data(), LK, n, s_ntt, target.data(), kind, param, e0, 2 * n, e0 + n,
                           2 * n);
        for (uint32_t l = 0; l < LK; ++l) gf[l] = mul_mod(gf[l], (u64)(((u128)1 << base_log) % m[l]), m[l]);
    }
}

void oracle_bounded_relin_key_generate_chacha(const uint64_t* q, uint32_t L, uint32_t n, uint32_t base_log,
                                              const int8_t* secret, int kind, double param, void* rng,
                                              uint64_t* key) {
    // bounded_key_switch.rs:28-104: entry j = encrypt_rns_raw_with_distribution_ntt_rng(B^j s^2), coefficient domain
    uint32_t D = digit_count(q, L, base_log);
    auto s_ntt = secret_ntt(q, L, n, secret);
    std::vector<u64> s2((size_t)L * n), target((size_t)L * n);
    for (uint32_t l = 0; l < L; ++l) {
        for (uint32_t c = 0; c < n; ++c) s2[(size_t)l * n + c] = mul_mod(s_ntt[(size_t)l * n + c], s_ntt[(size_t)l * n + c], q[l]);
        ntt_inverse_poly(q[l], n, &s2[(size_t)l * n]);
    }
    for (uint32_t j = 0; j < D; ++j) {
        for (uint32_t l = 0; l < L; ++l) {
            u64 f = 1, bm = ((u128)1 << base_log) % q[l];
            for (uint32_t t = 0; t < j; ++t) f = mul_mod(f, bm, q[l]);
            for (uint32_t c = 0; c < n; ++c) target[(size_t)l * n + c] = mul_mod(s2[(size_t)l * n + c], f, q[l]);
        }
        u64* e0 = key + (size_t)j * 2 * L * n;
        chacha_encrypt_ntt(*(OracleChaCha*)rng, q, L, n, s_ntt, target.data(), kind, param, e0, n, e0 + (size_t)L * n, n);
        for (uint32_t l = 0; l < L; ++l) {
            ntt_inverse_poly(q[l], n, e0 + (size_t)l * n);
            ntt_inverse_poly(q[l], n, e0 + (size_t)(L + l) * n);
        }
    }
}

void oracle_encrypt_chacha(const uint64_t* q, uint32_t L, uint32_t n, const int8_t* secret, int kind, double param,
                           void* rng, const uint64_t* message, uint64_t* ct) {
    // rns_key_switch.rs:278-387: one logical error, then per limb a uniform a (coefficients),
    // b = m + e - a s with a s the negacyclic product
    auto& r = *(OracleChaCha*)rng;
    std::vector<i64> e(n);
    chacha_error(r, n, kind, param, e.data());
    auto s_ntt = secret_ntt(q, L, n, secret);
    std::vector<u64> a(n), as(n);
    for (uint32_t l = 0; l < L; ++l) {
        chacha_uniform(r, n, q[l], a.data());
        std::copy(a.begin(), a.end(), ct + (size_t)(L + l) * n);
        as = a;
        ntt_forward_poly(q[l], n, as.data());
        for (uint32_t c = 0; c < n; ++c) as[c] = mul_mod(as[c], s_ntt[(size_t)l * n + c], q[l]);
        ntt_inverse_poly(q[l], n, as.data());
        for (uint32_t c = 0; c < n; ++c)
            ct[(size_t)l * n + c] =
                sub_mod(add_mod(message[(size_t)l * n + c], signed_mod(e[c], q[l]), q[l]), as[c], q[l]);
    }
}


// ccmm/park.rs:1405-1434 (park_matrix_mul_reference): per output, accumulate
// lhs[row][k] * rhs[k][col] in u128 and reduce mod q after every term.
void oracle_park_mod_pp_mm(const uint64_t* lhs, const uint64_t* rhs, uint32_t rows, uint32_t inner, uint32_t cols,
                           uint64_t q, uint64_t* out) {
    const u128 Q = q;
    for (uint32_t r = 0; r < rows; ++r)
        for (uint32_t c = 0; c < cols; ++c) {
            u128 acc = 0;
            for (uint32_t k = 0; k < inner; ++k) {
                acc += (u128)lhs[(size_t)r * inner + k] * rhs[(size_t)k * cols + c];
                acc %= Q;
            }
            out[(size_t)r * cols + c] = (uint64_t)acc;
        }
}

}  // extern "C"
