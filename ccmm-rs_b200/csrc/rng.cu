// rng.cu -- the reference's seeded sampling stream, restated on the host.
//
// Every random draw of the reference (secret, errors, uniform masks) comes
// from rand_chacha 0.3.1's ChaCha20Rng, seeded by rand_core 0.6.4's
// SeedableRng::seed_from_u64 and consumed through rand 0.8's RngCore /
// Rng::gen_range. The stream is sequential by construction (rejection
// sampling makes the position of every later draw depend on every earlier
// one), so it is produced here on the host; the arithmetic that consumes it
// (NTTs, products) runs on the GPU (keyswitch.cu, capi_rng.cu).
//
// Algorithms restated (published sources of the pinned crate versions):
//   ChaCha20 block function (D. J. Bernstein; RFC 8439 quarter round and
//     state layout) with rand_chacha's 64-bit block counter in words 12-13 and
//     64-bit stream id (0) in words 14-15; the RNG hands out the keystream as
//     little-endian 32-bit words in order (BlockRng: next_u32 = next word,
//     next_u64 = next two words, low word first, across buffer refills too).
//   seed_from_u64: PCG32 (state = state * 6364136223846793005 +
//     11634580027462260723, XSH-RR output) fills the 32-byte key four bytes
//     at a time, little endian.
//   gen_range for 8-bit and 64-bit integers (rand 0.8 UniformInt
//     sample_single_inclusive): widening multiply v * range, accepted when
//     the low half is at most the zone (for u8 the zone is computed in u32
//     with a modulus; for 64-bit types zone = (range << lz(range)) - 1).
// Reference call sites: rlwe/secret_key.rs:25-40 (ternary secret),
// rlwe/error.rs:33-156 (bounded-uniform and discrete-Gaussian errors),
// rlwe/uniform.rs:12-30 (rejection-sampled residues).
#include <cmath>
#include <cstring>
#include <vector>

#include "rng.cuh"

namespace {

inline u32 rotl32(u32 x, int r) { return (x << r) | (x >> (32 - r)); }

inline void quarter(u32& a, u32& b, u32& c, u32& d) {
    a += b; d ^= a; d = rotl32(d, 16);
    c += d; b ^= c; b = rotl32(b, 12);
    a += b; d ^= a; d = rotl32(d, 8);
    c += d; b ^= c; b = rotl32(b, 7);
}

}  // namespace

void chacha20_block(const u32 key[8], u64 counter, u64 stream, u32 out[16]) {
    u32 s[16] = {0x61707865u, 0x3320646eu, 0x79622d32u, 0x6b206574u, key[0], key[1], key[2], key[3],
                 key[4],      key[5],      key[6],      key[7],      (u32)counter, (u32)(counter >> 32),
                 (u32)stream, (u32)(stream >> 32)};
    u32 x[16];
    std::memcpy(x, s, sizeof(x));
    for (int r = 0; r < 10; ++r) {  // 20 rounds: column round, diagonal round
        quarter(x[0], x[4], x[8], x[12]);
        quarter(x[1], x[5], x[9], x[13]);
        quarter(x[2], x[6], x[10], x[14]);
        quarter(x[3], x[7], x[11], x[15]);
        quarter(x[0], x[5], x[10], x[15]);
        quarter(x[1], x[6], x[11], x[12]);
        quarter(x[2], x[7], x[8], x[13]);
        quarter(x[3], x[4], x[9], x[14]);
    }
    for (int i = 0; i < 16; ++i) out[i] = x[i] + s[i];
}

void ckks_rng::seed_u64(u64 state) {
    // rand_core 0.6.4 SeedableRng::seed_from_u64 (PCG32, XSH-RR)
    for (int i = 0; i < 8; ++i) {
        state = state * 6364136223846793005ull + 11634580027462260723ull;
        const u32 xorshifted = (u32)(((state >> 18) ^ state) >> 27);
        const u32 rot = (u32)(state >> 59);
        key[i] = (xorshifted >> rot) | (xorshifted << ((32 - rot) & 31));
    }
    pos = 0;
    block = ~0ull;
}

void ckks_rng::seed_bytes(const uint8_t seed[32]) {
    for (int i = 0; i < 8; ++i)
        key[i] = (u32)seed[4 * i] | ((u32)seed[4 * i + 1] << 8) | ((u32)seed[4 * i + 2] << 16) |
                 ((u32)seed[4 * i + 3] << 24);
    pos = 0;
    block = ~0ull;
}

u32 ckks_rng::next_u32() {
    const u64 b = pos >> 4;
    if (b != block) {
        chacha20_block(key, b, 0, buf);
        block = b;
    }
    return buf[pos++ & 15];
}

u64 ckks_rng::next_u64() {
    const u64 lo = next_u32();
    return lo | ((u64)next_u32() << 32);
}

void ckks_rng::fill_u32(u32* out, size_t n) {
    for (size_t i = 0; i < n; ++i) out[i] = next_u32();
}

// rand 0.8 UniformInt<u8>::sample_single(0..3) (rlwe/secret_key.rs:30): range 3 in u32,
// zone = u32::MAX - ((u32::MAX - range + 1) % range)
u32 ckks_rng::range_u8(u32 range) {
    const u32 reject = (u32)((0xFFFFFFFFull - range + 1) % range);
    const u32 zone = 0xFFFFFFFFu - reject;
    for (;;) {
        const u64 m = (u64)next_u32() * range;
        if ((u32)m <= zone) return (u32)(m >> 32);
    }
}

// rand 0.8 UniformInt<i64>::sample_single_inclusive(low, high) (rlwe/error.rs:48)
i64 ckks_rng::range_i64_inclusive(i64 low, i64 high) {
    const u64 range = (u64)high - (u64)low + 1;
    if (range == 0) return (i64)next_u64();
    const u64 zone = (range << __builtin_clzll(range)) - 1;
    for (;;) {
        const unsigned __int128 m = (unsigned __int128)next_u64() * range;
        if ((u64)m <= zone) return (i64)((u64)low + (u64)(m >> 64));
    }
}

// SecretKey::generate_with_rng (rlwe/secret_key.rs:25-40): 0 -> 0, 1 -> 1, 2 -> -1,
// redrawn whole when every coefficient is zero
void ckks_rng::ternary(u32 n, int8_t* out) {
    for (;;) {
        bool any = false;
        for (u32 i = 0; i < n; ++i) {
            const u32 v = range_u8(3);
            out[i] = v == 0 ? 0 : v == 1 ? 1 : -1;
            any = any || v != 0;
        }
        if (any || n == 0) return;
    }
}

// rlwe/uniform.rs:12-30: candidates below 2^64 mod q are rejected, the rest reduced mod q
void ckks_rng::uniform(u32 n, u64 q, u64* out) {
    const u64 threshold = (0 - q) % q;
    u32 k = 0;
    while (k < n) {
        const u64 c = next_u64();
        if (c >= threshold) out[k++] = c % q;
    }
}

GaussianTable::GaussianTable(double sigma) {
    // rlwe/error.rs:73-95: weights exp(-(x^2) / (2 sigma^2)) for |x| <= ceil(16 sigma),
    // summed in order
    tail = (i64)std::ceil(16.0 * sigma);
    weights.reserve((size_t)(2 * tail + 1));
    total = 0.0;
    for (i64 x = -tail; x <= tail; ++x) {
        const double xf = (double)x;
        const double w = std::exp(-(xf * xf) / (2.0 * sigma * sigma));
        weights.push_back(w);
        total += w;
    }
}

// rlwe/error.rs:97-113 with uniform_open_unit (:141-151): (u64 >> 11 + 0.5) 2^-53 * total,
// then the first x whose running sum exceeds it
i64 GaussianTable::sample(ckks_rng& rng) const {
    const u64 v = rng.next_u64() >> 11;
    const double target = ((double)v + 0.5) * (1.0 / 9007199254740992.0) * total;
    double cum = 0.0;
    for (size_t i = 0; i < weights.size(); ++i) {
        cum += weights[i];
        if (target < cum) return (i64)i - tail;
    }
    return tail;
}

// sample_error_coefficients (rlwe/error.rs:33-57)
int32_t ckks_rng::error(u32 n, int kind, double param, i64* out) {
    if (kind == CKKS_DIST_BOUNDED_UNIFORM) {
        const i64 bound = (i64)param;
        if (!(param >= 0) || (double)bound != param) return CKKS_ERR_BAD_ARG;
        for (u32 i = 0; i < n; ++i) out[i] = bound == 0 ? 0 : range_i64_inclusive(-bound, bound);
        return CKKS_OK;
    }
    if (kind == CKKS_DIST_GAUSSIAN) {
        if (!(param > 0) || !std::isfinite(param)) return CKKS_ERR_BAD_ARG;
        GaussianTable t(param);
        for (u32 i = 0; i < n; ++i) out[i] = t.sample(*this);
        return CKKS_OK;
    }
    return CKKS_ERR_BAD_ARG;
}
