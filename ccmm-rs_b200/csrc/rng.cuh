// rng.cuh -- host restatement of the reference's ChaCha20 sampling stream
// (rng.cu) behind the opaque ckks_rng handle of the C ABI.
#pragma once
#include <vector>

#include "context.cuh"

// One ChaCha20 block (20 rounds) of key[8], 64-bit block counter and stream id.
void chacha20_block(const u32 key[8], u64 counter, u64 stream, u32 out[16]);

// rand_chacha::ChaCha20Rng: the keystream as 32-bit words in order.
struct ckks_rng {
    u32 key[8] = {};
    u64 pos = 0;       // next keystream word
    u64 block = ~0ull;  // block held in buf
    u32 buf[16] = {};

    void seed_u64(u64 seed);             // SeedableRng::seed_from_u64
    void seed_bytes(const uint8_t s[32]);  // SeedableRng::from_seed
    u32 next_u32();
    u64 next_u64();
    void fill_u32(u32* out, size_t n);
    u32 range_u8(u32 range);                  // gen_range(0u8..range)
    i64 range_i64_inclusive(i64 low, i64 high);  // gen_range(low..=high)
    void ternary(u32 n, int8_t* out);
    void uniform(u32 n, u64 q, u64* out);
    int32_t error(u32 n, int kind, double param, i64* out);
};

// Discrete Gaussian table of rlwe/error.rs:64-113.
struct GaussianTable {
    std::vector<double> weights;
    double total = 0.0;
    i64 tail = 0;
    explicit GaussianTable(double sigma);
    i64 sample(ckks_rng& rng) const;
};
