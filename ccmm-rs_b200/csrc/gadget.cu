// gadget.cu -- exact gadget decompositions on the GPU.
//
// Bounded gadget (grafting/bounded_gadget.rs): per coefficient, exact CRT of
// the Q residues (mixed-radix Garner with Shoup constants), centring against
// floor(Q/2) (wide_crt.rs:96-111), conversion to a two's complement integer of
// W 64-bit words, then balanced base-2^b digits d_j in [-2^(b-1), 2^(b-1))
// extracted as chunk_j + carry (identical to the reference loop
// residue = value mod B; digit = residue - B if residue >= B/2;
// value = (value - digit) / B, bounded_gadget.rs:75-118).
#include <map>

#include "kernels.cuh"

namespace {

constexpr int kT = 128;

// Per Q-prefix constants: mixed-radix digits of floor(Q/2) and Q as words.
struct PrefixConst {
    u64* d_half_mr = nullptr;  // [q_limbs]
    u64* d_q_words = nullptr;  // [W]
    int W = 0;
    u32 bits = 0;
};

std::mutex g_prefix_mutex;
std::map<std::pair<const ckks_ctx*, u32>, PrefixConst> g_prefix;

typedef unsigned __int128 u128;

int words_for_bits(u32 bits) { return (int)(bits / 64) + 2; }
constexpr int kMaxWords = 66;  // widest k_bounded_decompose / k_crt_to_double instantiation

// Host helpers on little-endian word vectors.
void mul_small_add(std::vector<u64>& x, u64 m, u64 a) {
    u128 carry = a;
    for (auto& w : x) {
        u128 t = (u128)w * m + carry;
        w = (u64)t;
        carry = t >> 64;
    }
}

int32_t prefix_const(ckks_ctx* ctx, u32 q_limbs, PrefixConst* out) {
    std::lock_guard<std::mutex> lock(g_prefix_mutex);
    auto key = std::make_pair((const ckks_ctx*)ctx, q_limbs);
    auto it = g_prefix.find(key);
    if (it != g_prefix.end()) {
        *out = it->second;
        return CKKS_OK;
    }
    double lb = 0;
    for (u32 i = 0; i < q_limbs; ++i) lb += std::log2((double)ctx->moduli[i]);
    int W = words_for_bits((u32)lb + 1);
    std::vector<u64> Q(W, 0);
    Q[0] = 1;
    for (u32 i = 0; i < q_limbs; ++i) mul_small_add(Q, ctx->moduli[i], 0);
    u32 bits = 0;
    for (int i = W - 1; i >= 0; --i)
        if (Q[i]) { bits = (u32)(64 * i + 64 - __builtin_clzll(Q[i])); break; }
    // floor(Q/2) and its mixed-radix digits: v_i in [0, q_i), value = sum v_i prod_{j<i} q_j
    std::vector<u64> half(W);
    for (int i = 0; i < W; ++i) half[i] = (Q[i] >> 1) | (i + 1 < W ? (Q[i + 1] << 63) : 0);
    std::vector<u64> mr(q_limbs), rem = half;
    for (u32 i = 0; i < q_limbs; ++i) {  // repeated division by q_i
        u128 r = 0;
        for (int w = W - 1; w >= 0; --w) {
            u128 cur = (r << 64) | rem[w];
            rem[w] = (u64)(cur / ctx->moduli[i]);
            r = cur % ctx->moduli[i];
        }
        mr[i] = (u64)r;
    }
    PrefixConst pc;
    pc.W = W;
    pc.bits = bits;
    // Q as words, zero-padded to the widest kernel instantiation (kernels of
    // width W' >= W read all W' words)
    std::vector<u64> qpad(kMaxWords, 0);
    std::copy(Q.begin(), Q.end(), qpad.begin());
    if (cudaMalloc(&pc.d_half_mr, q_limbs * sizeof(u64)) != cudaSuccess ||
        cudaMalloc(&pc.d_q_words, kMaxWords * sizeof(u64)) != cudaSuccess) {
        cudaGetLastError();
        ckks_set_error("out of device memory for gadget constants");
        return CKKS_ERR_OOM;
    }
    cudaMemcpy(pc.d_half_mr, mr.data(), q_limbs * sizeof(u64), cudaMemcpyHostToDevice);
    cudaMemcpy(pc.d_q_words, qpad.data(), kMaxWords * sizeof(u64), cudaMemcpyHostToDevice);
    g_prefix[key] = pc;
    *out = pc;
    return CKKS_OK;
}

// bits [start, start + len) of a two's complement value, len <= 63
template <int W>
__device__ __forceinline__ u64 field(const u64 (&x)[W], u32 start, u32 len) {
    const u32 wi = start >> 6, off = start & 63;
    const u64 sign = (x[W - 1] >> 63) ? ~0ull : 0ull;
    u64 lo = wi < W ? x[wi] : sign;
    u64 hi = wi + 1 < W ? x[wi + 1] : sign;
    u64 v = off ? ((lo >> off) | (hi << (64 - off))) : lo;
    return v & ((1ull << len) - 1);
}

template <int W>
__global__ void __launch_bounds__(kT) k_bounded_decompose(const u64* __restrict__ poly, i64* __restrict__ digits,
                                                          u32* __restrict__ flags, const NttTab* __restrict__ tabs,
                                                          GarnerQ g, const u64* __restrict__ half_mr,
                                                          const u64* __restrict__ q_words, int q_limbs, int L,
                                                          int log_n, int base_log, int D, size_t poly_stride) {
    const u32 n = 1u << log_n;
    const u32 c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    const size_t pbase = (size_t)blockIdx.y * poly_stride;
    // mixed radix (Garner), v kept in registers/local memory
    u64 v[kMaxQ];
    bool neg = false;
    for (int i = 0; i < q_limbs; ++i) {
        const u64 qi = tabs[i].q;
        u64 acc = 0;
        for (int j = 0; j < i; ++j) acc = add_mod(acc, mul_shoup(v[j], g.gq[i * L + j], g.gq_q[i * L + j], qi), qi);
        v[i] = mul_shoup(sub_mod(poly[pbase + ((size_t)i << log_n) + c], acc, qi), g.ginv[i], g.ginv_q[i], qi);
    }
    for (int i = q_limbs - 1; i >= 0; --i) {
        u64 h = half_mr[i];
        if (v[i] != h) { neg = v[i] > h; break; }
    }
    // binary: x = v_{L-1}; x = x * q_i + v_i
    u64 x[W];
#pragma unroll
    for (int w = 0; w < W; ++w) x[w] = 0;
    x[0] = v[q_limbs - 1];
    for (int i = q_limbs - 2; i >= 0; --i) {
        const u64 qi = tabs[i].q;
        u64 carry = v[i];
#pragma unroll
        for (int w = 0; w < W; ++w) {
            u64 lo = x[w] * qi, hi = __umul64hi(x[w], qi);
            lo += carry;
            hi += lo < carry;
            x[w] = lo;
            carry = hi;
        }
    }
    if (neg) {  // x - Q, two's complement
        u64 borrow = 0;
#pragma unroll
        for (int w = 0; w < W; ++w) {
            u64 b = q_words[w] + borrow;
            u64 nb = (b < borrow) | (x[w] < b);
            x[w] -= b;
            borrow = nb;
        }
    }
    const i64 B = (i64)1 << base_log, half = B >> 1;
    i64 carry = 0;
    u32 flag = 0;
    const size_t dbase = (size_t)blockIdx.y * D << log_n;
    for (int j = 0; j < D; ++j) {
        i64 d = (i64)field<W>(x, (u32)j * base_log, base_log) + carry;
        if (d >= half) { d -= B; carry = 1; } else { carry = 0; }
        if (d == -half) flag = 1;
        digits[dbase + ((size_t)j << log_n) + c] = d;
    }
    if (flags && flag) {  // list of coefficients holding a -B/2 digit: [count][indices]
        u32* fl = flags + (size_t)blockIdx.y * (n + 1);
        u32 slot = atomicAdd(fl, 1u);
        fl[1 + slot] = c;
    }
}

// automorphism_hoisted (bounded_gadget.rs:273-312), output-driven:
// out[t] = digits of +-x[s], s = t * k^-1 mod 2N, negation re-normalised with carries.
__global__ void k_digits_automorphism(const i64* __restrict__ in, i64* __restrict__ out, int log_n, int D,
                                      int base_log, u64 k_inv) {
    const u32 n = 1u << log_n;
    const u32 t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const size_t pb = (size_t)blockIdx.y * D << log_n;
    const u64 s = ((u64)t * k_inv) & (2ull * n - 1);
    const u32 src = (u32)(s & (n - 1));
    if (s < n) {
        for (int j = 0; j < D; ++j) out[pb + ((size_t)j << log_n) + t] = in[pb + ((size_t)j << log_n) + src];
        return;
    }
    const i64 B = (i64)1 << base_log, half = B >> 1;
    i64 carry = 0;
    for (int j = 0; j < D; ++j) {
        i64 value = -in[pb + ((size_t)j << log_n) + src] + carry;
        i64 m = (value + half) & (B - 1);  // rem_euclid for a power-of-two base
        i64 normalized = m - half;
        out[pb + ((size_t)j << log_n) + t] = normalized;
        carry = (value - normalized) >> base_log;
    }
}

// Decode support (application_support/ckks.rs:106-130): per coefficient the
// exact CRT value, centred (wide_crt.rs:96-111), rounded to the nearest double
// (ties to even; 64 leading bits plus a sticky bit round exactly as the whole
// value) and divided by the scale.
template <int W>
__global__ void __launch_bounds__(kT) k_crt_to_double(const u64* __restrict__ poly, double* __restrict__ out,
                                                      const NttTab* __restrict__ tabs, GarnerQ g,
                                                      const u64* __restrict__ half_mr, const u64* __restrict__ q_words,
                                                      int q_limbs, int L, int log_n, double scale) {
    const u32 n = 1u << log_n;
    const u32 c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    const size_t pbase = (size_t)blockIdx.y * q_limbs << log_n;
    u64 v[kMaxQ];
    for (int i = 0; i < q_limbs; ++i) {
        const u64 qi = tabs[i].q;
        u64 acc = 0;
        for (int j = 0; j < i; ++j) acc = add_mod(acc, mul_shoup(v[j], g.gq[i * L + j], g.gq_q[i * L + j], qi), qi);
        v[i] = mul_shoup(sub_mod(poly[pbase + ((size_t)i << log_n) + c], acc, qi), g.ginv[i], g.ginv_q[i], qi);
    }
    bool neg = false;
    for (int i = q_limbs - 1; i >= 0; --i) {
        if (v[i] != half_mr[i]) { neg = v[i] > half_mr[i]; break; }
    }
    u64 x[W];
#pragma unroll
    for (int w = 0; w < W; ++w) x[w] = 0;
    x[0] = v[q_limbs - 1];
    for (int i = q_limbs - 2; i >= 0; --i) {
        const u64 qi = tabs[i].q;
        u64 carry = v[i];
#pragma unroll
        for (int w = 0; w < W; ++w) {
            u64 lo = x[w] * qi, hi = __umul64hi(x[w], qi);
            lo += carry;
            hi += lo < carry;
            x[w] = lo;
            carry = hi;
        }
    }
    if (neg) {  // magnitude Q - x
        u64 borrow = 0;
#pragma unroll
        for (int w = 0; w < W; ++w) {
            u64 b = x[w] + borrow;
            u64 nb = (b < borrow) | (q_words[w] < b);
            x[w] = q_words[w] - b;
            borrow = nb;
        }
    }
    int top = -1;
#pragma unroll
    for (int w = W - 1; w >= 0; --w)
        if (top < 0 && x[w]) top = w * 64 + 63 - __clzll(x[w]);
    double r = 0.0;
    if (top >= 0 && top < 64) {
        r = __ull2double_rn(x[0]);
    } else if (top >= 64) {
        const int shift = top - 63;
        const int wi = shift >> 6, off = shift & 63;
        u64 lead = off ? ((x[wi] >> off) | (x[wi + 1] << (64 - off))) : x[wi];
        bool sticky = off ? (x[wi] << (64 - off)) != 0 : false;
#pragma unroll
        for (int w = 0; w < W; ++w)
            if (w < wi && x[w]) sticky = true;
        if (sticky) lead |= 1;
        r = ldexp(__ull2double_rn(lead), shift);
    }
    r = neg ? -r : r;
    out[(size_t)blockIdx.y * n + c] = __ddiv_rn(r, scale);
}

u64 galois_inverse(u64 k, u32 n) {
    const u64 two_n = 2ull * n;
    k %= two_n;
    u64 r = 1, b = k, e = n - 1;
    while (e) {
        if (e & 1) r = (r * b) % two_n;
        b = (b * b) % two_n;
        e >>= 1;
    }
    return r;
}

}  // namespace

int32_t bounded_digit_count(ckks_ctx* ctx, u32 q_limbs, u32 base_log, u32* out) {
    CKKS_CHECK_ARG(base_log >= 1 && base_log <= 62, "bounded gadget base_log must be in [1, 62]");
    CKKS_CHECK_ARG(q_limbs >= 1 && q_limbs <= ctx->L, "bounded gadget: Q prefix outside the context basis");
    PrefixConst pc;
    if (int32_t rc = prefix_const(ctx, q_limbs, &pc)) return rc;
    *out = (pc.bits + 1 + base_log - 1) / base_log;  // ceil((bits(Q) + 1) / base_log), bounded_gadget.rs:24-29
    return CKKS_OK;
}

int32_t bounded_decompose_launch(ckks_ctx* ctx, const u64* poly, u32 n_polys, u32 q_limbs, u32 base_log, i64* digits,
                                 u32* flags, cudaStream_t st, size_t poly_stride) {
    if (!poly_stride) poly_stride = (size_t)q_limbs << ctx->log_n;
    u32 D;
    if (int32_t rc = bounded_digit_count(ctx, q_limbs, base_log, &D)) return rc;
    PrefixConst pc;
    if (int32_t rc = prefix_const(ctx, q_limbs, &pc)) return rc;
    if (!n_polys) return CKKS_OK;
    dim3 grid((ctx->n + kT - 1) / kT, n_polys);
#define CKKS_DECOMP(WW)                                                                                          \
    k_bounded_decompose<WW><<<grid, kT, 0, st>>>(poly, digits, flags, ctx->d_tabs, ctx->garner, pc.d_half_mr,     \
                                                 pc.d_q_words, q_limbs, ctx->L, ctx->log_n, base_log, D, poly_stride)
    if (pc.W <= 4) CKKS_DECOMP(4);
    else if (pc.W <= 8) CKKS_DECOMP(8);
    else if (pc.W <= 16) CKKS_DECOMP(16);
    else if (pc.W <= 24) CKKS_DECOMP(24);
    else if (pc.W <= 32) CKKS_DECOMP(32);
    else if (pc.W <= 48) CKKS_DECOMP(48);
    else CKKS_DECOMP(66);
#undef CKKS_DECOMP
    CKKS_CUDA_TRY(cudaGetLastError());
    return CKKS_OK;
}

int32_t digits_automorphism_launch(ckks_ctx* ctx, const i64* in, i64* out, u32 n_polys, u32 D, u32 base_log, u64 k,
                                   cudaStream_t st) {
    CKKS_CHECK_ARG(base_log >= 1 && base_log <= 62, "bounded gadget base_log must be in [1, 62]");
    CKKS_CHECK_ARG((k & 1) == 1, "Galois exponent must be odd");
    if (!n_polys || !D) return CKKS_OK;
    dim3 grid((ctx->n + kT - 1) / kT, n_polys);
    k_digits_automorphism<<<grid, kT, 0, st>>>(in, out, ctx->log_n, D, base_log, galois_inverse(k, ctx->n));
    CKKS_CUDA_TRY(cudaGetLastError());
    return CKKS_OK;
}

int32_t crt_to_double_launch(ckks_ctx* ctx, const u64* poly, u32 n_polys, u32 q_limbs, double scale, double* out,
                             cudaStream_t st) {
    CKKS_CHECK_ARG(q_limbs >= 1 && q_limbs <= ctx->L, "decode: Q prefix outside the context basis");
    PrefixConst pc;
    if (int32_t rc = prefix_const(ctx, q_limbs, &pc)) return rc;
    if (!n_polys) return CKKS_OK;
    dim3 grid((ctx->n + kT - 1) / kT, n_polys);
#define CKKS_CRT(WW)                                                                                                \
    k_crt_to_double<WW><<<grid, kT, 0, st>>>(poly, out, ctx->d_tabs, ctx->garner, pc.d_half_mr, pc.d_q_words,       \
                                             q_limbs, ctx->L, ctx->log_n, scale)
    if (pc.W <= 4) CKKS_CRT(4);
    else if (pc.W <= 8) CKKS_CRT(8);
    else if (pc.W <= 16) CKKS_CRT(16);
    else if (pc.W <= 24) CKKS_CRT(24);
    else if (pc.W <= 32) CKKS_CRT(32);
    else if (pc.W <= 48) CKKS_CRT(48);
    else CKKS_CRT(66);
#undef CKKS_CRT
    CKKS_CUDA_TRY(cudaGetLastError());
    return CKKS_OK;
}

// Drops the cached prefix constants of a context that is being destroyed (a
// later context may be created at the same address).
void gadget_release_ctx(const ckks_ctx* ctx) {
    std::lock_guard<std::mutex> lock(g_prefix_mutex);
    for (auto it = g_prefix.begin(); it != g_prefix.end();) {
        if (it->first.first == ctx) {
            cudaFree(it->second.d_half_mr);
            cudaFree(it->second.d_q_words);
            it = g_prefix.erase(it);
        } else {
            ++it;
        }
    }
}
