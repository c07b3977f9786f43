// embed.cu -- CKKS encode/decode on the GPU in FP64 with the reference's
// rounding: CkksCanonicalEmbedding::slots_to_coefficients /
// coefficients_to_slots (ckks/embedding.rs:57-349) with encode_rns
// (application_support/ckks.rs:39-62) and the CRT decode (:106-130).
//
// Every floating-point result equals the reference operation sequence bit for
// bit: the radix-2 decimation-in-time DFT performs the same butterflies with
// the same twiddle values (each stage's twiddles are the reference's running
// products tw_{o+1} = tw_o * root, and the twists its running powers of
// zeta^{+-1}), complex products are (ac - bd) + (ad + bc)i with every
// multiply and add rounded separately (no fused multiply-add), and roots come
// from the host's cos/sin exactly as the reference's Complex64::from_polar.
// Only the schedule differs: the bit-reversal permutation is folded into the
// placement of the inputs, and each stage is one launch over all butterflies.
#include <cmath>
#include <map>

#include "kernels.cuh"

namespace {

constexpr int kT = 256;

struct EmbedTables {
    u32* idx = nullptr;        // [N/2] slot -> root index (5^i mod 2N - 1) / 2
    double* tw_fwd = nullptr;  // [N-1][2] stage twiddles, sign -1 (stage len at offset len/2 - 1)
    double* tw_inv = nullptr;  // [N-1][2] stage twiddles, sign +1
    double* tw_enc = nullptr;  // [N][2] running powers of exp(-i pi / N)
    double* tw_dec = nullptr;  // [N][2] running powers of exp(+i pi / N)
};

std::mutex g_embed_mutex;
std::map<const ckks_ctx*, EmbedTables> g_embed;

struct C2 {
    double re, im;
};
C2 h_mul(C2 a, C2 b) {
    volatile double ac = a.re * b.re, bd = a.im * b.im, ad = a.re * b.im, bc = a.im * b.re;
    return C2{ac - bd, ad + bc};
}
C2 h_polar(double angle) { return C2{1.0 * std::cos(angle), 1.0 * std::sin(angle)}; }

int32_t embed_tables(ckks_ctx* ctx, EmbedTables* out) {
    std::lock_guard<std::mutex> lock(g_embed_mutex);
    auto it = g_embed.find(ctx);
    if (it != g_embed.end()) {
        *out = it->second;
        return CKKS_OK;
    }
    const u32 n = ctx->n;
    std::vector<u32> idx(n / 2);
    u64 e = 1;
    for (u32 i = 0; i < n / 2; ++i) {
        idx[i] = (u32)((e - 1) / 2);
        e = (e * 5) % (2ull * n);
    }
    std::vector<double> fwd(2 * (size_t)n), inv(2 * (size_t)n), enc(2 * (size_t)n), dec(2 * (size_t)n);
    for (int which = 0; which < 2; ++which) {
        const double sign = which ? 1.0 : -1.0;
        std::vector<double>& t = which ? inv : fwd;
        for (u32 len = 2; len <= n; len *= 2) {
            const double angle = sign * 2.0 * M_PI / (double)len;
            const C2 root = h_polar(angle);
            C2 tw{1.0, 0.0};
            for (u32 o = 0; o < len / 2; ++o) {
                t[2 * (len / 2 - 1 + o)] = tw.re;
                t[2 * (len / 2 - 1 + o) + 1] = tw.im;
                tw = h_mul(tw, root);
            }
        }
    }
    {
        const C2 izeta = h_polar(-M_PI / (double)n), zeta = h_polar(M_PI / (double)n);
        C2 a{1.0, 0.0}, b{1.0, 0.0};
        for (u32 c = 0; c < n; ++c) {
            enc[2 * c] = a.re;
            enc[2 * c + 1] = a.im;
            dec[2 * c] = b.re;
            dec[2 * c + 1] = b.im;
            a = h_mul(a, izeta);
            b = h_mul(b, zeta);
        }
    }
    EmbedTables T;
    const size_t tb = 2 * (size_t)n * sizeof(double);
    if (cudaMalloc(&T.idx, (n / 2) * sizeof(u32)) != cudaSuccess || cudaMalloc(&T.tw_fwd, tb) != cudaSuccess ||
        cudaMalloc(&T.tw_inv, tb) != cudaSuccess || cudaMalloc(&T.tw_enc, tb) != cudaSuccess ||
        cudaMalloc(&T.tw_dec, tb) != cudaSuccess) {
        cudaGetLastError();
        ckks_set_error("out of device memory for embedding tables");
        return CKKS_ERR_OOM;
    }
    CKKS_CUDA_TRY(cudaMemcpy(T.idx, idx.data(), (n / 2) * sizeof(u32), cudaMemcpyHostToDevice));
    CKKS_CUDA_TRY(cudaMemcpy(T.tw_fwd, fwd.data(), tb, cudaMemcpyHostToDevice));
    CKKS_CUDA_TRY(cudaMemcpy(T.tw_inv, inv.data(), tb, cudaMemcpyHostToDevice));
    CKKS_CUDA_TRY(cudaMemcpy(T.tw_enc, enc.data(), tb, cudaMemcpyHostToDevice));
    CKKS_CUDA_TRY(cudaMemcpy(T.tw_dec, dec.data(), tb, cudaMemcpyHostToDevice));
    g_embed[ctx] = T;
    *out = T;
    return CKKS_OK;
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(__dsub_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y)),
                        __dadd_rn(__dmul_rn(a.x, b.y), __dmul_rn(a.y, b.x)));
}

__device__ __forceinline__ u32 brev_n(u32 x, int log_n) { return __brev(x) >> (32 - log_n); }

// ev[brev(idx[i])] = s_i, ev[brev(N-1-idx[i])] = conj(s_i)   (embedding.rs:261-300)
__global__ void k_enc_place(const double2* __restrict__ slots, double2* __restrict__ ev, const u32* __restrict__ idx,
                            int log_n) {
    const u32 n = 1u << log_n;
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n / 2) return;
    const double2 s = slots[(size_t)blockIdx.y * (n / 2) + i];
    double2* v = ev + (size_t)blockIdx.y * n;
    v[brev_n(idx[i], log_n)] = s;
    v[brev_n(n - 1 - idx[i], log_n)] = make_double2(s.x, -s.y);
}

// One radix-2 DIT stage of span len over every message (embedding.rs:57-117).
__global__ void k_dit_stage(double2* __restrict__ ev, const double2* __restrict__ tw, int log_n, int log_len) {
    const u32 n = 1u << log_n, half = 1u << (log_len - 1);
    const u32 b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n / 2) return;
    const u32 o = b & (half - 1), s = (b >> (log_len - 1)) << log_len;
    double2* v = ev + (size_t)blockIdx.y * n;
    const double2 even = v[s + o];
    const double2 odd = cmul(v[s + o + half], tw[half - 1 + o]);
    v[s + o] = make_double2(__dadd_rn(even.x, odd.x), __dadd_rn(even.y, odd.y));
    v[s + o + half] = make_double2(__dsub_rn(even.x, odd.x), __dsub_rn(even.y, odd.y));
}

// The first stages (spans 2 .. 2^log_m) of every block of 2^log_m points in shared memory.
__global__ void k_dit_block(double2* __restrict__ ev, const double2* __restrict__ tw, int log_n, int log_m) {
    extern __shared__ double2 sv[];
    const u32 n = 1u << log_n, m = 1u << log_m;
    double2* v = ev + (size_t)blockIdx.y * n + (size_t)blockIdx.x * m;
    for (u32 i = threadIdx.x; i < m; i += blockDim.x) sv[i] = v[i];
    __syncthreads();
    for (int ll = 1; ll <= log_m; ++ll) {
        const u32 half = 1u << (ll - 1);
        for (u32 b = threadIdx.x; b < m / 2; b += blockDim.x) {
            const u32 o = b & (half - 1), s = (b >> (ll - 1)) << ll;
            const double2 even = sv[s + o];
            const double2 odd = cmul(sv[s + o + half], tw[half - 1 + o]);
            sv[s + o] = make_double2(__dadd_rn(even.x, odd.x), __dadd_rn(even.y, odd.y));
            sv[s + o + half] = make_double2(__dsub_rn(even.x, odd.x), __dsub_rn(even.y, odd.y));
        }
        __syncthreads();
    }
    for (u32 i = threadIdx.x; i < m; i += blockDim.x) v[i] = sv[i];
}

// Rust `f64 as i128` (saturating) of an integer-valued double, reduced mod q.
__device__ __forceinline__ u64 double_int_mod(double v, u64 q, const Barrett& bm) {
    const bool neg = v < 0;
    const double a = fabs(v);
    u64 r;
    if (a < 9223372036854775808.0) {  // 2^63
        const u64 m = (u64)a;
        r = m % q;
    } else {
        const u64 bits = (u64)__double_as_longlong(a);
        int e = (int)((bits >> 52) & 0x7ff) - 1075;          // a = m * 2^e
        u64 m = (bits & ((1ull << 52) - 1)) | (1ull << 52);
        if (e + 53 > 127) {                                  // saturates at 2^127 - 1
            // (2^127 - 1) mod q: 2^127 mod q minus one
            u64 p = 1 % q, b2 = 2 % q;
            for (int k = 0; k < 127; ++k) p = mul_barrett(p, b2, bm);
            r = p ? p - 1 : q - 1;
        } else {
            u64 p = m % q, b2 = 2 % q;
            for (int k = 0; k < e; ++k) p = mul_barrett(p, b2, bm);
            r = p;
        }
    }
    return (neg && r) ? q - r : r;
}

// coefficients: t = ev[c] * (1/N) componentwise, co = t * tw_enc[c]; out = round(co.re * scale) mod q_l
__global__ void k_enc_finish(const double2* __restrict__ ev, const double2* __restrict__ tw, u64* __restrict__ out,
                             const NttTab* __restrict__ tabs, int limbs, int log_n, double norm, double scale) {
    const u32 n = 1u << log_n;
    const u32 c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    const double2 e = ev[(size_t)blockIdx.y * n + c];
    const double2 t = make_double2(__dmul_rn(e.x, norm), __dmul_rn(e.y, norm));
    const double co = cmul(t, tw[c]).x;
    const double v = round(__dmul_rn(co, scale));
    for (int l = 0; l < limbs; ++l) {
        const NttTab& T = tabs[l];
        out[(((size_t)blockIdx.y * limbs + l) << log_n) + c] = double_int_mod(v, T.q, Barrett{T.q, T.mu_hi, T.mu_lo});
    }
}

// ev[brev(c)] = (coef[c], 0) * tw_dec[c]   (embedding.rs:174-220)
__global__ void k_dec_twist(const double* __restrict__ coef, const double2* __restrict__ tw, double2* __restrict__ ev,
                            int log_n) {
    const u32 n = 1u << log_n;
    const u32 c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    const double x = coef[(size_t)blockIdx.y * n + c];
    ev[(size_t)blockIdx.y * n + brev_n(c, log_n)] = cmul(make_double2(x, 0.0), tw[c]);
}

__global__ void k_dec_gather(const double2* __restrict__ ev, double2* __restrict__ slots, const u32* __restrict__ idx,
                             int log_n) {
    const u32 n = 1u << log_n;
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n / 2) return;
    slots[(size_t)blockIdx.y * (n / 2) + i] = ev[(size_t)blockIdx.y * n + idx[i]];
}

int32_t dit(ckks_ctx* ctx, double2* ev, const double* tw, u32 n_msg, cudaStream_t st) {
    const int log_n = (int)ctx->log_n;
    const u32 n = ctx->n;
    const int log_m = log_n < 10 ? log_n : 10;
    if (log_m >= 1) {
        dim3 g(n >> log_m, n_msg);
        k_dit_block<<<g, kT, sizeof(double2) << log_m, st>>>(ev, (const double2*)tw, log_n, log_m);
    }
    for (int ll = log_m + 1; ll <= log_n; ++ll) {
        dim3 g((n / 2 + kT - 1) / kT, n_msg);
        k_dit_stage<<<g, kT, 0, st>>>(ev, (const double2*)tw, log_n, ll);
    }
    CKKS_CUDA_TRY(cudaGetLastError());
    return CKKS_OK;
}

}  // namespace

int32_t encode_launch(ckks_ctx* ctx, const double* slots, u64* out, u32 n_msg, u32 q_limbs, double scale,
                      cudaStream_t st) {
    EmbedTables T;
    if (int32_t rc = embed_tables(ctx, &T)) return rc;
    const u32 n = ctx->n;
    Workspace<double2> ev;
    if (int32_t rc = ev.alloc((size_t)n * n_msg, st)) return rc;
    dim3 gh((n / 2 + kT - 1) / kT, n_msg), gn((n + kT - 1) / kT, n_msg);
    k_enc_place<<<gh, kT, 0, st>>>((const double2*)slots, ev.p, T.idx, (int)ctx->log_n);
    if (int32_t rc = dit(ctx, ev.p, T.tw_fwd, n_msg, st)) return rc;
    k_enc_finish<<<gn, kT, 0, st>>>(ev.p, (const double2*)T.tw_enc, out, ctx->d_tabs, (int)q_limbs, (int)ctx->log_n,
                                    1.0 / (double)n, scale);
    CKKS_CUDA_TRY(cudaGetLastError());
    return CKKS_OK;
}

int32_t decode_launch(ckks_ctx* ctx, const u64* poly, double* slots, u32 n_msg, u32 q_limbs, double scale,
                      cudaStream_t st) {
    EmbedTables T;
    if (int32_t rc = embed_tables(ctx, &T)) return rc;
    const u32 n = ctx->n;
    Workspace<double> coef;
    Workspace<double2> ev;
    int32_t rc;
    if ((rc = coef.alloc((size_t)n * n_msg, st)) || (rc = ev.alloc((size_t)n * n_msg, st))) return rc;
    if ((rc = crt_to_double_launch(ctx, poly, n_msg, q_limbs, scale, coef.p, st))) return rc;
    dim3 gh((n / 2 + kT - 1) / kT, n_msg), gn((n + kT - 1) / kT, n_msg);
    k_dec_twist<<<gn, kT, 0, st>>>(coef.p, (const double2*)T.tw_dec, ev.p, (int)ctx->log_n);
    if ((rc = dit(ctx, ev.p, T.tw_inv, n_msg, st))) return rc;
    k_dec_gather<<<gh, kT, 0, st>>>(ev.p, (double2*)slots, T.idx, (int)ctx->log_n);
    CKKS_CUDA_TRY(cudaGetLastError());
    return CKKS_OK;
}

// Drops the cached tables of a context that is being destroyed.
void embed_release_ctx(const ckks_ctx* ctx) {
    std::lock_guard<std::mutex> lock(g_embed_mutex);
    auto it = g_embed.find(ctx);
    if (it == g_embed.end()) return;
    cudaFree(it->second.idx);
    cudaFree(it->second.tw_fwd);
    cudaFree(it->second.tw_inv);
    cudaFree(it->second.tw_enc);
    cudaFree(it->second.tw_dec);
    g_embed.erase(it);
}
