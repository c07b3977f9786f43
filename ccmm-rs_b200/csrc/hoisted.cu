// hoisted.cu -- NTT-domain hoisting of the bounded hybrid-QP rotation.
//
// The reference hoists at the digit level (BoundedGadgetDecomposition::
// automorphism_hoisted, grafting/bounded_gadget.rs:273-312) and transforms the
// re-normalised digits for every Galois element. Those digits equal the
// signed automorphism of the digits of a, sigma(d_j), except at coefficients
// whose source value is negated and holds a digit equal to -B/2: there the
// carry re-normalisation changes a few digits by Delta. Since
// NTT(sigma(d_j)) is the NTT-domain permutation of NTT(d_j)
// (ring/ntt_galois_permutation.rs:5-19), the exact key-switch sum is
//   sum_j NTT(d_j)[pi(k)] K_j[k] + sum_{(t,j,Delta)} Delta psi^((2k+1) t) K_j[k],
// so the digit transforms are done once per ciphertext, and every Galois
// element costs one MAC pass plus the (rare, sparse) correction terms. A
// (ciphertext, Galois element) pair whose corrections exceed the list
// capacity is recomputed by the non-hoisted path, so every output word equals
// the reference's.
//
// The MAC streams each key slice once per group of G ciphertexts (evict-first
// loads) while the hoisted digit transforms of the group stay L2-resident
// and are gathered through the permutation.
#include "keyswitch.cuh"

#include <algorithm>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <vector>

namespace {

constexpr int kT = 256;

struct Exc {
    u32 t, j;
    i64 delta;
};


__device__ __forceinline__ u64 pow_mod_dev(u64 b, u64 e, const Barrett& m) {
    u64 r = 1;
    while (e) {
        if (e & 1) r = mul_barrett(r, b, m);
        b = mul_barrett(b, b, m);
        e >>= 1;
    }
    return r;
}

// Flagged source coefficients (a digit equals -B/2) of G ciphertexts ->
// exception lists per (ciphertext, key): entries (t, j, Delta) where the
// reference's re-normalised digit differs from -d_j[s].
__global__ void k_hoist_exceptions(const i64* __restrict__ digits, size_t dig_stride, const u32* __restrict__ flags,
                                   size_t flag_stride, const u64* __restrict__ exps, int n_keys, int D, int base_log,
                                   int log_n, Exc* __restrict__ exc, u32* __restrict__ exc_count, int cap) {
    const int c = blockIdx.z, g = blockIdx.y;
    const u32* fl = flags + c * flag_stride;
    const u32 nflag = fl[0];
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nflag) return;
    const u32 n = 1u << log_n;
    const u32 s = fl[1 + i];
    const u64 mapped = ((u64)s * exps[g]) & (2ull * n - 1);
    if (mapped < n) return;  // not negated: digits move unchanged
    const u32 t = (u32)(mapped - n);
    const i64* d = digits + c * dig_stride;
    const i64 B = (i64)1 << base_log, half = B >> 1;
    i64 carry = 0;
    Exc* list = exc + ((size_t)c * n_keys + g) * cap;
    u32* cnt = exc_count + (size_t)c * n_keys + g;
    for (int j = 0; j < D; ++j) {
        i64 dj = d[((size_t)j << log_n) + s];
        i64 value = -dj + carry;
        i64 m = (value + half) & (B - 1);
        i64 normalized = m - half;
        carry = (value - normalized) >> base_log;
        i64 delta = normalized + dj;  // reference digit minus the naive -d_j
        if (delta != 0) {
            u32 slot = atomicAdd(cnt, 1u);
            if ((int)slot < cap) list[slot] = Exc{t, (u32)j, delta};
        }
    }
}

// MAC in the permuted index s = pi_g(k) (keys are stored permuted):
// acc'[c][g][comp][l][s] = sum_j Yhat_c[j][l][s] key'_g[j][l][comp][s] + corrections
// so acc = perm_g(acc'); the caller applies sigma_g after the inverse transform
// and the inverse transform adds the base term P b in the coefficient domain
// (InvBase), so P NTT(b) is not accumulated here.
// Every load is contiguous: keys stream once per group (evict-first), the
// group's digit transforms are re-read from L2 by every key.
template <int G>
__global__ void __launch_bounds__(kT) k_mac_hoisted(const u64* __restrict__ Yhat, size_t y_stride,
                                                    const u64* const* __restrict__ keys,
                                                    const u64* __restrict__ exps_inv, u64* __restrict__ acc,
                                                    const NttTab* __restrict__ tabs, LimbMap lm, int n_ct, int n_keys,
                                                    int Lq, int LK, int D, int log_n, const Exc* __restrict__ exc,
                                                    const u32* __restrict__ exc_count, int cap,
                                                    const u64* __restrict__ psi) {
    const u32 n = 1u << log_n;
    const u32 s = blockIdx.x * blockDim.x + threadIdx.x;
    const int g = blockIdx.y, l = blockIdx.z;
    if (s >= n) return;
    const NttTab& T = tabs[lm(l)];
    const u64 q = T.q, mh = T.mu_hi, ml = T.mu_lo;
    const u64* key = keys[g];
    Acc128 ab[G], aa[G];
#pragma unroll
    for (int c = 0; c < G; ++c) ab[c] = aa[c] = Acc128{0, 0};
    int since = 0;
    for (int j = 0; j < D; ++j) {
        const size_t kofs = (((size_t)j * LK + l) * 2) << log_n;
        const u64 kb = __ldcs(key + kofs + s), ka = __ldcs(key + kofs + n + s);
        const size_t yofs = (((size_t)j * LK + l) << log_n) + s;
#pragma unroll
        for (int c = 0; c < G; ++c) {
            if (c < n_ct) {
                u64 y = __ldg(Yhat + c * y_stride + yofs);
                ab[c].mac(y, kb);
                aa[c].mac(y, ka);
            }
        }
        if (++since == 15) {
#pragma unroll
            for (int c = 0; c < G; ++c) {
                ab[c].fold(q, mh, ml);
                aa[c].fold(q, mh, ml);
            }
            since = 0;
        }
    }
    const Barrett bm{q, mh, ml};
#pragma unroll
    for (int c = 0; c < G; ++c) {
        if (c >= n_ct) break;
        ab[c].fold(q, mh, ml);
        aa[c].fold(q, mh, ml);
        u64 b = ab[c].lo, a = aa[c].lo;
        u32 cnt = exc_count[(size_t)c * n_keys + g];
        if (cnt > (u32)cap) cnt = 0;  // overflowed: recomputed by the exact fallback
        if (cnt) {
            const Exc* list = exc + ((size_t)c * n_keys + g) * cap;
            const u64 ps = psi[lm(l)];
            const u32 k = galois_src(s, exps_inv[g], log_n);  // unpermuted slot of s
            for (u32 e = 0; e < cnt; ++e) {
                const Exc x = list[e];
                // NTT of Delta * X^t at slot k: Delta * psi^((2k+1) t)
                u64 w = pow_mod_dev(ps, ((2ull * k + 1) * x.t) & (2ull * n - 1), bm);
                u64 dm = x.delta < 0 ? (u64)(-x.delta) % q : (u64)x.delta % q;
                if (x.delta < 0 && dm) dm = q - dm;
                u64 v = mul_barrett(w, dm, bm);
                const size_t kofs = (((size_t)x.j * LK + l) * 2) << log_n;
                b = add_mod(b, mul_barrett(v, key[kofs + s], bm), q);
                a = add_mod(a, mul_barrett(v, key[kofs + n + s], bm), q);
            }
        }
        const size_t obase = (((size_t)c * n_keys + g) * 2 * LK) << log_n;
        acc[obase + ((size_t)l << log_n) + s] = b;
        acc[obase + (((size_t)LK + l) << log_n) + s] = a;
    }
}

u64 galois_inverse_host(u64 k, u32 n) {
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

// Split-operand accumulator: with sb = ceil(bits(q - 1) / 2), an operand
// x < q is x1 * 2^sb + x0 (x0, x1 < 2^sb) and a product is
// x0 y0 + (x0 y1 + x1 y0) 2^sb + x1 y1 2^(2 sb). Three 64-bit partial sums
// take each 32 x 32 -> 64 multiply with accumulate (IMAD.WIDE.U32) without
// carry handling; they are reduced mod q every `fold` terms (chosen so the
// middle sum cannot overflow) and combined with 2^sb, 2^2sb mod q. The value
// is the canonical residue of the same exact sum of products.
struct SplitAcc {
    u64 s0, s1, s2;
    __device__ __forceinline__ void mac(u32 x0, u32 x1, u32 y0, u32 y1) {
        s0 += (u64)x0 * y0;
        s1 += (u64)x0 * y1;
        s1 += (u64)x1 * y0;
        s2 += (u64)x1 * y1;
    }
    // Reduce to the canonical residue, kept in s0 (s0 stays below
    // q + fold * 2^(2 sb) < 2^64 until the next fold).
    __device__ __forceinline__ void fold(u64 q, u64 one_q, u64 r1, u64 r1q, u64 r2, u64 r2q) {
        u64 t = reduce_2q(mul_shoup_lazy(s0, 1, one_q, q), q);
        t = add_mod(t, reduce_2q(mul_shoup_lazy(s1, r1, r1q, q), q), q);
        t = add_mod(t, reduce_2q(mul_shoup_lazy(s2, r2, r2q, q), q), q);
        s0 = t;
        s1 = s2 = 0;
    }
};

// Tiled MAC: one CTA owns (limb l, slot tile of kS slots) for G ciphertexts
// and every Galois key. The G x D x kS digit-transform tile is staged in
// shared memory once (pre-split into its two sb-bit halves); keys stream from
// HBM exactly once per group (evict-first), kU digits of key loads in flight
// per thread. Thread (s, lane) accumulates keys g = lane, lane + kLanes, ..
// for all G ciphertexts. Same sums as k_mac_hoisted.
constexpr int kS = 64, kLanes = 4, kU = 4;

template <int G>
__global__ void __launch_bounds__(kS * kLanes, 2) k_mac_tiled(const u64* __restrict__ Yhat, size_t y_stride,
                                                           const u64* const* __restrict__ keys,
                                                           const u64* __restrict__ exps_inv,
                                                           u64* __restrict__ acc, const NttTab* __restrict__ tabs,
                                                           LimbMap lm, int n_ct, int n_keys, int Lq, int LK, int D,
                                                           int log_n, const Exc* __restrict__ exc,
                                                           const u32* __restrict__ exc_count, int cap,
                                                           const u64* __restrict__ psi) {
    extern __shared__ u64 ytile[];  // [G][D][kS], each word (y >> sb) << 32 | (y & mask)
    const u32 n = 1u << log_n;
    const int l = blockIdx.y;
    const u32 s0 = blockIdx.x * kS;
    const int tid = threadIdx.x, si = tid % kS, lane = tid / kS;
    const u32 s = s0 + si;
    const NttTab& T = tabs[lm(l)];
    const u64 q = T.q, mh = T.mu_hi, ml = T.mu_lo;
    const int sb = (65 - __clzll(q - 1)) / 2;  // ceil(bits(q - 1) / 2)
    const u64 mask = (1ull << sb) - 1;
    // middle sum grows by < 2^(2 sb + 1) per product: fold before 2^64
    const u64 fold_lim = (~0ull) >> (2 * sb + 1);
    const int fold_every = fold_lim > 8191 ? 8191 : (int)fold_lim;
    const u64 one_q = shoup_quotient_dev(1, q);
    const u64 r1 = (1ull << sb) % q, r2 = mul_barrett(r1, r1, Barrett{q, mh, ml});
    const u64 r1q = shoup_quotient_dev(r1, q), r2q = shoup_quotient_dev(r2, q);
    for (int c = 0; c < G; ++c)
        for (int idx = tid; idx < D * kS; idx += blockDim.x) {
            const int j = idx / kS, x = idx % kS;
            u64 y = c < n_ct ? __ldg(Yhat + c * y_stride + (((size_t)j * LK + l) << log_n) + s0 + x) : 0;
            ytile[c * D * kS + idx] = ((y >> sb) << 32) | (y & mask);
        }
    __syncthreads();
    const Barrett bm{q, mh, ml};
    const size_t jstride = ((size_t)LK * 2) << log_n;
    for (int g = lane; g < n_keys; g += kLanes) {
        const u64* key = keys[g];
        const u64* kp = key + ((((size_t)l * 2) << log_n) + s);
        SplitAcc ab[G], aa[G];
#pragma unroll
        for (int c = 0; c < G; ++c) ab[c] = aa[c] = SplitAcc{0, 0, 0};
        int since = 0;
        for (int j0 = 0; j0 < D; j0 += kU) {
            u64 kb[kU], ka[kU];
#pragma unroll
            for (int u = 0; u < kU; ++u) {
                if (j0 + u < D) {
                    kb[u] = __ldcs(kp + (j0 + u) * jstride);
                    ka[u] = __ldcs(kp + (j0 + u) * jstride + n);
                }
            }
#pragma unroll
            for (int u = 0; u < kU; ++u) {
                if (j0 + u < D) {
                    const u32 b0 = (u32)(kb[u] & mask), b1 = (u32)(kb[u] >> sb);
                    const u32 a0 = (u32)(ka[u] & mask), a1 = (u32)(ka[u] >> sb);
#pragma unroll
                    for (int c = 0; c < G; ++c) {
                        const u64 y = ytile[(c * D + j0 + u) * kS + si];
                        const u32 y0 = (u32)y, y1 = (u32)(y >> 32);
                        ab[c].mac(y0, y1, b0, b1);
                        aa[c].mac(y0, y1, a0, a1);
                    }
                    if (++since == fold_every) {
#pragma unroll
                        for (int c = 0; c < G; ++c) {
                            ab[c].fold(q, one_q, r1, r1q, r2, r2q);
                            aa[c].fold(q, one_q, r1, r1q, r2, r2q);
                        }
                        since = 0;
                    }
                }
            }
        }
#pragma unroll
        for (int c = 0; c < G; ++c) {
            if (c >= n_ct) break;
            ab[c].fold(q, one_q, r1, r1q, r2, r2q);
            aa[c].fold(q, one_q, r1, r1q, r2, r2q);
            u64 b = ab[c].s0, a = aa[c].s0;
            u32 cnt = exc_count[(size_t)c * n_keys + g];
            if (cnt > (u32)cap) cnt = 0;  // overflowed: recomputed by the exact fallback
            if (cnt) {
                const Exc* list = exc + ((size_t)c * n_keys + g) * cap;
                const u64 ps = psi[lm(l)];
                const u32 k = galois_src(s, exps_inv[g], log_n);
                for (u32 e = 0; e < cnt; ++e) {
                    const Exc x = list[e];
                    u64 w = pow_mod_dev(ps, ((2ull * k + 1) * x.t) & (2ull * n - 1), bm);
                    u64 dm = x.delta < 0 ? (u64)(-x.delta) % q : (u64)x.delta % q;
                    if (x.delta < 0 && dm) dm = q - dm;
                    u64 v = mul_barrett(w, dm, bm);
                    const size_t kofs = (((size_t)x.j * LK + l) * 2) << log_n;
                    b = add_mod(b, mul_barrett(v, key[kofs + s], bm), q);
                    a = add_mod(a, mul_barrett(v, key[kofs + n + s], bm), q);
                }
            }
            const size_t obase = (((size_t)c * n_keys + g) * 2 * LK) << log_n;
            acc[obase + ((size_t)l << log_n) + s] = b;
            acc[obase + (((size_t)LK + l) << log_n) + s] = a;
        }
    }
}

}  // namespace

// The tensor-core MAC runs on compute capability 10.0 devices (the library is
// built for sm_100a only).
bool tc_enabled() {
    static int cached = -1;
    if (cached < 0) {
        int dev = 0, major = 0, minor = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
        cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev);
        cached = (major == 10 && minor == 0) ? 1 : 0;
    }
    return cached == 1;
}

namespace {

// ------------------------------------------------------------ packed key sets
// The tensor-core MAC reads the A operand of an item (tile of 4 slots of one
// limb, 32-key chunk, 4-digit chunk) as one contiguous block, brought into
// shared memory by a single bulk copy. Blocks are in the MAC's shared-memory
// image (K-major, no swizzle): row group rg (8 rows = 4 keys x 2 components) of
// 1 KB, then slot i (256 B), K chunk kk (128 B: digits 2 kk, 2 kk + 1), row
// (16 B), digit (8 B). Only the row groups of present keys are stored. Digit D
// (one past the gadget digits) holds P mod q_l in the b rows of the Q limbs and
// 0 elsewhere: paired with the NTT of the ciphertext's b it adds the base term
// P b of the rotation inside the same contraction. A set is packed once per
// ordered list of Galois keys and cached per context until a key of the set or
// the context is destroyed.
struct PackedSet {
    std::vector<const ckks_ksk*> keys;
    u64* d = nullptr;
    u32 rg = 0, n_kc = 0, n_chunks = 0;
    u32 g_max = 4;  // ciphertexts per group that fit the device next to the set (sized once, at packing)
};
constexpr u32 kGroupMax = 16;  // ciphertexts per tensor-core MAC group (tc::kCt)
std::mutex g_sets_mu;
std::map<const ckks_ctx*, std::vector<std::unique_ptr<PackedSet>>> g_sets;

__global__ void k_pack_keys(const u64* const* __restrict__ keys, int n_keys, int LK, int D, int log_n, u32 rg,
                            u32 n_kc, u32 n_chunks, const u64* __restrict__ pf, int Lq, u64* __restrict__ out,
                            size_t total) {
    const u32 block_words = rg * 128;
    const u32 tiles_s = (1u << log_n) >> 2;
    for (size_t w = (size_t)blockIdx.x * blockDim.x + threadIdx.x; w < total; w += (size_t)gridDim.x * blockDim.x) {
        const size_t block = w / block_words;
        const u32 off = (u32)(w - block * block_words);
        const u32 r = off & 127;
        const u32 m = ((off >> 7) << 3) | ((r >> 1) & 7);
        const u32 i = r >> 5, jj = (((r >> 4) & 1) << 1) | (r & 1);
        const u32 ch = (u32)(block % n_chunks);
        const size_t rest = block / n_chunks;
        const u32 kc = (u32)(rest % n_kc);
        const size_t tile = rest / n_kc;
        const u32 l = (u32)(tile / tiles_s), s = (u32)(tile % tiles_s) * 4 + i;
        const u32 g = kc * 32 + (m >> 1), comp = m & 1, j = ch * 4 + jj;
        u64 v = 0;
        if (g < (u32)n_keys) {
            if (j < (u32)D) v = __ldg(keys[g] + (((((size_t)j * LK + l) * 2 + comp) << log_n) + s));
            else if (j == (u32)D && comp == 0 && l < (u32)Lq) v = pf[l];
        }
        out[w] = v;
    }
}

// The packed set of these keys, packed on first use when device memory allows
// (null otherwise: the caller takes the CUDA-core MAC).
const PackedSet* packed_set_get(ckks_ctx* ctx, const ckks_ksk* const* keys, u32 n_keys, cudaStream_t st) {
    std::lock_guard<std::mutex> lock(g_sets_mu);
    std::vector<std::unique_ptr<PackedSet>>& sets = g_sets[ctx];
    for (const auto& p : sets)
        if (p->keys.size() == n_keys && std::equal(p->keys.begin(), p->keys.end(), keys)) return p.get();
    const ckks_ksk* k0 = keys[0];
    const u32 LK = ksk_limbs(k0), n = ctx->n;
    std::unique_ptr<PackedSet> pp(new PackedSet);
    PackedSet& p = *pp;
    p.keys.assign(keys, keys + n_keys);
    p.n_kc = (n_keys + 31) / 32;
    p.n_chunks = (k0->D + 1 + 3) / 4;  // gadget digits and the base digit
    p.rg = n_keys >= 32 ? 8 : (n_keys + 3) / 4;
    const size_t total = (size_t)LK * (n / 4) * p.n_kc * p.n_chunks * p.rg * 128;
    // unused stream-ordered workspace memory goes back to the device first
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, ctx->device) == cudaSuccess) {
        cudaStreamSynchronize(st);
        cudaMemPoolTrimTo(pool, 0);
    }
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) return nullptr;
    // keep a quarter of the device free for the rotation workspaces
    const size_t bytes = total * sizeof(u64);
    if (bytes > free_b || free_b - bytes < total_b / 4) return nullptr;
    std::vector<const u64*> hptr(n_keys);
    for (u32 g = 0; g < n_keys; ++g) hptr[g] = keys[g]->d_entries;
    const u64** d_ptr = nullptr;
    if (cudaMalloc(&p.d, bytes) != cudaSuccess || cudaMalloc(&d_ptr, n_keys * sizeof(u64*)) != cudaSuccess ||
        cudaMemcpy(d_ptr, hptr.data(), n_keys * sizeof(u64*), cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaGetLastError();
        if (p.d) cudaFree(p.d);
        if (d_ptr) cudaFree(d_ptr);
        return nullptr;
    }
    {  // group size: workspace per ciphertext (digit transforms, accumulators) within half the free memory
        const size_t per_ct = ((size_t)k0->D * LK * n + 4 * (size_t)n_keys * LK * n) * sizeof(u64);
        const size_t left = free_b - bytes;
        u32 g = kGroupMax;
        while (g > 4 && (size_t)g * per_ct > left / 2) g -= 4;
        p.g_max = g;
    }
    k_pack_keys<<<148 * 16, 256, 0, st>>>(d_ptr, (int)n_keys, (int)LK, (int)k0->D, (int)ctx->log_n, p.rg, p.n_kc,
                                          p.n_chunks, ctx->d_pmodq, (int)k0->q_limbs, p.d, total);
    // ready for every stream of the context
    const bool ok = cudaGetLastError() == cudaSuccess && cudaStreamSynchronize(st) == cudaSuccess;
    cudaFree(d_ptr);
    if (!ok) {
        cudaFree(p.d);
        return nullptr;
    }
    sets.push_back(std::move(pp));
    return sets.back().get();
}

}  // namespace

void keyset_release_ctx(const ckks_ctx* ctx) {
    std::lock_guard<std::mutex> lock(g_sets_mu);
    auto it = g_sets.find(ctx);
    if (it == g_sets.end()) return;
    for (auto& p : it->second) cudaFree(p->d);
    g_sets.erase(it);
}

void keyset_forget_key(const ckks_ksk* key) {
    std::lock_guard<std::mutex> lock(g_sets_mu);
    auto it = g_sets.find(key->ctx);
    if (it == g_sets.end()) return;
    auto& sets = it->second;
    bool synced = false;
    for (size_t i = 0; i < sets.size();) {
        if (std::find(sets[i]->keys.begin(), sets[i]->keys.end(), key) != sets[i]->keys.end()) {
            if (!synced) {
                cudaDeviceSynchronize();  // no launch may still read the set
                synced = true;
            }
            cudaFree(sets[i]->d);
            sets.erase(sets.begin() + i);
        } else {
            ++i;
        }
    }
}

namespace {

// CUDA-event phase timer (the analogue of the reference's HybridRotationTiming,
// ckks/hybrid_rns_galois_key.rs:323-336). Phases accumulate over groups.
struct PhaseTimer {
    double* out = nullptr;
    cudaStream_t st = nullptr;
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> spans;
    cudaEvent_t open_ev = nullptr;
    int open_phase = -1;
    void begin(int phase) {
        if (!out) return;
        cudaEventCreate(&open_ev);
        cudaEventRecord(open_ev, st);
        open_phase = phase;
    }
    void end() {
        if (!out || open_phase < 0) return;
        cudaEvent_t e;
        cudaEventCreate(&e);
        cudaEventRecord(e, st);
        spans.push_back({open_phase, {open_ev, e}});
        open_phase = -1;
    }
    void finish() {
        if (!out) return;
        for (auto& sp : spans) {
            float ms = 0;
            cudaEventSynchronize(sp.second.second);
            cudaEventElapsedTime(&ms, sp.second.first, sp.second.second);
            out[sp.first] += ms;
            cudaEventDestroy(sp.second.first);
            cudaEventDestroy(sp.second.second);
        }
        spans.clear();
    }
};

// ---------------------------------------------------------------------------
// Key-switch MAC on the tcgen05 INT8 tensor cores.
//
// For one limb l and slot s the MAC of a ciphertext group and a set of
// Galois keys is a matrix product over the digits j:
//   acc[c][g][comp] = sum_j Y[c][j] * K_g[j][comp]        (mod q_l)
// Both operands are split into bytes. With w_b = 2^(8b) Y mod q (canonical),
//   sum_j Y K = sum_j sum_b byte_b(K) 2^(8b) Y  ==  sum_(j,b) byte_b(K) w_b   (mod q)
// and w_b = sum_a 2^(8a) byte_a(w_b), so
//   acc[c][g][comp] == sum_a 2^(8a) P[(g,comp)][(c,a)]  (mod q),
//   P[(g,comp)][(c,a)] = sum_(j,b) byte_b(K_g[j][comp]) * byte_a(w_b(Y[c][j]))
// an exact unsigned 8-bit product with K = 8 D' terms (D' = D rounded up to a
// multiple of 4) and 32-bit accumulation (< 8 D' 255^2 < 2^31 for D' <= 4096).
// One tcgen05.mma.kind::i8 per (slot, 4 digits): M = 64 rows (32 keys x 2
// components), N = 128 columns (16 ciphertexts x 8 byte planes), K = 32 bytes.
// A (keys) is K-major: row (g, comp) holds the key words of 4 digits; B is
// MN-major: for each (digit j, weight b) the 16 words w_b(Y[c][j]) lie in
// order. Both use the no-swizzle canonical layout (8 x 16-byte core matrices).
//
// Warp roles of a persistent CTA (one per SM, all 512 TMEM columns):
//   producers  (warps kEpiWarps..11, groups of four taking alternate items):
//              for item t a group issues the bulk copy of the packed key block
//              and the cp.async of the digit transforms of item t + kAhead into
//              an 8-deep ring, then builds the B operand of item t (B stage
//              t % kBStages);
//   warp 12    issues the MMAs of item t once its operands are ready;
//   epilogue   (warps 0..kEpiWarps-1, warp w on TMEM lane quadrant w % 4; with
//              8 warps, warp w takes slot pair w / 4): TMEM -> exact combine of
//              the 8 planes, reduction mod q and sparse carry corrections, stores.
// An item is (tile of 4 slots of one limb, key chunk, 4-digit chunk); the
// accumulators of consecutive (tile, key chunk) units alternate between two
// TMEM column halves, so the epilogue of one unit overlaps the MMAs of the
// next. Stages are handed over with mbarriers (ready, empty, full, free);
// every wait is bounded and on a timeout the kernel records an error, drains
// and frees its TMEM.
namespace tc {

constexpr int kTS = 4;            // slots per tile
constexpr int kCt = 16;           // ciphertexts per group (N = 8 kCt = 128)
constexpr int kKeys = 32;         // keys per pass (M = 2 kKeys = 64)
// Digits per item (CKKS_TC_DIGITS): 4 (one K = 32 MMA per slot) or 8 (two, with
// half as many items, so the per-item waits and copy issue cover twice the work).
#ifndef CKKS_TC_DIGITS
#define CKKS_TC_DIGITS 4
#endif
constexpr int kJc = CKKS_TC_DIGITS;  // digits per item
constexpr int kSub = kJc / 4;        // MMAs (K = 32 bytes, 4 digits) per slot and item
static_assert(kJc == 4 || kJc == 8, "digits per item");
// Tuning (measured on B200, see the design notes): epilogue warps (4 or 8; the
// other 12 - kEpiWarps warps produce, in groups of 4 that take alternate items)
// and B stages (2 or 4; the prefetch distance is kRing - kBStages items).
#ifndef CKKS_TC_EPI_WARPS
#define CKKS_TC_EPI_WARPS 4
#endif
#ifndef CKKS_TC_BSTAGES
#define CKKS_TC_BSTAGES 2
#endif
#ifndef CKKS_TC_PROD_WARPS
#define CKKS_TC_PROD_WARPS 8
#endif
// Two CTAs per SM (CKKS_TC_TWO_CTAS): twice the warps to hide the latency
// chains of each role, at half the rings, 72 registers a thread and one TMEM
// accumulator buffer (256 columns) per CTA: the other CTA's MMAs overlap an
// epilogue instead of the CTA's own second buffer.
#ifndef CKKS_TC_TWO_CTAS
#define CKKS_TC_TWO_CTAS 0
#endif
constexpr int kCtasPerSm = CKKS_TC_TWO_CTAS ? 2 : 1;
constexpr int kAccBufs = CKKS_TC_TWO_CTAS ? 1 : 2;  // TMEM accumulator buffers (256 columns each)
constexpr int kEpiWarps = CKKS_TC_EPI_WARPS;
constexpr int kBStages = CKKS_TC_BSTAGES;      // B operand stages
constexpr int kRing = (CKKS_TC_TWO_CTAS || kJc == 8) ? 4 : 8;  // Y prefetch ring depth
constexpr int kAhead = kRing - kBStages;       // items whose Y is fetched ahead
#ifndef CKKS_TC_ARING
#define CKKS_TC_ARING ((CKKS_TC_TWO_CTAS || CKKS_TC_DIGITS == 8) ? 8 : 16)
#endif
constexpr int kARing = CKKS_TC_ARING;          // A (packed key block) ring depth
constexpr int kAAhead = kARing - 2 * kBStages;  // items whose A block is fetched ahead
constexpr int kGroups = CKKS_TC_PROD_WARPS / 4;  // producer groups of 4 warps
constexpr int kProdWarp0 = kEpiWarps, kMmaWarp = kEpiWarps + CKKS_TC_PROD_WARPS;
constexpr int kThreads = 32 * (kMmaWarp + 1);  // epilogue, producers, 1 MMA warp
constexpr int kGrp = 128, kEpi = 32 * kEpiWarps;  // threads per producer group, epilogue threads
constexpr int kBarGrp0 = 1, kBarEpi = 3;       // named barriers: producer groups 1, 2; epilogue 3
static_assert((kEpiWarps == 4 || kEpiWarps == 8) && (kBStages == 2 || kBStages == 4) &&
                  (CKKS_TC_PROD_WARPS == 4 || CKKS_TC_PROD_WARPS == 8), "tuning range");
static_assert(kAhead % kGroups == 0 && kAAhead % kGroups == 0 && kBStages % kGroups == 0,
              "a group prefetches and builds its own items");
static_assert((kARing & (kARing - 1)) == 0 && kAAhead >= kAhead, "A ring");
// A (packed key block, bulk-copied): row groups of 1 KB, slot i at 256 i, K
// chunks 128 B apart. B strides are padded (slot and digit strides off
// multiples of 128 B) so the producers' shared-memory stores spread over the banks.
constexpr u32 kSboA = 1024, kLboA = 128, kASlot = 256;
constexpr u32 kSboB = 128, kLboB = 1088;       // B: ciphertext pairs, digits
constexpr u32 kBSlot = kJc * kLboB + 16;       // digits x 8 weights x 128 B (+padding)
constexpr u32 kAStage = 8192 * kSub;           // 8 row groups per 4-digit block
constexpr u32 kYStage = kCt * kJc * kTS * 8;   // 2048: Y words [c][jj][i]
constexpr u32 kBStage = kTS * kBSlot;          // 17472
constexpr u32 kOffY = kARing * kAStage;                    // A ring
constexpr u32 kOffB = kOffY + kRing * kYStage;             // 16 KB of Y
constexpr u32 kOffCnt = kOffB + kBStages * kBStage;        // correction counts [c][g], g < kCntKeys
#ifndef CKKS_TC_CNT_KEYS
#define CKKS_TC_CNT_KEYS ((CKKS_TC_TWO_CTAS || CKKS_TC_DIGITS == 8) ? 64 : 256)
#endif
constexpr int kCntKeys = CKKS_TC_CNT_KEYS;  // keys whose correction counts are staged in shared memory
constexpr u32 kSmemBytes = kOffCnt + kCt * kCntKeys * 4;   // 197 KB (16 A slots, 2 B stages): one CTA per SM
static_assert(kSmemBytes * kCtasPerSm + kCtasPerSm * 2048 <= 228 * 1024, "shared memory per SM");
constexpr u32 kTmemCols = 256 * kAccBufs;
// Bounded waits: a waiting thread sleeps in mbarrier.try_wait (woken when the
// phase completes, at the latest after kSuspendNs) so spinning warps do not
// take issue slots from the working ones; it gives up after kWaitCycles.
#ifndef CKKS_TC_SUSPEND_NS
#define CKKS_TC_SUSPEND_NS 20000
#endif
constexpr u32 kSuspendNs = CKKS_TC_SUSPEND_NS;
constexpr long long kWaitCycles = 1ll << 31;   // about a second

__device__ __forceinline__ u32 smem_u32(const void* p) { return (u32)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t sdesc(u32 saddr, u32 lbo, u32 sbo) {
    uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version (sm_100); base offset 0, no swizzle
    return d;
}

// kind::i8 instruction descriptor: D s32, A u8 K-major, B u8 MN-major, N = 128, M = 64.
constexpr u32 kIdesc = (2u << 4) | (0u << 7) | (0u << 10) | (0u << 15) | (1u << 16) | ((128u >> 3) << 17) |
                       ((64u >> 4) << 24);

__device__ __forceinline__ void mma_i8(u32 d_tmem, uint64_t a, uint64_t b, u32 accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(kIdesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void commit(u32 bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

__device__ __forceinline__ void arrive(u32 bar) {
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}\n" ::"r"(bar) : "memory");
}

// true once the phase with the given parity has completed (bounded)
__device__ __forceinline__ bool wait_parity(u32 bar, u32 parity) {
    const long long t0 = clock64();
    do {
        u32 done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(bar), "r"(parity), "r"(kSuspendNs)
            : "memory");
        if (done) return true;
    } while (clock64() - t0 < kWaitCycles);
    return false;
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void named_sync(int id, int n) { asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory"); }
// barrier over the n threads of group `id` that returns the OR of v (one decision for the group)
__device__ __forceinline__ bool group_any(int id, int n, bool v) {
    u32 r;
    asm volatile("{\n\t.reg .pred p, q;\n\tsetp.ne.u32 p, %1, 0;\n\tbar.red.or.pred q, %2, %3, p;\n\t"
                 "selp.u32 %0, 1, 0, q;\n\t}\n"
                 : "=r"(r)
                 : "r"((u32)v), "r"(id), "r"(n)
                 : "memory");
    return r != 0;
}

// 16-byte asynchronous global -> shared copy; src_bytes 0 stores zeros
__device__ __forceinline__ void cp16(u32 dst, const void* src, u32 src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// 32 TMEM lanes x 32 columns: lane L of the warp gets columns 0 .. 31 of lane L.
// The wait is part of the same statement, so no use of r can be scheduled
// before the load has completed.
__device__ __forceinline__ void tmem_ld32(u32 taddr, u32 (&r)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
}

// Position in a CTA's item sequence (tile_local-th tile of the CTA, key chunk,
// digit chunk), advanced by counters instead of divisions.
struct Item {
    int tl, kc, ch;
    __device__ __forceinline__ void next(int n_kc, int n_chunks) {
        if (++ch == n_chunks) {
            ch = 0;
            if (++kc == n_kc) {
                kc = 0;
                ++tl;
            }
        }
    }
};

static_assert(kCt == (int)kGroupMax, "group size of the packed sets");
}  // namespace tc

// Same arguments and results as k_mac_tiled for bounded keys (up to 16
// ciphertexts per call, any number of keys, D < 4096, N >= 4); the A operand
// comes from the packed set of the keys (rg row groups per block).
__global__ void __launch_bounds__(tc::kThreads, tc::kCtasPerSm)
    k_mac_tc(const u64* __restrict__ Yhat, size_t y_stride, const u64* __restrict__ Bhat, size_t b_stride, int Lq,
             const u64* __restrict__ packed, int rg, const u64* const* __restrict__ keys,
             const u64* __restrict__ exps_inv, u64* __restrict__ acc, const NttTab* __restrict__ tabs, LimbMap lm,
             int n_ct, int n_keys, int LK, int D, int log_n, const Exc* __restrict__ exc,
             const u32* __restrict__ exc_count, int cap, const u64* __restrict__ psi, int* __restrict__ err) {
    using namespace tc;
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ u32 s_tmem;
    __shared__ int s_abort;
    // ready / empty: B stages (producer group -> MMA, MMA -> producer group);
    // full / free: TMEM accumulator halves (MMA -> epilogue, epilogue -> MMA);
    // afull: A ring slots (bulk copy -> MMA)
    __shared__ __align__(8) uint64_t s_ready[kBStages], s_empty[kBStages], s_full[kAccBufs], s_free[kAccBufs],
        s_afull[kARing];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const u32 n = 1u << log_n;
    const int n_tiles_s = (int)(n / kTS), lts = log_n - 2;  // tiles per limb (a power of two)
    const int n_tiles = LK * n_tiles_s;
    const int n_chunks = (D + 1 + kJc - 1) / kJc;  // gadget digits and the base digit (P b)
    const int n_kc = (n_keys + kKeys - 1) / kKeys;
    const int per_tile = n_kc * n_chunks;
    const int my_tiles = (int)blockIdx.x < n_tiles ? (n_tiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
    const int n_items = my_tiles * per_tile;
    const int n_units = my_tiles * n_kc;
    const bool cnt_staged = n_keys <= kCntKeys;
    if (tid == 0) {
        s_abort = 0;
        for (int i = 0; i < kBStages; ++i) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&s_ready[i])), "r"(1));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&s_empty[i])), "r"(1));
        }
        for (int i = 0; i < kAccBufs; ++i) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&s_full[i])), "r"(1));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&s_free[i])), "r"(1));
        }
        for (int i = 0; i < kARing; ++i)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&s_afull[i])), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == kMmaWarp) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                     "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    // zero the operand rings once: A rows of absent keys and B columns of
    // absent ciphertexts stay zero; stage the correction counts
    for (u32 i = tid; i < kOffCnt / 16; i += kThreads) ((uint4*)smem)[i] = make_uint4(0, 0, 0, 0);
    u32* s_cnt = (u32*)(smem + kOffCnt);
    if (cnt_staged)
        for (int w = tid; w < kCt * n_keys; w += kThreads)
            s_cnt[w] = w / n_keys < n_ct ? exc_count[(size_t)(w / n_keys) * n_keys + w % n_keys] : 0u;
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // zeros before the bulk copies
    fence_before();
    __syncthreads();
    fence_after();
    const u32 tmem = s_tmem;
    const u32 sbase = smem_u32(smem);

    if (warp >= kProdWarp0 && warp < kMmaWarp) {
        // ------------------------------------------------------------ producers
        const int ptid = tid - kProdWarp0 * 32;
        const int grp = ptid / kGrp, gtid = ptid % kGrp, bar = kBarGrp0 + grp;
        // A: one bulk copy of the item's packed key block (thread 0 of the group);
        // Y copies: 16 bytes (slots 2 ph, 2 ph + 1) of digit pjj of ciphertext
        // yc = gtid / 8 (Y words 2 gtid, 2 gtid + 1 of the stage, [c][jj][i]).
        static_assert(kGrp == 128 && kTS * kJc * kCt == 2 * kSub * kGrp, "producer work split");
        // kJc 4: 16 bytes (slots 2 ph, 2 ph + 1) of digit pjj; kJc 8: all 4 slots of digit pjj
        const int ph = kJc == 4 ? (gtid & 1) : 0, pjj = kJc == 4 ? ((gtid >> 1) & 3) : (gtid & 7);
        const int yc = gtid >> 3;
        const int n4 = (D + 1 + 3) / 4;  // 4-digit blocks of the packed set per tile and key chunk
        int last_issued = -1;  // last item whose block this thread copied (thread 0 of a group)
        // A block of item t into A slot t % kARing (thread 0 of the group)
        auto prefetch_a = [&](int t, const Item& it) {
            if (t < n_items && gtid == 0) {
                const int tile = (int)blockIdx.x + it.tl * (int)gridDim.x;
                const int b4 = it.ch * kSub;  // first 4-digit block of the item (consecutive in the set)
                const u32 a_bytes = (u32)((n4 - b4) < kSub ? (n4 - b4) : kSub) * (u32)rg * 1024u;
                const u64* src = packed + ((((size_t)tile * n_kc + it.kc) * n4 + b4) * (size_t)rg << 7);
                const u32 bar = smem_u32(&s_afull[t & (kARing - 1)]);
                asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}\n"
                             ::"r"(bar), "r"(a_bytes) : "memory");
                asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                             ::"r"(sbase + (u32)(t & (kARing - 1)) * kAStage), "l"(src), "r"(a_bytes), "r"(bar)
                             : "memory");
                last_issued = t;
            }
        };
        auto prefetch = [&](int t, const Item& it) {
            if (t < n_items) {
                const int tile = (int)blockIdx.x + it.tl * (int)gridDim.x;
                const int l = tile >> lts;
                const u32 s0 = (u32)(tile & (n_tiles_s - 1)) * kTS;
                // digit j < D: the digit transform; j == D: NTT(b) on the Q limbs
                const int j = it.ch * kJc + pjj;
                const bool jok = j < D, bok = j == D && l < Lq;
                const u64* ysrc = jok ? Yhat + ((((size_t)j * LK + l) << log_n) + s0 + 2 * ph)
                                      : bok ? Bhat + (((size_t)l << log_n) + s0 + 2 * ph) : Yhat;
                const size_t ystep = jok ? y_stride : b_stride;
                const u32 y_st = sbase + kOffY + (u32)(t & (kRing - 1)) * kYStage;
                // 16-byte aligned: s0 is a multiple of 4 slots and the workspaces are 256-byte aligned;
                // stage layout [c][jj][i]
                if (yc < n_ct) {
#pragma unroll
                    for (int h = 0; h < kSub; ++h)
                        cp16(y_st + (u32)(((yc * kJc + pjj) * kTS + 2 * ph + 2 * h) * 8),
                             ysrc + (jok || bok ? yc * ystep + 2 * h : 0), jok || bok ? 16u : 0u);
                }
            }
            cp_commit();
        };
        auto advance = [&](Item& x) {
#pragma unroll
            for (int k = 0; k < kGroups; ++k) x.next(n_kc, n_chunks);
        };
        Item it{0, 0, 0};
        if (grp) it.next(n_kc, n_chunks);
        Item ahead = it, ahead_a = it;
        for (int k = 0; k < kAAhead / kGroups; ++k) {
            prefetch_a(grp + kGroups * k, ahead_a);
            advance(ahead_a);
        }
        for (int k = 0; k < kAhead / kGroups; ++k) {
            prefetch(grp + kGroups * k, ahead);
            advance(ahead);
        }
        int f_limb = -1, q_bits = 0;
        bool near_pow2 = false;
        u64 q = 0, f256 = 0, f256q = 0;  // q_l, 2^8 mod q_l and its Shoup companion
        for (int t = grp; t < n_items; t += kGroups) {
            const int tile = (int)blockIdx.x + it.tl * (int)gridDim.x;
            const int l = tile >> lts;
            const int bst = t & (kBStages - 1);
            bool bad = false;
            // the MMAs of item t - kBStages released B stage bst and ring slot (t + kAhead) % kRing
            if (t >= kBStages) bad = !wait_parity(smem_u32(&s_empty[bst]), (u32)(((t / kBStages) - 1) & 1));
            if (group_any(bar, kGrp, bad || s_abort)) {  // one decision for the group
                if (gtid == 0) {
                    atomicExch(err, 1);
                    s_abort = 1;
                }
                break;
            }
            // the MMAs of item t - kBStages (and so of t + kAAhead - kARing) are done:
            // A slot (t + kAAhead) % kARing and Y slot (t + kAhead) % kRing are free
            prefetch_a(t + kAAhead, ahead_a);
            advance(ahead_a);
            prefetch(t + kAhead, ahead);
            advance(ahead);
            cp_wait<kAhead / kGroups>();  // this thread's copies of item t have landed
            named_sync(bar, kGrp);
            if (l != f_limb) {
                q = tabs[lm(l)].q;
                f256 = 256 % q;
                f256q = shoup_quotient_dev(f256, q);
                q_bits = 64 - __clzll(q);
                near_pow2 = q_bits <= 55 && ((1ull << q_bits) - q) < (1ull << (q_bits - 9));
                f_limb = l;
            }
            // B: w_b(Y[c][j]) == 2^(8b) Y (mod q), lazily reduced below 2^64, for the
            // units (c, slot, digit) and (c + 8, slot, digit): two independent chains.
            // The thread mapping (c & 1, slot, digit & 1 in the low bits) puts a
            // half-warp's 8-byte stores on distinct banks.
            {
                const u64* ys = (const u64*)(smem + kOffY + (t & (kRing - 1)) * kYStage);
                const int c = ((gtid >> 5) << 1) | (gtid & 1), i = (gtid >> 1) & 3, jj = (gtid >> 3) & 3;
                uint8_t* d0 = smem + kOffB + bst * kBStage + i * kBSlot + jj * kLboB + (c >> 1) * kSboB + (c & 1) * 8;
                uint8_t* d1 = d0 + 4 * kSboB;  // ciphertext c + 8
                const bool ok0 = c < n_ct, ok1 = c + 8 < n_ct;
#pragma unroll
                for (int h = 0; h < kSub; ++h) {  // digits jj and (kJc 8) jj + 4
                const int jh = jj + 4 * h;
                uint8_t* d0h = d0 + h * 4 * kLboB;
                uint8_t* d1h = d1 + h * 4 * kLboB;
                u64 w0 = ys[(c * kJc + jh) * kTS + i], w1 = ys[((c + 8) * kJc + jh) * kTS + i];
                if (near_pow2) {
                    // q in (2^e - 2^(e-9), 2^e), e <= 55: w < 2^(e+1) stays below 2^(e+1)
#pragma unroll
                    for (int b = 0; b < 8; ++b) {
                        if (ok0) *(u64*)(d0h + b * 16) = w0;
                        if (ok1) *(u64*)(d1h + b * 16) = w1;
                        const u64 x0 = w0 << 8, x1 = w1 << 8;
                        w0 = x0 - (x0 >> q_bits) * q;
                        w1 = x1 - (x1 >> q_bits) * q;
                    }
                } else {
#pragma unroll
                    for (int b = 0; b < 8; ++b) {
                        if (ok0) *(u64*)(d0h + b * 16) = w0;
                        if (ok1) *(u64*)(d1h + b * 16) = w1;
                        w0 = mul_shoup_lazy(w0, f256, f256q, q);
                        w1 = mul_shoup_lazy(w1, f256, f256q, q);
                    }
                }
                }
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            named_sync(bar, kGrp);
            if (gtid == 0) {
                // the item's key block has landed before its B operand is announced
                if (!wait_parity(smem_u32(&s_afull[t & (kARing - 1)]), (u32)((t / kARing) & 1))) {
                    atomicExch(err, 5);
                    s_abort = 1;  // ready is still announced; the MMA warp stops on the flag
                }
                arrive(smem_u32(&s_ready[bst]));
            }
            advance(it);
        }
        cp_wait<0>();
        // bulk copies still in flight (after an abort) land before the CTA exits:
        // only the group's last kAAhead / kGroups blocks can be outstanding
        if (gtid == 0)
            for (int k = 0; k < kAAhead / kGroups; ++k) {
                const int u = last_issued - kGroups * k;
                if (u >= 0) wait_parity(smem_u32(&s_afull[u & (kARing - 1)]), (u32)((u / kARing) & 1));
            }
    } else if (warp == kMmaWarp) {
        // ------------------------------------------------------------- MMA issue
        if (lane == 0) {
            Item it{0, 0, 0};
            int unit = -1, last_t = -1;
            const u32 a_block = (u32)rg * 1024u;  // one 4-digit block of the packed set
            // Every mbarrier wait costs the issuing thread a few hundred cycles even when the
            // phase is complete, and the MMAs of one item issue back to back: per item this
            // thread waits on `ready` only (the producers have already seen the key block
            // land), and on `free` (plus the tcgen05 fence for the TMEM reuse) once per unit.
            for (int t = 0; t < n_items; ++t, it.next(n_kc, n_chunks)) {
                const int bst = t & (kBStages - 1);
                if (!wait_parity(smem_u32(&s_ready[bst]), (u32)((t / kBStages) & 1))) {
                    atomicExch(err, 2);
                    s_abort = 1;
                    break;
                }
                if (it.ch == 0) {
                    ++unit;
                    if ((unit >= kAccBufs &&
                         !wait_parity(smem_u32(&s_free[unit % kAccBufs]), (u32)(((unit / kAccBufs) - 1) & 1))) ||
                        s_abort) {
                        atomicExch(err, 3);
                        s_abort = 1;
                        break;
                    }
                    fence_after();
                }
                const u32 a0 = sbase + (u32)(t & (kARing - 1)) * kAStage, b0 = sbase + kOffB + (u32)bst * kBStage;
                // accumulator of slot i: columns 256 buf + 128 (i / 2), TMEM lanes 16 (i % 2) + ..
                const u32 dbase = tmem + (u32)(256 * (unit % kAccBufs));
#pragma unroll
                for (int i = 0; i < kTS; ++i)
#pragma unroll
                    for (int h = 0; h < kSub; ++h)  // 4-digit block h of the item: A block h, B digits 4 h ..
                        mma_i8(dbase + ((u32)(16 * (i & 1)) << 16) + (u32)(i >> 1) * 128u,
                               sdesc(a0 + (u32)h * a_block + i * kASlot, kLboA, kSboA),
                               sdesc(b0 + i * kBSlot + (u32)h * 4 * kLboB, kLboB, kSboB),
                               (it.ch > 0 || h > 0) ? 1u : 0u);
                commit(smem_u32(&s_empty[bst]));
                if (it.ch == n_chunks - 1) commit(smem_u32(&s_full[unit % kAccBufs]));
                last_t = t;
            }
            // drain: the last commit covers every MMA issued
            if (last_t >= 0)
                wait_parity(smem_u32(&s_empty[last_t & (kBStages - 1)]), (u32)((last_t / kBStages) & 1));
        }
        __syncwarp();
    } else {
        // -------------------------------------------------------------- epilogue
        // TMEM lane quadrant (lanes 32 qd ..); slot pairs [pp0, pp1) of each unit
        const int qd = warp & 3;
        const int pp0 = kEpiWarps == 8 ? warp >> 2 : 0, pp1 = kEpiWarps == 8 ? pp0 + 1 : kTS / 2;
        int r_limb = -1;
        u64 q = 0, one_q = 0, r64 = 0, r64q = 0;  // q_l, floor(2^64 / q_l), 2^64 mod q_l, Shoup companion
        u64 r32 = 0, r32q = 0;                    // 2^32 mod q_l, Shoup companion
        bool wide_q = false;                      // q_l > 2^49.5: the two-half combine below applies
        Barrett bm{0, 0, 0};
        for (int u = 0; u < n_units; ++u) {
            const int tl = u / n_kc, kc = u - tl * n_kc;
            const int tile = (int)blockIdx.x + tl * (int)gridDim.x;
            const int l = tile >> lts;
            const u32 s0 = (u32)(tile & (n_tiles_s - 1)) * kTS;
            const int g0 = kc * kKeys;
            const int gn = n_keys - g0 < kKeys ? n_keys - g0 : kKeys;
            const bool bad = !wait_parity(smem_u32(&s_full[u % kAccBufs]), (u32)((u / kAccBufs) & 1));
            if (group_any(kBarEpi, kEpi, bad || s_abort)) {  // one decision for all epilogue threads
                if (tid == 0) {
                    atomicExch(err, 4);
                    s_abort = 1;
                }
                break;
            }
            fence_after();
            if (l != r_limb) {
                const NttTab& T = tabs[lm(l)];
                q = T.q;
                bm = Barrett{q, T.mu_hi, T.mu_lo};
                one_q = (~0ull) / q;                 // floor(2^64 / q), q odd
                r64 = (u64)(-(q * one_q));           // 2^64 mod q
                r64q = shoup_quotient_dev(r64, q);
                r32 = (1ull << 32) % q;
                r32q = shoup_quotient_dev(r32, q);
                wide_q = q > 0x2D413CCCFE779ull;  // floor(2^49.5)
                r_limb = l;
            }
            // lane L of warp qd: row m = 16 qd + (L % 16); slot 2 pp + (L / 16) of slot pair pp
            const u32 taddr = tmem + ((u32)(32 * qd) << 16) + (u32)(256 * (u % kAccBufs));
            const int m = 16 * qd + (lane & 15);
            const int gl = m >> 1, comp = m & 1, g = g0 + gl;
            const bool row_ok = gl < gn;
            // ciphertexts of this row whose (ciphertext, key) pair has carry corrections
            // (lists that overflowed are recomputed by the exact fallback: skipped here)
            u32 corr = 0;
            if (row_ok)
                for (int c = 0; c < n_ct; ++c) {
                    const u32 cnt = cnt_staged ? s_cnt[c * n_keys + g] : exc_count[(size_t)c * n_keys + g];
                    if (cnt && cnt <= (u32)cap) corr |= 1u << c;
                }
            // output word (c, s) at acc_row + c * c_stride + s
            u64* acc_row = acc + (((((size_t)g * 2 + comp) * LK + l) << log_n) + s0);
            const size_t c_stride = ((size_t)n_keys * 2 * LK) << log_n;
            // the 4 ciphertexts cb .. cb + 3 of slot 2 pp + (lane / 16) of this row, reduced
            auto slot_values = [&](int pp, int cb, u64 (&v)[4]) {
                const int i = 2 * pp + (lane >> 4);
                const u32 s = s0 + i;
                u32 r[32];
                __syncwarp();
                tmem_ld32(taddr + (u32)(pp * 128 + 8 * cb), r);
                // sum_a 2^(8a) P_a with P_a < 2^25 as L + 2^32 H (L, H < 2^49.01) for the
                // 4 ciphertexts at once: independent chains, no branches
                if (wide_q) {
#pragma unroll
                    for (int cc = 0; cc < 4; ++cc) {
                        const u32* P = r + 8 * cc;
                        const u64 L = (u64)P[0] + ((u64)P[1] << 8) + ((u64)P[2] << 16) + ((u64)P[3] << 24);
                        const u64 H = (u64)P[4] + ((u64)P[5] << 8) + ((u64)P[6] << 16) + ((u64)P[7] << 24);
                        // L < q: 2^32 H mod q lazily in [0, 2q), plus L, below 3q
                        u64 x = mul_shoup_lazy(H, r32, r32q, q) + L;
                        x = x >= 2 * q ? x - 2 * q : x;
                        v[cc] = x >= q ? x - q : x;
                    }
                } else {
#pragma unroll
                    for (int cc = 0; cc < 4; ++cc) {
                        const u32* P = r + 8 * cc;
                        const u64 L = (u64)P[0] + ((u64)P[1] << 8) + ((u64)P[2] << 16) + ((u64)P[3] << 24);
                        const u64 H = (u64)P[4] + ((u64)P[5] << 8) + ((u64)P[6] << 16) + ((u64)P[7] << 24);
                        const u64 lo = L + (H << 32), hi = (H >> 32) + (lo < L);  // exact 128-bit sum
                        v[cc] = add_mod(reduce_2q(mul_shoup_lazy(lo, 1, one_q, q), q), mul_shoup(hi, r64, r64q, q), q);
                    }
                }
                if ((corr >> cb) & 15) {  // rare: sparse carry corrections of the hoisted digits
                    const u64 ps = psi[lm(l)];
                    const u32 k = galois_src(s, exps_inv[g], log_n);
                    const u64* key = keys[g];
                    for (int cc = 0; cc < 4; ++cc) {
                        const int c = cb + cc;
                        if (!((corr >> c) & 1)) continue;
                        const u32 cnt = cnt_staged ? s_cnt[c * n_keys + g] : exc_count[(size_t)c * n_keys + g];
                        const Exc* list = exc + ((size_t)c * n_keys + g) * cap;
                        for (u32 e = 0; e < cnt; ++e) {
                            const Exc xe = list[e];
                            u64 wv = pow_mod_dev(ps, ((2ull * k + 1) * xe.t) & (2ull * n - 1), bm);
                            u64 dm = xe.delta < 0 ? (u64)(-xe.delta) % q : (u64)xe.delta % q;
                            if (xe.delta < 0 && dm) dm = q - dm;
                            const u64 tv = mul_barrett(wv, dm, bm);
                            const size_t kofs = (((size_t)xe.j * LK + l) * 2 + comp) << log_n;
                            v[cc] = add_mod(v[cc], mul_barrett(tv, key[kofs + s], bm), q);
                        }
                    }
                }
            };
            if (kEpiWarps == 4) {
                // Each (row, ciphertext) output is 4 consecutive slots, one 32-byte sector.
                // Lane L holds slots L / 16 and 2 + L / 16 of its row after both column
                // blocks; one exchange with lane L ^ 16 gives lane L < 16 slots 0, 1 and
                // lane L + 16 slots 2, 3, so every store instruction writes whole sectors
                // (16 bytes a lane) instead of half sectors completed by a later instruction.
                const bool lo_half = lane < 16;
                for (int cb = 0; cb < kCt; cb += 4) {
                    u64 va[4], vb[4];
                    slot_values(0, cb, va);
                    slot_values(1, cb, vb);
#pragma unroll
                    for (int cc = 0; cc < 4; ++cc) {
                        const u64 send = lo_half ? vb[cc] : va[cc];
                        const u64 got = ((u64)__shfl_xor_sync(0xffffffffu, (u32)(send >> 32), 16) << 32) |
                                        (u64)__shfl_xor_sync(0xffffffffu, (u32)send, 16);
                        const u64 x0 = lo_half ? va[cc] : got, x1 = lo_half ? got : vb[cc];
                        if (row_ok && cb + cc < n_ct) {
                            u64* dst = acc_row + (size_t)(cb + cc) * c_stride + (lo_half ? 0 : 2);
                            asm volatile("st.global.v2.u64 [%0], {%1, %2};" ::"l"(dst), "l"(x0), "l"(x1) : "memory");
                        }
                    }
                }
            } else {
                for (int pp = pp0; pp < pp1; ++pp) {
                    const int i = 2 * pp + (lane >> 4);
                    for (int cb = 0; cb < kCt; cb += 4) {
                        u64 v[4];
                        slot_values(pp, cb, v);
                        if (row_ok) {
#pragma unroll
                            for (int cc = 0; cc < 4; ++cc)
                                if (cb + cc < n_ct) acc_row[(size_t)(cb + cc) * c_stride + i] = v[cc];
                        }
                    }
                }
            }
            fence_before();
            named_sync(kBarEpi, kEpi);
            if (tid == 0) arrive(smem_u32(&s_free[u % kAccBufs]));
        }
    }
    // teardown: every role has left its loop (on abort, after a bounded wait)
    fence_before();
    __syncthreads();
    fence_after();
    if (warp == kMmaWarp) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
}

// A pinned status buffer from the context and an event marking when the
// device's copies into it are done. The buffer goes back to the context only
// after those copies have landed (also on early error returns).
struct StatusReadback {
    ckks_ctx* ctx;
    void* p = nullptr;
    size_t bytes = 0;
    cudaEvent_t ev = nullptr;
    StatusReadback(ckks_ctx* c, size_t want) : ctx(c) {
        p = pinned_take(ctx, want, &bytes);
        if (p && cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            ev = nullptr;
            pinned_give(ctx, p, bytes);
            p = nullptr;
        }
    }
    bool ok() const { return p && ev; }
    ~StatusReadback() {
        if (!ev) return;
        cudaEventSynchronize(ev);
        cudaEventDestroy(ev);
        pinned_give(ctx, p, bytes);
    }
};

}  // namespace

// sigma_g folded into the inverse transform (pass 1 permutes row columns, pass 2
// rows through shared memory) instead of gathered by ModDown. Measured at the
// 16 ct x 32 keys shape: inverse NTT +2.7 ms, ModDown -1.9 ms per step, so it
// stays off; kept for the fused inverse-transform + ModDown layout.
#ifndef CKKS_FOLD_SIGMA
#define CKKS_FOLD_SIGMA 0
#endif
constexpr bool kFoldSigma = CKKS_FOLD_SIGMA != 0;
// Inverse transform's second pass fused with ModDown on the tensor-core path
// (ntt_inverse_moddown_launch): the Q limbs' inverse-transform output stays on chip.
#ifndef CKKS_FUSE_MODDOWN
#define CKKS_FUSE_MODDOWN 1
#endif
constexpr bool kFuseModDown = CKKS_FUSE_MODDOWN != 0;

// Hoisted hybrid rotations of n_ct ciphertexts by n_keys Galois keys (bounded
// or RNS-block gadget), out [n_ct][n_keys][2][Lq][N]. Ciphertexts are
// processed in groups of up to 4 sharing each streamed key slice.
int32_t rotate_hoisted_ntt(ckks_ctx* ctx, const ckks_ksk* const* keys, u32 n_keys, const u64* ct_in,
                                   u64* ct_out, u32 n_ct, cudaStream_t st, double* phase_ms) {
    PhaseTimer pt;
    pt.out = phase_ms;
    pt.st = st;
    const ckks_ksk* k0 = keys[0];
    const u32 Lq = k0->q_limbs, LK = ksk_limbs(k0), D = k0->D, n = ctx->n;
    const size_t ct_words = (size_t)2 * Lq * n;
    const bool bounded = k0->kind == CKKS_KSK_HYBRID_BOUNDED;
    // Bounded keys use the tensor-core MAC with up to 16 ciphertexts per group
    // (each key word read once per group), as far as device memory allows;
    // otherwise groups of 4 on the CUDA-core tiled MAC.
    bool use_tc = bounded && n >= (u32)tc::kTS && D < 4096 && ctx->tensor_cores && tc_enabled();
    // the tensor-core MAC reads the keys' packed set (made on first use)
    const PackedSet* pset = use_tc ? packed_set_get(ctx, keys, n_keys, st) : nullptr;
    use_tc = pset != nullptr;
    ctx->last_mac_path = use_tc ? 1 : 0;
    u32 G = n_ct >= 4 ? 4 : n_ct;
    if (use_tc) G = n_ct < pset->g_max ? n_ct : pset->g_max;
    const int cap = 1024;
    const LimbMap lqp = LimbMap::qp(ctx, Lq);
    const size_t y_stride = (size_t)D * LK * n, d_stride = (size_t)D * n, f_stride = (size_t)n + 1,
                 b_stride = (size_t)Lq * n;
    Workspace<u64> Y, Bh, acc, Z, karr;
    Workspace<i64> dig;
    Workspace<u32> flags, cnt;
    Workspace<Exc> exc;
    Workspace<int> terr;
    int32_t rc;
    if ((rc = terr.alloc(1, st))) return rc;
    CKKS_CUDA_TRY(cudaMemsetAsync(terr.p, 0, sizeof(int), st));
    // the group size was sized against the free memory when the key set was packed; if the
    // workspaces do not fit now, smaller groups are taken (same words, keys read more often)
    for (;;) {
        if (!(rc = Y.alloc(G * y_stride, st)) && !(use_tc && (rc = Bh.alloc(G * b_stride, st))) &&
            !(rc = acc.alloc((size_t)G * n_keys * 2 * LK * n, st)) &&
            !(rc = Z.alloc((size_t)G * n_keys * 2 * LK * n, st)) &&
            !(rc = karr.alloc(3 * (size_t)n_keys + ctx->moduli.size(), st)) && !(rc = dig.alloc(G * d_stride, st)) &&
            !(rc = flags.alloc(G * f_stride, st)) && !(rc = cnt.alloc((size_t)G * n_keys, st)) &&
            !(rc = exc.alloc((size_t)G * n_keys * cap, st)))
            break;
        if (rc != CKKS_ERR_OOM || G <= 1) return rc;
        Y.release(), Bh.release(), acc.release(), Z.release(), karr.release(), dig.release(), flags.release();
        cnt.release(), exc.release();
        G = G > 4 ? G - 4 : G / 2;
    }
    // the tensor-core path fuses the inverse transform's second pass with ModDown
    // (FP64 networks and ModDown); its P-CRT words
    // (and zp, the K auxiliary limbs of pass 2) need G * n_keys * 2 * N * (4 + K)
    // words, which the accumulators' buffer holds once pass 1 has read it
    const bool fuse_md = use_tc && kFuseModDown && ntt_inverse_moddown_supported(ctx, Lq);
    Workspace<u64> wsp;
    double* words = nullptr;
    u64* zp = nullptr;
    if (fuse_md) {
        const size_t per = (size_t)G * n_keys * 2 * n;
        u64* base = acc.p;
        if (LK < 4 + ctx->K) {
            if ((rc = wsp.alloc(per * (4 + ctx->K), st))) return rc;
            base = wsp.p;
        }
        words = reinterpret_cast<double*>(base);
        zp = base + per * 4;
    }
    // key pointers, exponents and psi per modulus
    std::vector<u64> hk(3 * (size_t)n_keys + ctx->moduli.size());
    for (u32 g = 0; g < n_keys; ++g) {
        hk[g] = (u64)(uintptr_t)keys[g]->d_entries;
        hk[n_keys + g] = keys[g]->exponent;
        hk[2 * n_keys + ctx->moduli.size() + g] = galois_inverse_host(keys[g]->exponent, n);
    }
    for (size_t i = 0; i < ctx->moduli.size(); ++i) hk[2 * n_keys + i] = ctx->psi[i];
    // through a pinned buffer: a copy from pageable memory would first wait for
    // the stream to drain (the previous call's inverse transforms and ModDown),
    // leaving the device idle while this call is enqueued
    StatusReadback up(ctx, hk.size() * 8);
    if (up.ok()) {
        std::memcpy(up.p, hk.data(), hk.size() * 8);
        CKKS_CUDA_TRY(cudaMemcpyAsync(karr.p, up.p, hk.size() * 8, cudaMemcpyHostToDevice, st));
        CKKS_CUDA_TRY(cudaEventRecord(up.ev, st));
    } else {
        CKKS_CUDA_TRY(cudaMemcpyAsync(karr.p, hk.data(), hk.size() * 8, cudaMemcpyHostToDevice, st));
    }
    const u64* const* d_keys = (const u64* const*)karr.p;
    const u64* d_exps = karr.p + n_keys;
    const u64* d_psi = karr.p + 2 * n_keys;
    const u64* d_exps_inv = karr.p + 2 * n_keys + ctx->moduli.size();
    std::vector<u32> overflow;
    std::vector<u32> h_cnt((size_t)G * n_keys);
    // the correction-list counts and the MAC's error flag come back through pinned
    // memory behind the MAC, and the host waits for that event only: the call
    // returns while the inverse transforms and ModDown of the last group still
    // run, so back-to-back calls keep the device busy
    StatusReadback rb(ctx, ((size_t)G * n_keys + 1) * sizeof(u32));
    for (u32 c0 = 0; c0 < n_ct; c0 += G) {
        const u32 gn = (n_ct - c0) < G ? (n_ct - c0) : G;
        CKKS_CUDA_TRY(cudaMemsetAsync(flags.p, 0, G * f_stride * sizeof(u32), st));
        CKKS_CUDA_TRY(cudaMemsetAsync(cnt.p, 0, (size_t)G * n_keys * sizeof(u32), st));
        pt.begin(0);
        if (bounded) {  // the group's decompositions and digit transforms in one launch each
            const u64* in0 = ct_in + (size_t)c0 * ct_words;
            if ((rc = bounded_decompose_launch(ctx, in0 + (size_t)Lq * n, gn, Lq, k0->base_log, dig.p, flags.p, st,
                                               ct_words)))
                return rc;
            if ((rc = ntt_forward_digits_launch(ctx, dig.p, Y.p, D * gn, lqp, LK, st))) return rc;
            if (use_tc) {  // the tensor-core MAC takes P b as one more digit: NTT(b) on the Q limbs
                CKKS_CUDA_TRY(cudaMemcpy2DAsync(Bh.p, b_stride * sizeof(u64), in0, ct_words * sizeof(u64),
                                                b_stride * sizeof(u64), gn, cudaMemcpyDeviceToDevice, st));
                if ((rc = ntt_forward_launch_map(ctx, Bh.p, Bh.p, gn, LimbMap::range(0, Lq), Lq, st))) return rc;
            }
        }
        for (u32 c = 0; c < gn && !bounded; ++c) {
            const u64* in = ct_in + (size_t)(c0 + c) * ct_words;
            {  // RNS blocks: ModUp of a, then transform (the permutation is the whole automorphism)
                if ((rc = rnsblock_modup_launch(ctx, k0, in + (size_t)Lq * n, Y.p + c * y_stride, st))) return rc;
                if ((rc = ntt_forward_launch_map(ctx, Y.p + c * y_stride, Y.p + c * y_stride, D, lqp, LK, st))) return rc;
            }
        }
        pt.end();
        pt.begin(2);
        if (bounded) {
            dim3 g((n + kT - 1) / kT, n_keys, gn);
            k_hoist_exceptions<<<g, kT, 0, st>>>(dig.p, d_stride, flags.p, f_stride, d_exps, n_keys, D,
                                                 k0->base_log, ctx->log_n, exc.p, cnt.p, cap);
        }
        pt.end();
        pt.begin(3);
        if (use_tc) {
            int n_sm = 0;
            CKKS_CUDA_TRY(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, ctx->device));
            const int n_tiles = (int)(LK * (n / tc::kTS));
            CKKS_CUDA_TRY(cudaFuncSetAttribute(k_mac_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)tc::kSmemBytes));
            if (tc::kCtasPerSm > 1)  // the whole carveout as shared memory, so two CTAs fit an SM
                CKKS_CUDA_TRY(cudaFuncSetAttribute(k_mac_tc, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
            const int n_cta = n_sm * tc::kCtasPerSm;
            k_mac_tc<<<n_tiles < n_cta ? n_tiles : n_cta, tc::kThreads, tc::kSmemBytes, st>>>(
                Y.p, y_stride, Bh.p, b_stride, (int)Lq, pset->d, (int)pset->rg, d_keys, d_exps_inv, acc.p,
                ctx->d_tabs, lqp, (int)gn,
                (int)n_keys, (int)LK, (int)D, (int)ctx->log_n, exc.p, cnt.p, cap, d_psi, terr.p);
        } else {
            const size_t smem = (size_t)(G >= 3 ? 4 : G) * D * kS * sizeof(u64);
            if (n >= (u32)kS && smem <= 200 * 1024) {
                dim3 g(n / kS, LK);
#define CKKS_MACT(GG)                                                                                              \
    do {                                                                                                           \
        cudaFuncSetAttribute(k_mac_tiled<GG>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);            \
        k_mac_tiled<GG><<<g, kS * kLanes, (size_t)GG * D * kS * sizeof(u64), st>>>(                              \
            Y.p, y_stride, d_keys, d_exps_inv, acc.p, ctx->d_tabs, lqp, gn, n_keys, Lq, LK, D, ctx->log_n, exc.p,  \
            cnt.p, cap, d_psi);                                                                                    \
    } while (0)
                if (G >= 3) CKKS_MACT(4);
                else if (G == 2) CKKS_MACT(2);
                else CKKS_MACT(1);
#undef CKKS_MACT
            } else {
                dim3 g((n + kT - 1) / kT, n_keys, LK);
#define CKKS_MAC(GG)                                                                                               \
    k_mac_hoisted<GG><<<g, kT, 0, st>>>(Y.p, y_stride, d_keys, d_exps_inv, acc.p, ctx->d_tabs, lqp, gn, n_keys, Lq, \
                                        LK, D, ctx->log_n, exc.p, cnt.p, cap, d_psi)
                if (G >= 3) CKKS_MAC(4);
                else if (G == 2) CKKS_MAC(2);
                else CKKS_MAC(1);
#undef CKKS_MAC
            }
        }
        CKKS_CUDA_TRY(cudaGetLastError());
        pt.end();
        if (rb.ok()) {
            u32* hc = (u32*)rb.p;
            CKKS_CUDA_TRY(cudaMemcpyAsync(hc, cnt.p, (size_t)gn * n_keys * sizeof(u32), cudaMemcpyDeviceToHost, st));
            CKKS_CUDA_TRY(cudaMemcpyAsync(hc + (size_t)G * n_keys, terr.p, sizeof(int), cudaMemcpyDeviceToHost, st));
            CKKS_CUDA_TRY(cudaEventRecord(rb.ev, st));
        }
        pt.begin(4);
        // inverse transform; the b components get P b of their ciphertext added on the
        // Q limbs (ModDown(x + P b) = ModDown(x) + b: the base term of the rotation)
        InvBase ib;  // the tensor-core MAC already added P NTT(b) (base digit)
        ib.b = use_tc ? nullptr : ct_in + (size_t)c0 * ct_words;
        ib.b_stride = ct_words;
        ib.n_keys = n_keys;
        ib.q_limbs = Lq;
        ib.pf = ctx->d_pmodq;
        ib.pf_q = ctx->d_pmodq + ctx->L;
        // the tensor-core path folds sigma_g into the inverse transform (ModDown then
        // streams without a gather); the CUDA-core path adds P b in the inverse
        // transform and applies sigma_g in ModDown
        GaloisOut go;
        if (use_tc && kFoldSigma) {
            go.exps = d_exps;
            go.exps_inv = d_exps_inv;
            go.n_keys = n_keys;
        }
        if (fuse_md) {
            // sigma folded into pass 1; pass 2 of the auxiliary limbs leaves the P-CRT
            // words (in the accumulators' buffer, which pass 1 has consumed) and pass 2
            // of each Q limb writes its ModDown output directly
            GaloisOut gf;
            gf.exps = d_exps;
            gf.exps_inv = d_exps_inv;
            gf.n_keys = n_keys;
            if ((rc = ntt_inverse_moddown_launch(ctx, acc.p, Z.p, words, zp, ct_out + (size_t)c0 * n_keys * ct_words,
                                                 gn * n_keys * 2, Lq, gf, st)))
                return rc;
            pt.end();
            pt.begin(5);
            pt.end();
        } else {
            if ((rc = ntt_inverse_base_launch(ctx, acc.p, Z.p, gn * n_keys * 2, lqp, LK, ib, st, go))) return rc;
            pt.end();
            pt.begin(5);
            // ModDown of every (ciphertext, key) pair (and sigma_g unless folded above), into the output
            if ((rc = mod_down_sigma_multi(ctx, Z.p, ct_out + (size_t)c0 * n_keys * ct_words, gn * n_keys * 2, Lq,
                                           go.exps ? nullptr : d_exps_inv, n_keys, st)))
                return rc;
            pt.end();
        }
        // pairs whose correction lists overflowed are recomputed exactly
        int h_err = 0;
        if (rb.ok()) {
            CKKS_CUDA_TRY(cudaEventSynchronize(rb.ev));
            const u32* hc = (const u32*)rb.p;
            std::memcpy(h_cnt.data(), hc, (size_t)gn * n_keys * sizeof(u32));
            std::memcpy(&h_err, hc + (size_t)G * n_keys, sizeof(int));
        } else {  // no pinned memory: pageable copies and a stream synchronisation
            CKKS_CUDA_TRY(cudaMemcpyAsync(h_cnt.data(), cnt.p, (size_t)G * n_keys * sizeof(u32),
                                          cudaMemcpyDeviceToHost, st));
            CKKS_CUDA_TRY(cudaMemcpyAsync(&h_err, terr.p, sizeof(int), cudaMemcpyDeviceToHost, st));
            CKKS_CUDA_TRY(cudaStreamSynchronize(st));
        }
        if (h_err) {
            ckks_set_error("key-switch MAC: a tensor-core pipeline wait timed out");
            return CKKS_ERR_TIMEOUT;
        }
        for (u32 c = 0; c < gn; ++c)
            for (u32 g = 0; g < n_keys; ++g)
                if (h_cnt[(size_t)c * n_keys + g] > (u32)cap) overflow.push_back(((c0 + c) << 16) | g);
    }
    pt.finish();
    for (u32 code : overflow) {
        const u32 c = code >> 16, g = code & 0xffff;
        if ((rc = rotate_hybrid(ctx, keys[g], ct_in + (size_t)c * ct_words,
                                ct_out + ((size_t)c * n_keys + g) * ct_words, 1, st)))
            return rc;
    }
    return CKKS_OK;
}
