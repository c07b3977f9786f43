// park.cu -- Park et al. modular plaintext matrix product (Mod-PP-MM) on the GPU.
//
// park_mod_pp_mm (ccmm/park.rs:1634-1647) multiplies two u64 matrices modulo an
// arbitrary modulus q > 1: out = (lhs x rhs) mod q, lhs rows x inner, rhs
// inner x cols, row-major. Every backend of the reference
// (park_matrix_mul_{reference,transposed_rhs,wide_accumulator,parallel_wide},
// :1405-1620) returns the canonical residue of the exact integer dot product,
// and so do both device backends here.
//
// Tensor cores (default). With nb = bytes of q - 1, a = sum_i 2^(8i) a_i
// (bytes of lhs mod q) and the weights W_i = 2^(8i) (rhs mod q) mod q split into
// bytes w_ij,
//   sum_k lhs[r][k] rhs[k][c] == sum_j 2^(8j) P_j[r][c]              (mod q),
//   P_j[r][c] = sum_(k,i) a_i[r][k] w_ij[k][c],
// exact unsigned 8-bit products summed in 32 bits on tcgen05.mma.kind::i8 (an
// inner chunk keeps nb * 32 * blocks * 255^2 below 2^31; longer inner sums take
// several launches that add their residues). Two packing kernels write both
// operands as 32-byte inner steps in the canonical K-major core-matrix order
// (A: 128 rows x 32 bytes; B: nb x ct rows (j, column) x 32 bytes, ct output
// columns per tile with nb ct <= 256), so each pipeline stage is two bulk
// copies. The GEMM is a persistent kernel: one producer thread (bulk copies
// into 4 stages of 4 inner steps), one MMA thread (M = 128, N = nb ct, K = 32 per step),
// four epilogue warps (plane combine, one reduction per output); the two TMEM
// accumulator sets let a tile's epilogue overlap the next tile's MMAs.
//
// CUDA cores. A CTA computes a 64 x 64 block of outputs with 256 threads (4 x 4
// outputs each, strided by 16 so a warp's loads of a staged tile row are
// consecutive), staging 16-deep slices of both operands in shared memory; each
// dot product is summed exactly in 192 bits (any u64 inputs, up to 2^64 terms)
// and reduced once.
#include "context.cuh"
#include "kernels.cuh"
#include "tcgen05.cuh"

namespace {

constexpr int kTile = 64, kDepth = 16, kThreads = 256;

typedef unsigned __int128 u128;

struct Acc192 {
    u64 lo, mid, hi;
    __device__ __forceinline__ void add(u64 a, u64 b) {
        const u64 pl = a * b, ph = __umul64hi(a, b);
        asm("add.cc.u64 %0, %0, %3;\n\taddc.cc.u64 %1, %1, %4;\n\taddc.u64 %2, %2, 0;"
            : "+l"(lo), "+l"(mid), "+l"(hi)
            : "l"(pl), "l"(ph));
    }
};

// (hi 2^128 + mid 2^64 + lo) mod q with r64 = 2^64 mod q, r128 = 2^128 mod q
__device__ __forceinline__ u64 reduce192(const Acc192& a, u64 q, u64 r64, u64 r128) {
    const u128 Q = q;
    u128 t = (u128)(a.hi % q) * r128 % Q;
    t = (t + (u128)(a.mid % q) * r64 % Q) % Q;
    t = (t + a.lo % q) % Q;
    return (u64)t;
}

__global__ void __launch_bounds__(kThreads) k_park_mm(const u64* __restrict__ A, const u64* __restrict__ B,
                                                      u64* __restrict__ C, int rows, int inner, int cols, u64 q,
                                                      u64 r64, u64 r128) {
    __shared__ u64 sa[kDepth][kTile + 1];  // sa[k][r]: lhs[row0 + r][k0 + k]
    __shared__ u64 sb[kDepth][kTile];      // sb[k][c]: rhs[k0 + k][col0 + c]
    const int tid = threadIdx.x;
    const int tr = tid >> 4, tc = tid & 15;  // outputs (tr + 16 i, tc + 16 j)
    const int row0 = blockIdx.y * kTile, col0 = blockIdx.x * kTile;
    Acc192 acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = Acc192{0, 0, 0};
    for (int k0 = 0; k0 < inner; k0 += kDepth) {
        // stage lhs [64 x 16] (transposed) and rhs [16 x 64]; zeros outside the matrices
        for (int w = tid; w < kTile * kDepth; w += kThreads) {
            const int r = w / kDepth, k = w % kDepth;
            const int gr = row0 + r, gk = k0 + k;
            sa[k][r] = (gr < rows && gk < inner) ? A[(size_t)gr * inner + gk] : 0;
            const int kk = w / kTile, c = w % kTile;
            const int gk2 = k0 + kk, gc = col0 + c;
            sb[kk][c] = (gk2 < inner && gc < cols) ? B[(size_t)gk2 * cols + gc] : 0;
        }
        __syncthreads();
#pragma unroll 4
        for (int k = 0; k < kDepth; ++k) {
            u64 a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = sa[k][tr + 16 * i];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = sb[k][tc + 16 * j];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j].add(a[i], b[j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int gr = row0 + tr + 16 * i;
        if (gr >= rows) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int gc = col0 + tc + 16 * j;
            if (gc < cols) C[(size_t)gr * cols + gc] = reduce192(acc[i][j], q, r64, r128);
        }
    }
}

// ----------------------------------------------------------------- tensor cores
namespace ptc {

using namespace tcg;

constexpr int kEpiWarps = 4, kProdWarp = 4, kMmaWarp = 5, kThreads = 32 * 6;
constexpr int kEpi = 32 * kEpiWarps, kBarEpi = 1;
#ifndef CKKS_PARK_STEPS
#define CKKS_PARK_STEPS 4
#endif
// inner steps of 32 bytes per stage (one barrier wait per kSteps MMAs), stages in 192 KB
constexpr int kSteps = CKKS_PARK_STEPS, kStages = 16 / kSteps;
static_assert(kSteps == 1 || kSteps == 2 || kSteps == 4 || kSteps == 8, "inner steps per stage");
constexpr u32 kATile = 128 * 32;        // A step: 128 rows x 32 bytes
constexpr u32 kOffB = kSteps * kATile;  // B steps after the stage's A steps (up to 256 rows x 32 bytes each)
constexpr u32 kStageBytes = kOffB + kSteps * 256 * 32;
constexpr u32 kSmemBytes = kStages * kStageBytes;  // 192 KB: one CTA per SM
constexpr u32 kTmemCols = 512;                                     // two accumulator sets of <= 256 columns
constexpr u32 kLbo = 128, kSbo = 256;  // K-major, no swizzle: K halves 128 B apart, 8-row groups 256 B

// output columns per tile for nb bytes per residue: nb * ct <= 256, a multiple of 16
constexpr int cols_per_tile(int nb) {
    return ((256 / nb) / 8 * 8 * nb) % 16 ? (256 / nb) / 8 * 8 - 8 : (256 / nb) / 8 * 8;
}
// inner 32-blocks per launch: every P_j stays below 2^31
constexpr int blocks_per_launch(int nb) { return (int)(0x7FFFFFFFull / (65025ull * (u64)nb) / 32); }

// tile order: row tiles vary fastest (CTAs that run together share column tiles of B'')
#ifndef CKKS_PARK_COLS_FIRST
#define CKKS_PARK_COLS_FIRST 0
#endif
__device__ __forceinline__ int tile_row(int t, int n_mt, int n_nt) { return CKKS_PARK_COLS_FIRST ? t / n_nt : t % n_mt; }
__device__ __forceinline__ int tile_col(int t, int n_mt, int n_nt) { return CKKS_PARK_COLS_FIRST ? t % n_nt : t / n_mt; }

__device__ __forceinline__ u32 core_off(int row, int half) { return (u32)((row >> 3) * 256 + half * 128 + (row & 7) * 16); }

// bytes `shift` .. of 16 values as one 16-byte core-matrix row
__device__ __forceinline__ uint4 pack16(const u64 (&v)[16], int shift) {
    u32 w[4];
#pragma unroll
    for (int g = 0; g < 4; ++g)
        w[g] = (u32)((v[4 * g] >> shift) & 255) | (u32)((v[4 * g + 1] >> shift) & 255) << 8 |
               (u32)((v[4 * g + 2] >> shift) & 255) << 16 | (u32)((v[4 * g + 3] >> shift) & 255) << 24;
    return make_uint4(w[0], w[1], w[2], w[3]);
}

// A' [n_mt][n_kb][nb][128 x 32 bytes]: step (kb, i) of row tile mt holds byte i of
// lhs[128 mt + row][32 kb + k] mod q. One thread per (row, 16-deep run).
__global__ void k_pack_a(const u64* __restrict__ A, uint8_t* __restrict__ Ap, int rows, int inner, u64 q, int nb,
                         int n_mt, int n_kb) {
    const size_t runs = (size_t)2 * n_kb, total = (size_t)n_mt * 128 * runs;
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const int row = (int)(t / runs), h = (int)(t % runs);
        u64 v[16];
#pragma unroll
        for (int e = 0; e < 16; ++e) {
            const int k = 16 * h + e;
            const u64 x = (row < rows && k < inner) ? A[(size_t)row * inner + k] : 0;
            v[e] = x < q ? x : x % q;
        }
        uint8_t* dst = Ap + ((size_t)(row >> 7) * n_kb + (h >> 1)) * nb * kATile + core_off(row & 127, h & 1);
        for (int i = 0; i < nb; ++i) *(uint4*)(dst + (size_t)i * kATile) = pack16(v, 8 * i);
    }
}

// B'' [n_nt][n_kb][nb][nb ct x 32 bytes]: step (kb, i), row j ct + c holds byte j of
// 2^(8i) (rhs[32 kb + k][ct nt + c] mod q) mod q. One thread per (column, 16-deep run).
// f256q = floor(2^72 / q): the weights step by a Shoup product with 256 when
// 256 < q <= 2^63 (f256q != 0), else by a 128-bit remainder.
__global__ void k_pack_b(const u64* __restrict__ B, uint8_t* __restrict__ Bp, int inner, int cols, u64 q, int nb,
                         int ct, int n_nt, int n_kb, u64 f256q) {
    const int cpad = n_nt * ct;
    const size_t total = (size_t)cpad * 2 * n_kb;
    const u32 b_step = (u32)(nb * ct) * 32;
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const int c = (int)(t % cpad), h = (int)(t / cpad);
        const int nt = c / ct, cl = c - nt * ct;
        u64 w[16];
#pragma unroll
        for (int e = 0; e < 16; ++e) {
            const int k = 16 * h + e;
            const u64 x = (c < cols && k < inner) ? B[(size_t)k * cols + c] : 0;
            w[e] = x < q ? x : x % q;
        }
        uint8_t* base = Bp + ((size_t)nt * n_kb + (h >> 1)) * nb * b_step;
        for (int i = 0; i < nb; ++i) {
            if (i > 0 && f256q) {
#pragma unroll
                for (int e = 0; e < 16; ++e) w[e] = mul_shoup(w[e], 256, f256q, q);
            } else if (i > 0) {
#pragma unroll
                for (int e = 0; e < 16; ++e) w[e] = (u64)(((u128)w[e] << 8) % q);
            }
            for (int j = 0; j < nb; ++j)
                *(uint4*)(base + (size_t)i * b_step + core_off(j * ct + cl, h & 1)) = pack16(w, 8 * j);
        }
    }
}

// Inner blocks kb0 .. kb1 - 1 of every (row tile, column tile); accumulate: add
// the residues already in C. `err` receives the role of a timed-out wait.
template <int NB>
__global__ void __launch_bounds__(kThreads, 1)
    k_park_tc(const uint8_t* __restrict__ Ap, const uint8_t* __restrict__ Bp, u64* __restrict__ C, int rows,
              int cols, u64 q, int n_mt, int n_nt, int n_kb, int kb0, int kb1, int accumulate, int* __restrict__ err) {
    constexpr int kCt = cols_per_tile(NB), kRows = NB * kCt;
    constexpr u32 kBStep = (u32)kRows * 32;
    constexpr u32 kIdesc = idesc_i8(128, kRows, false);
    static_assert(kRows <= 256 && kRows % 16 == 0 && kCt % 8 == 0, "tile shape");
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ u32 s_tmem;
    __shared__ int s_abort;
    __shared__ __align__(8) uint64_t s_full[kStages], s_empty[kStages], s_tfull[2], s_tfree[2];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int n_tiles = n_mt * n_nt;
    const int my_tiles = (int)blockIdx.x < n_tiles ? (n_tiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
    const int steps = (kb1 - kb0) * NB;
    const u64 mu = ~0ull / q;
    if (tid == 0) {
        s_abort = 0;
        for (int i = 0; i < kStages; ++i) {
            mbar_init(smem_u32(&s_full[i]), 1);
            mbar_init(smem_u32(&s_empty[i]), 1);
        }
        for (int i = 0; i < 2; ++i) {
            mbar_init(smem_u32(&s_tfull[i]), 1);
            mbar_init(smem_u32(&s_tfree[i]), 1);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == kMmaWarp) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                     "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    fence_before();
    __syncthreads();
    fence_after();
    const u32 tmem = s_tmem, sbase = smem_u32(smem);

    if (warp == kProdWarp) {
        // ------------------------------------------------------------ producer
        if (lane == 0) {
            int g = 0;
            bool bad = false;
            for (int lt = 0; lt < my_tiles && !bad; ++lt) {
                const int t = (int)blockIdx.x + lt * (int)gridDim.x;
                const int mt = tile_row(t, n_mt, n_nt), nt = tile_col(t, n_mt, n_nt);
                const uint8_t* a = Ap + ((size_t)mt * n_kb + kb0) * NB * kATile;
                const uint8_t* b = Bp + ((size_t)nt * n_kb + kb0) * NB * kBStep;
                for (int s = 0; s < steps; s += kSteps, ++g) {
                    const int st = g % kStages;
                    const u32 n = (u32)(steps - s < kSteps ? steps - s : kSteps);
                    if ((g >= kStages && !wait_parity(smem_u32(&s_empty[st]), (u32)(((g / kStages) - 1) & 1))) ||
                        s_abort) {
                        atomicExch(err, 1);
                        s_abort = 1;
                        bad = true;
                        break;
                    }
                    const u32 bar = smem_u32(&s_full[st]), dst = sbase + (u32)st * kStageBytes;
                    expect_tx(bar, n * (kATile + kBStep));
                    bulk_g2s(dst, a + (size_t)s * kATile, n * kATile, bar);
                    bulk_g2s(dst + kOffB, b + (size_t)s * kBStep, n * kBStep, bar);
                }
            }
            // every copy issued has landed before the CTA can leave (bounded)
            for (int x = g - kStages < 0 ? 0 : g - kStages; x < g; ++x)
                wait_parity(smem_u32(&s_full[x % kStages]), (u32)((x / kStages) & 1));
        }
        __syncwarp();
    } else if (warp == kMmaWarp) {
        // ------------------------------------------------------------ MMA issue
        if (lane == 0) {
            int g = 0, last = -1;
            bool bad = false;
            for (int lt = 0; lt < my_tiles && !bad; ++lt) {
                const int buf = lt & 1;
                if (lt >= 2 && !wait_parity(smem_u32(&s_tfree[buf]), (u32)(((lt >> 1) - 1) & 1))) {
                    atomicExch(err, 3);
                    s_abort = 1;
                    break;
                }
                fence_after();
                for (int s = 0; s < steps; s += kSteps, ++g) {
                    const int st = g % kStages;
                    const int n = steps - s < kSteps ? steps - s : kSteps;
                    if (!wait_parity(smem_u32(&s_full[st]), (u32)((g / kStages) & 1)) || s_abort) {
                        atomicExch(err, 2);
                        s_abort = 1;
                        bad = true;
                        break;
                    }
                    fence_after();
                    const u32 a_addr = sbase + (u32)st * kStageBytes, b_addr = a_addr + kOffB;
#pragma unroll
                    for (int u = 0; u < kSteps; ++u)
                        if (u < n)
                            mma_i8(tmem + (u32)buf * 256u, sdesc(a_addr + (u32)u * kATile, kLbo, kSbo),
                                   sdesc(b_addr + (u32)u * kBStep, kLbo, kSbo), kIdesc, (s + u) > 0 ? 1u : 0u);
                    commit(smem_u32(&s_empty[st]));
                    last = g;
                }
                if (!bad) commit(smem_u32(&s_tfull[buf]));
            }
            // the last commit covers every MMA issued
            if (last >= 0) wait_parity(smem_u32(&s_empty[last % kStages]), (u32)((last / kStages) & 1));
        }
        __syncwarp();
    } else if (warp < kEpiWarps) {
        // ------------------------------------------------------------- epilogue
        for (int lt = 0; lt < my_tiles; ++lt) {
            const int buf = lt & 1;
            const int t = (int)blockIdx.x + lt * (int)gridDim.x;
            const int mt = tile_row(t, n_mt, n_nt), nt = tile_col(t, n_mt, n_nt);
            const bool bad = !wait_parity(smem_u32(&s_tfull[buf]), (u32)((lt >> 1) & 1));
            if (group_any(kBarEpi, kEpi, bad || s_abort)) {
                if (tid == 0) {
                    atomicExch(err, 4);
                    s_abort = 1;
                }
                break;
            }
            fence_after();
            const int row = 128 * mt + 32 * warp + lane, cmax = cols - nt * kCt;
            const u32 taddr = tmem + ((u32)(32 * warp) << 16) + (u32)buf * 256u;
            u64* out = C + (size_t)row * cols + (size_t)nt * kCt;
#pragma unroll 1
            for (int c0 = 0; c0 < kCt; c0 += 8) {
                u64 r[8];
                if constexpr (NB <= 5) {  // sum_j 2^(8j) P_j < 2^63.01
                    u64 v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
                    for (int j = 0; j < NB; ++j) {
                        u32 P[8];
                        tmem_ld8(taddr + (u32)(j * kCt + c0), P);
#pragma unroll
                        for (int cc = 0; cc < 8; ++cc) v[cc] += (u64)P[cc] << (8 * j);
                    }
#pragma unroll
                    for (int cc = 0; cc < 8; ++cc) {  // v - floor(v mu / 2^64) q < 3q
                        u64 x = v[cc] - __umul64hi(v[cc], mu) * q;
                        x = x >= q ? x - q : x;
                        r[cc] = x >= q ? x - q : x;
                    }
                } else {
                    u128 v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
                    for (int j = 0; j < NB; ++j) {
                        u32 P[8];
                        tmem_ld8(taddr + (u32)(j * kCt + c0), P);
#pragma unroll
                        for (int cc = 0; cc < 8; ++cc) v[cc] += (u128)P[cc] << (8 * j);
                    }
#pragma unroll
                    for (int cc = 0; cc < 8; ++cc) r[cc] = (u64)(v[cc] % q);
                }
                if (row < rows) {
#pragma unroll
                    for (int cc = 0; cc < 8; ++cc) {
                        if (c0 + cc >= cmax) break;
                        u64 x = r[cc];
                        if (accumulate) {
                            const u64 y = x + out[c0 + cc];
                            x = (y < x || y >= q) ? y - q : y;
                        }
                        out[c0 + cc] = x;
                    }
                }
            }
            fence_before();
            named_sync(kBarEpi, kEpi);  // every lane of the set read
            if (tid == 0) arrive(smem_u32(&s_tfree[buf]));
        }
    }
    // teardown: every role has left its loop (on abort, after a bounded wait)
    fence_before();
    __syncthreads();
    fence_after();
    if (warp == kMmaWarp) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
}

// CUDA events around the packing and the GEMM launches of this thread's last
// tensor-core call (created per thread and device on first use)
struct Timing {
    int dev = -1;
    cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
    float pack_ms = -1.f, gemm_ms = -1.f;
};
thread_local Timing t_timing;

int32_t timing_events(int dev) {
    Timing& t = t_timing;
    if (t.dev == dev) return CKKS_OK;
    for (auto& e : t.ev)
        if (e) cudaEventDestroy(e), e = nullptr;
    t.dev = -1;
    for (auto& e : t.ev) CKKS_CUDA_TRY(cudaEventCreate(&e));
    t.dev = dev;
    return CKKS_OK;
}

template <int NB>
int32_t launch(const u64* lhs, const u64* rhs, u64* out, u32 rows, u32 inner, u32 cols, u64 q, cudaStream_t st) {
    constexpr int kCt = cols_per_tile(NB), kRows = NB * kCt, kChunk = blocks_per_launch(NB);
    const int n_mt = (int)((rows + 127) / 128), n_nt = (int)((cols + kCt - 1) / kCt), n_kb = (int)((inner + 31) / 32);
    int dev = 0, n_sm = 0;
    CKKS_CUDA_TRY(cudaGetDevice(&dev));
    CKKS_CUDA_TRY(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev));
    {  // keep the freed packed operands cached in the device pool between calls
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
            uint64_t thr = ~0ull;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
        }
    }
    Workspace<uint8_t> ap, bp;
    Workspace<int> err;
    int32_t rc;
    if ((rc = ap.alloc((size_t)n_mt * n_kb * NB * kATile, st)) ||
        (rc = bp.alloc((size_t)n_nt * n_kb * NB * kRows * 32, st)) || (rc = err.alloc(1, st)))
        return rc;
    CKKS_CUDA_TRY(cudaMemsetAsync(err.p, 0, sizeof(int), st));
    if ((rc = timing_events(dev))) return rc;
    t_timing.pack_ms = t_timing.gemm_ms = -1.f;
    CKKS_CUDA_TRY(cudaEventRecord(t_timing.ev[0], st));
    auto grid_of = [&](size_t threads) {
        const size_t g = (threads + 255) / 256, cap = (size_t)n_sm * 16;
        return (int)(g < cap ? g : cap);
    };
    k_pack_a<<<grid_of((size_t)n_mt * 128 * 2 * n_kb), 256, 0, st>>>(lhs, ap.p, (int)rows, (int)inner, q, NB, n_mt,
                                                                       n_kb);
    CKKS_CUDA_TRY(cudaGetLastError());
    const u64 f256q = (q > 256 && q <= (1ull << 63)) ? (u64)(((u128)256 << 64) / q) : 0;
    k_pack_b<<<grid_of((size_t)n_nt * kCt * 2 * n_kb), 256, 0, st>>>(rhs, bp.p, (int)inner, (int)cols, q, NB, kCt,
                                                                      n_nt, n_kb, f256q);
    CKKS_CUDA_TRY(cudaGetLastError());
    CKKS_CUDA_TRY(cudaFuncSetAttribute(k_park_tc<NB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBytes));
    const int n_tiles = n_mt * n_nt, grid = n_tiles < n_sm ? n_tiles : n_sm;
    CKKS_CUDA_TRY(cudaEventRecord(t_timing.ev[1], st));
    for (int kb0 = 0; kb0 < n_kb; kb0 += kChunk) {
        const int kb1 = kb0 + kChunk < n_kb ? kb0 + kChunk : n_kb;
        k_park_tc<NB><<<grid, kThreads, kSmemBytes, st>>>(ap.p, bp.p, out, (int)rows, (int)cols, q, n_mt, n_nt, n_kb,
                                                          kb0, kb1, kb0 > 0 ? 1 : 0, err.p);
        CKKS_CUDA_TRY(cudaGetLastError());
    }
    CKKS_CUDA_TRY(cudaEventRecord(t_timing.ev[2], st));
    int h_err = 0;
    CKKS_CUDA_TRY(cudaMemcpyAsync(&h_err, err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    CKKS_CUDA_TRY(cudaStreamSynchronize(st));
    CKKS_CUDA_TRY(cudaEventElapsedTime(&t_timing.pack_ms, t_timing.ev[0], t_timing.ev[1]));
    CKKS_CUDA_TRY(cudaEventElapsedTime(&t_timing.gemm_ms, t_timing.ev[1], t_timing.ev[2]));
    if (h_err) {
        ckks_set_error("ckks_park_mod_pp_mm: a tensor-core pipeline wait timed out (role " + std::to_string(h_err) +
                       ")");
        return CKKS_ERR_TIMEOUT;
    }
    return CKKS_OK;
}

// the tensor-core form covers every modulus; tile counts stay within int
bool supported(u32 rows, u32 cols, u64 q) {
    const int nb = (64 - __builtin_clzll(q - 1) + 7) / 8;
    const u64 n_mt = (rows + 127) / 128, n_nt = (cols + (u64)cols_per_tile(nb) - 1) / (u64)cols_per_tile(nb);
    return n_mt * n_nt < (1ull << 31);
}

int32_t run(const u64* lhs, const u64* rhs, u64* out, u32 rows, u32 inner, u32 cols, u64 q, cudaStream_t st) {
    switch ((64 - __builtin_clzll(q - 1) + 7) / 8) {
        case 1: return launch<1>(lhs, rhs, out, rows, inner, cols, q, st);
        case 2: return launch<2>(lhs, rhs, out, rows, inner, cols, q, st);
        case 3: return launch<3>(lhs, rhs, out, rows, inner, cols, q, st);
        case 4: return launch<4>(lhs, rhs, out, rows, inner, cols, q, st);
        case 5: return launch<5>(lhs, rhs, out, rows, inner, cols, q, st);
        case 6: return launch<6>(lhs, rhs, out, rows, inner, cols, q, st);
        case 7: return launch<7>(lhs, rhs, out, rows, inner, cols, q, st);
        default: return launch<8>(lhs, rhs, out, rows, inner, cols, q, st);
    }
}

}  // namespace ptc

int32_t check_dims(uint32_t rows, uint32_t inner, uint32_t cols, uint64_t q, const char* who) {
    // the reference asserts non-empty operands and a modulus above one (ccmm/park.rs:1489-1505)
    if (rows == 0 || inner == 0 || cols == 0 || q < 2 || rows > 0x7FFFFFFFu || cols > 0x7FFFFFFFu ||
        inner > 0x7FFFFFFFu || (u64)((rows + kTile - 1) / kTile) > 65535u) {
        ckks_set_error(std::string(who) + ": empty operand, modulus below 2 or matrix too large");
        return CKKS_ERR_BAD_ARG;
    }
    return CKKS_OK;
}

}  // namespace

extern "C" {

int32_t ckks_park_mod_pp_mm_with_backend(const uint64_t* lhs, const uint64_t* rhs, uint64_t* out, uint32_t rows,
                                         uint32_t inner, uint32_t cols, uint64_t modulus, int32_t backend,
                                         void* stream) {
    if (int32_t rc = check_dims(rows, inner, cols, modulus, "ckks_park_mod_pp_mm")) return rc;
    CKKS_CHECK_ARG(lhs && rhs && out, "ckks_park_mod_pp_mm: null matrix");
    const bool tc_ok = tc_enabled() && ptc::supported(rows, cols, modulus);
    if (backend == CKKS_PARK_AUTO) backend = tc_ok ? CKKS_PARK_TENSOR_CORES : CKKS_PARK_CUDA_CORES;
    const cudaStream_t st = (cudaStream_t)stream;
    if (backend == CKKS_PARK_TENSOR_CORES) {
        CKKS_CHECK_ARG(tc_ok, "ckks_park_mod_pp_mm: the tensor-core backend needs a compute capability 10.0 device "
                              "and fewer than 2^31 output tiles");
        return ptc::run(lhs, rhs, out, rows, inner, cols, modulus, st);
    }
    CKKS_CHECK_ARG(backend == CKKS_PARK_CUDA_CORES, "ckks_park_mod_pp_mm: unknown backend");
    const u64 r64 = (u64)(((u128)1 << 64) % modulus);
    const u64 r128 = (u64)((u128)r64 * r64 % modulus);
    dim3 grid((cols + kTile - 1) / kTile, (rows + kTile - 1) / kTile);
    k_park_mm<<<grid, kThreads, 0, st>>>(lhs, rhs, out, (int)rows, (int)inner, (int)cols, modulus, r64, r128);
    CKKS_CUDA_TRY(cudaGetLastError());
    return CKKS_OK;
}

int32_t ckks_park_last_timing(float* pack_ms, float* gemm_ms) {
    CKKS_CHECK_ARG(pack_ms && gemm_ms, "ckks_park_last_timing: null output");
    CKKS_CHECK_ARG(ptc::t_timing.gemm_ms >= 0.f, "ckks_park_last_timing: no tensor-core call on this thread");
    *pack_ms = ptc::t_timing.pack_ms;
    *gemm_ms = ptc::t_timing.gemm_ms;
    return CKKS_OK;
}

int32_t ckks_park_mod_pp_mm(const uint64_t* lhs, const uint64_t* rhs, uint64_t* out, uint32_t rows, uint32_t inner,
                            uint32_t cols, uint64_t modulus, void* stream) {
    return ckks_park_mod_pp_mm_with_backend(lhs, rhs, out, rows, inner, cols, modulus, CKKS_PARK_AUTO, stream);
}

int32_t ckks_park_mod_pp_mm_host(const uint64_t* lhs, const uint64_t* rhs, uint64_t* out, uint32_t rows,
                                 uint32_t inner, uint32_t cols, uint64_t modulus) {
    if (int32_t rc = check_dims(rows, inner, cols, modulus, "ckks_park_mod_pp_mm_host")) return rc;
    CKKS_CHECK_ARG(lhs && rhs && out, "ckks_park_mod_pp_mm_host: null matrix");
    const size_t na = (size_t)rows * inner, nb = (size_t)inner * cols, nc = (size_t)rows * cols;
    u64 *dA = nullptr, *dB = nullptr, *dC = nullptr;
    int32_t rc = CKKS_OK;
    if (cudaMalloc(&dA, na * 8) != cudaSuccess || cudaMalloc(&dB, nb * 8) != cudaSuccess ||
        cudaMalloc(&dC, nc * 8) != cudaSuccess) {
        cudaGetLastError();
        ckks_set_error("ckks_park_mod_pp_mm_host: out of device memory");
        rc = CKKS_ERR_OOM;
    }
    if (rc == CKKS_OK && (cudaMemcpy(dA, lhs, na * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
                          cudaMemcpy(dB, rhs, nb * 8, cudaMemcpyHostToDevice) != cudaSuccess)) {
        ckks_set_error("ckks_park_mod_pp_mm_host: copy to the device failed");
        rc = CKKS_ERR_CUDA;
    }
    if (rc == CKKS_OK) rc = ckks_park_mod_pp_mm(dA, dB, dC, rows, inner, cols, modulus, nullptr);
    if (rc == CKKS_OK && cudaMemcpy(out, dC, nc * 8, cudaMemcpyDeviceToHost) != cudaSuccess) {
        ckks_set_error(std::string("ckks_park_mod_pp_mm_host: ") + cudaGetErrorString(cudaGetLastError()));
        rc = CKKS_ERR_CUDA;
    }
    cudaFree(dA);
    cudaFree(dB);
    cudaFree(dC);
    return rc;
}

}  // extern "C"
