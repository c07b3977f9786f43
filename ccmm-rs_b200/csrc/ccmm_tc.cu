// ccmm_tc.cu -- the per-(limb, slot) matrix products of the structured CCMM on
// the tcgen05 INT8 tensor cores.
//
// For one limb l and NTT slot s the tensor sum of the structured CCMM
// (matrix/rns_ckks_ciphertext.rs:220-318) is three small modular products of the
// entries' residues (m x k times k x n):
//   C0 = Ab Bb,  C1 = Ab Ba + Aa Bb,  C2 = Aa Ba            (mod q_l)
// Both operands are split into bytes. With w_b = 2^(8b) B mod q (lazily reduced
// below 2^64),
//   sum_t A[r][t] B[t][c] == sum_(t,b) byte_b(A[r][t]) w_b(B[t][c])
//                          == sum_a 2^(8a) P[r][(c,a)]               (mod q),
//   P[r][(c,a)] = sum_(t,b) byte_b(A[r][t]) byte_a(w_b(B[t][c]))
// an exact unsigned 8-bit product summed in 32 bits: K = 8 k <= 512 terms of at
// most 255^2, so P < 2^25 (k <= 64). One MMA per (16-column block, 4 inner
// indices): M = 128 rows [Ab; Aa] (64 rows each), N = 256 columns [Bb | Ba] x 16
// columns x 8 byte planes, K = 32 bytes. The accumulator of a column block holds
// Ab Bb (C0) and Ab Ba in the upper 64 lanes and Aa Bb, Aa Ba (C2) in the lower;
// the epilogue adds the two halves of C1 through shared memory.
//
// A (K-major): the entry A[comp][r][t] is K bytes 8t..8t+7 of row 64 comp + r,
// so the operand is the entries themselves in the canonical core-matrix order;
// it is copied once per slot (cp.async, double-buffered across slots). B
// (MN-major) is built per item by the producers from the raw entries (8-byte
// cp.async ring): entry B[comp][t][c] gives 8 weights w_b, one u64 per K row
// (t, b) at N bytes 128 comp + 8 c.. (its 8 bytes are the planes a).
//
// Warps: 0-3 epilogue (TMEM lane quadrants), 4-7 producers, 8 the MMA issuer.
// Every wait is bounded (about a second); on a timeout the kernel records an
// error, leaves its loops, drains its copies and MMAs and frees its TMEM.
#include "keyswitch.cuh"
#include "tcgen05.cuh"

namespace {

using namespace tcg;

constexpr int kEpiWarps = 4, kProdWarps = 4, kMmaWarp = kEpiWarps + kProdWarps;
constexpr int kThreads = 32 * (kMmaWarp + 1);
constexpr int kProd = 32 * kProdWarps, kEpi = 32 * kEpiWarps;
constexpr int kBarProd = 1, kBarEpi = 2;  // named barriers
constexpr int kCB = 16;                   // columns per block (N = 2 x 16 x 8 = 256)
#ifndef CKKS_CCMM_TC_KT
#define CKKS_CCMM_TC_KT 8
#endif
constexpr int kKT = CKKS_CCMM_TC_KT;      // inner indices per item (kKT / 4 MMAs of K = 32 bytes)
constexpr int kSubK = kKT / 4;
static_assert(kKT == 4 || kKT == 8 || kKT == 16, "inner indices per item");
#ifndef CKKS_CCMM_TC_BSTAGES
#define CKKS_CCMM_TC_BSTAGES 2
#endif
constexpr int kRing = kKT == 16 ? 4 : 8, kBStages = CKKS_CCMM_TC_BSTAGES, kAhead = kRing - kBStages;
static_assert((kBStages & (kBStages - 1)) == 0 && kAhead >= 2, "B stages: a power of two below the raw ring");
constexpr u32 kRingSlot = 1024 * kSubK;   // raw entries of one item: 128 producers x kSubK x 8 bytes
// A: 128 rows x 512 K bytes; core matrices 8 rows x 16 B, K chunks 128 B apart, row groups 4 KB
constexpr u32 kLboA = 128, kSboA = 4096, kABytes = 65536;
// B stage: kKT K groups (inner index) x 16 N chunks; strides chosen so the
// producers' 8-byte stores take two wavefronts per warp (no bank conflicts)
constexpr u32 kSboB = 144, kLboB = 2304, kBBytes = kKT * kLboB;
constexpr u32 kOffA = 0, kOffRing = 2 * kABytes, kOffB = kOffRing + kRing * kRingSlot,
              kOffX = kOffB + kBStages * kBBytes;
constexpr u32 kSmemBytes = kOffX + 64 * kCB * 8;  // 188 KB at kKT 8: one CTA per SM
static_assert(kSmemBytes <= 227 * 1024, "shared memory per CTA");
constexpr u32 kTmemCols = 512;
constexpr u32 kIdesc = idesc_i8(128, 256, true);

__device__ __forceinline__ u64 combine_planes(const u32* P, u64 q, bool wide, u64 r32, u64 r32q, u64 one_q, u64 r64,
                                              u64 r64q) {
    // sum_a 2^(8a) P_a with P_a < 2^25 as L + 2^32 H (L, H < 2^49.01)
    const u64 L = (u64)P[0] + ((u64)P[1] << 8) + ((u64)P[2] << 16) + ((u64)P[3] << 24);
    const u64 H = (u64)P[4] + ((u64)P[5] << 8) + ((u64)P[6] << 16) + ((u64)P[7] << 24);
    if (wide) {  // q > 2^49.5 > L: 2^32 H mod q lazily in [0, 2q), plus L, below 3q
        u64 x = mul_shoup_lazy(H, r32, r32q, q) + L;
        x = x >= 2 * q ? x - 2 * q : x;
        return x >= q ? x - q : x;
    }
    const u64 lo = L + (H << 32), hi = (H >> 32) + (lo < L);  // exact 128-bit sum
    return add_mod(reduce_2q(mul_shoup_lazy(lo, 1, one_q, q), q), mul_shoup(hi, r64, r64q, q), q);
}

// At, Bt: slot-major canonical entries [L * N][2][m * kd] (entry r + t m) and
// [L * N][2][kd * nd] (entry t + c kd); Ct [L * N][3][m * nc] (entry c m + r,
// columns c_begin .. c_begin + nc). m, kd <= 64.
__global__ void __launch_bounds__(kThreads, 1)
    k_ccmm_tc(const u64* __restrict__ At, const u64* __restrict__ Bt, u64* __restrict__ Ct,
              const NttTab* __restrict__ tabs, int m, int kd, int nd, int c_begin, int nc, int log_n, int n_limbs,
              int* __restrict__ err) {
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ u32 s_tmem;
    __shared__ int s_abort;
    __shared__ __align__(8) uint64_t s_ready[kBStages], s_empty[kBStages], s_full[2], s_free[2], s_aempty[2];
    const int tid = threadIdx.x, warp = tid >> 5;
    const long long n_slots = (long long)n_limbs << log_n;
    const int my_slots = (long long)blockIdx.x < n_slots
                             ? (int)((n_slots - 1 - (long long)blockIdx.x) / (long long)gridDim.x + 1)
                             : 0;
    const int ncb = (nc + kCB - 1) / kCB, nkt = (kd + kKT - 1) / kKT;
    const int per_slot = ncb * nkt;
    const int n_items = my_slots * per_slot, n_units = my_slots * ncb;
    const size_t a_ent = (size_t)m * kd, b_ent = (size_t)kd * nd, c_ent = (size_t)m * nc;
    if (tid == 0) {
        s_abort = 0;
        for (int i = 0; i < kBStages; ++i) {
            mbar_init(smem_u32(&s_ready[i]), 1);
            mbar_init(smem_u32(&s_empty[i]), 1);
        }
        for (int i = 0; i < 2; ++i) {
            mbar_init(smem_u32(&s_full[i]), 1);
            mbar_init(smem_u32(&s_free[i]), 1);
            mbar_init(smem_u32(&s_aempty[i]), 1);
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
    const u32 tmem = s_tmem;
    const u32 sbase = smem_u32(smem);
    auto slot_of = [&](int j) { return (long long)blockIdx.x + (long long)j * gridDim.x; };

    if (warp >= kEpiWarps && warp < kMmaWarp) {
        // ------------------------------------------------------------ producers
        const int gtid = tid - 32 * kEpiWarps, pw = gtid >> 5, lane = gtid & 31;
        // entries (comp, inner t_loc and t_loc + 4, column c_loc) of each item
        const int c_loc = lane & 15, t_loc = (lane >> 4) + 2 * (pw & 1), comp = pw >> 1;
        // A of slot j into buffer j & 1: 8192 words, destination word w holds entry
        // (row 8 (w / 512) + (w % 16) / 2, inner index 2 ((w % 512) / 16) + w % 2)
        auto load_a = [&](int j) {
            const long long gs = slot_of(j);
            const u64* src = At + (size_t)gs * 2 * a_ent;
            const u32 dst = sbase + kOffA + (u32)(j & 1) * kABytes;
            for (int w = gtid; w < (int)(kABytes / 8); w += kProd) {
                const int rowm = 8 * (w >> 9) + ((w & 15) >> 1), t = 2 * ((w & 511) >> 4) + (w & 1);
                const int cmp = rowm >> 6, r = rowm & 63;
                const bool ok = r < m && t < kd;
                cp8(dst + (u32)w * 8, ok ? src + (size_t)cmp * a_ent + r + (size_t)t * m : src, ok ? 8u : 0u);
            }
        };
        // raw entry of this thread for item `it` (slot j, block cb, inner chunk t) into the ring.
        // Every call commits one cp.async group, so group g holds item g's entries (and
        // an A image issued just before): waiting for all but the kAhead newest groups
        // completes item `it` and everything issued before it.
        struct Pos {
            int j = 0, cb = 0, t = 0, pos = 0;  // slot, column block, inner chunk, item within the slot
        };
        auto prefetch_b = [&](int it, const Pos& p) {
            if (it < n_items) {
                const long long gs = slot_of(p.j);
                const int c = kCB * p.cb + c_loc;
#pragma unroll
                for (int h = 0; h < kSubK; ++h) {
                    const int tt = kKT * p.t + t_loc + 4 * h;
                    const bool ok = tt < kd && c < nc;
                    const u64* src = Bt + (size_t)gs * 2 * b_ent + (size_t)comp * b_ent + tt + (size_t)(c_begin + c) * kd;
                    cp8(sbase + kOffRing + (u32)(it & (kRing - 1)) * kRingSlot + (u32)(h * kProd + gtid) * 8,
                        ok ? src : Bt, ok ? 8u : 0u);
                }
            }
            cp_commit();
        };
        auto advance = [&](Pos& p) {
            ++p.pos;
            if (++p.t == nkt) {
                p.t = 0;
                if (++p.cb == ncb) {
                    p.cb = 0;
                    p.pos = 0;
                    ++p.j;
                }
            }
        };
        // The A of slot j + 1 is loaded at item a_pos of slot j, into the buffer of
        // slot j - 1: by then the MMAs of slot j - 1 have completed (the B-stage wait
        // of item a_pos covers them), so the wait on that buffer does not drain the
        // pipeline. It joins group it0(j) + a_pos + kAhead, which completes by the
        // first item of slot j + 1 when a slot has at least kRing items; shorter
        // slots wait for every copy.
        const int a_pos = per_slot - 1 < kBStages ? per_slot - 1 : kBStages;
        const bool wait_all = per_slot < kRing;
        if (my_slots > 0) load_a(0);
        Pos ahead;
        for (int k = 0; k < kAhead; ++k) {
            prefetch_b(k, ahead);
            advance(ahead);
        }
        Pos cur;
        int f_limb = -1, q_bits = 0;
        bool near_pow2 = false;
        u64 q = 0, f256 = 0, f256q = 0;
        for (int it = 0; it < n_items; ++it) {
            const int bst = it & (kBStages - 1);
            const bool next_a = cur.pos == a_pos && cur.j + 1 < my_slots;
            bool bad = false;
            if (it >= kBStages) bad = !wait_parity(smem_u32(&s_empty[bst]), (u32)(((it / kBStages) - 1) & 1));
            // the buffer of slot j - 1 (the MMAs of its last item committed s_aempty)
            if (!bad && next_a && cur.j >= 1)
                bad = !wait_parity(smem_u32(&s_aempty[(cur.j + 1) & 1]), (u32)((((cur.j + 1) >> 1) - 1) & 1));
            if (group_any(kBarProd, kProd, bad || s_abort)) {
                if (gtid == 0) {
                    atomicExch(err, 1);
                    s_abort = 1;
                }
                break;
            }
            if (next_a) load_a(cur.j + 1);
            prefetch_b(it + kAhead, ahead);
            advance(ahead);
            if (wait_all) cp_wait<0>();
            else cp_wait<kAhead>();
            const int l = (int)(slot_of(cur.j) >> log_n);
            if (l != f_limb) {
                q = tabs[l].q;
                f256 = 256 % q;
                f256q = shoup_quotient_dev(f256, q);
                q_bits = 64 - __clzll(q);
                near_pow2 = q_bits <= 55 && ((1ull << q_bits) - q) < (1ull << (q_bits - 9));
                f_limb = l;
            }
            {   // the 8 weights of this thread's entries: K rows (t_loc + 4 h, b), N bytes 128 comp + 8 c_loc
                const uint8_t* ring = smem + kOffRing + (it & (kRing - 1)) * kRingSlot;
                uint8_t* d0 = smem + kOffB + bst * kBBytes + t_loc * kLboB + (comp * 8 + (c_loc >> 1)) * kSboB +
                              (c_loc & 1) * 8;
                u64 w[kSubK];
#pragma unroll
                for (int h = 0; h < kSubK; ++h) w[h] = *(const u64*)(ring + (h * kProd + gtid) * 8);
                if (near_pow2) {  // q in (2^e - 2^(e-9), 2^e), e <= 55: w < 2^(e+1) stays below 2^(e+1)
#pragma unroll
                    for (int b = 0; b < 8; ++b) {
#pragma unroll
                        for (int h = 0; h < kSubK; ++h) {
                            *(u64*)(d0 + h * 4 * kLboB + b * 16) = w[h];
                            const u64 x = w[h] << 8;
                            w[h] = x - (x >> q_bits) * q;
                        }
                    }
                } else {
#pragma unroll
                    for (int b = 0; b < 8; ++b) {
#pragma unroll
                        for (int h = 0; h < kSubK; ++h) {
                            *(u64*)(d0 + h * 4 * kLboB + b * 16) = w[h];
                            w[h] = mul_shoup_lazy(w[h], f256, f256q, q);
                        }
                    }
                }
            }
            fence_async_smem();  // generic-proxy writes (B, and the cp.async A) before the MMA reads them
            named_sync(kBarProd, kProd);
            if (gtid == 0) arrive(smem_u32(&s_ready[bst]));
            advance(cur);
        }
        cp_wait<0>();
    } else if (warp == kMmaWarp) {
        // ------------------------------------------------------------- MMA issue
        if ((tid & 31) == 0) {
            int j = 0, cb = 0, t = 0, u = 0, last = -1;
            for (int it = 0; it < n_items; ++it) {
                const int bst = it & (kBStages - 1);
                if (!wait_parity(smem_u32(&s_ready[bst]), (u32)((it / kBStages) & 1)) || s_abort) {
                    atomicExch(err, 2);
                    s_abort = 1;
                    break;
                }
                if (t == 0) {
                    if (u >= 2 && !wait_parity(smem_u32(&s_free[u & 1]), (u32)(((u >> 1) - 1) & 1))) {
                        atomicExch(err, 3);
                        s_abort = 1;
                        break;
                    }
                    fence_after();
                }
                // kSubK MMAs of 4 inner indices each: A K chunks (2 inner indices of 16 bytes)
                // 2 (kSubK t + h) .., B K groups 4 h ..
#pragma unroll
                for (int h = 0; h < kSubK; ++h) {
                    const uint64_t a = sdesc(sbase + kOffA + (u32)(j & 1) * kABytes + (u32)(kSubK * t + h) * 2 * kLboA,
                                             kLboA, kSboA);
                    const uint64_t b = sdesc(sbase + kOffB + (u32)bst * kBBytes + (u32)h * 4 * kLboB, kLboB, kSboB);
                    mma_i8(tmem + (u32)(u & 1) * 256u, a, b, kIdesc, (t > 0 || h > 0) ? 1u : 0u);
                }
                commit(smem_u32(&s_empty[bst]));
                last = it;
                if (++t == nkt) {
                    commit(smem_u32(&s_full[u & 1]));
                    t = 0;
                    ++u;
                    if (++cb == ncb) {
                        commit(smem_u32(&s_aempty[j & 1]));
                        cb = 0;
                        ++j;
                    }
                }
            }
            // drain: the last commit covers every MMA issued
            if (last >= 0) wait_parity(smem_u32(&s_empty[last & (kBStages - 1)]), (u32)((last / kBStages) & 1));
        }
        __syncwarp();
    } else {
        // -------------------------------------------------------------- epilogue
        const int lane = tid & 31, qd = warp & 3;
        const int rowm = 32 * qd + lane, ca = rowm >> 6, r = rowm & 63;  // row of [Ab; Aa]
        u64* xch = (u64*)(smem + kOffX);                                 // Aa Bb of the block, [c][r]
        int r_limb = -1;
        bool wide = false;
        u64 q = 0, one_q = 0, r64 = 0, r64q = 0, r32 = 0, r32q = 0;
        for (int u = 0; u < n_units; ++u) {
            const int j = u / ncb, cb = u - j * ncb;
            const long long gs = slot_of(j);
            const int l = (int)(gs >> log_n);
            const bool bad = !wait_parity(smem_u32(&s_full[u & 1]), (u32)((u >> 1) & 1));
            if (group_any(kBarEpi, kEpi, bad || s_abort)) {
                if (tid == 0) {
                    atomicExch(err, 4);
                    s_abort = 1;
                }
                break;
            }
            fence_after();
            if (l != r_limb) {
                q = tabs[l].q;
                one_q = (~0ull) / q;
                r64 = (u64)(-(q * one_q));
                r64q = shoup_quotient_dev(r64, q);
                r32 = (1ull << 32) % q;
                r32q = shoup_quotient_dev(r32, q);
                wide = q > 0x2D413CCCFE779ull;  // floor(2^49.5)
                r_limb = l;
            }
            u64* out = Ct + (size_t)gs * 3 * c_ent;
            const u32 taddr = tmem + ((u32)(32 * qd) << 16) + (u32)(256 * (u & 1));
            u64 x1[kCB];  // Ab Ba of this row (upper half)
#pragma unroll
            for (int part = 0; part < 2; ++part) {
#pragma unroll
                for (int h = 0; h < 4; ++h) {  // 4 columns x 8 planes per load
                    u32 P[32];
                    tmem_ld32(taddr + (u32)(part * 128 + h * 32), P);
#pragma unroll
                    for (int cc = 0; cc < 4; ++cc) {
                        const int cl = 4 * h + cc, c = kCB * cb + cl;
                        const u64 v = combine_planes(P + 8 * cc, q, wide, r32, r32q, one_q, r64, r64q);
                        if (part == 0 && ca == 0) {  // C0 = Ab Bb
                            if (r < m && c < nc) out[(size_t)c * m + r] = v;
                        } else if (part == 0) {      // Aa Bb, half of C1
                            xch[cl * 64 + r] = v;
                        } else if (ca == 0) {        // Ab Ba, half of C1
                            x1[cl] = v;
                        } else {                     // C2 = Aa Ba
                            if (r < m && c < nc) out[2 * c_ent + (size_t)c * m + r] = v;
                        }
                    }
                }
            }
            named_sync(kBarEpi, kEpi);
            if (ca == 0) {
#pragma unroll
                for (int cl = 0; cl < kCB; ++cl) {
                    const int c = kCB * cb + cl;
                    if (r < m && c < nc) out[c_ent + (size_t)c * m + r] = add_mod(x1[cl], xch[cl * 64 + r], q);
                }
            }
            fence_before();
            named_sync(kBarEpi, kEpi);  // TMEM half and exchange buffer free
            if (tid == 0) arrive(smem_u32(&s_free[u & 1]));
        }
    }
    // teardown: every role has left its loop (on abort, after a bounded wait)
    fence_before();
    __syncthreads();
    fence_after();
    if (warp == kMmaWarp) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
}

}  // namespace

bool ccmm_tc_supported(const ckks_ctx* ctx, u32 m, u32 kd) {
    return ctx->tensor_cores && tc_enabled() && m >= 1 && m <= 64 && kd >= 1 && kd <= 64;
}

// One launch per output column chunk; `err` (device, zeroed by the caller)
// receives the stage of a timed-out wait. The grid is one persistent CTA per SM.
int32_t ccmm_slot_tc_launch(ckks_ctx* ctx, const u64* At, const u64* Bt, u64* Ct, u32 L, u32 m, u32 kd, u32 nd,
                            u32 c_begin, u32 nc, int* err, cudaStream_t st) {
    int n_sm = 0;
    CKKS_CUDA_TRY(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, ctx->device));
    const long long slots = (long long)L << ctx->log_n;
    const int grid = slots < n_sm ? (int)slots : n_sm;
    CKKS_CUDA_TRY(cudaFuncSetAttribute(k_ccmm_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBytes));
    k_ccmm_tc<<<grid, kThreads, kSmemBytes, st>>>(At, Bt, Ct, ctx->d_tabs, (int)m, (int)kd, (int)nd, (int)c_begin,
                                                  (int)nc, (int)ctx->log_n, (int)L, err);
    CKKS_CUDA_TRY(cudaGetLastError());
    return CKKS_OK;
}
