// rnsblock.cu -- RNS-block ("dnum") gadget ModUp: for each block i of
// consecutive Q limbs, the canonical digit x mod Q_i (grafting/rns_gadget.rs:
// 143-228, decompose_block_local) is formed in mixed radix from the block's
// residues (Garner) and reduced into every QP limb as
//   digit mod m = sum_b v_b * (q_s .. q_{s+b-1} mod m)  (exact: the digit is
//   the integer sum_b v_b prod_{c<b} q_{s+c} < Q_i).
// This is the basis-conversion product [N x alpha] x [alpha x (L+K)].
#include "keyswitch.cuh"

namespace {

constexpr int kT = 128;
constexpr int kMaxBlock = 16;

typedef unsigned __int128 u128;
u64 mm(u64 a, u64 b, u64 q) { return (u64)((u128)a * b % q); }
u64 pw(u64 b, u64 e, u64 q) {
    u64 r = 1 % q;
    b %= q;
    while (e) {
        if (e & 1) r = mm(r, b, q);
        b = mm(b, b, q);
        e >>= 1;
    }
    return r;
}

// Constant layout per block i (offset i * stride):
//   gq[a][b], gq_q[a][b]  (kMaxBlock^2 each): (q_s..q_{s+b-1}) mod q_{s+a}
//   ginv[a], ginv_q[a]    (kMaxBlock each)
//   pre[l][b], pre_q[l][b] (LK * kMaxBlock each): (q_s..q_{s+b-1}) mod m_l
__global__ void k_rnsblock_modup(const u64* __restrict__ a, u64* __restrict__ Y, const u64* __restrict__ cst,
                                 const u32* __restrict__ starts, const u32* __restrict__ sizes,
                                 const NttTab* __restrict__ tabs, LimbMap lm, int LK, int log_n, size_t stride) {
    const u32 n = 1u << log_n;
    const u32 c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    const int i = blockIdx.y;
    const u32 s = starts[i], alpha = sizes[i];
    const u64* gq = cst + i * stride;
    const u64* gq_q = gq + kMaxBlock * kMaxBlock;
    const u64* ginv = gq_q + kMaxBlock * kMaxBlock;
    const u64* ginv_q = ginv + kMaxBlock;
    const u64* pre = ginv_q + kMaxBlock;
    const u64* pre_q = pre + (size_t)LK * kMaxBlock;
    u64 v[kMaxBlock];
    for (u32 x = 0; x < alpha; ++x) {
        const u64 qx = tabs[s + x].q;
        u64 acc = 0;
        for (u32 y = 0; y < x; ++y) acc = add_mod(acc, mul_shoup(v[y], gq[x * kMaxBlock + y], gq_q[x * kMaxBlock + y], qx), qx);
        v[x] = mul_shoup(sub_mod(a[((size_t)(s + x) << log_n) + c], acc, qx), ginv[x], ginv_q[x], qx);
    }
    for (int l = 0; l < LK; ++l) {
        const u64 m = tabs[lm(l)].q;
        u64 r = 0;
        for (u32 b = 0; b < alpha; ++b) r = add_mod(r, mul_shoup(v[b], pre[l * kMaxBlock + b], pre_q[l * kMaxBlock + b], m), m);
        Y[(((size_t)i * LK + l) << log_n) + c] = r;
    }
}

}  // namespace

int32_t rnsblock_prepare(ckks_ctx* ctx, ckks_ksk* key) {
    const u32 LK = ksk_limbs(key), nb = (u32)key->blocks.size();
    const size_t stride = 2 * kMaxBlock * kMaxBlock + 2 * kMaxBlock + 2 * (size_t)LK * kMaxBlock;
    std::vector<u64> h(stride * nb + 2 * nb, 0);
    const LimbMap lm = LimbMap::qp(ctx, key->q_limbs);
    u32 s = 0;
    std::vector<u32> starts(nb), sizes(nb);
    for (u32 i = 0; i < nb; ++i) {
        u32 alpha = key->blocks[i];
        if (alpha == 0 || alpha > kMaxBlock) {
            ckks_set_error("RNS gadget blocks must hold 1..16 limbs");
            return CKKS_ERR_BAD_ARG;
        }
        starts[i] = s;
        sizes[i] = alpha;
        u64* gq = h.data() + i * stride;
        u64* gq_q = gq + kMaxBlock * kMaxBlock;
        u64* ginv = gq_q + kMaxBlock * kMaxBlock;
        u64* ginv_q = ginv + kMaxBlock;
        u64* pre = ginv_q + kMaxBlock;
        u64* pre_q = pre + (size_t)LK * kMaxBlock;
        for (u32 x = 0; x < alpha; ++x) {
            u64 qx = ctx->moduli[s + x], p = 1 % qx;
            for (u32 y = 0; y < alpha; ++y) {
                gq[x * kMaxBlock + y] = p;
                gq_q[x * kMaxBlock + y] = shoup_quotient_host(p, qx);
                if (y < x) p = mm(p, ctx->moduli[s + y] % qx, qx);
            }
            ginv[x] = pw(gq[x * kMaxBlock + x], qx - 2, qx);
            ginv_q[x] = shoup_quotient_host(ginv[x], qx);
        }
        for (u32 l = 0; l < LK; ++l) {
            u64 m = ctx->moduli[lm((int)l)], p = 1 % m;
            for (u32 b = 0; b < alpha; ++b) {
                pre[l * kMaxBlock + b] = p;
                pre_q[l * kMaxBlock + b] = shoup_quotient_host(p, m);
                p = mm(p, ctx->moduli[s + b] % m, m);
            }
        }
        s += alpha;
    }
    if (s != key->q_limbs) {
        ckks_set_error("RNS gadget blocks must cover the Q basis exactly");
        return CKKS_ERR_BASIS_MISMATCH;
    }
    size_t bytes = h.size() * 8;
    if (cudaMalloc(&key->d_block_const, bytes) != cudaSuccess) {
        cudaGetLastError();
        ckks_set_error("out of device memory for RNS gadget constants");
        return CKKS_ERR_OOM;
    }
    u32* tail = (u32*)(h.data() + stride * nb);
    for (u32 i = 0; i < nb; ++i) {
        tail[i] = starts[i];
        tail[nb + i] = sizes[i];
    }
    CKKS_CUDA_TRY(cudaMemcpy(key->d_block_const, h.data(), bytes, cudaMemcpyHostToDevice));
    return CKKS_OK;
}

int32_t rnsblock_modup_launch(ckks_ctx* ctx, const ckks_ksk* key, const u64* a, u64* Y, cudaStream_t st) {
    const u32 LK = ksk_limbs(key), nb = (u32)key->blocks.size();
    const size_t stride = 2 * kMaxBlock * kMaxBlock + 2 * kMaxBlock + 2 * (size_t)LK * kMaxBlock;
    const u32* tail = (const u32*)(key->d_block_const + stride * nb);
    dim3 g((ctx->n + kT - 1) / kT, nb);
    k_rnsblock_modup<<<g, kT, 0, st>>>(a, Y, key->d_block_const, tail, tail + nb, ctx->d_tabs,
                                       LimbMap::qp(ctx, key->q_limbs), LK, ctx->log_n, stride);
    CKKS_CUDA_TRY(cudaGetLastError());
    return CKKS_OK;
}
