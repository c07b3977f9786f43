// context.cu -- context creation (moduli validation, psi search, NTT table
// construction and upload), scratch management and error reporting.
#include <cstring>
#include <thread>

#include "context.cuh"
#include "kernels.cuh"

namespace {

thread_local std::string g_last_error;

typedef unsigned __int128 u128;

u64 mulmod(u64 a, u64 b, u64 q) { return (u64)((u128)a * b % q); }
u64 powmod(u64 b, u64 e, u64 q) {
    u64 r = 1 % q;
    b %= q;
    while (e) {
        if (e & 1) r = mulmod(r, b, q);
        b = mulmod(b, b, q);
        e >>= 1;
    }
    return r;
}
u64 invmod(u64 a, u64 q) { return powmod(a, q - 2, q); }

// Deterministic Miller-Rabin for u64 (witness set of ring/ntt_prime.rs:28).
bool is_prime(u64 n) {
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
    for (u64 a : wit) {
        a %= n;
        if (!a) continue;
        u64 x = powmod(a, d, n);
        if (x == 1 || x == n - 1) continue;
        bool comp = true;
        for (int i = 1; i < s; ++i) {
            x = mulmod(x, x, n);
            if (x == n - 1) { comp = false; break; }
            if (x == 1) return false;
        }
        if (comp) return false;
    }
    return true;
}

// Smallest generator candidate g >= 2 with psi = g^((q-1)/2N), psi^N = -1
// (the reference's find_negacyclic_root, ring/ntt_params.rs:16-50).
u64 find_root(u64 q, u32 n) {
    u64 e = (q - 1) / (2ull * n);
    for (u64 g = 2; g < q; ++g) {
        u64 psi = powmod(g, e, q);
        if (powmod(psi, n, q) == q - 1) return psi;
    }
    return 0;
}

u32 brev(u32 x, int bits) {
    u32 r = 0;
    for (int i = 0; i < bits; ++i) { r = (r << 1) | (x & 1); x >>= 1; }
    return r;
}

// Host tables of one modulus, in the order of the device layout.
struct HostTables {
    std::vector<u64> psiA, psiA_inv, psiB, psiB_inv, mid, midi;
};

void build_tables(u64 q, u64 psi, u32 log_n, HostTables& t) {
    const u32 la = log_n - log_n / 2, lb = log_n / 2, A = 1u << la, B = 1u << lb, N = A * B;
    const u64 two_n = 2ull * N;
    std::vector<u64> pw(two_n);
    u64 v = 1;
    for (u64 e = 0; e < two_n; ++e) {
        pw[e] = v;
        v = mulmod(v, psi, q);
    }
    auto P = [&](u64 e) { return pw[e % two_n]; };
    t.psiA.resize(A);
    t.psiA_inv.resize(A);
    for (u32 i = 0; i < A; ++i) {  // psi_A = psi^B
        u64 r = brev(i, (int)la);
        t.psiA[i] = P((u64)B * r);
        t.psiA_inv[i] = P(two_n - ((u64)B * r) % two_n);
    }
    t.psiB.resize(B);
    t.psiB_inv.resize(B);
    for (u32 i = 0; i < B; ++i) {  // psi_2B = psi^A
        u64 r = brev(i, (int)lb);
        t.psiB[i] = P((u64)A * r);
        t.psiB_inv[i] = P(two_n - ((u64)A * r) % two_n);
    }
    u64 ninv = invmod(N % q, q);
    t.mid.resize(N);
    t.midi.resize(N);
    for (u32 jl = 0; jl < B; ++jl)
        for (u32 ka = 0; ka < A; ++ka) {
            // exponent (2k_a + 1 - A) j_lo mod 2N
            u64 e = ((2ull * ka + 1 + two_n - A) % two_n) * jl % two_n;
            t.mid[(size_t)jl * A + ka] = P(e);
            t.midi[(size_t)ka * B + jl] = mulmod(ninv, P((two_n - e) % two_n), q);
        }
}

// Rescale, ModDown, P-factor and Q-Garner constants (device copies).
int32_t build_constants(ckks_ctx* ctx) {
    const u32 L = ctx->L, K = ctx->K;
    const std::vector<u64>& m = ctx->moduli;
    // layout: rescale [L][2][L] | pmodq [2][L] | md.q [L] | pre, pre_q [L][kMaxAux] x2 | p_mod_q [L] |
    //         pinv_mod_q [L] | pinv_mod_q_q [L] | gq, gq_q [L][L] x2 | ginv, ginv_q [L] x2
    const size_t n_res = (size_t)L * 2 * L, n_pm = 2 * (size_t)L, n_md = (size_t)L * (4 + 2 * kMaxAux),
                 n_g = 2 * (size_t)L * L + 2 * (size_t)L, n_f = (size_t)L * 12;
    std::vector<u64> h(n_res + n_pm + n_md + n_g + n_f, 0);
    u64* res = h.data();
    for (u32 d = 1; d < L; ++d)
        for (u32 i = 0; i < d; ++i) {
            u64 inv = invmod(m[d] % m[i], m[i]);
            res[(size_t)d * 2 * L + i] = inv;
            res[(size_t)d * 2 * L + L + i] = shoup_quotient_host(inv, m[i]);
        }
    u64* pm = res + n_res;
    for (u32 i = 0; i < L; ++i) {
        u64 pf = 1 % m[i];
        for (u32 k = 0; k < K; ++k) pf = mulmod(pf, m[L + k] % m[i], m[i]);
        pm[i] = pf;
        pm[L + i] = shoup_quotient_host(pf, m[i]);
    }
    u64* mdq = pm + n_pm;
    u64* pre = mdq + L;
    u64* pre_q = pre + (size_t)L * kMaxAux;
    u64* pmq = pre_q + (size_t)L * kMaxAux;
    u64* pinvq = pmq + L;
    u64* pinvq_q = pinvq + L;
    ModDownConst& md = ctx->mod_down;
    md.K = (int)K;
    for (u32 i = 0; i < K; ++i) {
        u64 pi = m[L + i], pp = 1 % pi;
        md.p[i] = pi;
        for (u32 j = 0; j < K; ++j) {
            md.pp[i][j] = pp;
            md.pp_q[i][j] = shoup_quotient_host(pp, pi);
            if (j < i) pp = mulmod(pp, m[L + j] % pi, pi);
        }
        md.pinv[i] = invmod(md.pp[i][i], pi);
        md.pinv_q[i] = shoup_quotient_host(md.pinv[i], pi);
    }
    if (K) {  // mixed-radix digits of floor(P/2): P = prod p_i, P/2 via digits of (P-1)/2
        // (P-1)/2 has mixed-radix digits ((p_i - 1)/2 ... ) only when computed exactly:
        // do a long division of the words of P by 2 then repeated division by p_i.
        std::vector<u64> P(K + 2, 0);
        P[0] = 1;
        for (u32 k = 0; k < K; ++k) {
            unsigned __int128 c = 0;
            for (auto& w : P) {
                unsigned __int128 t = (unsigned __int128)w * m[L + k] + c;
                w = (u64)t;
                c = t >> 64;
            }
        }
        std::vector<u64> half(P.size());
        for (size_t i = 0; i < P.size(); ++i) half[i] = (P[i] >> 1) | (i + 1 < P.size() ? (P[i + 1] << 63) : 0);
        for (u32 k = 0; k < K; ++k) {
            unsigned __int128 r = 0;
            for (size_t w = half.size(); w-- > 0;) {
                unsigned __int128 cur = (r << 64) | half[w];
                half[w] = (u64)(cur / m[L + k]);
                r = cur % m[L + k];
            }
            md.half[k] = (u64)r;
        }
    }
    for (u32 i = 0; i < L; ++i) {
        mdq[i] = m[i];
        u64 pp = 1 % m[i];
        for (u32 j = 0; j < K; ++j) {
            pre[(size_t)i * kMaxAux + j] = pp;
            pre_q[(size_t)i * kMaxAux + j] = shoup_quotient_host(pp, m[i]);
            pp = mulmod(pp, m[L + j] % m[i], m[i]);
        }
        pmq[i] = pp;  // P mod q_i
        pinvq[i] = K ? invmod(pp, m[i]) : 1;
        pinvq_q[i] = shoup_quotient_host(pinvq[i], m[i]);
    }
    u64* gq = pinvq_q + L;
    u64* gq_q = gq + (size_t)L * L;
    u64* ginv = gq_q + (size_t)L * L;
    u64* ginv_q = ginv + L;
    for (u32 i = 0; i < L; ++i) {
        u64 pp = 1 % m[i];
        for (u32 j = 0; j < L; ++j) {
            gq[(size_t)i * L + j] = pp;
            gq_q[(size_t)i * L + j] = shoup_quotient_host(pp, m[i]);
            if (j < i) pp = mulmod(pp, m[j] % m[i], m[i]);
        }
        ginv[i] = invmod(gq[(size_t)i * L + i], m[i]);
        ginv_q[i] = shoup_quotient_host(ginv[i], m[i]);
    }
    {  // FP64 ModDown constants: P in three words and, per Q limb, (value, value / q) pairs
        std::vector<u64> Pw(4, 0);
        Pw[0] = 1;
        for (u32 k = 0; k < K && K <= 3; ++k) {
            unsigned __int128 c = 0;
            for (auto& w : Pw) {
                unsigned __int128 t = (unsigned __int128)w * m[L + k] + c;
                w = (u64)t;
                c = t >> 64;
            }
        }
        for (int w = 0; w < 3; ++w) md.P3[w] = Pw[w];
        double* fc = (double*)(h.data() + n_res + n_pm + n_md + n_g);
        for (u32 i = 0; i < L; ++i) {
            const u64 qi = m[i];
            double* c = fc + (size_t)i * 12;
            c[0] = (double)qi;
            c[1] = 1.0 / (double)qi;
            const u64 pinv = pinvq[i] % qi;
            c[2] = (double)pinv;
            c[3] = (double)pinv / (double)qi;
            u64 r = 1 % qi;  // 2^(47 k) mod q
            for (int k = 0; k < 4; ++k) {
                const u64 v = mulmod(r, pinv, qi);
                c[4 + 2 * k] = (double)v;
                c[5 + 2 * k] = (double)v / (double)qi;
                r = mulmod(r, (1ull << 47) % qi, qi);
            }
        }
    }
    if (cudaMalloc(&ctx->d_const_mem, h.size() * sizeof(u64)) != cudaSuccess) {
        cudaGetLastError();
        return CKKS_ERR_OOM;
    }
    if (cudaMemcpy(ctx->d_const_mem, h.data(), h.size() * sizeof(u64), cudaMemcpyHostToDevice) != cudaSuccess)
        return CKKS_ERR_CUDA;
    u64* d = ctx->d_const_mem;
    ctx->d_rescale_inv = d;
    ctx->d_pmodq = d + n_res;
    u64* dmd = d + n_res + n_pm;
    md.q = dmd;
    md.pre = dmd + L;
    md.pre_q = md.pre + (size_t)L * kMaxAux;
    md.p_mod_q = md.pre_q + (size_t)L * kMaxAux;
    md.pinv_mod_q = md.p_mod_q + L;
    md.pinv_mod_q_q = md.pinv_mod_q + L;
    u64* dg = d + n_res + n_pm + n_md;
    ctx->garner.gq = dg;
    ctx->garner.gq_q = dg + (size_t)L * L;
    ctx->garner.ginv = dg + 2 * (size_t)L * L;
    ctx->garner.ginv_q = ctx->garner.ginv + L;
    md.f64c = (const double*)(d + n_res + n_pm + n_md + n_g);
    return CKKS_OK;
}

}  // namespace

void ckks_set_error(const std::string& msg) { g_last_error = msg; }

void ntt_set_smem_limits();

extern "C" {

const char* ckks_last_error_string(void) { return g_last_error.c_str(); }
const char* ckks_version(void) { return "ckks_b200 0.1 (sm_100a)"; }

int32_t ckks_ctx_create(uint32_t log_n, const uint64_t* q, uint32_t L, const uint64_t* p, uint32_t K,
                        ckks_ctx** out) {
    CKKS_CHECK_ARG(out != nullptr, "ckks_ctx_create: out is null");
    *out = nullptr;
    CKKS_CHECK_ARG(log_n >= 2 && log_n <= 17, "ckks_ctx_create: log_n must be in [2, 17]");
    CKKS_CHECK_ARG(L >= 1 && (q != nullptr), "ckks_ctx_create: need at least one Q limb");
    CKKS_CHECK_ARG(K == 0 || p != nullptr, "ckks_ctx_create: p is null");
    CKKS_CHECK_ARG(L + K <= 64, "ckks_ctx_create: at most 64 limbs");
    const u32 n = 1u << log_n;
    std::vector<u64> mod(q, q + L);
    if (K) mod.insert(mod.end(), p, p + K);
    for (size_t i = 0; i < mod.size(); ++i) {
        u64 m = mod[i];
        if (m >= (1ull << 62) || m < 3 || !(m & 1) || (m - 1) % (2ull * n) != 0 || !is_prime(m)) {
            ckks_set_error("ckks_ctx_create: modulus " + std::to_string(m) +
                           " must be an odd prime below 2^62 with q = 1 mod 2N");
            return CKKS_ERR_BAD_ARG;
        }
        for (size_t j = 0; j < i; ++j)
            if (mod[j] == m) {
                ckks_set_error("ckks_ctx_create: moduli must be pairwise distinct");
                return CKKS_ERR_BAD_ARG;
            }
    }
    auto* ctx = new ckks_ctx();
    ctx->log_n = log_n;
    ctx->n = n;
    ctx->log_n2 = log_n / 2;
    ctx->log_n1 = log_n - ctx->log_n2;
    ctx->L = L;
    ctx->K = K;
    ctx->moduli = mod;
    cudaGetDevice(&ctx->device);
    const size_t M = mod.size();
    ctx->psi.resize(M);
    std::vector<HostTables> ht(M);
    {
        std::vector<std::thread> th;
        for (size_t i = 0; i < M; ++i)
            th.emplace_back([&, i]() {
                ctx->psi[i] = find_root(mod[i], n);
                build_tables(mod[i], ctx->psi[i], ctx->log_n, ht[i]);
            });
        for (auto& t : th) t.join();
    }
    // per modulus: value + Shoup of psiA, psiA_inv (A), psiB, psiB_inv (B), mid, midi (N)
    const size_t per = 4 * ((size_t)(1u << ctx->log_n1) + (1u << ctx->log_n2) + n);
    std::vector<u64> host(per * M);
    ctx->h_tabs.resize(M);
    if (cudaMalloc(&ctx->d_table_mem, host.size() * sizeof(u64)) != cudaSuccess ||
        cudaMalloc(&ctx->d_tabs, M * sizeof(NttTab)) != cudaSuccess) {
        cudaGetLastError();
        ckks_ctx_destroy(ctx);
        ckks_set_error("ckks_ctx_create: out of device memory for NTT tables");
        return CKKS_ERR_OOM;
    }
    // FP64 networks: primes below 2^50 when both transform halves have at most
    // 2^8 points (four register stages on each side of the exchange)
    const bool f64_shape = ctx->log_n1 <= 8 && ctx->log_n2 <= 8;
    const size_t fper = 2 * ((size_t)(1u << ctx->log_n1) + (1u << ctx->log_n2) + n);
    size_t n_f64 = 0;
    for (size_t i = 0; i < M; ++i) n_f64 += f64_shape && mod[i] < (1ull << 50);
    std::vector<double2> fhost(fper * n_f64);
    if (n_f64 && cudaMalloc(&ctx->d_ftable_mem, fhost.size() * sizeof(double2)) != cudaSuccess) {
        cudaGetLastError();
        ckks_ctx_destroy(ctx);
        ckks_set_error("ckks_ctx_create: out of device memory for NTT tables");
        return CKKS_ERR_OOM;
    }
    size_t foff = 0;
    for (size_t i = 0; i < M; ++i) {
        u64 m = mod[i];
        size_t off = per * i;
        NttTab& T = ctx->h_tabs[i];
        T.f64 = f64_shape && m < (1ull << 50);
        T.qd = (double)m;
        T.qinv = 1.0 / (double)m;
        if (T.f64) {
            auto fput = [&](const std::vector<u64>& v, const double2** dst) {
                for (size_t k = 0; k < v.size(); ++k) fhost[foff + k] = make_double2((double)v[k], (double)v[k] / (double)m);
                *dst = ctx->d_ftable_mem + foff;
                foff += v.size();
            };
            fput(ht[i].psiA, &T.fA);
            fput(ht[i].psiA_inv, &T.fA_inv);
            fput(ht[i].psiB, &T.fB);
            fput(ht[i].psiB_inv, &T.fB_inv);
            fput(ht[i].mid, &T.fmid);
            fput(ht[i].midi, &T.fmidi);
        }
        T.q = m;
        barrett_host(m, &T.mu_hi, &T.mu_lo);
        auto put = [&](const std::vector<u64>& v, const u64** val, const u64** quo) {
            for (size_t k = 0; k < v.size(); ++k) {
                host[off + k] = v[k];
                host[off + v.size() + k] = shoup_quotient_host(v[k], m);
            }
            *val = ctx->d_table_mem + off;
            *quo = ctx->d_table_mem + off + v.size();
            off += 2 * v.size();
        };
        put(ht[i].psiA, &T.psiA, &T.psiA_q);
        put(ht[i].psiA_inv, &T.psiA_inv, &T.psiA_inv_q);
        put(ht[i].psiB, &T.psiB, &T.psiB_q);
        put(ht[i].psiB_inv, &T.psiB_inv, &T.psiB_inv_q);
        put(ht[i].mid, &T.mid, &T.mid_q);
        put(ht[i].midi, &T.midi, &T.midi_q);
    }
    if (cudaMemcpy(ctx->d_table_mem, host.data(), host.size() * sizeof(u64), cudaMemcpyHostToDevice) != cudaSuccess ||
        (n_f64 && cudaMemcpy(ctx->d_ftable_mem, fhost.data(), fhost.size() * sizeof(double2),
                             cudaMemcpyHostToDevice) != cudaSuccess) ||
        cudaMemcpy(ctx->d_tabs, ctx->h_tabs.data(), M * sizeof(NttTab), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
        std::string e = cudaGetErrorString(cudaGetLastError());
        ckks_ctx_destroy(ctx);
        ckks_set_error("ckks_ctx_create: " + e);
        return CKKS_ERR_CUDA;
    }
    if (K > (u32)kMaxAux) {
        ckks_ctx_destroy(ctx);
        ckks_set_error("ckks_ctx_create: at most 8 auxiliary limbs");
        return CKKS_ERR_BAD_ARG;
    }
    if (int32_t rc = build_constants(ctx)) {
        ckks_ctx_destroy(ctx);
        ckks_set_error("ckks_ctx_create: cannot upload constants");
        return rc;
    }
    {  // keep freed stream-ordered workspaces cached in the device pool
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, ctx->device) == cudaSuccess) {
            uint64_t thr = ~0ull;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
        }
    }
    ntt_set_smem_limits();
    *out = ctx;
    return CKKS_OK;
}

uint64_t ckks_find_negacyclic_root(uint64_t q, uint32_t degree) {
    if (degree < 2 || (degree & (degree - 1)) || q < 3 || (q - 1) % (2ull * degree) != 0) return 0;
    return find_root(q, degree);
}

int32_t ckks_is_prime(uint64_t value) { return is_prime(value) ? 1 : 0; }

int32_t ckks_primes_below_bits(uint32_t bits, uint32_t degree, uint32_t count, uint64_t* out) {
    CKKS_CHECK_ARG(out != nullptr, "ckks_primes_below_bits: out is null");
    CKKS_CHECK_ARG(bits >= 2 && bits <= 62 && degree >= 2 && !(degree & (degree - 1)),
                   "ckks_primes_below_bits: bits must be in [2, 62] and degree a power of two");
    u64 two_n = 2ull * degree;
    u64 cand = (1ull << bits) - 1;
    cand -= (cand - 1) % two_n;
    uint32_t found = 0;
    while (cand > two_n + 1 && found < count) {
        if (is_prime(cand)) out[found++] = cand;
        cand -= two_n;
    }
    if (found != count) {
        ckks_set_error("ckks_primes_below_bits: not enough NTT-friendly primes below 2^bits");
        return CKKS_ERR_BAD_ARG;
    }
    return CKKS_OK;
}

int32_t ckks_ctx_set_tensor_cores(ckks_ctx* ctx, int32_t enable) {
    CKKS_CHECK_ARG(ctx != nullptr, "ckks_ctx_set_tensor_cores: ctx is null");
    ctx->tensor_cores = enable != 0;
    return CKKS_OK;
}

int32_t ckks_ctx_autotune(ckks_ctx* ctx, uint32_t limbs, uint32_t polys, void* stream) {
    if (int32_t rc = ckks_require_device(ctx, "ckks_ctx_autotune")) return rc;
    cudaStream_t st = ckks_stream(ctx, stream);
    const int32_t rc = ntt_autotune(ctx, limbs, polys, st);
    if (rc == CKKS_OK) CKKS_CUDA_TRY(cudaStreamSynchronize(st));
    return rc;
}

int32_t ckks_ctx_tuning_report(const ckks_ctx* ctx, char* buf, uint64_t len) {
    CKKS_CHECK_ARG(ctx != nullptr && buf != nullptr && len > 0, "ckks_ctx_tuning_report: bad arguments");
    const std::string& r = ctx->tuning_report.empty() ? std::string("NTT: built-in tile choices (not tuned)\n")
                                                      : ctx->tuning_report;
    const size_t n = r.size() < len - 1 ? r.size() : (size_t)(len - 1);
    memcpy(buf, r.data(), n);
    buf[n] = 0;
    return CKKS_OK;
}

int32_t ckks_ctx_tensor_cores(const ckks_ctx* ctx) {
    if (!ctx) return 0;
    return ctx->tensor_cores && tc_enabled() ? 1 : 0;
}

int32_t ckks_ctx_last_mac_path(const ckks_ctx* ctx) {
    if (!ctx) return -1;
    return ctx->last_mac_path;
}

}  // extern "C"

int32_t ckks_require_device(const ckks_ctx* ctx, const char* who) {
    if (!ctx) {
        ckks_set_error(std::string(who) + ": null context");
        return CKKS_ERR_BAD_ARG;
    }
    int dev = -1;
    CKKS_CUDA_TRY(cudaGetDevice(&dev));
    if (dev != ctx->device) {
        ckks_set_error(std::string(who) + ": the current CUDA device (" + std::to_string(dev) +
                       ") is not the context's device (" + std::to_string(ctx->device) + ")");
        return CKKS_ERR_BAD_ARG;
    }
    return CKKS_OK;
}

void* pinned_take(ckks_ctx* ctx, size_t bytes, size_t* got) {
    {
        std::lock_guard<std::mutex> lock(ctx->pinned_mu);
        for (size_t i = 0; i < ctx->pinned_free.size(); ++i)
            if (ctx->pinned_free[i].second >= bytes) {
                auto b = ctx->pinned_free[i];
                ctx->pinned_free.erase(ctx->pinned_free.begin() + (long)i);
                *got = b.second;
                return b.first;
            }
    }
    const size_t sz = bytes < 4096 ? 4096 : (bytes + 4095) / 4096 * 4096;
    void* p = nullptr;
    if (cudaHostAlloc(&p, sz, cudaHostAllocDefault) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    *got = sz;
    return p;
}

void pinned_give(ckks_ctx* ctx, void* p, size_t bytes) {
    if (!p) return;
    std::lock_guard<std::mutex> lock(ctx->pinned_mu);
    ctx->pinned_free.emplace_back(p, bytes);
}

extern "C" {

int32_t ckks_ctx_destroy(ckks_ctx* ctx) {
    if (!ctx) return CKKS_OK;
    cudaDeviceSynchronize();
    gadget_release_ctx(ctx);
    embed_release_ctx(ctx);
    keyset_release_ctx(ctx);
    if (ctx->d_tabs) cudaFree(ctx->d_tabs);
    if (ctx->d_table_mem) cudaFree(ctx->d_table_mem);
    if (ctx->d_ftable_mem) cudaFree(ctx->d_ftable_mem);
    if (ctx->d_const_mem) cudaFree(ctx->d_const_mem);
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    for (auto& b : ctx->pinned_free) cudaFreeHost(b.first);
    delete ctx;
    return CKKS_OK;
}

int32_t ckks_ctx_psi(const ckks_ctx* ctx, uint64_t* psi_host) {
    CKKS_CHECK_ARG(ctx && psi_host, "ckks_ctx_psi: null argument");
    std::memcpy(psi_host, ctx->psi.data(), ctx->psi.size() * sizeof(u64));
    return CKKS_OK;
}

}  // extern "C"
