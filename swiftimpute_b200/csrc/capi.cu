// capi.cu — the C ABI (include/swiftimpute_b200.h) over the device kernels.
#include "fb_typed.hpp"
#include "si_internal.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <thread>

namespace si {

si_status fail(si_ctx* ctx, si_status s, const std::string& msg) {
    if (ctx) ctx->err = msg;
    return s;
}

si_status cuda_fail(si_ctx* ctx, cudaError_t e, const char* what) {
    std::string m = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
    return fail(ctx, e == cudaErrorMemoryAllocation ? SI_ERR_OUT_OF_MEMORY : SI_ERR_CUDA, m);
}

si_status dev_alloc(si_ctx* ctx, DeviceBuffer& buf, size_t bytes) {
    dev_free(ctx, buf);
    if (bytes == 0) bytes = 16;
    bytes = (bytes + 255) & ~size_t(255);
    if (ctx->used + bytes > ctx->budget)
        return fail(ctx, SI_ERR_BUDGET, "HBM budget exceeded: need " + std::to_string(bytes) + " more bytes, " +
                                            std::to_string(ctx->budget - ctx->used) + " left");
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) { cudaGetLastError(); return cuda_fail(ctx, e, "cudaMalloc"); }
    buf.ptr = p;
    buf.bytes = bytes;
    ctx->used += bytes;
    return SI_OK;
}

void dev_free(si_ctx* ctx, DeviceBuffer& buf) {
    if (buf.ptr) {
        cudaFree(buf.ptr);
        ctx->used -= buf.bytes;
    }
    buf.ptr = nullptr;
    buf.bytes = 0;
}

si_status dev_reserve(si_ctx* ctx, DeviceBuffer& buf, size_t bytes) {
    if (buf.ptr && buf.bytes >= bytes) return SI_OK;
    if (buf.ptr) {
        // regrowing: take half again the old size when the budget allows, so
        // slowly rising sizes do not reallocate (and synchronise) every call
        const size_t roomy = std::max(bytes, buf.bytes + buf.bytes / 2);
        const uint64_t after = ctx->used - buf.bytes + ((roomy + 255) & ~size_t(255));
        if (roomy > bytes && after <= ctx->budget) return dev_alloc(ctx, buf, roomy);
    }
    return dev_alloc(ctx, buf, bytes);
}

}  // namespace si

using namespace si;

#define SI_CUDA(ctx, call, what)                           \
    do {                                                   \
        cudaError_t e_ = (call);                           \
        if (e_ != cudaSuccess) return cuda_fail(ctx, e_, what); \
    } while (0)
#define SI_TRY(x)                      \
    do {                               \
        si_status st_ = (x);           \
        if (st_ != SI_OK) return st_;  \
    } while (0)

namespace {

si_status set_device(si_ctx* ctx) {
    SI_CUDA(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");
    return SI_OK;
}

void reset_index(si_ctx* ctx) {
    dev_free(ctx, ctx->head);
    dev_free(ctx, ctx->prefix);
    dev_free(ctx, ctx->row_hash);
    dev_free(ctx, ctx->rank_bits);
    dev_free(ctx, ctx->rank_zeros);
    for (auto& kv : ctx->sel) {
        dev_free(ctx, kv.second.pairs);
        dev_free(ctx, kv.second.masks);
        dev_free(ctx, kv.second.g2);
        dev_free(ctx, kv.second.raw);
    }
    ctx->sel.clear();
    for (auto& kv : ctx->region_sel) {
        dev_free(ctx, kv.second.masks);
        dev_free(ctx, kv.second.g2);
        dev_free(ctx, kv.second.raw);
    }
    ctx->region_sel.clear();
    ctx->has_index = false;
    ctx->pbwt_flags = 0;
}

void clear_exceptions(si_ctx* ctx) {
    dev_free(ctx, ctx->ex_off);
    dev_free(ctx, ctx->ex_ent);
    ctx->n_ex = 0;
}

// Alleles other than 0 and 1 of a u8 panel [M][N], per marker in haplotype
// order: off[M + 1] and entries h << 8 | byte. Rows are scanned eight bytes at
// a time on several host threads; a 0/1 panel yields none.
void panel_exceptions(const uint8_t* a, uint32_t M, uint32_t N, std::vector<unsigned long long>& off,
                      std::vector<uint32_t>& ent) {
    off.assign((size_t)M + 1, 0);
    ent.clear();
    const uint32_t nt = std::max(1u, std::min<uint32_t>({std::thread::hardware_concurrency(), 16u, M}));
    std::vector<std::vector<uint32_t>> part(nt);
    auto scan = [&](uint32_t t) {
        const uint32_t r0 = (uint32_t)((uint64_t)M * t / nt), r1 = (uint32_t)((uint64_t)M * (t + 1) / nt);
        for (uint32_t m = r0; m < r1; ++m) {
            const uint8_t* row = a + (size_t)m * N;
            uint64_t n = 0;
            uint32_t h = 0;
            for (; h + 8 <= N; h += 8) {
                uint64_t w;
                std::memcpy(&w, row + h, 8);
                if (!(w & 0xFEFEFEFEFEFEFEFEull)) continue;
                for (uint32_t j = 0; j < 8; ++j)
                    if (row[h + j] > 1) { part[t].push_back((h + j) << 8 | row[h + j]); ++n; }
            }
            for (; h < N; ++h)
                if (row[h] > 1) { part[t].push_back(h << 8 | row[h]); ++n; }
            off[m + 1] = n;
        }
    };
    std::vector<std::thread> th;
    for (uint32_t t = 1; t < nt; ++t) th.emplace_back(scan, t);
    scan(0);
    for (auto& x : th) x.join();
    for (uint32_t m = 0; m < M; ++m) off[m + 1] += off[m];
    ent.reserve(off[M]);
    for (auto& p : part) ent.insert(ent.end(), p.begin(), p.end());
}

// Li–Stephens transition between genetic positions (Morgans), as
// compute_transition_probs_kernel (transition.cu:83-115): FP64 maths, log10
// values rounded to float, then read by natural-log recursions, so the linear
// weights are exp(log10 value).
LinTrans lin_trans(double gd0, double gd1, double ne, double rho_rate) {
    double dist = gd1 - gd0;
    if (dist < 0.0) dist = 0.0;
    const double exponent = -4.0 * ne * dist * rho_rate;
    double rho = 1.0 - std::exp(exponent);
    if (rho < 0.0) rho = 0.0;
    if (rho > 1.0) rho = 1.0;
    const double stay = (1.0 - rho) + rho / (2.0 * ne);
    const double sw = rho / (2.0 * ne);
    const float t_diag = (float)std::log10(stay);
    const float t_off = (sw < 1e-300) ? -999.0f : (float)std::log10(sw);
    const double c = std::exp((double)t_off), d = std::exp((double)t_diag);
    return LinTrans{(float)c, (float)(d - c)};
}

si_status ensure_trans(si_ctx* ctx, const si_impute_params* p) {
    if (!ctx->has_map) return fail(ctx, SI_ERR_STATE, "marker positions not set (si_panel_set_map)");
    uint64_t key = (uint64_t)p->transition_mode * 0x9E3779B97F4A7C15ull;
    double pr[2] = {(double)p->ne, p->rho_rate};
    uint64_t bits[2];
    std::memcpy(bits, pr, sizeof bits);
    key ^= bits[0] * 0xBF58476D1CE4E5B9ull ^ bits[1] * 0x94D049BB133111EBull;
    if (ctx->trans.ptr && ctx->trans_key == key) return SI_OK;
    const uint32_t M = ctx->M;
    std::vector<LinTrans> t(M);
    const double ne = (double)p->ne;
    LinTrans t0 = M >= 2 ? lin_trans(ctx->morgans[0], ctx->morgans[1], ne, p->rho_rate) : LinTrans{1.f, 0.f};
    for (uint32_t m = 0; m < M; ++m) {
        if (p->transition_mode == SI_TRANS_PER_GAP && m >= 1)
            t[m] = lin_trans(ctx->morgans[m - 1], ctx->morgans[m], ne, p->rho_rate);
        else
            t[m] = t0;
        if (m >= 1 && !(t[m].c >= 1e-30f))
            return fail(ctx, SI_ERR_UNSUPPORTED,
                        "switch weight exp(log10 switch) = " + std::to_string(t[m].c) + " at marker " +
                            std::to_string(m) +
                            " is below 1e-30 (zero genetic distance); the FP32 linear-space kernel needs a "
                            "representable switch weight");
    }
    SI_TRY(dev_reserve(ctx, ctx->trans, sizeof(LinTrans) * M));
    SI_CUDA(ctx, cudaMemcpy(ctx->trans.ptr, t.data(), sizeof(LinTrans) * M, cudaMemcpyHostToDevice), "copy trans");
    ctx->trans0 = t0;
    ctx->trans_key = key;
    return SI_OK;
}

si_status ensure_selection(si_ctx* ctx, uint32_t L, int kind, SelectionCache** out, bool force = false,
                           cudaStream_t s = nullptr) {
    if (L == 0 || L > kHead) return fail(ctx, SI_ERR_INVALID_ARG, "L must be in 1..128");
    if (kind == SI_SEL_TARGET)
        return fail(ctx, SI_ERR_UNSUPPORTED,
                    "target-aware selection (SI_SEL_TARGET) is per target: si_impute, si_impute_device and "
                    "si_select_states_target only");
    if (kind == SI_SEL_FIRST_PAIRS) {
        if ((uint64_t)2 * L > ctx->N)
            return fail(ctx, SI_ERR_UNSUPPORTED, "first-pairs selection needs N >= 2L haplotypes");
    } else {
        if (!ctx->has_index) return fail(ctx, SI_ERR_STATE, "PBWT index not built (si_pbwt_build)");
        if (kind == SI_SEL_AUTO) kind = (L <= 32 && ctx->N <= 10000) ? SI_SEL_WARP : SI_SEL_INSERTION;
        if (kind != SI_SEL_WARP && kind != SI_SEL_INSERTION)
            return fail(ctx, SI_ERR_INVALID_ARG, "bad selection kind");
    }
    auto& c = ctx->sel[{L, kind}];
    if (!c.pairs.ptr || force) {
        c.L = L;
        c.kind = kind;
        if (!c.pairs.ptr) {
            SI_TRY(dev_alloc(ctx, c.pairs, (size_t)ctx->M * L * 2 * sizeof(uint32_t)));
            SI_TRY(dev_alloc(ctx, c.masks, (size_t)ctx->M * sizeof(SlotMasks)));
            SI_TRY(dev_alloc(ctx, c.g2, (size_t)ctx->M * fb_lmax(L) * sizeof(float2)));
            if (ctx->n_ex) SI_TRY(dev_alloc(ctx, c.raw, (size_t)ctx->M * fb_lmax(L) * 2));
        }
        SI_CUDA(ctx,
                launch_select((const uint32_t*)ctx->head.ptr, (const uint32_t*)ctx->panel.ptr, ctx->M, ctx->N, ctx->W,
                              L, kind, (const unsigned long long*)ctx->ex_off.ptr, (const uint32_t*)ctx->ex_ent.ptr,
                              (uint32_t*)c.pairs.ptr, (SlotMasks*)c.masks.ptr, (float2*)c.g2.ptr, (uint8_t*)c.raw.ptr,
                              fb_lmax(L), s ? s : ctx->stream),
                "select kernel");
    }
    *out = &c;
    return SI_OK;
}

si_status check_params(si_ctx* ctx, const si_impute_params* p) {
    if (!p) return fail(ctx, SI_ERR_INVALID_ARG, "params is NULL");
    if (p->num_states == 0 || p->num_states > 32)
        return fail(ctx, SI_ERR_UNSUPPORTED, "num_states must be 1..32 (the reference sampler holds 32 slots)");
    if (p->ne == 0) return fail(ctx, SI_ERR_INVALID_ARG, "ne must be positive");
    if (p->transition_mode != SI_TRANS_MATRIX0 && p->transition_mode != SI_TRANS_PER_GAP)
        return fail(ctx, SI_ERR_INVALID_ARG, "bad transition_mode");
    if (p->sampling != SI_SAMPLE_ARGMAX && p->sampling != SI_SAMPLE_PHILOX)
        return fail(ctx, SI_ERR_INVALID_ARG, "bad sampling mode");
    if (!(p->tie_eps >= 0.0 && p->tie_eps < 1.0)) return fail(ctx, SI_ERR_INVALID_ARG, "tie_eps must be in [0, 1)");
    if (p->checkpoint_interval > 32) return fail(ctx, SI_ERR_UNSUPPORTED, "checkpoint_interval must be <= 32");
    if (p->flags & ~(uint32_t)(SI_IMPUTE_RESELECT | SI_IMPUTE_FULL_CHAIN | SI_IMPUTE_CODES_2BIT | SI_IMPUTE_HAPS_BITS))
        return fail(ctx, SI_ERR_INVALID_ARG, "unknown flag bits");
    if (p->block_threads && (p->block_threads % 32 || p->block_threads > 128))
        return fail(ctx, SI_ERR_UNSUPPORTED, "block_threads must be a multiple of 32, <= 128");
    if (!ctx->panel.ptr) return fail(ctx, SI_ERR_STATE, "no panel uploaded");
    return SI_OK;
}

// Tile choice per slot count: chains per CTA and markers per segment. The
// alpha tile of a segment (C * Lmax * T floats) sits in shared memory.
void default_tiles(uint32_t L, uint32_t* T, uint32_t* C) {
    const uint32_t lm = fb_lmax(L);
    *C = lm >= 32 ? 16 : 32;
    *T = lm <= 8 ? 64 : 32;
}

constexpr uint32_t kTabN = 4096;

// Closed-form run coefficients for (c, delta, L) in FP64 (fb_typed.hpp),
// cached per (transition, L).
si_status tables_for(si_ctx* ctx, const LinTrans& t0, uint32_t L, TypedTables* out) {
    uint64_t key = 0;
    std::memcpy(&key, &t0, 8);
    key = key * 0x9E3779B97F4A7C15ull ^ (uint64_t)L;
    auto& ts = ctx->tables[key];
    if (!ts.QS.ptr) {
        const double c = (double)t0.c, dl = (double)t0.delta;
        const double rho = dl + (double)L * c;
        const double q = dl / rho;
        const double lq = q > 0.0 ? std::log(q) : -INFINITY;
        const double lr = std::log(rho);
        const int regime = std::fabs(rho - 1.0) < 1e-15 ? 2 : (rho < 1.0 ? 0 : 1);
        const double lgc = regime == 0 ? std::log1p(-rho) : (regime == 1 ? std::log(rho - 1.0) : 0.0);
        // QS [n] {Q, S}; then the pair tables {Q_n, Q_n+1, S_n, S_n+1} and
        // {Q_n, Q_n-1, S_n, S_n-1} (index 0: Q_0, S_0 twice) for two consecutive cells
        std::vector<float> QS(2 * kTabN + 12 * kTabN);
        std::vector<double> G(kTabN);
        std::vector<float> qf(kTabN + 1), sf(kTabN + 1);
        for (uint32_t n = 0; n <= kTabN; ++n) {
            const double qn = (n == 0) ? 1.0 : (q > 0.0 ? std::exp((double)n * lq) : 0.0);
            const double om = (n == 0) ? 0.0 : (q > 0.0 ? -std::expm1((double)n * lq) : 1.0);
            qf[n] = (float)qn;
            sf[n] = (float)(om / (double)L);
        }
        float* up = QS.data() + 2 * kTabN;
        float* dn = up + 4 * kTabN;
        for (uint32_t n = 0; n < kTabN; ++n) {
            QS[2 * n] = qf[n];
            QS[2 * n + 1] = sf[n];
            up[4 * n] = qf[n]; up[4 * n + 1] = qf[n + 1]; up[4 * n + 2] = sf[n]; up[4 * n + 3] = sf[n + 1];
            const uint32_t b = n ? n - 1 : 0;
            dn[4 * n] = qf[n]; dn[4 * n + 1] = qf[b]; dn[4 * n + 2] = sf[n]; dn[4 * n + 3] = sf[b];
            if (n == 0) G[n] = -INFINITY;
            else if (regime == 0) G[n] = -(double)n * lr + std::log(-std::expm1((double)n * lr)) - lgc;
            else if (regime == 1) G[n] = std::log(-std::expm1(-(double)n * lr)) - lgc;
            else G[n] = std::log((double)n);
        }
        // Gdn [n] {hi G_n, hi G_n-1, lo G_n, lo G_n-1}: G as a float pair, so the floor's
        // log farg' + G_j (nearly cancelling where the floor matters) is formed in FP32
        float* gd = dn + 4 * kTabN;
        auto hi = [&](uint32_t n) { return n == 0 ? -1e30f : (float)G[n]; };
        auto lo = [&](uint32_t n) { return n == 0 ? 0.f : (float)(G[n] - (double)(float)G[n]); };
        for (uint32_t n = 0; n < kTabN; ++n) {
            const uint32_t b = n ? n - 1 : 0;
            gd[4 * n] = hi(n); gd[4 * n + 1] = hi(b); gd[4 * n + 2] = lo(n); gd[4 * n + 3] = lo(b);
        }
        si_status st = dev_alloc(ctx, ts.QS, QS.size() * 4);
        if (st == SI_OK) st = dev_alloc(ctx, ts.G, kTabN * 8);
        if (st != SI_OK) {
            dev_free(ctx, ts.QS); dev_free(ctx, ts.G);
            ctx->tables.erase(key);
            return st;
        }
        SI_CUDA(ctx, cudaMemcpy(ts.QS.ptr, QS.data(), QS.size() * 4, cudaMemcpyHostToDevice), "copy tables");
        SI_CUDA(ctx, cudaMemcpy(ts.G.ptr, G.data(), kTabN * 8, cudaMemcpyHostToDevice), "copy tables");
        ts.consts[0] = q > 0.0 ? std::log2(q) : -INFINITY;
        ts.consts[1] = lr;
        ts.consts[2] = lgc;
        ts.consts[3] = regime;
    }
    out->QS = (const float2*)ts.QS.ptr; out->G = (const double*)ts.G.ptr;
    out->QSup = (const float4*)((const float*)ts.QS.ptr + 2 * kTabN);
    out->QSdn = out->QSup + kTabN;
    out->Gdn = out->QSdn + kTabN;
    out->NT = kTabN; out->log2q = (float)ts.consts[0]; out->invL = 1.0f / (float)L;
    out->lr = ts.consts[1]; out->lgc = ts.consts[2]; out->regime = (int)ts.consts[3];
    return SI_OK;
}

// The typed-marker pipeline once the per-sample views are set in `a`
// (geno, B, M, regions/samples or reg0, sampling, outputs): anchor lists,
// chain, posterior. Waits once on `s` for the list totals.
si_status run_typed(si_ctx* ctx, const si_impute_params* p, TypedArgs& a, uint32_t lmax, bool all_full,
                    cudaStream_t s) {
    a.C = p->checkpoint_interval ? p->checkpoint_interval : typed_default_window(lmax);
    a.threads = p->block_threads ? p->block_threads : typed_default_threads(lmax);
    if (typed_post_smem_bytes(lmax, a.threads, a.C) > 227u * 1024u)
        return fail(ctx, SI_ERR_UNSUPPORTED, "posterior tile needs more than 227 KB of shared memory");
    if (!ctx->pinned_totals) {
        SI_CUDA(ctx, cudaHostAlloc(&ctx->pinned_totals, 4 * sizeof(unsigned long long), cudaHostAllocMapped),
                "pinned totals");
        SI_CUDA(ctx, cudaHostGetDevicePointer(&ctx->pinned_totals_dev, ctx->pinned_totals, 0), "pinned totals");
    }
    if (!ctx->totals_ev) SI_CUDA(ctx, cudaEventCreateWithFlags(&ctx->totals_ev, cudaEventDisableTiming), "event");
    a.host_totals = ctx->pinned_totals_dev;
    a.K = kPostGroup;
    const uint32_t B = a.B, G = typed_groups(B);
    a.nseg = typed_nseg(a.max_len);
    SI_TRY(dev_reserve(ctx, ctx->t_counts, (size_t)B * 4));
    SI_TRY(dev_reserve(ctx, ctx->t_segc, (size_t)B * a.nseg * 4));
    a.segc = (uint32_t*)ctx->t_segc.ptr;
    SI_TRY(dev_reserve(ctx, ctx->t_aoff, ((size_t)G + 1) * 8));
    SI_TRY(dev_reserve(ctx, ctx->t_woff, ((size_t)G + 1) * 8));
    a.cap = nullptr;
    a.counts = (uint32_t*)ctx->t_counts.ptr;
    a.aoff = (unsigned long long*)ctx->t_aoff.ptr;
    a.woff = (unsigned long long*)ctx->t_woff.ptr;
    SI_CUDA(ctx, launch_anchor_lists_count(a, s), "anchor count");
    SI_CUDA(ctx, cudaEventRecord(ctx->totals_ev, s), "event");
    SI_CUDA(ctx, cudaEventSynchronize(ctx->totals_ev), "anchor count");
    const volatile unsigned long long* tot = ctx->pinned_totals;
    const unsigned long long NA = tot[0], NW = tot[1];
    a.max_windows = (uint32_t)tot[2];
    SI_TRY(dev_reserve(ctx, ctx->t_apos, (size_t)NA * 4));
    SI_TRY(dev_reserve(ctx, ctx->t_aem, (size_t)NA * 4));
    SI_TRY(dev_reserve(ctx, ctx->t_ckF, (size_t)NW * lmax * 4));
    SI_TRY(dev_reserve(ctx, ctx->t_ckB, (size_t)NW * lmax * 4));
    SI_TRY(dev_reserve(ctx, ctx->t_ckU, (size_t)NW * 8));
    a.apos = (uint32_t*)ctx->t_apos.ptr;
    a.aem = (uint32_t*)ctx->t_aem.ptr;
    a.total_windows = NW;
    a.ckptF = (float*)ctx->t_ckF.ptr;
    a.ckptB = (float*)ctx->t_ckB.ptr;
    a.ckptU = (double*)ctx->t_ckU.ptr;
    SI_CUDA(ctx, launch_anchor_lists_fill(a, s), "anchor fill");
    SI_CUDA(ctx, cudaEventRecord(ctx->kev[2], s), "event");
    a.ev_chain_done = ctx->kev[3];
    SI_CUDA(ctx, launch_typed_fb(a, lmax, all_full, s), "typed forward-backward");
    SI_CUDA(ctx, cudaEventRecord(ctx->kev[4], s), "event");
    return SI_OK;
}

// Typed-marker forward-backward for a plain batch (every sample over all M markers).
si_status run_device_typed(si_ctx* ctx, const si_impute_params* p, const SelectionCache* sel, const uint8_t* d_geno,
                           uint32_t B, float* d_dosage, float* d_hprob, uint8_t* d_haps, cudaStream_t s) {
    TypedArgs a{};
    a.geno = d_geno;
    a.B = B;
    a.M = ctx->M;
    a.max_len = ctx->M;
    a.sampling = p->sampling;
    a.tie_eps = (float)p->tie_eps;
    a.seed = p->seed;
    a.sid_base = p->sample_id_base;
    a.reg0.masks = (const SlotMasks*)sel->masks.ptr;
    a.reg0.g2 = (const float2*)sel->g2.ptr;
    a.reg0.raw = (const uint8_t*)sel->raw.ptr;
    a.reg0.gs = fb_lmax(p->num_states);
    a.reg0.L = p->num_states;
    SI_TRY(tables_for(ctx, ctx->trans0, p->num_states, &a.reg0.tabs));
    a.dosage = d_dosage;
    a.hprob = d_hprob;
    a.haps = d_haps;
    const uint32_t lmax = fb_lmax(p->num_states);
    return run_typed(ctx, p, a, lmax, lmax == p->num_states, s);
}

// Target-aware selection of B targets (codes d_geno [B][M]) on stream s: the
// rank tables on first use, then each target's slot masks into ctx->smasks
// [M][B] and, when d_pairs is given, its pairs [B][M][L][2].
si_status run_target_select(si_ctx* ctx, uint32_t L, const uint8_t* d_geno, uint32_t B, uint32_t* d_pairs,
                            cudaStream_t s) {
    if (!ctx->has_index) return fail(ctx, SI_ERR_STATE, "PBWT index not built (si_pbwt_build)");
    if (!ctx->prefix.ptr)
        return fail(ctx, SI_ERR_STATE,
                    "target-aware selection reads the full prefix rows: build the index with SI_PBWT_STORE_INDEX");
    if (ctx->n_ex) return fail(ctx, SI_ERR_UNSUPPORTED, "target-aware selection needs a panel of 0/1 alleles");
    if (L == 0 || L > 32) return fail(ctx, SI_ERR_UNSUPPORTED, "target-aware selection takes 1..32 states");
    const uint32_t M = ctx->M, N = ctx->N, W = ctx->W;
    if (!ctx->rank_bits.ptr) {
        SI_TRY(dev_alloc(ctx, ctx->rank_bits, (size_t)M * W * 4));
        si_status st = dev_alloc(ctx, ctx->rank_zeros, (size_t)M * (W + 1) * 4);
        if (st != SI_OK) {
            dev_free(ctx, ctx->rank_bits);
            return st;
        }
        SI_CUDA(ctx,
                launch_target_ranks((const uint32_t*)ctx->prefix.ptr, (const uint32_t*)ctx->panel.ptr, M, N, W,
                                    (uint32_t*)ctx->rank_bits.ptr, (uint32_t*)ctx->rank_zeros.ptr, ctx->stream),
                "target rank tables");
        SI_CUDA(ctx, cudaStreamSynchronize(ctx->stream), "target rank tables");
    }
    SI_TRY(dev_reserve(ctx, ctx->smasks, (size_t)M * B * sizeof(SlotMasks)));
    SI_CUDA(ctx,
            launch_target_select(d_geno, B, M, N, W, L, (const uint32_t*)ctx->prefix.ptr,
                                 (const uint32_t*)ctx->panel.ptr, (const uint32_t*)ctx->rank_bits.ptr,
                                 (const uint32_t*)ctx->rank_zeros.ptr, (SlotMasks*)ctx->smasks.ptr, d_pairs, s),
            "target-aware selection");
    return SI_OK;
}

// Device part of an imputation over B chains whose inputs/outputs are device
// pointers; queued on stream s.
si_status run_device(si_ctx* ctx, const si_impute_params* p, const uint8_t* d_geno, uint32_t B, float* d_dosage,
                     float* d_hprob, uint8_t* d_haps, cudaStream_t s) {
    SelectionCache* sel = nullptr;
    const bool target = p->selection_kind == SI_SEL_TARGET;  // per-target slots: the full-chain kernel
    SI_CUDA(ctx, cudaEventRecord(ctx->kev[0], s), "event");
    if (target) SI_TRY(run_target_select(ctx, p->num_states, d_geno, B, nullptr, s));
    else SI_TRY(ensure_selection(ctx, p->num_states, p->selection_kind, &sel, (p->flags & SI_IMPUTE_RESELECT) != 0, s));
    SI_CUDA(ctx, cudaEventRecord(ctx->kev[1], s), "event");
    ctx->kernel_pending = true;
    if (s != ctx->stream && !(p->flags & SI_IMPUTE_RESELECT)) {
        // a cached table may have been built on the ctx stream: order it before s
        SI_CUDA(ctx, cudaEventRecord(ctx->ev[3], ctx->stream), "event");
        SI_CUDA(ctx, cudaStreamWaitEvent(s, ctx->ev[3], 0), "stream wait");
    }
    SI_TRY(ensure_trans(ctx, p));
    if (!target && p->transition_mode == SI_TRANS_MATRIX0 && !(p->flags & SI_IMPUTE_FULL_CHAIN)) {
        SI_CUDA(ctx, cudaEventRecord(ctx->ev[1], s), "event");
        SI_TRY(run_device_typed(ctx, p, sel, d_geno, B, d_dosage, d_hprob, d_haps, s));
        SI_CUDA(ctx, cudaEventRecord(ctx->ev[2], s), "event");
        ctx->timings_pending = true;
        return SI_OK;
    }
    uint32_t T, C;
    default_tiles(p->num_states, &T, &C);
    // one chain per thread: a batch that fills fewer than two CTAs per SM takes 32-chain CTAs
    // (the CTA size changes nothing numerically)
    if (T > 32 && (B + T - 1) / T < 2u * 148u) T = 32;
    if (p->checkpoint_interval) C = p->checkpoint_interval;
    if (p->block_threads) T = p->block_threads;
    if (fb_smem_bytes(p->num_states, T, C) > 227u * 1024u)
        return fail(ctx, SI_ERR_UNSUPPORTED,
                    "tile (" + std::to_string(T) + " chains x " + std::to_string(C) + " markers) needs " +
                        std::to_string(fb_smem_bytes(p->num_states, T, C)) + " bytes of shared memory (max 227 KB)");
    SI_TRY(dev_reserve(ctx, ctx->ckpt, fb_ckpt_bytes(B, ctx->M, p->num_states, C)));
    FbLaunch l;
    l.geno = d_geno;
    l.masks = target ? nullptr : (const SlotMasks*)sel->masks.ptr;
    l.smasks = target ? (const SlotMasks*)ctx->smasks.ptr : nullptr;
    l.raw = target ? nullptr : (const uint8_t*)sel->raw.ptr;
    l.trans = (const LinTrans*)ctx->trans.ptr;
    l.B = B; l.M = ctx->M; l.L = p->num_states; l.C = C; l.threads = T;
    l.sampling = p->sampling; l.tie_eps = (float)p->tie_eps; l.seed = p->seed; l.sample_id_base = p->sample_id_base;
    l.ckpt = (float*)ctx->ckpt.ptr; l.dosage = d_dosage; l.hprob = d_hprob; l.haps = d_haps;
    SI_CUDA(ctx, cudaEventRecord(ctx->ev[1], s), "event");
    SI_CUDA(ctx, cudaEventRecord(ctx->kev[2], s), "event");
    SI_CUDA(ctx, cudaEventRecord(ctx->kev[3], s), "event");
    SI_CUDA(ctx, launch_fb(l, s), "forward-backward kernel");
    SI_CUDA(ctx, cudaEventRecord(ctx->kev[4], s), "event");
    SI_CUDA(ctx, cudaEventRecord(ctx->ev[2], s), "event");
    ctx->timings_pending = true;
    return SI_OK;
}

}  // namespace

namespace si {

// Arguments of an uneven batch (si_impute_jobs_device, si_plan_create).
bool region_first_gap_ok(const si_ctx* ctx, const si_impute_params* p, uint32_t m_begin, uint32_t m_end) {
    if (m_end - m_begin < 2) return true;
    const LinTrans t0 = lin_trans(ctx->morgans[m_begin], ctx->morgans[m_begin + 1], (double)p->ne, p->rho_rate);
    return t0.c >= 1e-30f;
}

si_status check_jobs_args(si_ctx* ctx, const si_impute_params* p, const si_region* regions, uint32_t n_regions,
                          const si_job* jobs, uint32_t n_jobs) {
    if (!ctx) return SI_ERR_INVALID_ARG;
    if (!p || !regions || !jobs || n_regions == 0 || n_jobs == 0)
        return fail(ctx, SI_ERR_INVALID_ARG, "NULL argument or empty batch");
    if (p->transition_mode != SI_TRANS_MATRIX0)
        return fail(ctx, SI_ERR_UNSUPPORTED, "uneven batches use the first-gap transition (SI_TRANS_MATRIX0)");
    if (!ctx->panel.ptr) return fail(ctx, SI_ERR_STATE, "no panel uploaded");
    if (!ctx->has_map) return fail(ctx, SI_ERR_STATE, "marker positions not set (si_panel_set_map)");
    if (p->sampling != SI_SAMPLE_ARGMAX && p->sampling != SI_SAMPLE_PHILOX)
        return fail(ctx, SI_ERR_INVALID_ARG, "bad sampling mode");
    if (!(p->tie_eps >= 0.0 && p->tie_eps < 1.0)) return fail(ctx, SI_ERR_INVALID_ARG, "tie_eps must be in [0, 1)");
    if (p->checkpoint_interval > 32) return fail(ctx, SI_ERR_UNSUPPORTED, "checkpoint_interval must be <= 32");
    if (p->block_threads && (p->block_threads % 32 || p->block_threads > 128))
        return fail(ctx, SI_ERR_UNSUPPORTED, "block_threads must be a multiple of 32, <= 128");
    return SI_OK;
}

// Region tables of an uneven batch: region-local sweeps and selections not
// cached yet (one launch for all), global-origin selections, run tables; and
// the per-job descriptors.
si_status prepare_jobs(si_ctx* ctx, const si_impute_params* p, const si_region* regions, uint32_t n_regions,
                       const si_job* jobs, uint32_t n_jobs, cudaStream_t s, std::vector<TypedRegion>& tr,
                       std::vector<TypedSample>& ts, uint32_t& lmax, bool& all_full) {
    const uint32_t N = ctx->N, W = ctx->W;
    lmax = 4;
    bool need_global = false;
    for (uint32_t r = 0; r < n_regions; ++r) {
        const si_region& g = regions[r];
        if (g.m_begin >= g.m_end || g.m_end > ctx->M)
            return fail(ctx, SI_ERR_INVALID_ARG, "region " + std::to_string(r) + " is empty or outside the panel");
        if (g.num_states == 0 || g.num_states > 32)
            return fail(ctx, SI_ERR_UNSUPPORTED, "region " + std::to_string(r) + ": num_states must be 1..32");
        if (g.index_origin != SI_INDEX_GLOBAL && g.index_origin != SI_INDEX_REGION)
            return fail(ctx, SI_ERR_INVALID_ARG, "bad index_origin");
        lmax = std::max(lmax, fb_lmax(g.num_states));
        need_global |= g.index_origin == SI_INDEX_GLOBAL;
    }
    all_full = true;
    for (uint32_t r = 0; r < n_regions; ++r) all_full &= regions[r].num_states == lmax;
    if (need_global) SI_TRY(ensure_trans(ctx, p));  // panel-wide first-gap transition (trans0)
    tr.assign(n_regions, TypedRegion{});
    // region-local sweeps that are not cached yet, all in one launch
    std::vector<SweepJob> sweeps;
    std::vector<uint32_t> sweep_region;
    uint64_t head_rows = 0;
    for (uint32_t r = 0; r < n_regions; ++r) {
        const si_region& g = regions[r];
        if (g.index_origin != SI_INDEX_REGION) continue;
        const uint32_t L = g.num_states;
        const int kind = (L <= 32 && N <= 10000) ? SI_SEL_WARP : SI_SEL_INSERTION;
        auto key = std::make_tuple(g.m_begin, g.m_end, L, kind);
        if (ctx->region_sel.count(key)) continue;
        bool dup = false;
        for (uint32_t q : sweep_region)
            if (regions[q].m_begin == g.m_begin && regions[q].m_end == g.m_end) dup = true;
        if (dup) continue;
        sweeps.push_back(SweepJob{g.m_begin, g.m_end - g.m_begin, head_rows * kHead, kIota});
        sweep_region.push_back(r);
        head_rows += g.m_end - g.m_begin;
    }
    if (!sweeps.empty()) {
        DeviceBuffer head, perm, jb;
        SI_TRY(dev_alloc(ctx, head, head_rows * kHead * 4));
        si_status st = dev_alloc(ctx, perm, (size_t)sweeps.size() * 2 * N * 4);
        if (st == SI_OK) st = dev_alloc(ctx, jb, sweeps.size() * sizeof(SweepJob));
        cudaError_t e = cudaSuccess;
        if (st == SI_OK) e = cudaMemsetAsync(head.ptr, 0, head_rows * kHead * 4, s);
        if (st == SI_OK && e == cudaSuccess)
            e = cudaMemcpyAsync(jb.ptr, sweeps.data(), sweeps.size() * sizeof(SweepJob), cudaMemcpyHostToDevice, s);
        if (st == SI_OK && e == cudaSuccess)
            e = launch_pbwt_sweep((const uint32_t*)ctx->panel.ptr, (const SweepJob*)jb.ptr, (uint32_t)sweeps.size(),
                                  N, W, nullptr, (uint32_t*)head.ptr, nullptr, nullptr, (uint32_t*)perm.ptr, s);
        // selection tables of every region (and slot count) that uses these sweeps
        for (uint32_t r = 0; st == SI_OK && e == cudaSuccess && r < n_regions; ++r) {
            const si_region& g = regions[r];
            if (g.index_origin != SI_INDEX_REGION) continue;
            const uint32_t L = g.num_states;
            const int kind = (L <= 32 && N <= 10000) ? SI_SEL_WARP : SI_SEL_INSERTION;
            auto key = std::make_tuple(g.m_begin, g.m_end, L, kind);
            if (ctx->region_sel.count(key)) continue;
            size_t j = 0;
            while (j < sweeps.size() && !(sweeps[j].m0 == g.m_begin && sweeps[j].len == g.m_end - g.m_begin)) ++j;
            if (j == sweeps.size()) continue;  // cached already under another slot count? swept above
            auto& rs = ctx->region_sel[key];
            st = dev_alloc(ctx, rs.masks, (size_t)(g.m_end - g.m_begin) * sizeof(SlotMasks));
            if (st == SI_OK) st = dev_alloc(ctx, rs.g2, (size_t)(g.m_end - g.m_begin) * fb_lmax(L) * sizeof(float2));
            if (st == SI_OK && ctx->n_ex) st = dev_alloc(ctx, rs.raw, (size_t)(g.m_end - g.m_begin) * fb_lmax(L) * 2);
            if (st != SI_OK) {
                dev_free(ctx, rs.masks);
                dev_free(ctx, rs.g2);
                ctx->region_sel.erase(key);
                break;
            }
            e = launch_select((const uint32_t*)head.ptr + sweeps[j].head_off,
                              (const uint32_t*)ctx->panel.ptr + (size_t)g.m_begin * W, g.m_end - g.m_begin, N, W, L,
                              kind, ctx->n_ex ? (const unsigned long long*)ctx->ex_off.ptr + g.m_begin : nullptr,
                              (const uint32_t*)ctx->ex_ent.ptr, nullptr, (SlotMasks*)rs.masks.ptr, (float2*)rs.g2.ptr,
                              (uint8_t*)rs.raw.ptr, fb_lmax(L), s);
        }
        if (st == SI_OK && e == cudaSuccess) e = cudaStreamSynchronize(s);  // scratch reuse below
        dev_free(ctx, head);
        dev_free(ctx, perm);
        dev_free(ctx, jb);
        if (st != SI_OK) return st;
        if (e != cudaSuccess) return cuda_fail(ctx, e, "region sweep");
    }
    for (uint32_t r = 0; r < n_regions; ++r) {
        const si_region& g = regions[r];
        const uint32_t L = g.num_states;
        tr[r].L = L;
        if (g.index_origin == SI_INDEX_GLOBAL) {
            SelectionCache* sel = nullptr;
            SI_TRY(ensure_selection(ctx, L, p->selection_kind, &sel, false, s));
            tr[r].masks = (const SlotMasks*)sel->masks.ptr + g.m_begin;
            tr[r].g2 = (const float2*)sel->g2.ptr + (size_t)g.m_begin * fb_lmax(L);
            tr[r].raw = sel->raw.ptr ? (const uint8_t*)sel->raw.ptr + (size_t)g.m_begin * fb_lmax(L) * 2 : nullptr;
            tr[r].gs = fb_lmax(L);
            SI_TRY(tables_for(ctx, ctx->trans0, L, &tr[r].tabs));
        } else {
            const int kind = (L <= 32 && N <= 10000) ? SI_SEL_WARP : SI_SEL_INSERTION;
            const auto& rs = ctx->region_sel[std::make_tuple(g.m_begin, g.m_end, L, kind)];
            tr[r].masks = (const SlotMasks*)rs.masks.ptr;
            tr[r].g2 = (const float2*)rs.g2.ptr;
            tr[r].raw = (const uint8_t*)rs.raw.ptr;
            tr[r].gs = fb_lmax(L);
            if (!region_first_gap_ok(ctx, p, g.m_begin, g.m_end))
                return fail(ctx, SI_ERR_UNSUPPORTED, "region " + std::to_string(r) +
                                                         ": zero genetic distance in its first gap");
            const LinTrans t0 = (g.m_end - g.m_begin >= 2)
                                    ? lin_trans(ctx->morgans[g.m_begin], ctx->morgans[g.m_begin + 1], (double)p->ne,
                                                p->rho_rate)
                                    : LinTrans{1.f, 0.f};
            SI_TRY(tables_for(ctx, t0, L, &tr[r].tabs));
        }
    }
    ts.assign(n_jobs, TypedSample{});
    for (uint32_t j = 0; j < n_jobs; ++j) {
        if (jobs[j].region >= n_regions) return fail(ctx, SI_ERR_INVALID_ARG, "job region out of range");
        const si_region& g = regions[jobs[j].region];
        ts[j].geno_off = jobs[j].geno_offset;
        ts[j].out_off = jobs[j].out_offset;
        ts[j].sample_id = jobs[j].sample_id;
        ts[j].m0 = g.m_begin;
        ts[j].len = g.m_end - g.m_begin;
        ts[j].region = jobs[j].region;
        ts[j].pad = 0;
    }
    // Launch order: longest slices first, a region's jobs together, so the 32
    // lanes of a warp (one group of the interleaved anchor lists) share their
    // slice length and, for targets of one array, their typed positions. Each
    // job still writes at its own offsets with its own sample id.
    std::stable_sort(ts.begin(), ts.end(), [](const TypedSample& x, const TypedSample& y) {
        return x.len != y.len ? x.len > y.len : x.region < y.region;
    });
    return SI_OK;
}

}  // namespace si

extern "C" {

int si_abi_version(void) { return SI_ABI_VERSION; }

const char* si_status_string(si_status s) {
    switch (s) {
        case SI_OK: return "ok";
        case SI_ERR_INVALID_ARG: return "invalid argument";
        case SI_ERR_CUDA: return "CUDA error";
        case SI_ERR_OUT_OF_MEMORY: return "out of device memory";
        case SI_ERR_UNSUPPORTED: return "unsupported";
        case SI_ERR_STATE: return "bad call order";
        case SI_ERR_TIMEOUT: return "timeout";
        case SI_ERR_BUDGET: return "HBM budget exceeded";
        case SI_ERR_CANCELLED: return "cancelled";
    }
    return "unknown status";
}

si_status si_ctx_create(int device, uint64_t hbm_budget_bytes, si_ctx** out) {
    if (!out) return SI_ERR_INVALID_ARG;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) { cudaGetLastError(); return SI_ERR_CUDA; }
    if (device < 0 || device >= n) return SI_ERR_INVALID_ARG;
    si_ctx* ctx = new (std::nothrow) si_ctx();
    if (!ctx) return SI_ERR_OUT_OF_MEMORY;
    ctx->device = device;
    if (cudaSetDevice(device) != cudaSuccess) { delete ctx; return SI_ERR_CUDA; }
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) { delete ctx; return SI_ERR_CUDA; }
    ctx->budget = hbm_budget_bytes ? hbm_budget_bytes : (uint64_t)free_b;
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) { delete ctx; return SI_ERR_CUDA; }
    for (auto& e : ctx->ev)
        if (cudaEventCreate(&e) != cudaSuccess) { delete ctx; return SI_ERR_CUDA; }
    for (auto& e : ctx->kev)
        if (cudaEventCreate(&e) != cudaSuccess) { delete ctx; return SI_ERR_CUDA; }
    *out = ctx;
    return SI_OK;
}

si_status si_ctx_destroy(si_ctx* ctx) {
    if (!ctx) return SI_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    reset_index(ctx);
    dev_free(ctx, ctx->panel);
    dev_free(ctx, ctx->trans);
    dev_free(ctx, ctx->ckpt);
    dev_free(ctx, ctx->smasks);
    dev_free(ctx, ctx->io_geno);
    dev_free(ctx, ctx->io_dosage);
    dev_free(ctx, ctx->io_hprob);
    dev_free(ctx, ctx->io_haps);
    dev_free(ctx, ctx->io_geno2);
    dev_free(ctx, ctx->io_hbits);
    for (si::DeviceBuffer* b : {&ctx->t_counts, &ctx->t_segc, &ctx->t_aoff, &ctx->t_woff, &ctx->t_apos, &ctx->t_aem,
                                &ctx->t_ckF, &ctx->t_ckB, &ctx->t_ckU, &ctx->job_regions,
                                &ctx->job_samples})
        dev_free(ctx, *b);
    for (auto& kv : ctx->tables) {
        dev_free(ctx, kv.second.QS);
        dev_free(ctx, kv.second.G);
    }
    for (auto& kv : ctx->region_sel) {
        dev_free(ctx, kv.second.masks);
        dev_free(ctx, kv.second.g2);
        dev_free(ctx, kv.second.raw);
    }
    dev_free(ctx, ctx->ex_off);
    dev_free(ctx, ctx->ex_ent);
    if (ctx->pinned_totals) cudaFreeHost(ctx->pinned_totals);
    if (ctx->totals_ev) cudaEventDestroy(ctx->totals_ev);
    for (auto& e : ctx->ev) if (e) cudaEventDestroy(e);
    for (auto& e : ctx->kev) if (e) cudaEventDestroy(e);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    if (ctx->copy_in) cudaStreamDestroy(ctx->copy_in);
    if (ctx->copy_out) cudaStreamDestroy(ctx->copy_out);
    delete ctx;
    return SI_OK;
}

const char* si_last_error(const si_ctx* ctx) { return ctx ? ctx->err.c_str() : "no context"; }

si_status si_ctx_memory(const si_ctx* ctx, uint64_t* used_bytes, uint64_t* budget_bytes) {
    if (!ctx) return SI_ERR_INVALID_ARG;
    if (used_bytes) *used_bytes = ctx->used;
    if (budget_bytes) *budget_bytes = ctx->budget;
    return SI_OK;
}

si_status si_panel_upload_packed(si_ctx* ctx, const uint32_t* words, uint32_t M, uint32_t N,
                                 uint32_t words_per_row) {
    if (!ctx) return SI_ERR_INVALID_ARG;
    if (!words || M == 0 || N < 2 || words_per_row < (N + 31) / 32)
        return fail(ctx, SI_ERR_INVALID_ARG, "bad packed panel arguments (need M >= 1, N >= 2)");
    if (M >= kMaxMarkers) return fail(ctx, SI_ERR_UNSUPPORTED, "panels hold at most 2^31 - 1 markers");
    SI_TRY(set_device(ctx));
    reset_index(ctx);
    clear_exceptions(ctx);
    const uint32_t W = words_per_row_pad(N);
    SI_TRY(dev_alloc(ctx, ctx->panel, (size_t)M * W * 4));
    SI_CUDA(ctx,
            cudaMemcpy2D(ctx->panel.ptr, (size_t)W * 4, words, (size_t)words_per_row * 4, (size_t)((N + 31) / 32) * 4,
                         M, cudaMemcpyHostToDevice),
            "copy packed panel");
    if (W > (N + 31) / 32)
        SI_CUDA(ctx,
                cudaMemset2D((char*)ctx->panel.ptr + (size_t)((N + 31) / 32) * 4, (size_t)W * 4, 0,
                             (size_t)(W - (N + 31) / 32) * 4, M),
                "pad panel");
    // clear bits past N in the last word of every row
    if (N % 32) {
        std::vector<uint32_t> last(M);
        SI_CUDA(ctx,
                cudaMemcpy2D(last.data(), 4, (char*)ctx->panel.ptr + (size_t)(N / 32) * 4, (size_t)W * 4, 4, M,
                             cudaMemcpyDeviceToHost),
                "read last words");
        const uint32_t keep = (1u << (N % 32)) - 1u;
        for (auto& v : last) v &= keep;
        SI_CUDA(ctx,
                cudaMemcpy2D((char*)ctx->panel.ptr + (size_t)(N / 32) * 4, (size_t)W * 4, last.data(), 4, 4, M,
                             cudaMemcpyHostToDevice),
                "write last words");
    }
    ctx->M = M; ctx->N = N; ctx->W = W;
    ctx->has_map = false;
    ctx->trans_key = ~0ull;
    return SI_OK;
}

si_status si_panel_upload_u8(si_ctx* ctx, const uint8_t* alleles, uint32_t M, uint32_t N) {
    if (!ctx) return SI_ERR_INVALID_ARG;
    if (!alleles || M == 0 || N < 2) return fail(ctx, SI_ERR_INVALID_ARG, "bad panel arguments (need M >= 1, N >= 2)");
    if (M >= kMaxMarkers) return fail(ctx, SI_ERR_UNSUPPORTED, "panels hold at most 2^31 - 1 markers");
    SI_TRY(set_device(ctx));
    reset_index(ctx);
    clear_exceptions(ctx);
    std::vector<unsigned long long> ex_off;
    std::vector<uint32_t> ex_ent;
    panel_exceptions(alleles, M, N, ex_off, ex_ent);
    if (!ex_ent.empty() && N >= (1u << 24))
        return fail(ctx, SI_ERR_UNSUPPORTED, "panels with alleles other than 0/1 need N < 2^24 haplotypes");
    const uint32_t W = words_per_row_pad(N);
    SI_TRY(dev_alloc(ctx, ctx->panel, (size_t)M * W * 4));
    SI_CUDA(ctx, cudaMemsetAsync(ctx->panel.ptr, 0, (size_t)M * W * 4, ctx->stream), "memset panel");
    // stream the u8 panel through a bounded staging buffer
    const size_t row_bytes = N;
    const uint32_t rows_per_chunk = (uint32_t)std::max<size_t>(1, std::min<size_t>(M, (256u << 20) / row_bytes));
    DeviceBuffer stage;
    SI_TRY(dev_alloc(ctx, stage, (size_t)rows_per_chunk * row_bytes));
    cudaError_t e = cudaSuccess;
    for (uint32_t m0 = 0; m0 < M && e == cudaSuccess; m0 += rows_per_chunk) {
        const uint32_t rows = std::min(rows_per_chunk, M - m0);
        e = cudaMemcpyAsync(stage.ptr, alleles + (size_t)m0 * N, (size_t)rows * N, cudaMemcpyHostToDevice, ctx->stream);
        if (e == cudaSuccess)
            e = launch_pack_panel((const uint8_t*)stage.ptr, rows, N, W, (uint32_t*)ctx->panel.ptr + (size_t)m0 * W,
                                  ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);  // staging buffer reuse
    }
    dev_free(ctx, stage);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "panel upload");
    if (!ex_ent.empty()) {
        si_status st = dev_alloc(ctx, ctx->ex_off, ex_off.size() * 8);
        if (st == SI_OK) st = dev_alloc(ctx, ctx->ex_ent, ex_ent.size() * 4);
        if (st != SI_OK) {
            clear_exceptions(ctx);
            dev_free(ctx, ctx->panel);
            return st;
        }
        SI_CUDA(ctx, cudaMemcpy(ctx->ex_off.ptr, ex_off.data(), ex_off.size() * 8, cudaMemcpyHostToDevice), "copy exceptions");
        SI_CUDA(ctx, cudaMemcpy(ctx->ex_ent.ptr, ex_ent.data(), ex_ent.size() * 4, cudaMemcpyHostToDevice), "copy exceptions");
        ctx->n_ex = ex_ent.size();
    }
    ctx->M = M; ctx->N = N; ctx->W = W;
    ctx->has_map = false;
    ctx->trans_key = ~0ull;
    return SI_OK;
}

si_status si_panel_exception_count(const si_ctx* ctx, uint64_t* count) {
    if (!ctx || !count) return SI_ERR_INVALID_ARG;
    *count = ctx->n_ex;
    return SI_OK;
}

si_status si_panel_set_map(si_ctx* ctx, const uint64_t* pos, const double* cM) {
    if (!ctx) return SI_ERR_INVALID_ARG;
    if (!ctx->panel.ptr) return fail(ctx, SI_ERR_STATE, "no panel uploaded");
    if (!pos) return fail(ctx, SI_ERR_INVALID_ARG, "pos is NULL");
    ctx->morgans.resize(ctx->M);
    for (uint32_t m = 0; m < ctx->M; ++m)
        ctx->morgans[m] = (cM && cM[m] > 0.0) ? cM[m] / 100.0 : (double)pos[m] / 1e8;
    ctx->has_map = true;
    ctx->trans_key = ~0ull;
    return SI_OK;
}

si_status si_pbwt_build(si_ctx* ctx, uint32_t flags) {
    Range range("si_pbwt_build");
    if (!ctx) return SI_ERR_INVALID_ARG;
    if (!ctx->panel.ptr) return fail(ctx, SI_ERR_STATE, "no panel uploaded");
    SI_TRY(set_device(ctx));
    reset_index(ctx);
    const uint32_t M = ctx->M, N = ctx->N;
    SI_TRY(dev_alloc(ctx, ctx->head, (size_t)M * kHead * 4));
    SI_CUDA(ctx, cudaMemsetAsync(ctx->head.ptr, 0, (size_t)M * kHead * 4, ctx->stream), "memset head");
    if (flags & SI_PBWT_STORE_INDEX) SI_TRY(dev_alloc(ctx, ctx->prefix, (size_t)M * N * 4));
    if (flags & SI_PBWT_ROW_HASHES) {
        SI_TRY(dev_alloc(ctx, ctx->row_hash, (size_t)M * 8));
        SI_CUDA(ctx, cudaMemsetAsync(ctx->row_hash.ptr, 0, (size_t)M * 8, ctx->stream), "memset hash");
    }
    // Segments of at least kMinSegment markers, one per SM: the groups pass and
    // the final sweep run every segment on its own CTA, the composition of the
    // segments' start orders runs once per segment (pbwt_kernels.cu).
    constexpr uint32_t kMinSegment = 64;
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, ctx->device);
    const uint32_t S0 = std::max(1u, std::min<uint32_t>((uint32_t)nsm, M / kMinSegment));
    const uint32_t Lseg = (M + S0 - 1) / S0;
    const uint32_t S = (M + Lseg - 1) / Lseg;
    std::vector<SweepJob> jobs(S);
    for (uint32_t j = 0; j < S; ++j)
        jobs[j] = SweepJob{j * Lseg, std::min(Lseg, M - j * Lseg), (uint64_t)j * Lseg * kHead,
                           j == 0 ? kIota : (uint64_t)j * N};
    int max_optin = 0;
    cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device);
    const bool sweep_global = pbwt_sweep_smem_bytes(N, ctx->W) > (size_t)max_optin;
    const bool group_global = S > 1 && pbwt_group_smem_bytes(N, ctx->W) > (size_t)max_optin;
    const size_t scratch_words = std::max<size_t>(sweep_global ? (size_t)2 * N * S : 0,
                                                  group_global ? (size_t)4 * N * (S - 1) : 0);
    DeviceBuffer scratch, jobbuf, orders, gid, sortbuf;
    si_status st = dev_alloc(ctx, jobbuf, S * sizeof(SweepJob));
    if (st == SI_OK && scratch_words) st = dev_alloc(ctx, scratch, scratch_words * 4);
    if (st == SI_OK && S > 1) st = dev_alloc(ctx, orders, (size_t)S * N * 4);
    if (st == SI_OK && S > 1) st = dev_alloc(ctx, gid, (size_t)(S - 1) * N * 4);
    if (st == SI_OK && S > 1) st = dev_alloc(ctx, sortbuf, (size_t)4 * N * 4);
    cudaError_t e = cudaSuccess;
    if (st == SI_OK) {
        e = cudaMemcpy(jobbuf.ptr, jobs.data(), S * sizeof(SweepJob), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaEventRecord(ctx->ev[0], ctx->stream);
        const uint32_t* panel = (const uint32_t*)ctx->panel.ptr;
        const SweepJob* dj = (const SweepJob*)jobbuf.ptr;
        uint32_t* ord = (uint32_t*)orders.ptr;
        if (e == cudaSuccess && S > 1) {
            e = launch_iota(ord, N, ctx->stream);
            if (e == cudaSuccess)
                e = launch_pbwt_groups(panel, dj, S - 1, N, ctx->W, (uint32_t*)gid.ptr, (uint32_t*)scratch.ptr,
                                       ctx->stream);
            for (uint32_t j = 0; e == cudaSuccess && j + 1 < S; ++j)
                e = launch_pbwt_compose(ord + (size_t)j * N, (const uint32_t*)gid.ptr + (size_t)j * N,
                                        ord + (size_t)(j + 1) * N, N, (uint32_t*)sortbuf.ptr, ctx->stream);
        }
        if (e == cudaSuccess)
            e = launch_pbwt_sweep(panel, dj, S, N, ctx->W, ord, (uint32_t*)ctx->head.ptr,
                                  (uint32_t*)ctx->prefix.ptr, (unsigned long long*)ctx->row_hash.ptr,
                                  (uint32_t*)scratch.ptr, ctx->stream);
        if (e == cudaSuccess) e = cudaEventRecord(ctx->ev[1], ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ctx->pbwt_ms, ctx->ev[0], ctx->ev[1]);
    }
    for (DeviceBuffer* b : {&scratch, &jobbuf, &orders, &gid, &sortbuf}) dev_free(ctx, *b);
    if (st != SI_OK) return st;
    if (e != cudaSuccess) return cuda_fail(ctx, e, "PBWT sweep");
    ctx->has_index = true;
    ctx->pbwt_flags = flags;
    return SI_OK;
}

namespace {

// Stored index: header {magic, M, N, head width, panel checksum} then the
// head rows [M][kHead] u32, the only part of the index selection reads.
struct StoredIndexHeader {
    char magic[8];
    uint32_t M, N, head;
    uint32_t reserved;
    uint64_t checksum;
};

si_status panel_checksum(si_ctx* ctx, uint64_t* out) {
    DeviceBuffer d;
    SI_TRY(dev_alloc(ctx, d, 8));
    cudaError_t e = launch_panel_checksum((const uint32_t*)ctx->panel.ptr, (uint64_t)ctx->M * ctx->W,
                                          (unsigned long long*)d.ptr, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, d.ptr, 8, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    dev_free(ctx, d);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "panel checksum");
    return SI_OK;
}

}  // namespace

si_status si_pbwt_stored_bytes(const si_ctx* ctx, uint64_t* bytes) {
    if (!ctx || !bytes) return SI_ERR_INVALID_ARG;
    *bytes = sizeof(StoredIndexHeader) + (uint64_t)ctx->M * kHead * 4;
    return SI_OK;
}

si_status si_pbwt_save(si_ctx* ctx, void* out, uint64_t bytes) {
    Range range("si_pbwt_save");
    if (!ctx) return SI_ERR_INVALID_ARG;
    if (!ctx->has_index) return fail(ctx, SI_ERR_STATE, "PBWT index not built (si_pbwt_build)");
    const uint64_t need = sizeof(StoredIndexHeader) + (uint64_t)ctx->M * kHead * 4;
    if (!out || bytes < need) return fail(ctx, SI_ERR_INVALID_ARG, "output smaller than si_pbwt_stored_bytes");
    SI_TRY(set_device(ctx));
    StoredIndexHeader h{};
    std::memcpy(h.magic, "SIINDEX1", 8);
    h.M = ctx->M; h.N = ctx->N; h.head = kHead;
    SI_TRY(panel_checksum(ctx, &h.checksum));
    std::memcpy(out, &h, sizeof h);
    SI_CUDA(ctx, cudaMemcpy((char*)out + sizeof h, ctx->head.ptr, (size_t)ctx->M * kHead * 4, cudaMemcpyDeviceToHost),
            "copy index");
    return SI_OK;
}

si_status si_pbwt_load(si_ctx* ctx, const void* in, uint64_t bytes) {
    Range range("si_pbwt_load");
    if (!ctx) return SI_ERR_INVALID_ARG;
    if (!ctx->panel.ptr) return fail(ctx, SI_ERR_STATE, "no panel uploaded");
    StoredIndexHeader h{};
    if (!in || bytes < sizeof h) return fail(ctx, SI_ERR_INVALID_ARG, "stored index too short");
    std::memcpy(&h, in, sizeof h);
    if (std::memcmp(h.magic, "SIINDEX1", 8) != 0) return fail(ctx, SI_ERR_INVALID_ARG, "not a stored PBWT index");
    if (h.M != ctx->M || h.N != ctx->N || h.head != kHead)
        return fail(ctx, SI_ERR_INVALID_ARG, "stored index shape differs from the uploaded panel");
    if (bytes < sizeof h + (uint64_t)h.M * kHead * 4) return fail(ctx, SI_ERR_INVALID_ARG, "stored index truncated");
    SI_TRY(set_device(ctx));
    uint64_t sum = 0;
    SI_TRY(panel_checksum(ctx, &sum));
    if (sum != h.checksum)
        return fail(ctx, SI_ERR_INVALID_ARG, "stored index was built on a different panel (checksum differs)");
    reset_index(ctx);
    SI_TRY(dev_alloc(ctx, ctx->head, (size_t)ctx->M * kHead * 4));
    SI_CUDA(ctx, cudaMemcpy(ctx->head.ptr, (const char*)in + sizeof h, (size_t)ctx->M * kHead * 4,
                            cudaMemcpyHostToDevice), "copy index");
    ctx->has_index = true;
    ctx->pbwt_flags = 0;
    return SI_OK;
}

si_status si_pbwt_get_prefix_rows(si_ctx* ctx, uint32_t m0, uint32_t count, uint32_t* out) {
    if (!ctx) return SI_ERR_INVALID_ARG;
    if (!ctx->has_index || !ctx->prefix.ptr)
        return fail(ctx, SI_ERR_STATE, "full prefix index not stored (build with SI_PBWT_STORE_INDEX)");
    if (!out || (uint64_t)m0 + count > ctx->M) return fail(ctx, SI_ERR_INVALID_ARG, "row range out of bounds");
    SI_TRY(set_device(ctx));
    SI_CUDA(ctx,
            cudaMemcpy(out, (uint32_t*)ctx->prefix.ptr + (size_t)m0 * ctx->N, (size_t)count * ctx->N * 4,
                       cudaMemcpyDeviceToHost),
            "copy prefix rows");
    return SI_OK;
}

si_status si_pbwt_row_hashes(si_ctx* ctx, uint64_t* out) {
    if (!ctx) return SI_ERR_INVALID_ARG;
    if (!ctx->has_index || !ctx->row_hash.ptr)
        return fail(ctx, SI_ERR_STATE, "row hashes not stored (build with SI_PBWT_ROW_HASHES)");
    if (!out) return fail(ctx, SI_ERR_INVALID_ARG, "out is NULL");
    SI_TRY(set_device(ctx));
    SI_CUDA(ctx, cudaMemcpy(out, ctx->row_hash.ptr, (size_t)ctx->M * 8, cudaMemcpyDeviceToHost), "copy hashes");
    return SI_OK;
}

si_status si_pbwt_last_ms(const si_ctx* ctx, float* ms) {
    if (!ctx || !ms) return SI_ERR_INVALID_ARG;
    *ms = ctx->pbwt_ms;
    return SI_OK;
}

si_status si_select_states(si_ctx* ctx, uint32_t L, int32_t kind, uint32_t m0, uint32_t m1, uint32_t* out_pairs) {
    Range range("si_select_states");
    if (!ctx) return SI_ERR_INVALID_ARG;
    if (!out_pairs || m0 > m1 || m1 > ctx->M) return fail(ctx, SI_ERR_INVALID_ARG, "bad marker range");
    SI_TRY(set_device(ctx));
    SelectionCache* c = nullptr;
    SI_TRY(ensure_selection(ctx, L, kind, &c));
    SI_CUDA(ctx, cudaStreamSynchronize(ctx->stream), "selection");
    SI_CUDA(ctx,
            cudaMemcpy(out_pairs, (uint32_t*)c->pairs.ptr + (size_t)m0 * L * 2, (size_t)(m1 - m0) * L * 2 * 4,
                       cudaMemcpyDeviceToHost),
            "copy pairs");
    return SI_OK;
}

si_status si_select_states_target(si_ctx* ctx, uint32_t L, const uint8_t* geno_codes, uint32_t B, uint32_t* out_pairs) {
    Range range("si_select_states_target");
    if (!ctx) return SI_ERR_INVALID_ARG;
    if (!geno_codes || !out_pairs || B == 0) return fail(ctx, SI_ERR_INVALID_ARG, "NULL argument or empty batch");
    if (!ctx->panel.ptr) return fail(ctx, SI_ERR_STATE, "no panel uploaded");
    SI_TRY(set_device(ctx));
    const size_t cells = (size_t)B * ctx->M, npairs = cells * L * 2;
    DeviceBuffer g, pr;
    SI_TRY(dev_alloc(ctx, g, cells));
    si_status st = dev_alloc(ctx, pr, npairs * 4);
    cudaError_t e = cudaSuccess;
    if (st == SI_OK) e = cudaMemcpyAsync(g.ptr, geno_codes, cells, cudaMemcpyHostToDevice, ctx->stream);
    if (st == SI_OK && e == cudaSuccess)
        st = run_target_select(ctx, L, (const uint8_t*)g.ptr, B, (uint32_t*)pr.ptr, ctx->stream);
    if (st == SI_OK && e == cudaSuccess)
        e = cudaMemcpyAsync(out_pairs, pr.ptr, npairs * 4, cudaMemcpyDeviceToHost, ctx->stream);
    if (st == SI_OK && e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    dev_free(ctx, g);
    dev_free(ctx, pr);
    if (st != SI_OK) return st;
    if (e != cudaSuccess) return cuda_fail(ctx, e, "target-aware selection");
    return SI_OK;
}

si_status si_impute_params_default(si_impute_params* p) {
    if (!p) return SI_ERR_INVALID_ARG;
    std::memset(p, 0, sizeof *p);
    p->num_states = 8;         // HMMParameters defaults, core/types.hpp:84-89
    p->ne = 10000;
    p->rho_rate = 4.0;
    p->theta = 0.001;
    p->transition_mode = SI_TRANS_MATRIX0;
    p->selection_kind = SI_SEL_AUTO;
    p->sampling = SI_SAMPLE_ARGMAX;
    p->tie_eps = 1e-4;
    p->seed = 12345;           // the reference's fixed cuRAND seed, sampling.cu:302
    return SI_OK;
}

si_status si_impute_device(si_ctx* ctx, const si_impute_params* p, const uint8_t* d_geno, uint32_t B,
                           float* d_dosage, float* d_hprob, uint8_t* d_haps, void* stream) {
    Range range("si_impute_device");
    if (!ctx) return SI_ERR_INVALID_ARG;
    SI_TRY(check_params(ctx, p));
    if (!d_geno || B == 0) return fail(ctx, SI_ERR_INVALID_ARG, "geno is NULL or B == 0");
    if (p->flags & (SI_IMPUTE_CODES_2BIT | SI_IMPUTE_HAPS_BITS))
        return fail(ctx, SI_ERR_UNSUPPORTED, "compact formats are formats of host buffers (si_impute)");
    SI_TRY(set_device(ctx));
    cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
    SI_CUDA(ctx, cudaEventRecord(ctx->ev[0], s), "event");
    return run_device(ctx, p, d_geno, B, d_dosage, d_hprob, d_haps, s);
}

si_status si_impute(si_ctx* ctx, const si_impute_params* p, const uint8_t* geno, uint32_t B, float* dosage,
                    float* hap_prob, uint8_t* haps) {
    Range range("si_impute");
    if (!ctx) return SI_ERR_INVALID_ARG;
    SI_TRY(check_params(ctx, p));
    if (!geno || B == 0) return fail(ctx, SI_ERR_INVALID_ARG, "geno is NULL or B == 0");
    SI_TRY(set_device(ctx));
    const uint32_t M = ctx->M;
    const size_t cells = (size_t)B * M;
    const bool codes2 = (p->flags & SI_IMPUTE_CODES_2BIT) != 0, hbits = (p->flags & SI_IMPUTE_HAPS_BITS) != 0;
    if (hbits && ctx->n_ex)
        return fail(ctx, SI_ERR_UNSUPPORTED, "haplotype bits hold 0/1 alleles: this panel has others (use bytes)");
    const size_t Mb = (M + 3) / 4, Mw = (M + 31) / 32;  // bytes of a 2-bit row, words of a bit row
    cudaStream_t s = ctx->stream;
    if (!ctx->copy_in) SI_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->copy_in, cudaStreamNonBlocking), "copy stream");
    if (!ctx->copy_out) SI_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->copy_out, cudaStreamNonBlocking), "copy stream");
    SI_TRY(dev_reserve(ctx, ctx->io_geno, cells));
    if (dosage) SI_TRY(dev_reserve(ctx, ctx->io_dosage, cells * 4));
    if (hap_prob) SI_TRY(dev_reserve(ctx, ctx->io_hprob, cells * 8));
    if (haps) SI_TRY(dev_reserve(ctx, ctx->io_haps, cells * 2));
    if (codes2) SI_TRY(dev_reserve(ctx, ctx->io_geno2, (size_t)B * Mb));
    if (haps && hbits) SI_TRY(dev_reserve(ctx, ctx->io_hbits, (size_t)B * 2 * Mw * 4));
    // Samples in chunks of about 64 MB of codes: chunk k's codes go in on the
    // copy-in stream, it is imputed on the ctx stream, and its outputs come
    // back on the copy-out stream while chunk k+1 is imputed. A chunk keeps the
    // global sample ids of its rows, so its draws do not depend on the split.
    // (64 MB of the codes as they cross the link: 2-bit rows make fewer, larger chunks)
    const size_t row_in = codes2 ? Mb : (size_t)M;
    const uint32_t per = (uint32_t)std::max<size_t>(1, std::min<size_t>(B, ((size_t)64 << 20) / std::max<size_t>(row_in, 1)));
    const uint32_t K = (B + per - 1) / per;
    std::vector<cudaEvent_t> ev(2 * (size_t)K + 2, nullptr);
    for (auto& x : ev) SI_CUDA(ctx, cudaEventCreateWithFlags(&x, cudaEventDefault), "event");
    auto cleanup = [&] {
        for (auto& x : ev)
            if (x) cudaEventDestroy(x);
    };
    si_status st = SI_OK;
    cudaError_t e = cudaEventRecord(ev[2 * K], s);  // start
    if (e == cudaSuccess) e = cudaStreamWaitEvent(ctx->copy_in, ev[2 * K], 0);
    for (uint32_t k = 0; k < K && e == cudaSuccess; ++k) {
        const size_t r0 = (size_t)k * per, rows = std::min<size_t>(per, B - r0);
        if (codes2)
            e = cudaMemcpyAsync((uint8_t*)ctx->io_geno2.ptr + r0 * Mb, geno + r0 * Mb, rows * Mb,
                                cudaMemcpyHostToDevice, ctx->copy_in);
        else
            e = cudaMemcpyAsync((uint8_t*)ctx->io_geno.ptr + r0 * M, geno + r0 * M, rows * M, cudaMemcpyHostToDevice,
                                ctx->copy_in);
        if (e == cudaSuccess) e = cudaEventRecord(ev[k], ctx->copy_in);
    }
    for (uint32_t k = 0; k < K && e == cudaSuccess && st == SI_OK; ++k) {
        const size_t r0 = (size_t)k * per, rows = std::min<size_t>(per, B - r0);
        e = cudaStreamWaitEvent(s, ev[k], 0);
        if (e == cudaSuccess && codes2)
            e = launch_unpack_codes((const uint8_t*)ctx->io_geno2.ptr + r0 * Mb, rows, M,
                                    (uint8_t*)ctx->io_geno.ptr + r0 * M, s);
        if (e != cudaSuccess) break;
        if (k + 1 == K) e = cudaEventRecord(ctx->ev[0], s);  // stage timings describe the last chunk
        if (e != cudaSuccess) break;
        si_impute_params pk = *p;
        pk.flags &= ~(uint32_t)(SI_IMPUTE_CODES_2BIT | SI_IMPUTE_HAPS_BITS);
        pk.sample_id_base = p->sample_id_base + r0;
        if (k) pk.flags &= ~(uint32_t)SI_IMPUTE_RESELECT;  // the first chunk rebuilt the selection
        st = run_device(ctx, &pk, (const uint8_t*)ctx->io_geno.ptr + r0 * M, (uint32_t)rows,
                        dosage ? (float*)ctx->io_dosage.ptr + r0 * M : nullptr,
                        hap_prob ? (float*)ctx->io_hprob.ptr + 2 * r0 * M : nullptr,
                        haps ? (uint8_t*)ctx->io_haps.ptr + 2 * r0 * M : nullptr, s);
        if (st != SI_OK) break;
        if (haps && hbits)
            e = launch_pack_haps((const uint8_t*)ctx->io_haps.ptr + 2 * r0 * M, 2 * rows, M,
                                 (uint32_t*)ctx->io_hbits.ptr + 2 * r0 * Mw, s);
        if (e != cudaSuccess) break;
        e = cudaEventRecord(ev[K + k], s);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(ctx->copy_out, ev[K + k], 0);
        if (e == cudaSuccess && dosage)
            e = cudaMemcpyAsync(dosage + r0 * M, (const float*)ctx->io_dosage.ptr + r0 * M, rows * M * 4,
                                cudaMemcpyDeviceToHost, ctx->copy_out);
        if (e == cudaSuccess && hap_prob)
            e = cudaMemcpyAsync(hap_prob + 2 * r0 * M, (const float*)ctx->io_hprob.ptr + 2 * r0 * M, rows * M * 8,
                                cudaMemcpyDeviceToHost, ctx->copy_out);
        if (e == cudaSuccess && haps && hbits)
            e = cudaMemcpyAsync(haps + 2 * r0 * Mw * 4, (const uint32_t*)ctx->io_hbits.ptr + 2 * r0 * Mw,
                                rows * Mw * 8, cudaMemcpyDeviceToHost, ctx->copy_out);
        else if (e == cudaSuccess && haps)
            e = cudaMemcpyAsync(haps + 2 * r0 * M, (const uint8_t*)ctx->io_haps.ptr + 2 * r0 * M, rows * M * 2,
                                cudaMemcpyDeviceToHost, ctx->copy_out);
    }
    if (e == cudaSuccess) e = cudaEventRecord(ev[2 * K + 1], ctx->copy_out);  // end
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->copy_out);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (st == SI_OK && e != cudaSuccess) st = cuda_fail(ctx, e, "imputation");
    if (st != SI_OK) {
        cudaStreamSynchronize(ctx->copy_in);  // no copy may outlive the call
        cudaStreamSynchronize(ctx->copy_out);
        cudaStreamSynchronize(s);
        cleanup();
        return st;
    }
    // timings of the last chunk's stages; [2] is the whole call, copies included
    cudaEventElapsedTime(&ctx->last_ms[0], ctx->ev[0], ctx->ev[1]);
    cudaEventElapsedTime(&ctx->last_ms[1], ctx->ev[1], ctx->ev[2]);
    cudaEventElapsedTime(&ctx->last_ms[2], ev[2 * K], ev[2 * K + 1]);
    ctx->timings_pending = false;
    cleanup();
    return SI_OK;
}

si_status si_impute_gl(si_ctx* ctx, const si_impute_params* p, const float* gl, uint32_t B, float* dosage,
                       float* hap_prob, uint8_t* haps) {
    if (!ctx) return SI_ERR_INVALID_ARG;
    if (!gl || B == 0) return fail(ctx, SI_ERR_INVALID_ARG, "gl is NULL or B == 0");
    const size_t cells = (size_t)B * ctx->M;
    std::vector<uint8_t> codes(cells);
    for (size_t i = 0; i < cells; ++i) {
        const float a = gl[3 * i], b = gl[3 * i + 1], c = gl[3 * i + 2];
        if (a == b && b == c) codes[i] = SI_GENO_MISSING;
        else if (a == 0.f && b == -999.f && c == -999.f) codes[i] = 0;
        else if (a == -999.f && b == 0.f && c == -999.f) codes[i] = 1;
        else if (a == -999.f && b == -999.f && c == 0.f) codes[i] = 2;
        else
            return fail(ctx, SI_ERR_UNSUPPORTED,
                        "genotype likelihood triple at cell " + std::to_string(i) +
                            " is not a hard call {0,-999,-999} pattern or missing");
    }
    return si_impute(ctx, p, codes.data(), B, dosage, hap_prob, haps);
}

si_status si_last_timings(si_ctx* ctx, float* ms3) {
    if (!ctx || !ms3) return SI_ERR_INVALID_ARG;
    if (ctx->timings_pending) {
        SI_CUDA(ctx, cudaEventSynchronize(ctx->ev[2]), "wait for kernels");
        cudaEventElapsedTime(&ctx->last_ms[0], ctx->ev[0], ctx->ev[1]);
        cudaEventElapsedTime(&ctx->last_ms[1], ctx->ev[1], ctx->ev[2]);
        ctx->last_ms[2] = 0.f;
        ctx->timings_pending = false;
    }
    for (int i = 0; i < 3; ++i) ms3[i] = ctx->last_ms[i];
    return SI_OK;
}

si_status si_impute_jobs_device(si_ctx* ctx, const si_impute_params* p, const si_region* regions, uint32_t n_regions,
                                const si_job* jobs, uint32_t n_jobs, const uint8_t* d_geno, float* d_dosage,
                                float* d_hap_prob, uint8_t* d_haps, void* stream) {
    Range range("si_impute_jobs_device");
    if (!ctx) return SI_ERR_INVALID_ARG;
    SI_TRY(check_jobs_args(ctx, p, regions, n_regions, jobs, n_jobs));
    if (!d_geno) return fail(ctx, SI_ERR_INVALID_ARG, "NULL genotype buffer");
    SI_TRY(set_device(ctx));
    cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
    SI_CUDA(ctx, cudaEventRecord(ctx->kev[0], s), "event");
    std::vector<TypedRegion> tr;
    std::vector<TypedSample> ts;
    uint32_t lmax = 4;
    bool all_full = true;
    SI_TRY(prepare_jobs(ctx, p, regions, n_regions, jobs, n_jobs, s, tr, ts, lmax, all_full));
    SI_TRY(dev_reserve(ctx, ctx->job_regions, tr.size() * sizeof(TypedRegion)));
    SI_TRY(dev_reserve(ctx, ctx->job_samples, ts.size() * sizeof(TypedSample)));
    SI_CUDA(ctx, cudaMemcpyAsync(ctx->job_regions.ptr, tr.data(), tr.size() * sizeof(TypedRegion),
                                 cudaMemcpyHostToDevice, s), "copy regions");
    SI_CUDA(ctx, cudaMemcpyAsync(ctx->job_samples.ptr, ts.data(), ts.size() * sizeof(TypedSample),
                                 cudaMemcpyHostToDevice, s), "copy jobs");
    SI_CUDA(ctx, cudaEventRecord(ctx->kev[1], s), "event");
    ctx->kernel_pending = true;
    TypedArgs a{};
    a.geno = d_geno;
    a.B = n_jobs;
    a.M = 0;
    a.max_len = ts.empty() ? 0u : ts.front().len;  // jobs are ordered longest first
    a.sampling = p->sampling;
    a.tie_eps = (float)p->tie_eps;
    a.seed = p->seed;
    a.sid_base = 0;
    a.regions = (const TypedRegion*)ctx->job_regions.ptr;
    a.samples = (const TypedSample*)ctx->job_samples.ptr;
    a.dosage = d_dosage;
    a.hprob = d_hap_prob;
    a.haps = d_haps;
    SI_CUDA(ctx, cudaEventRecord(ctx->ev[1], s), "event");
    SI_TRY(run_typed(ctx, p, a, lmax, all_full, s));
    SI_CUDA(ctx, cudaEventRecord(ctx->ev[2], s), "event");
    ctx->timings_pending = true;
    // host copies of tr/ts must outlive the async copies: wait before returning
    SI_CUDA(ctx, cudaStreamSynchronize(s), "uneven batch");
    return SI_OK;
}

si_status si_last_kernel_ms(si_ctx* ctx, float* ms4) {
    if (!ctx || !ms4) return SI_ERR_INVALID_ARG;
    if (ctx->kernel_pending) {
        SI_CUDA(ctx, cudaEventSynchronize(ctx->kev[4]), "wait for kernels");
        for (int i = 0; i < 4; ++i) cudaEventElapsedTime(&ctx->kernel_ms[i], ctx->kev[i], ctx->kev[i + 1]);
        ctx->kernel_pending = false;
    }
    for (int i = 0; i < 4; ++i) ms4[i] = ctx->kernel_ms[i];
    return SI_OK;
}

}  // extern "C"
