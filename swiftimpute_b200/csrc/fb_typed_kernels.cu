// fb_typed_kernels.cu — forward-backward over typed markers only.
//
// Same model as fb_kernels.cu (the reference's recurrences restated in linear
// space, with beta's e^-999 logsumexp floor), specialised to one transition
// for every gap (the reference reads matrix 0 for all gaps,
// forward_backward.cu:108,201,234,269). Untyped markers have emission 1 in
// every slot, and T = c 11^T + delta I, so a run of n untyped markers has a
// closed form (rho = delta + L c, q = delta / rho):
//   forward   alpha_{p+n}  ~  q^n a + sum(a) (1 - q^n) / L
//   backward  beta_{t-n}   ~  q^n w + sum(w) (1 - q^n) / L + e^-999 / U * G(n)
//             with w = E_t . beta_t at typed marker t, U its scale and
//             G(n) = sum_{k=1..n} rho^-k (the floor accumulated over the run).
// The sequential chain therefore steps over typed markers ("anchors") only,
// and every cell's posterior follows from its two bracketing anchors, so the
// per-cell work runs in parallel. Kernels:
//   anchor_count / anchor_scan / anchor_fill   per-sample anchor lists (marker 0
//                                              is always an anchor)
//   anchor_chain     one thread per sample: forward and backward over anchors,
//                    checkpoints every C anchors
//   anchor_posterior one thread per (sample, window of C anchors): rebuilds the
//                    window's anchors from the checkpoints and writes dosage,
//                    P(hap=1) and haplotypes for every cell of the window.
#include "fb_typed.hpp"
#include "philox.cuh"

namespace si {
namespace {

__device__ __forceinline__ int exp2_of(float x) { return ((__float_as_int(x) >> 23) & 0xff) - 127; }
__device__ __forceinline__ float pow2_neg(int e) { return __int_as_float((127 - e) << 23); }

__device__ __forceinline__ uint32_t emission_mask(uint32_t g, SlotMasks mk, uint32_t lmask, uint32_t* shift) {
    uint32_t mg;
    if (g == 0) mg = ~(mk.a0 | mk.a1);
    else if (g == 1) mg = mk.a0 ^ mk.a1;
    else if (g == 2) mg = mk.a0 & mk.a1;
    else { *shift = 0; return lmask; }
    mg &= lmask;
    *shift = mg ? 0u : 1u;
    return mg ? mg : lmask;
}

using Tabs = TypedTables;

// Per-sample view: a plain batch is B rows of M codes sharing reg0; an uneven
// batch reads its sample and region descriptors.
struct View {
    const uint8_t* geno;
    uint64_t out;
    uint64_t sid;
    uint32_t m0, len;
    TypedRegion r;
};

__device__ __forceinline__ View view_of(const TypedArgs& A, uint32_t s) {
    View v;
    if (A.samples) {
        const TypedSample d = A.samples[s];
        v.geno = A.geno + d.geno_off;
        v.out = d.out_off;
        v.sid = d.sample_id;
        v.m0 = d.m0;
        v.len = d.len;
        v.r = A.regions[d.region];
    } else {
        v.geno = A.geno + (uint64_t)s * A.M;
        v.out = (uint64_t)s * A.M;
        v.sid = A.sid_base + s;
        v.m0 = 0;
        v.len = A.M;
        v.r = A.reg0;
    }
    return v;
}

__device__ __forceinline__ uint32_t lmask_of(uint32_t L) { return L >= 32 ? 0xffffffffu : ((1u << L) - 1u); }

__device__ __forceinline__ float tabQ(const Tabs& t, uint32_t n) {
    return n < t.NT ? __ldg(t.Q + n) : exp2f((float)n * t.log2q);
}
__device__ __forceinline__ float tabS(const Tabs& t, uint32_t n) {
    return n < t.NT ? __ldg(t.S + n) : (1.0f - exp2f((float)n * t.log2q)) * t.invL;
}
__device__ __forceinline__ double tabG(const Tabs& t, uint32_t n) {
    if (n < t.NT) return __ldg(t.G + n);
    if (t.regime == 0) return -(double)n * t.lr + log1p(-exp((double)n * t.lr)) - t.lgc;
    if (t.regime == 1) return log(-expm1(-(double)n * t.lr)) - t.lgc;
    return log((double)n);
}

// ---------------------------------------------------------------- anchor lists

constexpr uint32_t kWarpsPerBlock = 8;

// 16 consecutive codes per lane: bit j set when code j < 3 (typed).
__device__ __forceinline__ uint32_t typed_bits16(const uint8_t* g, uint32_t base, uint32_t len, bool vec) {
    uint32_t bits = 0;
    if (vec && base + 16 <= len) {
        const uint4 w = *reinterpret_cast<const uint4*>(g + base);
        const uint32_t ww[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const uint32_t lt = __vcmpltu4(ww[q], 0x03030303u);  // 0xff in each byte below 3
#pragma unroll
            for (int b = 0; b < 4; ++b) bits |= ((lt >> (8 * b + 7)) & 1u) << (4 * q + b);
        }
    } else {
        for (uint32_t j = 0; j < 16 && base + j < len; ++j) bits |= (g[base + j] < 3 ? 1u : 0u) << j;
    }
    return bits;
}

__global__ void anchor_count_kernel(TypedArgs A) {
    const uint32_t s = blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
    const uint32_t lane = threadIdx.x & 31;
    if (s >= A.B) return;
    const View v = view_of(A, s);
    const bool vec = (reinterpret_cast<uintptr_t>(v.geno) & 15u) == 0;
    uint32_t n = 0;
    for (uint32_t base = lane * 16; base < v.len; base += 512) {
        uint32_t bits = typed_bits16(v.geno, base, v.len, vec);
        if (base == 0) bits |= 1u;  // marker 0 is always an anchor
        n += __popc(bits);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) n += __shfl_xor_sync(0xffffffffu, n, o);
    if (lane == 0) A.counts[s] = n;
}

// Exclusive scans of anchor counts and window counts (ceil(count / C)) in one
// CTA; entry B holds the totals.
__global__ void __launch_bounds__(1024) anchor_scan_kernel(const uint32_t* __restrict__ counts, uint32_t B,
                                                           uint32_t C, unsigned long long* __restrict__ aoff,
                                                           unsigned long long* __restrict__ woff) {
    __shared__ unsigned long long sa[32], sw[32];
    const uint32_t t = threadIdx.x, T = blockDim.x, lane = t & 31, warp = t >> 5;
    const uint32_t per = (B + T - 1) / T;
    const uint32_t b0 = min(B, t * per), b1 = min(B, b0 + per);
    unsigned long long la = 0, lw = 0;
    for (uint32_t b = b0; b < b1; ++b) { la += counts[b]; lw += (counts[b] + C - 1) / C; }
    unsigned long long ia = la, iw = lw;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long ya = __shfl_up_sync(0xffffffffu, ia, o), yw = __shfl_up_sync(0xffffffffu, iw, o);
        if (lane >= (uint32_t)o) { ia += ya; iw += yw; }
    }
    if (lane == 31) { sa[warp] = ia; sw[warp] = iw; }
    __syncthreads();
    if (warp == 0) {
        unsigned long long xa = lane < (T >> 5) ? sa[lane] : 0, xw = lane < (T >> 5) ? sw[lane] : 0;
        unsigned long long pa = xa, pw = xw;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long ya = __shfl_up_sync(0xffffffffu, pa, o), yw = __shfl_up_sync(0xffffffffu, pw, o);
            if (lane >= (uint32_t)o) { pa += ya; pw += yw; }
        }
        sa[lane] = pa - xa;
        sw[lane] = pw - xw;
    }
    __syncthreads();
    unsigned long long ra = sa[warp] + ia - la, rw = sw[warp] + iw - lw;
    for (uint32_t b = b0; b < b1; ++b) {
        aoff[b] = ra;
        woff[b] = rw;
        ra += counts[b];
        rw += (counts[b] + C - 1) / C;
    }
    if (t == T - 1) { aoff[B] = ra; woff[B] = rw; }
}

// Anchor lists: marker position, emission mask over the slots and the
// "no slot matches" flag (which scales every slot by e^-999, counted in
// beta's unit), in marker order; marker 0 is always an anchor.
__global__ void anchor_fill_kernel(TypedArgs A) {
    const uint32_t s = blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
    const uint32_t lane = threadIdx.x & 31;
    if (s >= A.B) return;
    const View v = view_of(A, s);
    const uint32_t lmask = lmask_of(v.r.L);
    const bool vec = (reinterpret_cast<uintptr_t>(v.geno) & 15u) == 0;
    unsigned long long o = A.aoff[s];
    for (uint32_t b0 = 0; b0 < v.len; b0 += 512) {
        const uint32_t base = b0 + lane * 16;
        uint32_t bits = base < v.len ? typed_bits16(v.geno, base, v.len, vec) : 0u;
        if (base == 0) bits |= 1u;
        const uint32_t cnt = __popc(bits);
        uint32_t incl = cnt;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= (uint32_t)d) incl += y;
        }
        unsigned long long at = o + incl - cnt;
        while (bits) {
            const uint32_t j = __ffs(bits) - 1;
            bits &= bits - 1;
            const uint32_t m = base + j;
            uint32_t sh;
            A.apos[at] = m;
            A.aem[at] = emission_mask(v.geno[m], v.r.masks[m], lmask, &sh);
            A.ashift[at] = (uint8_t)sh;
            ++at;
        }
        o += __shfl_sync(0xffffffffu, incl, 31);
    }
    for (unsigned long long w = A.woff[s] + lane; w < A.woff[s + 1]; w += 32) A.wsample[w] = s;
}

// ---------------------------------------------------------------- chain

template <int LM>
__device__ __forceinline__ float vsum(const float (&v)[LM]) {
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < LM; ++k) s += v[k];
    return s;
}

// beta anchor at the last anchor (marker p): beta_{M-1} = 1, n = M-1-p untyped
// steps give the uniform value rho^n + e^-999 sum_{i<n} rho^i.
__device__ __forceinline__ double chain_end_logU(const Tabs& tb, uint32_t n) {
    if (n == 0) return 0.0;
    const double f = -999.0 + tabG(tb, n);
    return (double)n * tb.lr + (f > 30.0 ? f + log1p(exp(-f)) : log1p(exp(f)));
}

template <int LM>
__device__ __forceinline__ void backward_step(const Tabs& tb, uint32_t n, float (&w)[LM], double& logU, uint32_t em,
                                              uint32_t sh, uint32_t lmask) {
    const float Qn = tabQ(tb, n), Sn = tabS(tb, n);
    const float sw = vsum<LM>(w);
    const double fterm = -999.0 - logU + tabG(tb, n);
    if (fterm > 0.0) {
        // the floor dominates: unit becomes U rho^n e^fterm
        const float g = expf(-(float)fmin(fterm, 100.0));
        const float base = fmaf(g * sw, Sn, 1.0f);
        const float gq = g * Qn;
#pragma unroll
        for (int k = 0; k < LM; ++k) w[k] = ((em >> k) & 1u) ? fmaf(gq, w[k], base) : 0.f;
        logU += (double)n * tb.lr + fterm;
    } else {
        const float F = fterm > -104.0 ? expf((float)fterm) : 0.f;
        const float base = fmaf(sw, Sn, F);
#pragma unroll
        for (int k = 0; k < LM; ++k) w[k] = ((em >> k) & 1u) ? fmaf(Qn, w[k], base) : 0.f;
        logU += (double)n * tb.lr;
    }
    (void)lmask;
    logU -= 999.0 * (double)sh;
    const float s = vsum<LM>(w);
    const int e = exp2_of(s);
    const float sc = pow2_neg(e);
#pragma unroll
    for (int k = 0; k < LM; ++k) w[k] *= sc;
    logU += (double)e * 0.69314718055994530942;
}

template <int LM>
__device__ __forceinline__ void forward_step(const Tabs& tb, uint32_t n, float (&a)[LM], uint32_t em) {
    const float Qn = tabQ(tb, n), Sn = tabS(tb, n);
    const float base = vsum<LM>(a) * Sn;
#pragma unroll
    for (int k = 0; k < LM; ++k) a[k] = ((em >> k) & 1u) ? fmaf(Qn, a[k], base) : 0.f;
    const int e = exp2_of(vsum<LM>(a));
    const float sc = pow2_neg(e);
#pragma unroll
    for (int k = 0; k < LM; ++k) a[k] *= sc;
}

template <int LM>
__device__ __forceinline__ void init_forward(float (&a)[LM], uint32_t em) {
#pragma unroll
    for (int k = 0; k < LM; ++k) a[k] = ((em >> k) & 1u) ? 1.f : 0.f;
}

constexpr int kPrefetch = 8;  // anchors whose list entries are loaded ahead of the chain step

// A CTA of 128 threads serves 64 samples: warps 0-1 run their forward chains
// and warps 2-3 their backward chains at the same time (the two directions
// are independent). Anchor entries are loaded one group of kPrefetch ahead.
template <int LM>
__global__ void __launch_bounds__(128) anchor_chain_kernel(TypedArgs A) {
    const uint32_t s = blockIdx.x * 64 + (threadIdx.x & 63);
    const bool forward = threadIdx.x < 64;
    if (s >= A.B) return;
    const View v = view_of(A, s);
    const Tabs& tb = v.r.tabs;
    const unsigned long long base = A.aoff[s], NA = A.aoff[s + 1] - base, wb = A.woff[s];
    const uint32_t* pos = A.apos + base;
    const uint32_t* aem = A.aem + base;
    const uint8_t* ash = A.ashift + base;
    const uint32_t C = A.C;
    if (forward) {
        float a[LM];
        init_forward<LM>(a, aem[0]);
        forward_step<LM>(tb, 0, a, 0xffffffffu);  // normalise
#pragma unroll
        for (int k = 0; k < LM; ++k) A.ckptF[wb * LM + k] = a[k];
        uint32_t prev = pos[0];
        uint32_t pp[kPrefetch], ee[kPrefetch];
#pragma unroll
        for (int j = 0; j < kPrefetch; ++j) {
            const unsigned long long k = 1 + j;
            pp[j] = k < NA ? pos[k] : 0u;
            ee[j] = k < NA ? aem[k] : 0u;
        }
        for (unsigned long long k0 = 1; k0 < NA; k0 += kPrefetch) {
            uint32_t pn[kPrefetch], en[kPrefetch];
#pragma unroll
            for (int j = 0; j < kPrefetch; ++j) {  // next group, in flight during this one
                const unsigned long long k = k0 + kPrefetch + j;
                pn[j] = k < NA ? pos[k] : 0u;
                en[j] = k < NA ? aem[k] : 0u;
            }
#pragma unroll
            for (int j = 0; j < kPrefetch; ++j) {
                const unsigned long long k = k0 + j;
                if (k < NA) {
                    forward_step<LM>(tb, pp[j] - prev, a, ee[j]);
                    prev = pp[j];
                    if (k % C == 0)
#pragma unroll
                        for (int l = 0; l < LM; ++l) A.ckptF[(wb + k / C) * LM + l] = a[l];
                }
            }
#pragma unroll
            for (int j = 0; j < kPrefetch; ++j) { pp[j] = pn[j]; ee[j] = en[j]; }
        }
    } else {
        float w[LM];
        uint32_t nextp = pos[NA - 1];
        double logU = chain_end_logU(tb, v.len - 1 - nextp);
        init_forward<LM>(w, aem[NA - 1]);
        logU -= 999.0 * (double)ash[NA - 1];
        if ((NA - 1) % C == 0) {
#pragma unroll
            for (int l = 0; l < LM; ++l) A.ckptB[(wb + (NA - 1) / C) * LM + l] = w[l];
            A.ckptU[wb + (NA - 1) / C] = logU;
        }
        uint32_t pp[kPrefetch], ee[kPrefetch], hh[kPrefetch];
#pragma unroll
        for (int j = 0; j < kPrefetch; ++j) {
            const long long k = (long long)NA - 2 - j;
            pp[j] = k >= 0 ? pos[k] : 0u;
            ee[j] = k >= 0 ? aem[k] : 0u;
            hh[j] = k >= 0 ? ash[k] : 0u;
        }
        for (long long k0 = (long long)NA - 2; k0 >= 0; k0 -= kPrefetch) {
            uint32_t pn[kPrefetch], en[kPrefetch], hn[kPrefetch];
#pragma unroll
            for (int j = 0; j < kPrefetch; ++j) {
                const long long k = k0 - kPrefetch - j;
                pn[j] = k >= 0 ? pos[k] : 0u;
                en[j] = k >= 0 ? aem[k] : 0u;
                hn[j] = k >= 0 ? ash[k] : 0u;
            }
#pragma unroll
            for (int j = 0; j < kPrefetch; ++j) {
                const long long k = k0 - j;
                if (k >= 0) {
                    backward_step<LM>(tb, nextp - pp[j], w, logU, ee[j], hh[j], 0u);
                    nextp = pp[j];
                    if (k % C == 0) {
#pragma unroll
                        for (int l = 0; l < LM; ++l) A.ckptB[(wb + k / C) * LM + l] = w[l];
                        A.ckptU[wb + k / C] = logU;
                    }
                }
            }
#pragma unroll
            for (int j = 0; j < kPrefetch; ++j) { pp[j] = pn[j]; ee[j] = en[j]; hh[j] = hn[j]; }
        }
    }
}

// ---------------------------------------------------------------- posterior

// Per-warp output staging: each thread computes 32 consecutive cells of its
// window into shared memory, then the warp writes every thread's 32 cells as
// one coalesced row segment (128 B of dosage, 2 x 32 B of alleles).
constexpr uint32_t kStageD = 33;  // floats per staged dosage row (32 + pad)
constexpr uint32_t kStageH = 36;  // bytes per staged allele row (32 + pad)

// nibble of slot bits -> four 0/1 floats (shared-memory table)
__device__ __forceinline__ float4 nib(const float4* lut, uint32_t bits, int j) { return lut[(bits >> (4 * j)) & 15u]; }

// kFull: every sample of the launch uses all LM slots (no active-slot masking).
template <int LM, bool kFull>
__global__ void __launch_bounds__(128) anchor_posterior_kernel(TypedArgs A) {
    extern __shared__ __align__(16) unsigned char smem[];
    const uint32_t T = blockDim.x, t = threadIdx.x, C = A.C, lane = t & 31, warp = t >> 5;
    float4* lut = reinterpret_cast<float4*>(smem);                                  // [16]
    float* bw = reinterpret_cast<float*>(smem + 256);                               // [C][LM][T]
    double* bu = reinterpret_cast<double*>(smem + 256 + (size_t)C * LM * T * 4);   // [C][T]
    unsigned char* stage = smem + 256 + (size_t)C * LM * T * 4 + (size_t)C * T * 8;
    float* sd = reinterpret_cast<float*>(stage) + (size_t)warp * 32 * kStageD;      // [32][kStageD] of this warp
    uint8_t* sh8 = stage + (size_t)(T / 32) * 32 * kStageD * 4 + (size_t)warp * 64 * kStageH;  // [32][2][kStageH]
    if (t < 16) lut[t] = make_float4((float)(t & 1), (float)((t >> 1) & 1), (float)((t >> 2) & 1), (float)(t >> 3));
    __syncthreads();

    const unsigned long long g = (unsigned long long)blockIdx.x * T + t;
    const bool live = g < A.total_windows;

    uint32_t s = 0, cstart = 0, ncells = 0;
    View v{};
    unsigned long long NA = 0, k0 = 0, k1 = 0;
    const uint32_t* pos = nullptr;
    const uint32_t* aem = nullptr;
    float a[LM];
#pragma unroll
    for (int l = 0; l < LM; ++l) a[l] = 0.f;
    if (live) {
        s = A.wsample[g];
        v = view_of(A, s);
        const Tabs& tb = v.r.tabs;
        const unsigned long long base = A.aoff[s], wb = A.woff[s], w = g - wb;
        NA = A.aoff[s + 1] - base;
        pos = A.apos + base;
        aem = A.aem + base;
        const uint8_t* ash = A.ashift + base;
        k0 = w * C;
        k1 = min(k0 + C, NA);
        // backward anchors k in (k0, k1], at slot k - k0 - 1
        float bv[LM];
        double logU;
        long long kstart;
        if (k1 < NA) {
#pragma unroll
            for (int l = 0; l < LM; ++l) bv[l] = A.ckptB[(wb + w + 1) * LM + l];
            logU = A.ckptU[wb + w + 1];
            kstart = (long long)k1;
        } else {
            logU = chain_end_logU(tb, v.len - 1 - pos[NA - 1]) - 999.0 * (double)ash[NA - 1];
            init_forward<LM>(bv, aem[NA - 1]);
            kstart = (long long)NA - 1;
        }
        for (long long k = kstart;; --k) {
            if (k > (long long)k0) {
                const uint32_t slot = (uint32_t)(k - (long long)k0 - 1);
#pragma unroll
                for (int l = 0; l < LM; ++l) bw[((size_t)slot * LM + l) * T + t] = bv[l];
                bu[(size_t)slot * T + t] = logU;
            }
            if (k - 1 <= (long long)k0) break;
            backward_step<LM>(tb, pos[k] - pos[k - 1], bv, logU, aem[k - 1], ash[k - 1], 0u);
        }
#pragma unroll
        for (int l = 0; l < LM; ++l) a[l] = A.ckptF[(wb + w) * LM + l];
        cstart = pos[k0];
        ncells = (k1 < NA ? pos[k1] : v.len) - cstart;
    }
    const Tabs& tb = v.r.tabs;
    const uint32_t lmask = lmask_of(v.r.L);
    float act[LM];  // 1 for the region's slots, 0 beyond L (only read when !kFull)
#pragma unroll
    for (int l = 0; l < LM; ++l) act[l] = ((lmask >> l) & 1u) ? 1.f : 0.f;

    // interval state (current anchor k, cells [p0, p1))
    unsigned long long k = k0;
    uint32_t p0 = cstart, p1 = 0, n = 0;
    float Sa = 0.f, Sw = 0.f;
    double farg = 0.0;
    int mode = 2;  // 0: exact floor per cell, 1: floor negligible, 2: beta uniform
    float wv[LM];
    auto open_interval = [&]() {
        const bool has_next = k + 1 < NA;
        p1 = has_next ? pos[k + 1] : v.len;
        n = p1 - p0;
        Sa = vsum<LM>(a);
        mode = 2;
        if (has_next) {
            const uint32_t slot = (uint32_t)(k - k0);
#pragma unroll
            for (int l = 0; l < LM; ++l) wv[l] = bw[((size_t)slot * LM + l) * T + t];
            Sw = vsum<LM>(wv);
            farg = -999.0 - bu[(size_t)slot * T + t];
            if (farg + tabG(tb, n) < -104.0) mode = 1;
            else if (farg + tabG(tb, 1) > 60.0) mode = 2;
            else mode = 0;
        } else {
#pragma unroll
            for (int l = 0; l < LM; ++l) wv[l] = 0.f;
        }
    };
    if (live) open_interval();

    const float keep = 1.0f - A.tie_eps;
    const uint32_t max_cells = __reduce_max_sync(0xffffffffu, ncells);
    for (uint32_t cb = 0; cb < max_cells; cb += 32) {
        for (uint32_t c = 0; c < 32; ++c) {
            const uint32_t idx = cb + c;
            if (idx >= ncells) break;
            const uint32_t m = cstart + idx;
            if (m == p1) {  // next anchor: forward step with its emission, open its interval
                forward_step<LM>(tb, n, a, aem[k + 1]);
                ++k;
                p0 = p1;
                open_interval();
            }
            const uint32_t i = m - p0;
            const float xf = tabQ(tb, i), yf = Sa * tabS(tb, i);
            float xb = 0.f, yb = 1.f;
            if (mode != 2) {
                const uint32_t j1 = n - i;
                const float Qj = tabQ(tb, j1), Sj = tabS(tb, j1);
                if (mode == 1) {
                    xb = Qj;
                    yb = Sw * Sj;
                } else {
                    const double ft = farg + tabG(tb, j1);
                    if (ft > 0.0) {
                        const float gg = expf(-(float)fmin(ft, 100.0));
                        xb = gg * Qj;
                        yb = fmaf(gg * Sw, Sj, 1.0f);
                    } else {
                        xb = Qj;
                        yb = fmaf(Sw, Sj, ft > -104.0 ? expf((float)ft) : 0.f);
                    }
                }
            }
            const SlotMasks mk = v.r.masks[m];
            // p_l = (xf a_l + yf)(xb w_l + yb), two slots per packed FP32x2 op
            float pr[LM];
            const float2 XF = make_float2(xf, xf), YF = make_float2(yf, yf);
            const float2 XB = make_float2(xb, xb), YB = make_float2(yb, yb);
            float2 tot2 = make_float2(0.f, 0.f), q02 = tot2, q12 = tot2;
#pragma unroll
            for (int l = 0; l < LM; l += 2) {
                const float2 al = __ffma2_rn(XF, make_float2(a[l], a[l + 1]), YF);
                const float2 be = __ffma2_rn(XB, make_float2(wv[l], wv[l + 1]), YB);
                float2 pp = __fmul2_rn(al, be);
                if (!kFull) pp = __fmul2_rn(pp, make_float2(act[l], act[l + 1]));
                pr[l] = pp.x;
                pr[l + 1] = pp.y;
                tot2 = __fadd2_rn(tot2, pp);
            }
#pragma unroll
            for (int j = 0; j < LM / 4; ++j) {
                const float4 m0 = nib(lut, mk.a0, j), m1 = nib(lut, mk.a1, j);
                const float2 p01 = make_float2(pr[4 * j], pr[4 * j + 1]), p23 = make_float2(pr[4 * j + 2], pr[4 * j + 3]);
                q02 = __ffma2_rn(p01, make_float2(m0.x, m0.y), q02);
                q02 = __ffma2_rn(p23, make_float2(m0.z, m0.w), q02);
                q12 = __ffma2_rn(p01, make_float2(m1.x, m1.y), q12);
                q12 = __ffma2_rn(p23, make_float2(m1.z, m1.w), q12);
            }
            const float tot = tot2.x + tot2.y, q0 = q02.x + q02.y, q1 = q12.x + q12.y;
            uint32_t pick;
            if (A.sampling == SI_SAMPLE_ARGMAX) {
                float pmax = pr[0];
#pragma unroll
                for (int l = 1; l < LM; ++l) pmax = fmaxf(pmax, pr[l]);
                const float thr = pmax * keep;
                pick = 0;
#pragma unroll
                for (int l = LM - 1; l >= 1; --l) pick = (pr[l] >= thr) ? (uint32_t)l : pick;
                if (pr[0] >= thr) pick = 0;
            } else {
                const float target = cell_uniform(A.seed, v.sid, v.m0 + m) * tot;
                float cum = 0.f;
                uint32_t last_nz = 0;
                pick = LM;
#pragma unroll
                for (int l = 0; l < LM; ++l) {
                    cum += pr[l];
                    if (pr[l] > 0.f) last_nz = (uint32_t)l;
                    if (pick == LM && target < cum) pick = (uint32_t)l;
                }
                if (pick == LM) pick = last_nz;
            }
            const float inv = __frcp_rn(tot);
            sd[lane * kStageD + c] = (q0 + q1) * inv;
            sh8[(lane * 2 + 0) * kStageH + c] = (uint8_t)((mk.a0 >> pick) & 1u);
            sh8[(lane * 2 + 1) * kStageH + c] = (uint8_t)((mk.a1 >> pick) & 1u);
            if (A.hprob) reinterpret_cast<float2*>(A.hprob)[v.out + m] = make_float2(q0 * inv, q1 * inv);
        }
        __syncwarp();
        // flush: row r = the 32 cells thread r just staged
        const int mine = (int)min(32u, ncells > cb ? ncells - cb : 0u);
        for (int r = 0; r < 32; ++r) {
            const int cnt = __shfl_sync(0xffffffffu, mine, r);
            if (cnt <= 0) continue;
            const unsigned long long out = __shfl_sync(0xffffffffu, (unsigned long long)v.out, r);
            const uint32_t len = __shfl_sync(0xffffffffu, v.len, r);
            const uint32_t m0 = __shfl_sync(0xffffffffu, cstart + cb, r);
            if ((int)lane < cnt) {
                if (A.dosage) A.dosage[out + m0 + lane] = sd[r * kStageD + lane];
                if (A.haps) {
                    A.haps[2 * out + m0 + lane] = sh8[(r * 2 + 0) * kStageH + lane];
                    A.haps[2 * out + len + m0 + lane] = sh8[(r * 2 + 1) * kStageH + lane];
                }
            }
        }
        __syncwarp();
    }
}

template <int LM>
size_t post_smem(uint32_t T, uint32_t C) {
    return 256 + (size_t)C * LM * T * 4 + (size_t)C * T * 8 + (size_t)(T / 32) * 32 * kStageD * 4 +
           (size_t)(T / 32) * 64 * kStageH;
}

template <int LM, bool kFull>
cudaError_t launch_post(const TypedArgs& a, cudaStream_t s) {
    const uint32_t T = a.threads;
    const size_t sm = post_smem<LM>(T, a.C);
    cudaError_t e = cudaFuncSetAttribute(anchor_posterior_kernel<LM, kFull>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    const unsigned long long grid = (a.total_windows + T - 1) / T;
    if (grid == 0) return cudaSuccess;
    if (grid > 0x7fffffffull) return cudaErrorInvalidConfiguration;
    anchor_posterior_kernel<LM, kFull><<<(uint32_t)grid, T, sm, s>>>(a);
    return cudaGetLastError();
}

template <int LM>
cudaError_t launch_typed_lm(const TypedArgs& a, bool full, cudaStream_t s) {
    anchor_chain_kernel<LM><<<(a.B + 63) / 64, 128, 0, s>>>(a);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (a.ev_chain_done && (e = cudaEventRecord(a.ev_chain_done, s)) != cudaSuccess) return e;
    return full ? launch_post<LM, true>(a, s) : launch_post<LM, false>(a, s);
}

}  // namespace

size_t typed_post_smem_bytes(uint32_t L, uint32_t T, uint32_t C) {
    switch (fb_lmax(L)) {
        case 4: return post_smem<4>(T, C);
        case 8: return post_smem<8>(T, C);
        case 16: return post_smem<16>(T, C);
        default: return post_smem<32>(T, C);
    }
}

cudaError_t launch_anchor_lists_count(const TypedArgs& a, cudaStream_t s) {
    anchor_count_kernel<<<(a.B + kWarpsPerBlock - 1) / kWarpsPerBlock, kWarpsPerBlock * 32, 0, s>>>(a);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    anchor_scan_kernel<<<1, 1024, 0, s>>>(a.counts, a.B, a.C, a.aoff, a.woff);
    return cudaGetLastError();
}

cudaError_t launch_anchor_lists_fill(const TypedArgs& a, cudaStream_t s) {
    anchor_fill_kernel<<<(a.B + kWarpsPerBlock - 1) / kWarpsPerBlock, kWarpsPerBlock * 32, 0, s>>>(a);
    return cudaGetLastError();
}

// lmax: slots held per thread (every region's L <= lmax); the fast variant
// runs when every region uses exactly lmax slots.
cudaError_t launch_typed_fb(const TypedArgs& a, uint32_t lmax, bool all_full, cudaStream_t s) {
    switch (lmax) {
        case 4: return launch_typed_lm<4>(a, all_full, s);
        case 8: return launch_typed_lm<8>(a, all_full, s);
        case 16: return launch_typed_lm<16>(a, all_full, s);
        default: return launch_typed_lm<32>(a, all_full, s);
    }
}

}  // namespace si
