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

struct Tabs {
    const float* Q;   // q^n
    const float* S;   // (1 - q^n) / L
    const double* G;  // log G(n)
    uint32_t NT;
    float log2q;
    float invL;
    double lr;        // log rho
    double lgc;       // log(1 - rho) (rho < 1) or log(rho - 1) (rho > 1)
    int regime;       // 0: rho < 1, 1: rho > 1, 2: rho == 1
};

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

__global__ void anchor_count_kernel(const uint8_t* __restrict__ geno, uint32_t B, uint32_t M,
                                    uint32_t* __restrict__ counts) {
    const uint32_t s = blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
    const uint32_t lane = threadIdx.x & 31;
    if (s >= B) return;
    const uint8_t* row = geno + (uint64_t)s * M;
    uint32_t n = 0;
    for (uint32_t m = lane; m < M; m += 32) n += (m == 0 || row[m] < 3) ? 1u : 0u;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) n += __shfl_xor_sync(0xffffffffu, n, o);
    if (lane == 0) counts[s] = n;
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

__global__ void anchor_fill_kernel(const uint8_t* __restrict__ geno, uint32_t B, uint32_t M,
                                   const unsigned long long* __restrict__ aoff,
                                   const unsigned long long* __restrict__ woff, uint32_t* __restrict__ apos,
                                   uint8_t* __restrict__ acode, uint32_t* __restrict__ wsample) {
    const uint32_t s = blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
    const uint32_t lane = threadIdx.x & 31;
    if (s >= B) return;
    const uint8_t* row = geno + (uint64_t)s * M;
    unsigned long long o = aoff[s];
    for (uint32_t m0 = 0; m0 < M; m0 += 32) {
        const uint32_t m = m0 + lane;
        uint8_t g = 3;
        bool a = false;
        if (m < M) {
            g = row[m];
            a = (m == 0) || g < 3;
        }
        const uint32_t bal = __ballot_sync(0xffffffffu, a);
        if (a) {
            const unsigned long long at = o + __popc(bal & ((1u << lane) - 1u));
            apos[at] = m;
            acode[at] = g > 3 ? 3 : g;
        }
        o += __popc(bal);
    }
    for (unsigned long long w = woff[s] + lane; w < woff[s + 1]; w += 32) wsample[w] = s;
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

template <int LM>
__global__ void __launch_bounds__(128) anchor_chain_kernel(TypedArgs A, Tabs tb) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= A.B) return;
    const uint32_t lmask = A.L >= 32 ? 0xffffffffu : ((1u << A.L) - 1u);
    const unsigned long long base = A.aoff[s], NA = A.aoff[s + 1] - base, wb = A.woff[s];
    const uint32_t* pos = A.apos + base;
    const uint8_t* code = A.acode + base;
    const uint32_t C = A.C;
    uint32_t sh;
    // forward
    float a[LM];
    init_forward<LM>(a, emission_mask(code[0], A.masks[0], lmask, &sh));
    forward_step<LM>(tb, 0, a, lmask);  // normalise (n = 0: q^0 = 1, S = 0)
#pragma unroll
    for (int k = 0; k < LM; ++k) A.ckptF[wb * LM + k] = a[k];
    for (unsigned long long k = 1; k < NA; ++k) {
        const uint32_t p = pos[k];
        forward_step<LM>(tb, p - pos[k - 1], a, emission_mask(code[k], A.masks[p], lmask, &sh));
        if (k % C == 0)
#pragma unroll
            for (int l = 0; l < LM; ++l) A.ckptF[(wb + k / C) * LM + l] = a[l];
    }
    // backward
    float w[LM];
    const uint32_t plast = pos[NA - 1];
    double logU = chain_end_logU(tb, A.M - 1 - plast);
    {
        const uint32_t em = emission_mask(code[NA - 1], A.masks[plast], lmask, &sh);
        init_forward<LM>(w, em);
        logU -= 999.0 * (double)sh;
    }
    if ((NA - 1) % C == 0) {
#pragma unroll
        for (int l = 0; l < LM; ++l) A.ckptB[(wb + (NA - 1) / C) * LM + l] = w[l];
        A.ckptU[wb + (NA - 1) / C] = logU;
    }
    for (long long k = (long long)NA - 2; k >= 0; --k) {
        const uint32_t p = pos[k];
        const uint32_t em = emission_mask(code[k], A.masks[p], lmask, &sh);
        backward_step<LM>(tb, pos[k + 1] - p, w, logU, em, sh, lmask);
        if (k % C == 0) {
#pragma unroll
            for (int l = 0; l < LM; ++l) A.ckptB[(wb + k / C) * LM + l] = w[l];
            A.ckptU[wb + k / C] = logU;
        }
    }
}

// ---------------------------------------------------------------- posterior

template <int LM>
__global__ void __launch_bounds__(128) anchor_posterior_kernel(TypedArgs A, Tabs tb) {
    extern __shared__ __align__(16) unsigned char smem[];
    const uint32_t T = blockDim.x, t = threadIdx.x, C = A.C;
    float* bw = reinterpret_cast<float*>(smem);                                  // [C][LM][T]
    double* bu = reinterpret_cast<double*>(smem + (size_t)C * LM * T * 4);      // [C][T]
    const unsigned long long g = (unsigned long long)blockIdx.x * T + t;
    if (g >= A.total_windows) return;
    const uint32_t s = A.wsample[g];
    const unsigned long long base = A.aoff[s], NA = A.aoff[s + 1] - base, wb = A.woff[s];
    const unsigned long long w = g - wb;
    const uint32_t* pos = A.apos + base;
    const uint8_t* code = A.acode + base;
    const unsigned long long k0 = w * C, k1 = min(k0 + C, NA);
    const uint32_t lmask = A.L >= 32 ? 0xffffffffu : ((1u << A.L) - 1u);
    const uint32_t M = A.M;
    uint32_t sh;

    // backward anchors k in (k0, k1], stored at slot k - k0 - 1
    {
        float v[LM];
        double logU;
        long long kstart;
        if (k1 < NA) {
#pragma unroll
            for (int l = 0; l < LM; ++l) v[l] = A.ckptB[(wb + w + 1) * LM + l];
            logU = A.ckptU[wb + w + 1];
            kstart = (long long)k1;
        } else {
            const uint32_t plast = pos[NA - 1];
            logU = chain_end_logU(tb, M - 1 - plast);
            const uint32_t em = emission_mask(code[NA - 1], A.masks[plast], lmask, &sh);
            init_forward<LM>(v, em);
            logU -= 999.0 * (double)sh;
            kstart = (long long)NA - 1;
        }
        for (long long k = kstart;; --k) {
            if (k > (long long)k0) {
                const uint32_t slot = (uint32_t)(k - (long long)k0 - 1);
#pragma unroll
                for (int l = 0; l < LM; ++l) bw[((size_t)slot * LM + l) * T + t] = v[l];
                bu[(size_t)slot * T + t] = logU;
            }
            if (k - 1 <= (long long)k0) break;
            const uint32_t p = pos[k - 1];
            const uint32_t em = emission_mask(code[k - 1], A.masks[p], lmask, &sh);
            backward_step<LM>(tb, pos[k] - p, v, logU, em, sh, lmask);
        }
    }

    // forward sweep over the window's intervals with the fused epilogue
    float a[LM];
#pragma unroll
    for (int l = 0; l < LM; ++l) a[l] = A.ckptF[(wb + w) * LM + l];
    const float keep = 1.0f - A.tie_eps;
    for (unsigned long long k = k0; k < k1; ++k) {
        const uint32_t p0 = pos[k];
        const bool has_next = k + 1 < NA;
        const uint32_t p1 = has_next ? pos[k + 1] : M;
        const uint32_t n = p1 - p0;
        const float Sa = vsum<LM>(a);
        float wv[LM];
        float Sw = 0.f;
        double farg = 0.0;
        int mode = 2;  // 0: exact floor per cell, 1: floor negligible, 2: beta uniform
        if (has_next) {
            const uint32_t slot = (uint32_t)(k - k0);
#pragma unroll
            for (int l = 0; l < LM; ++l) wv[l] = bw[((size_t)slot * LM + l) * T + t];
            Sw = vsum<LM>(wv);
            farg = -999.0 - bu[(size_t)slot * T + t];
            if (farg + tabG(tb, n) < -104.0) mode = 1;
            else if (farg + tabG(tb, 1) > 60.0) mode = 2;
            else mode = 0;
        }
        for (uint32_t i = 0; i < n; ++i) {
            const uint32_t m = p0 + i;
            const float xf = tabQ(tb, i), yf = Sa * tabS(tb, i);
            float xb = 0.f, yb = 1.f;
            if (mode != 2) {
                const uint32_t j1 = n - i;  // j + 1
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
            const SlotMasks mk = A.masks[m];
            float pr[LM];
            float tot = 0.f, q0 = 0.f, q1 = 0.f, pmax = 0.f;
#pragma unroll
            for (int l = 0; l < LM; ++l) {
                const float al = fmaf(xf, a[l], yf);
                const float be = fmaf(xb, has_next ? wv[l] : 0.f, yb);
                pr[l] = ((lmask >> l) & 1u) ? al * be : 0.f;
                tot += pr[l];
                q0 += ((mk.a0 >> l) & 1u) ? pr[l] : 0.f;
                q1 += ((mk.a1 >> l) & 1u) ? pr[l] : 0.f;
                pmax = fmaxf(pmax, pr[l]);
            }
            uint32_t pick;
            if (A.sampling == SI_SAMPLE_ARGMAX) {
                const float thr = pmax * keep;
                pick = LM;
#pragma unroll
                for (int l = LM - 1; l >= 0; --l) pick = (pr[l] >= thr) ? (uint32_t)l : pick;
                if (pick >= LM) pick = 0;
            } else {
                const float target = cell_uniform(A.seed, A.sid_base + s, m) * tot;
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
            const float inv = 1.0f / tot;
            const uint64_t cell = (uint64_t)s * M + m;
            if (A.dosage) A.dosage[cell] = (q0 + q1) * inv;
            if (A.hprob) reinterpret_cast<float2*>(A.hprob)[cell] = make_float2(q0 * inv, q1 * inv);
            if (A.haps) {
                A.haps[(uint64_t)s * 2 * M + m] = (uint8_t)((mk.a0 >> pick) & 1u);
                A.haps[(uint64_t)s * 2 * M + M + m] = (uint8_t)((mk.a1 >> pick) & 1u);
            }
        }
        if (has_next) forward_step<LM>(tb, n, a, emission_mask(code[k + 1], A.masks[p1], lmask, &sh));
    }
}

template <int LM>
size_t post_smem(uint32_t T, uint32_t C) {
    return (size_t)C * LM * T * 4 + (size_t)C * T * 8;
}

template <int LM>
cudaError_t launch_typed_lm(const TypedArgs& a, const Tabs& tb, cudaStream_t s) {
    anchor_chain_kernel<LM><<<(a.B + 127) / 128, 128, 0, s>>>(a, tb);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (a.ev_chain_done && (e = cudaEventRecord(a.ev_chain_done, s)) != cudaSuccess) return e;
    const uint32_t T = a.threads;
    const size_t sm = post_smem<LM>(T, a.C);
    e = cudaFuncSetAttribute(anchor_posterior_kernel<LM>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    const unsigned long long grid = (a.total_windows + T - 1) / T;
    if (grid == 0) return cudaSuccess;
    if (grid > 0x7fffffffull) return cudaErrorInvalidConfiguration;
    anchor_posterior_kernel<LM><<<(uint32_t)grid, T, sm, s>>>(a, tb);
    return cudaGetLastError();
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

cudaError_t launch_anchor_lists_count(const uint8_t* geno, uint32_t B, uint32_t M, uint32_t C, uint32_t* counts,
                                      unsigned long long* aoff, unsigned long long* woff, cudaStream_t s) {
    anchor_count_kernel<<<(B + kWarpsPerBlock - 1) / kWarpsPerBlock, kWarpsPerBlock * 32, 0, s>>>(geno, B, M, counts);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    anchor_scan_kernel<<<1, 1024, 0, s>>>(counts, B, C, aoff, woff);
    return cudaGetLastError();
}

cudaError_t launch_anchor_lists_fill(const uint8_t* geno, uint32_t B, uint32_t M, const unsigned long long* aoff,
                                     const unsigned long long* woff, uint32_t* apos, uint8_t* acode, uint32_t* wsample,
                                     cudaStream_t s) {
    anchor_fill_kernel<<<(B + kWarpsPerBlock - 1) / kWarpsPerBlock, kWarpsPerBlock * 32, 0, s>>>(
        geno, B, M, aoff, woff, apos, acode, wsample);
    return cudaGetLastError();
}

cudaError_t launch_typed_fb(const TypedArgs& a, const TypedTables& t, cudaStream_t s) {
    Tabs tb;
    tb.Q = t.Q; tb.S = t.S; tb.G = t.G; tb.NT = t.NT; tb.log2q = t.log2q; tb.invL = t.invL;
    tb.lr = t.lr; tb.lgc = t.lgc; tb.regime = t.regime;
    switch (fb_lmax(a.L)) {
        case 4: return launch_typed_lm<4>(a, tb, s);
        case 8: return launch_typed_lm<8>(a, tb, s);
        case 16: return launch_typed_lm<16>(a, tb, s);
        default: return launch_typed_lm<32>(a, tb, s);
    }
}

}  // namespace si
