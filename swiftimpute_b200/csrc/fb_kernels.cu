// fb_kernels.cu — fused emission / forward-backward / posterior epilogue.
//
// Model (the reference's recurrences, restated in linear space):
//   emission   E_m[k] = exp(GL[a(h0_k) + a(h1_k)])         emission.cu:35-54
//              GL is {0, -999, -999}-style (imputer.cpp:244-295): slots whose
//              pair sum equals the call get 1, the others e^-999 (= 0 here);
//              a call no slot matches scales every slot by e^-999 alike.
//   transition T = c + delta * I, c = exp(log10 switch),   transition.cu:98-115
//              c + delta = exp(log10 stay) (log10 values fed to natural-log
//              recursions, logsumexp.cuh:67-70).
//   forward    alpha_m = E_m . (T^T alpha_{m-1})             forward_backward.cu:92-131
//   backward   beta_m  = e^-999 + T (E_{m+1} . beta_{m+1})   forward_backward.cu:221-241
//              The e^-999 term is the LOG_ZERO seed of every logsumexp2
//              chain; beta is never rescaled in the reference, so the term
//              matters once beta decays near e^-999. beta's absolute scale is
//              therefore tracked exactly as 2^Kb * e^(-999 nb); when the floor
//              dominates the unit switches to e^-999 itself.
//   posterior  P_m(k) = softmax(log alpha + log beta)       sampling.cu:80-100
// FP32 values, exact power-of-two rescaling every marker (no rounding from
// the rescale), the floor term computed from the integer scale in FP64.
//
// One thread carries one target chain with all L slots in registers (the
// transition is rank-1 plus diagonal, so a step is O(L), not O(L^2)). The
// forward pass stores alpha at the end of every C-marker segment (HBM); the
// backward pass recomputes a segment's alpha into shared memory, then walks
// beta back through it and writes dosage, P(hap=1) and haplotypes. Inputs and
// outputs of a segment are staged in shared memory so global traffic is
// coalesced row segments.
#include "philox.cuh"
#include "si_internal.hpp"
#include "slots.cuh"

namespace si {
namespace {

struct FbArgs {
    const uint8_t* geno;
    const SlotMasks* masks;
    const SlotMasks* smasks;  // per-target [M][B] (target-aware selection), else null
    const uint8_t* raw;
    const LinTrans* trans;
    uint32_t B, M, L, C, nseg;
    int sampling;
    float tie_eps;
    uint64_t seed, sid_base;
    float* ckpt;
    float* dosage;
    float* hprob;
    uint8_t* haps;
};

__device__ __forceinline__ int exp2_of(float x) {  // floor(log2 x) for positive normal x
    return ((__float_as_int(x) >> 23) & 0xff) - 127;
}
__device__ __forceinline__ float pow2_neg(int e) {  // 2^-e, |e| <= 126
    return __int_as_float((127 - e) << 23);
}

template <int LM>
__device__ __forceinline__ void forward_step(float (&al)[LM], float& S, uint32_t em, LinTrans tr, bool first) {
    if (first) {
#pragma unroll
        for (int k = 0; k < LM; ++k) al[k] = ((em >> k) & 1u) ? 1.0f : 0.0f;
    } else {
        const float sc = pow2_neg(exp2_of(S));
        const float cS = tr.c * (S * sc);
        const float dl = tr.delta * sc;
#pragma unroll
        for (int k = 0; k < LM; ++k) al[k] = ((em >> k) & 1u) ? fmaf(dl, al[k], cS) : 0.0f;
    }
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < LM; ++k) s += al[k];
    S = s;
}

template <int LM>
__global__ void __launch_bounds__(128) fb_chain_kernel(FbArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    const uint32_t T = blockDim.x, C = a.C;
    const uint32_t GS = C + 4;          // code row stride (bytes)
    const uint32_t DS = C + 1;          // dosage row stride (floats)
    const uint32_t HS = 2 * C + 1;      // hprob row stride (floats)
    const uint32_t PS = C + 4;          // hap row stride (bytes, per phase)
    float* abuf = reinterpret_cast<float*>(smem);                       // [C][LM][T]
    float* dbuf = abuf + (size_t)C * LM * T;                            // [T][DS]
    float* hbuf = dbuf + (size_t)T * DS;                                // [T][HS]
    SlotMasks* mseg = reinterpret_cast<SlotMasks*>(hbuf + (size_t)T * HS);  // [C]
    LinTrans* tseg = reinterpret_cast<LinTrans*>(mseg + C);             // [C]
    uint8_t* gbuf = reinterpret_cast<uint8_t*>(tseg + C);               // [T][GS]
    uint8_t* pbuf = gbuf + (size_t)T * GS;                              // [T][2][PS]

    const uint32_t t = threadIdx.x, lane = t & 31, warp = t >> 5, nwarps = T >> 5;
    const uint32_t s0 = blockIdx.x * T;
    const uint32_t s = s0 + t;
    const bool live = s < a.B;
    const uint32_t M = a.M, L = a.L;
    const uint32_t lmask = (L >= 32) ? 0xffffffffu : ((1u << L) - 1u);

    // stage codes, masks and transitions of markers [m0, m0 + cl)
    auto stage = [&](uint32_t m0, uint32_t cl) {
        for (uint32_t r = warp; r < T; r += nwarps) {
            const uint32_t sr = s0 + r;
            if (sr < a.B && lane < cl) gbuf[r * GS + lane] = a.geno[(uint64_t)sr * M + m0 + lane];
        }
        for (uint32_t i = t; i < cl; i += T) {
            if (!a.smasks) mseg[i] = a.masks[m0 + i];
            tseg[i] = a.trans[m0 + i];
        }
    };
    // the slot masks of marker m (staged at i): per marker, or this target's own
    auto mask_at = [&](uint32_t i, uint32_t m) {
        if (!a.smasks) return mseg[i];
        return live ? a.smasks[(uint64_t)m * a.B + s] : SlotMasks{0u, 0u, 0u, 0u};
    };

    float al[LM];
    float S = 0.f;

    // ---------------- forward: checkpoints at segment ends ----------------
    for (uint32_t j = 0; j < a.nseg; ++j) {
        const uint32_t m0 = j * C, cl = min(C, M - m0);
        __syncthreads();
        stage(m0, cl);
        __syncthreads();
        for (uint32_t i = 0; i < cl; ++i) {
            uint32_t sh;
            const uint32_t em = emission_mask(gbuf[t * GS + i], mask_at(i, m0 + i), lmask, &sh);
            forward_step<LM>(al, S, em, tseg[i], m0 + i == 0);
        }
        if (live && j + 1 < a.nseg) {
#pragma unroll
            for (int k = 0; k < LM; ++k) a.ckpt[((uint64_t)j * LM + k) * a.B + s] = al[k];
        }
    }

    // ---------------- backward with fused posterior epilogue ----------------
    float be[LM];
    int Kb = 0, nb = 0;                  // |beta| = 2^Kb * e^(-999 nb) * be
    uint32_t em_next = 0, sh_next = 0;   // emission of marker m + 1
    LinTrans tr_next = {0.f, 0.f};       // transition into marker m + 1
    const float keep = 1.0f - a.tie_eps;

    for (int jj = (int)a.nseg - 1; jj >= 0; --jj) {
        const uint32_t j = (uint32_t)jj;
        const uint32_t m0 = j * C, cl = min(C, M - m0);
        __syncthreads();
        stage(m0, cl);
        __syncthreads();
        // recompute alpha over the segment
        if (j > 0) {
            S = 0.f;
#pragma unroll
            for (int k = 0; k < LM; ++k) {
                al[k] = live ? a.ckpt[((uint64_t)(j - 1) * LM + k) * a.B + s] : 0.f;
                S += al[k];
            }
            if (!live) S = 1.f;
        }
        for (uint32_t i = 0; i < cl; ++i) {
            uint32_t sh;
            const uint32_t em = emission_mask(gbuf[t * GS + i], mask_at(i, m0 + i), lmask, &sh);
            forward_step<LM>(al, S, em, tseg[i], m0 + i == 0);
#pragma unroll
            for (int k = 0; k < LM; ++k) abuf[((size_t)i * LM + k) * T + t] = al[k];
        }
        // beta walk and epilogue
        for (int ii = (int)cl - 1; ii >= 0; --ii) {
            const uint32_t i = (uint32_t)ii, m = m0 + i;
            if (m == M - 1) {
#pragma unroll
                for (int k = 0; k < LM; ++k) be[k] = ((lmask >> k) & 1u) ? 1.0f : 0.0f;
                Kb = 0; nb = 0;
            } else {
                float w[LM];
                float sw = 0.f;
#pragma unroll
                for (int k = 0; k < LM; ++k) { w[k] = ((em_next >> k) & 1u) ? be[k] : 0.0f; sw += w[k]; }
                // beta_m = e^-999 + U * (c sw + delta w), U = 2^Kb e^(-999 (nb + sh)): the
                // floor in units of U is exp(farg)
                const double farg = 999.0 * (double)(nb + (int)sh_next - 1) - (double)Kb * 0.69314718055994530942;
                if (farg > 0.0) {
                    // the floor dominates: switch the unit to e^-999 (Kb = 0, nb = 1),
                    // beta_m = e^-999 (1 + exp(-farg) (c sw + delta w))
                    const float g = expf(-(float)fmin(farg, 100.0));
                    const float cs = tr_next.c * sw;
#pragma unroll
                    for (int k = 0; k < LM; ++k)
                        be[k] = ((lmask >> k) & 1u) ? fmaf(g, fmaf(tr_next.delta, w[k], cs), 1.0f) : 0.0f;
                    Kb = 0;
                    nb = 1;
                } else {
                    const float F = farg > -104.0 ? expf((float)farg) : 0.0f;
                    const float base = fmaf(tr_next.c, sw, F);  // common part of every slot, >= c
                    const int e = exp2_of(base);
                    const float sc = pow2_neg(e);
                    const float b2 = base * sc;
                    const float dl = tr_next.delta * sc;
#pragma unroll
                    for (int k = 0; k < LM; ++k) be[k] = ((lmask >> k) & 1u) ? fmaf(dl, w[k], b2) : 0.0f;
                    Kb += e;
                    nb += (int)sh_next;
                }
            }
            // posterior at m
            const SlotMasks mk = mask_at(i, m);
            float p[LM];
            float tot = 0.f, q0 = 0.f, q1 = 0.f, pmax = 0.f;
#pragma unroll
            for (int k = 0; k < LM; ++k) {
                p[k] = abuf[((size_t)i * LM + k) * T + t] * be[k];
                tot += p[k];
                q0 += ((mk.a0 >> k) & 1u) ? p[k] : 0.f;
                q1 += ((mk.a1 >> k) & 1u) ? p[k] : 0.f;
                pmax = fmaxf(pmax, p[k]);
            }
            uint32_t pick = 0;
            if (a.sampling == SI_SAMPLE_ARGMAX) {
                const float thr = pmax * keep;
                pick = LM;
#pragma unroll
                for (int k = LM - 1; k >= 0; --k) pick = (p[k] >= thr) ? (uint32_t)k : pick;
                if (pick >= LM) pick = 0;
            } else {
                const float target = cell_uniform(a.seed, a.sid_base + s, m) * tot;
                float cum = 0.f;
                uint32_t last_nz = 0;
                pick = LM;
#pragma unroll
                for (int k = 0; k < LM; ++k) {
                    cum += p[k];
                    if (p[k] > 0.f) last_nz = (uint32_t)k;
                    if (pick == LM && target < cum) pick = (uint32_t)k;
                }
                if (pick == LM) pick = last_nz;
            }
            const float inv = 1.0f / tot;
            dbuf[t * DS + i] = (q0 + q1) * inv;
            hbuf[t * HS + 2 * i] = q0 * inv;
            hbuf[t * HS + 2 * i + 1] = q1 * inv;
            const uint32_t hv = slot_alleles(mk, a.raw, fb_lmax(L), m, pick);
            pbuf[(t * 2 + 0) * PS + i] = (uint8_t)(hv & 0xffu);
            pbuf[(t * 2 + 1) * PS + i] = (uint8_t)(hv >> 8);
            // this marker's emission/transition drive beta_{m-1}
            uint32_t sh;
            em_next = emission_mask(gbuf[t * GS + i], mk, lmask, &sh);
            sh_next = sh;
            tr_next = tseg[i];
        }
        __syncthreads();
        // flush the segment's outputs as coalesced row segments
        for (uint32_t r = warp; r < T; r += nwarps) {
            const uint32_t sr = s0 + r;
            if (sr >= a.B) continue;
            const uint64_t row = (uint64_t)sr * M + m0;
            if (lane < cl) {
                if (a.dosage) a.dosage[row + lane] = dbuf[r * DS + lane];
                if (a.haps) {
                    a.haps[(uint64_t)sr * 2 * M + m0 + lane] = pbuf[(r * 2 + 0) * PS + lane];
                    a.haps[(uint64_t)sr * 2 * M + M + m0 + lane] = pbuf[(r * 2 + 1) * PS + lane];
                }
            }
            if (a.hprob)
                for (uint32_t l = lane; l < 2 * cl; l += 32) a.hprob[row * 2 + l] = hbuf[r * HS + l];
        }
    }
}

template <int LM>
size_t smem_bytes(uint32_t T, uint32_t C) {
    return (size_t)C * LM * T * 4 + (size_t)T * (C + 1) * 4 + (size_t)T * (2 * C + 1) * 4 +
           (size_t)C * (sizeof(SlotMasks) + sizeof(LinTrans)) +
           (size_t)T * (C + 4) + (size_t)T * 2 * (C + 4) + 16;
}

template <int LM>
cudaError_t launch_lm(const FbArgs& fa, uint32_t T, cudaStream_t s) {
    const size_t sm = smem_bytes<LM>(T, fa.C);
    if (sm > 227u * 1024u) return cudaErrorInvalidValue;
    cudaError_t e = cudaFuncSetAttribute(fb_chain_kernel<LM>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    const uint32_t grid = (fa.B + T - 1) / T;
    fb_chain_kernel<LM><<<grid, T, sm, s>>>(fa);
    return cudaGetLastError();
}

}  // namespace


size_t fb_smem_bytes(uint32_t L, uint32_t T, uint32_t C) {
    switch (fb_lmax(L)) {
        case 4: return smem_bytes<4>(T, C);
        case 8: return smem_bytes<8>(T, C);
        case 16: return smem_bytes<16>(T, C);
        default: return smem_bytes<32>(T, C);
    }
}

size_t fb_ckpt_bytes(uint32_t B, uint32_t M, uint32_t L, uint32_t C) {
    const uint32_t nseg = (M + C - 1) / C;
    return (size_t)(nseg > 1 ? nseg - 1 : 1) * fb_lmax(L) * B * sizeof(float);
}

cudaError_t launch_fb(const FbLaunch& l, cudaStream_t s) {
    FbArgs fa;
    fa.geno = l.geno; fa.masks = l.masks; fa.smasks = l.smasks; fa.raw = l.raw; fa.trans = l.trans;
    fa.B = l.B; fa.M = l.M; fa.L = l.L; fa.C = l.C; fa.nseg = (l.M + l.C - 1) / l.C;
    fa.sampling = l.sampling; fa.tie_eps = l.tie_eps; fa.seed = l.seed; fa.sid_base = l.sample_id_base;
    fa.ckpt = l.ckpt; fa.dosage = l.dosage; fa.hprob = l.hprob; fa.haps = l.haps;
    if (l.C == 0 || l.C > 32 || l.threads == 0 || l.threads % 32 || l.threads > 128) return cudaErrorInvalidValue;
    switch (fb_lmax(l.L)) {
        case 4: return launch_lm<4>(fa, l.threads, s);
        case 8: return launch_lm<8>(fa, l.threads, s);
        case 16: return launch_lm<16>(fa, l.threads, s);
        default: return launch_lm<32>(fa, l.threads, s);
    }
}

}  // namespace si
