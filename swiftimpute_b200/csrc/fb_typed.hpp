// fb_typed.hpp — launch interface of the typed-marker forward-backward.
#pragma once
#include "si_internal.hpp"

namespace si {

// Closed-form coefficients for runs of untyped markers under one transition
// (c, delta), computed in FP64 on the host: q = delta / rho, rho = delta + L c,
// Q[n] = q^n, S[n] = (1 - q^n) / L, G[n] = log sum_{k=1..n} rho^-k.
struct TypedTables {
    const float* Q;
    const float* S;
    const double* G;
    uint32_t NT;
    float log2q;
    float invL;
    double lr;
    double lgc;
    int regime;  // 0: rho < 1, 1: rho > 1, 2: rho == 1
};

struct TypedArgs {
    const SlotMasks* masks;
    uint32_t B, M, L, C, threads;
    int sampling;
    float tie_eps;
    uint64_t seed, sid_base;
    const unsigned long long* aoff;  // [B+1] anchor offsets
    const unsigned long long* woff;  // [B+1] window offsets
    const uint32_t* apos;            // anchor marker positions
    const uint8_t* acode;            // anchor genotype codes
    const uint32_t* wsample;         // window -> sample
    unsigned long long total_windows;
    float* ckptF;                    // [windows][Lmax] forward anchor at each window's first anchor
    float* ckptB;                    // [windows][Lmax] backward anchor (E . beta, scaled)
    double* ckptU;                   // [windows] log of the backward anchor's unit
    float* dosage;
    float* hprob;
    uint8_t* haps;
    cudaEvent_t ev_chain_done;       // recorded between the chain and the posterior kernel (may be null)
};

cudaError_t launch_anchor_lists_count(const uint8_t* geno, uint32_t B, uint32_t M, uint32_t C, uint32_t* counts,
                                      unsigned long long* aoff, unsigned long long* woff, cudaStream_t s);
cudaError_t launch_anchor_lists_fill(const uint8_t* geno, uint32_t B, uint32_t M, const unsigned long long* aoff,
                                     const unsigned long long* woff, uint32_t* apos, uint8_t* acode, uint32_t* wsample,
                                     cudaStream_t s);
cudaError_t launch_typed_fb(const TypedArgs& a, const TypedTables& t, cudaStream_t s);
size_t typed_post_smem_bytes(uint32_t L, uint32_t T, uint32_t C);

}  // namespace si
