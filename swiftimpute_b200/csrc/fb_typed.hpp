// fb_typed.hpp — launch interface of the typed-marker forward-backward.
#pragma once
#include "si_internal.hpp"
#include "slots.cuh"

namespace si {

// Closed-form coefficients for runs of untyped markers under one transition
// (c, delta), computed in FP64 on the host: q = delta / rho, rho = delta + L c,
// QS[n] = {Q[n], S[n]} = {q^n, (1 - q^n) / L}, G[n] = log sum_{k=1..n} rho^-k;
// for two consecutive cells QSup[n] = {Q[n], Q[n+1], S[n], S[n+1]} and
// QSdn[n] = {Q[n], Q[n-1], S[n], S[n-1]}; Gdn[n] = {hi G[n], hi G[n-1],
// lo G[n], lo G[n-1]}, G as a float pair hi + lo (G[0] = -inf stands as -1e30).
struct TypedTables {
    const float2* QS;
    const float4* QSup;
    const float4* QSdn;
    const float4* Gdn;
    const double* G;
    uint32_t NT;
    float log2q;
    float invL;
    double lr;
    double lgc;
    int regime;  // 0: rho < 1, 1: rho > 1, 2: rho == 1
};

// A panel slice imputed with L slots: its slot masks, per-slot ALT counts at
// m and m + 1 g2 [marker][gs] and allele bytes raw [marker][gs][2] (null for a
// 0/1 panel; index 0 = the slice's first marker), and the closed-form tables
// of its transition.
struct TypedRegion {
    const SlotMasks* masks;
    const float2* g2;
    const uint8_t* raw;
    uint32_t gs;
    uint32_t L;
    TypedTables tabs;
};

// One target of an uneven batch.
struct TypedSample {
    uint64_t geno_off;   // codes at geno + geno_off, len bytes
    uint64_t out_off;    // outputs packed at out_off (dosage), 2 out_off (haps)
    uint64_t sample_id;  // Philox counter
    uint32_t m0;         // absolute panel marker of the slice's first marker
    uint32_t len;
    uint32_t region;
    uint32_t pad;
};

struct TypedArgs {
    const uint8_t* geno;
    uint32_t B;                      // samples
    uint32_t M;                      // markers per sample of a plain batch
    uint32_t C, threads;             // anchors per window (backward checkpoints), posterior CTA size
    uint32_t K;                      // windows per posterior group (forward checkpoints every K windows)
    uint32_t max_windows;            // most windows of any sample (posterior grid)
    int sampling;
    float tie_eps;
    uint64_t seed, sid_base;
    TypedRegion reg0;                // the region of a plain batch
    const TypedRegion* regions;      // device array, uneven batches (else null)
    const TypedSample* samples;      // device array, uneven batches (else null)
    // Anchor lists and window checkpoints are interleaved over groups of 32
    // consecutive samples (a warp's lanes): entry k of sample s sits at
    // aoff[s / 32] + 32 k + s % 32, window w at woff[s / 32] + 32 w + s % 32,
    // so the lanes of a warp reading the same anchor share cache lines.
    unsigned long long* aoff;        // [G+1] list offsets of the groups (32 x the group's most anchors, or capacities)
    unsigned long long* woff;        // [G+1] window offsets of the groups (likewise)
    uint32_t* counts;                // [B] anchors of each job (written by the count kernel)
    uint32_t* segc;                  // [B][nseg] anchors in each segment of kFillSeg markers (count kernel)
    uint32_t nseg;                   // segments of the longest job: ceil(max_len / kFillSeg)
    uint32_t max_len;                // markers of the longest job (M for a plain batch)
    const uint32_t* cap;             // [B] anchor capacity of each job (a plan), else null: every anchor is listed
    uint32_t* err;                   // device flag: bit 0 set when a job had more anchors than its capacity
    unsigned long long* host_totals; // mapped host memory: anchors, windows, most windows of a sample (may be null)
    uint32_t* apos;                  // anchor position within the slice | 1 << 31 where no slot matches the call
                                     // (every slot scaled by e^-999)
    uint32_t* aem;                   // anchor emission masks over the slots
    unsigned long long total_windows;
    float* ckptF;                    // [windows][Lmax] forward anchor at the first anchor of every K-th window
    float* ckptB;                    // [windows][Lmax] backward anchor (E . beta, scaled)
    double* ckptU;                   // [windows] log of the backward anchor's unit
    float* dosage;
    float* hprob;
    uint8_t* haps;
    cudaEvent_t ev_chain_done;       // recorded between the chain and the posterior kernel (may be null)
};

cudaError_t launch_anchor_lists_count(const TypedArgs& a, cudaStream_t s);  // count + offset scan
cudaError_t launch_anchor_count_only(const TypedArgs& a, cudaStream_t s);   // count (capacity offsets)
cudaError_t launch_anchor_lists_fill(const TypedArgs& a, cudaStream_t s);
cudaError_t launch_typed_fb(const TypedArgs& a, uint32_t lmax, bool all_full, cudaStream_t s);
size_t typed_post_smem_bytes(uint32_t L, uint32_t T, uint32_t C);
inline uint32_t typed_groups(uint32_t B) { return (B + 31) / 32; }  // 32-sample groups of the interleaved lists
constexpr uint32_t kShiftBit = 0x80000000u;                         // apos: no slot matches the call
constexpr uint32_t kFillSeg = 4096;                                 // markers per warp of the list fill (x 512)
inline uint32_t typed_nseg(uint32_t max_len) { return (max_len + kFillSeg - 1) / kFillSeg; }
// Uneven batches (capi.cu): argument checks, and the region tables and job
// descriptors of a batch (region sweeps and selections not cached yet run on s).
si_status check_jobs_args(si_ctx* ctx, const si_impute_params* p, const si_region* regions, uint32_t n_regions,
                          const si_job* jobs, uint32_t n_jobs);
si_status prepare_jobs(si_ctx* ctx, const si_impute_params* p, const si_region* regions, uint32_t n_regions,
                       const si_job* jobs, uint32_t n_jobs, cudaStream_t s, std::vector<TypedRegion>& tr,
                       std::vector<TypedSample>& ts, uint32_t& lmax, bool& all_full);

uint32_t typed_default_window(uint32_t lmax);   // anchors per window when the caller gives none
constexpr uint32_t kPostGroup = 16;             // windows per posterior group (fixed: rounding restarts there)
uint32_t typed_default_threads(uint32_t lmax);  // posterior CTA size when the caller gives none

}  // namespace si
