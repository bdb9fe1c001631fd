// select_kernels.cu — per-marker L-state selection with fused pair expansion.
//
// Every divergence entry of the reference index at marker m equals m
// (pbwt_index.cpp:173-191), so the reference selectors' top-L by divergence
// reduces to fixed positions of the marker's prefix row, identical for every
// target sample:
//   warp kernel (pbwt_selector.cu:212-312, used for L <= 32 and N <= 10000):
//     slot r = prefix[m][32 r] for r < min(4, ceil(N / 32)), else r % N;
//   insertion kernels (pbwt_selector.cu:320-394 and, in its defined case,
//     :47-204): slot r = prefix[m][r] for r < min(N, L), else r % N.
// Each slot h becomes the pair (h, (h + 1) % N) (imputer.cpp:863-874). The
// reference computes this per (sample, marker) by scanning whole N-long rows
// (B * M * N * 8 bytes); here it is one thread per marker reading at most L
// entries of the head rows the sweep kept.
#include "si_internal.hpp"

namespace si {
namespace {

// Allele byte of haplotype h in a panel row: 0 for a clear bit; for a set bit
// the row's exception entry (sorted by haplotype) if there is one, else 1.
__device__ __forceinline__ uint32_t allele_of(const uint32_t* prow, uint32_t h, const uint32_t* ex, uint32_t nex) {
    if (!((prow[h >> 5] >> (h & 31)) & 1u)) return 0u;
    uint32_t lo = 0, hi = nex;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if ((ex[mid] >> 8) < h) lo = mid + 1;
        else hi = mid;
    }
    return (lo < nex && (ex[lo] >> 8) == h) ? (ex[lo] & 0xffu) : 1u;
}

// The slot haplotype of slot k at marker m (before the pair expansion).
__device__ __forceinline__ uint32_t slot_hap(const uint32_t* hrow, uint32_t N, uint32_t L, int kind, uint32_t k) {
    const uint32_t lane0 = min(4u, (N + 31) / 32);
    const uint32_t top = min(N, L);
    if (kind == SI_SEL_WARP) return (k < lane0) ? hrow[32 * k] : (k % N);
    if (kind == SI_SEL_FIRST_PAIRS) return 2 * k;  // imputer.cpp:938-939, host checks N >= 2L
    return (k < top) ? hrow[k] : (k % N);
}

// Outputs (each may be null): pairs [M][L][2]; masks [M]; g2 [M][gs] float2,
// for each slot the number of non-zero alleles of its pair at m and at m + 1
// (0 past L and past the last marker), which the posterior pass weighs by slot
// to form the dosage of two consecutive cells; raw [M][gs][2], the pair's
// allele bytes (panels with alleles other than 0/1).
__global__ void select_kernel(const uint32_t* __restrict__ head, const uint32_t* __restrict__ panel, uint32_t M,
                              uint32_t N, uint32_t W, uint32_t L, int kind,
                              const unsigned long long* __restrict__ ex_off, const uint32_t* __restrict__ ex_ent,
                              uint32_t* __restrict__ pairs, SlotMasks* __restrict__ masks, float2* __restrict__ g2,
                              uint8_t* __restrict__ raw, uint32_t gs) {
    const uint32_t m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= M) return;
    auto alleles = [&](uint32_t mm, uint32_t k, uint32_t* v0, uint32_t* v1, uint32_t* h0, uint32_t* h1) {
        const uint32_t* hrow = head ? head + (uint64_t)mm * kHead : nullptr;
        const uint32_t* prow = panel + (uint64_t)mm * W;
        const uint32_t* ex = ex_ent ? ex_ent + ex_off[mm] : nullptr;
        const uint32_t nex = ex_ent ? (uint32_t)(ex_off[mm + 1] - ex_off[mm]) : 0u;
        *h0 = slot_hap(hrow, N, L, kind, k);
        *h1 = (*h0 + 1) % N;
        *v0 = allele_of(prow, *h0, ex, nex);
        *v1 = allele_of(prow, *h1, ex, nex);
    };
    uint32_t a0 = 0, a1 = 0, x = 0;
    for (uint32_t k = 0; k < L; ++k) {
        uint32_t v0, v1, h, h1;
        alleles(m, k, &v0, &v1, &h, &h1);
        if (pairs) {
            pairs[((uint64_t)m * L + k) * 2 + 0] = h;
            pairs[((uint64_t)m * L + k) * 2 + 1] = h1;
        }
        if (k < 32) {
            a0 |= (v0 != 0u ? 1u : 0u) << k;
            a1 |= (v1 != 0u ? 1u : 0u) << k;
            x |= (v0 > 1u || v1 > 1u ? 1u : 0u) << k;
        }
        if (k < gs) {
            if (raw) {
                raw[((uint64_t)m * gs + k) * 2 + 0] = (uint8_t)v0;
                raw[((uint64_t)m * gs + k) * 2 + 1] = (uint8_t)v1;
            }
            if (g2) {
                float next = 0.f;
                if (m + 1 < M) {
                    uint32_t w0, w1, hh, hh1;
                    alleles(m + 1, k, &w0, &w1, &hh, &hh1);
                    next = (float)((w0 != 0u) + (w1 != 0u));
                }
                g2[(uint64_t)m * gs + k] = make_float2((float)((v0 != 0u) + (v1 != 0u)), next);
            }
        }
    }
    if (masks) masks[m] = SlotMasks{a0, a1, x, 0u};
    for (uint32_t k = L; k < gs; ++k) {
        if (g2) g2[(uint64_t)m * gs + k] = make_float2(0.f, 0.f);
        if (raw) {
            raw[((uint64_t)m * gs + k) * 2 + 0] = 0;
            raw[((uint64_t)m * gs + k) * 2 + 1] = 0;
        }
    }
}

// ---------------------------------------------------------------- target-aware selection (opt-in)
//
// The reference's selection ignores the target (every divergence is m, so the
// slots are fixed positions of the prefix row). SI_SEL_TARGET instead follows
// each target through the index as Durbin's PBWT follows an inserted sequence:
// the target's pseudo-haplotype carries allele 0 at a homozygous-reference call
// (code 0), 1 at a homozygous-alternate call (code 2), and elsewhere the allele
// of the panel haplotype at its current position in the order; its position p
// in the order of marker m counts the haplotypes whose reversed prefix sorts
// before its own (the target goes before equal keys), so with Z zeros at m and
// z(p) zeros among the first p entries of the previous order,
//   p' = z(p) (allele 0),   p' = Z + p - z(p) (allele 1).
// The slots are the L haplotypes at positions clamp(p - L/2, 0, N - L) .. + L
// of marker m's order (r % N when L > N), as pairs (h, (h + 1) % N).
//
// Rank tables, built once from the stored prefix rows: rank_bits[m][w] holds
// bit i = the allele at m of entry 32 w + i of the previous order (the order
// before marker 0 is 0 .. N-1); rank_zeros[m][w] = zeros among entries
// [0, 32 w), rank_zeros[m][W] = Z. One CTA per marker.
__global__ void target_rank_kernel(const uint32_t* __restrict__ prefix, const uint32_t* __restrict__ panel,
                                   uint32_t M, uint32_t N, uint32_t W, uint32_t* __restrict__ rank_bits,
                                   uint32_t* __restrict__ rank_zeros) {
    const uint32_t m = blockIdx.x;
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const uint32_t* prev = m ? prefix + (uint64_t)(m - 1) * N : nullptr;
    const uint32_t* prow = panel + (uint64_t)m * W;
    uint32_t* bits = rank_bits + (uint64_t)m * W;
    uint32_t* zeros = rank_zeros + (uint64_t)m * (W + 1);
    const uint32_t nwords = (N + 31) / 32;
    for (uint32_t w = warp; w < W; w += nw) {
        const uint32_t i = 32 * w + lane;
        uint32_t b = 0;
        if (i < N) {
            const uint32_t h = prev ? prev[i] : i;
            b = (prow[h >> 5] >> (h & 31)) & 1u;
        }
        const uint32_t word = __ballot_sync(0xffffffffu, b);
        if (lane == 0) bits[w] = word;
    }
    __syncthreads();
    if (warp == 0) {  // exclusive scan of per-word zero counts
        uint32_t carry = 0;
        for (uint32_t w0 = 0; w0 < W; w0 += 32) {
            const uint32_t w = w0 + lane;
            uint32_t z = 0;
            if (w < nwords) {
                const uint32_t valid = (w + 1 < nwords || N % 32 == 0) ? 0xffffffffu : ((1u << (N % 32)) - 1u);
                z = __popc(~bits[w] & valid);
            }
            uint32_t incl = z;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= (uint32_t)o) incl += y;
            }
            if (w < W) zeros[w] = carry + incl - z;
            carry += __shfl_sync(0xffffffffu, incl, 31);
        }
        if (lane == 0) zeros[W] = carry;
    }
}

// One thread per target: the walk over all M markers, writing each marker's
// slot masks (a0, a1 bits of the pairs' two haplotypes) at smasks[m][s] and,
// when pairs is given, the pairs at pairs[s][m][L][2].
__global__ void target_select_kernel(const uint8_t* __restrict__ geno, uint32_t B, uint32_t M, uint32_t N,
                                     uint32_t W, uint32_t L, const uint32_t* __restrict__ prefix,
                                     const uint32_t* __restrict__ panel, const uint32_t* __restrict__ rank_bits,
                                     const uint32_t* __restrict__ rank_zeros, SlotMasks* __restrict__ smasks,
                                     uint32_t* __restrict__ pairs) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= B) return;
    const uint8_t* g = geno + (uint64_t)s * M;
    uint32_t p = 0;
    for (uint32_t m = 0; m < M; ++m) {
        const uint32_t* bits = rank_bits + (uint64_t)m * W;
        const uint32_t* zeros = rank_zeros + (uint64_t)m * (W + 1);
        const uint32_t Z = zeros[W];
        const uint32_t zb = p < N ? zeros[p >> 5] + __popc(~bits[p >> 5] & ((1u << (p & 31)) - 1u)) : Z;
        const uint32_t q = p < N ? p : N - 1;
        const uint32_t code = g[m];
        const uint32_t xt = code == 0 ? 0u : code == 2 ? 1u : ((bits[q >> 5] >> (q & 31)) & 1u);
        p = xt ? Z + (p - zb) : zb;
        const uint32_t* row = prefix + (uint64_t)m * N;
        const uint32_t* prow = panel + (uint64_t)m * W;
        uint32_t s0 = 0;
        if (L <= N) s0 = min(p > L / 2 ? p - L / 2 : 0u, N - L);
        uint32_t a0 = 0, a1 = 0;
        for (uint32_t r = 0; r < L; ++r) {
            const uint32_t h0 = L <= N ? row[s0 + r] : row[r % N];
            const uint32_t h1 = (h0 + 1) % N;
            a0 |= ((prow[h0 >> 5] >> (h0 & 31)) & 1u) << r;
            a1 |= ((prow[h1 >> 5] >> (h1 & 31)) & 1u) << r;
            if (pairs) {
                uint32_t* o = pairs + (((uint64_t)s * M + m) * L + r) * 2;
                o[0] = h0;
                o[1] = h1;
            }
        }
        smasks[(uint64_t)m * B + s] = SlotMasks{a0, a1, 0u, 0u};
    }
}

}  // namespace

cudaError_t launch_select(const uint32_t* d_head, const uint32_t* d_panel, uint32_t M, uint32_t N, uint32_t W,
                          uint32_t L, int kind, const unsigned long long* d_ex_off, const uint32_t* d_ex_ent,
                          uint32_t* d_pairs, SlotMasks* d_masks, float2* d_g2, uint8_t* d_raw, uint32_t gs,
                          cudaStream_t s) {
    const uint32_t bs = 128;
    select_kernel<<<(M + bs - 1) / bs, bs, 0, s>>>(d_head, d_panel, M, N, W, L, kind, d_ex_off, d_ex_ent, d_pairs,
                                                   d_masks, d_g2, d_raw, gs);
    return cudaGetLastError();
}

cudaError_t launch_target_ranks(const uint32_t* d_prefix, const uint32_t* d_panel, uint32_t M, uint32_t N, uint32_t W,
                                uint32_t* d_bits, uint32_t* d_zeros, cudaStream_t s) {
    if (M == 0) return cudaSuccess;
    target_rank_kernel<<<M, 256, 0, s>>>(d_prefix, d_panel, M, N, W, d_bits, d_zeros);
    return cudaGetLastError();
}

cudaError_t launch_target_select(const uint8_t* d_geno, uint32_t B, uint32_t M, uint32_t N, uint32_t W, uint32_t L,
                                 const uint32_t* d_prefix, const uint32_t* d_panel, const uint32_t* d_bits,
                                 const uint32_t* d_zeros, SlotMasks* d_smasks, uint32_t* d_pairs, cudaStream_t s) {
    if (B == 0) return cudaSuccess;
    target_select_kernel<<<(B + 127) / 128, 128, 0, s>>>(d_geno, B, M, N, W, L, d_prefix, d_panel, d_bits, d_zeros,
                                                        d_smasks, d_pairs);
    return cudaGetLastError();
}

}  // namespace si
