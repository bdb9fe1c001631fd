// pbwt_kernels.cu — panel bit-packing and the PBWT prefix sweep.
//
// The reference builds the index on the CPU, one std::vector partition per
// marker (PBWTBuilder::build_marker, pbwt_index.cpp:153-208), and copies both
// [M][N] u32 arrays to the device (pbwt_selector.cu:487-513). Here the sweep
// runs on the device over the bit-packed panel: one CTA carries the whole
// permutation in shared memory and performs the stable allele partition of
// each marker as a block-wide exclusive scan of per-thread zero counts.
#include "si_internal.hpp"

namespace si {
namespace {

// u8 [M][N] -> bit-packed [M][W]: bit set for a non-zero allele, the side
// the reference's sweep sends it to (pbwt_index.cpp:183). One warp builds one
// 32-haplotype word with a ballot, so loads are coalesced bytes. Alleles other
// than 0 and 1 are kept beside the bits in the panel's exception lists.
__global__ void pack_panel_kernel(const uint8_t* __restrict__ u8, uint32_t M, uint32_t N, uint32_t W,
                                  uint32_t* __restrict__ words) {
    const uint64_t gtid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t word = gtid >> 5;
    const uint32_t lane = threadIdx.x & 31;
    if (word >= (uint64_t)M * W) return;  // whole warps exit together (blockDim multiple of 32)
    const uint32_t m = (uint32_t)(word / W), w = (uint32_t)(word % W);
    const uint32_t h = w * 32 + lane;
    uint8_t v = 0;
    if (h < N) v = u8[(uint64_t)m * N + h];
    const uint32_t bits = __ballot_sync(0xffffffffu, v != 0);
    if (lane == 0) words[word] = bits;
}

__device__ __forceinline__ unsigned long long mix_entry(uint32_t value, uint32_t pos) {
    unsigned long long x = (unsigned long long)value + (unsigned long long)pos * 0x9E3779B97F4A7C15ull;
    x ^= x >> 30; x *= 0xBF58476D1CE4E5B9ull;
    x ^= x >> 27; x *= 0x94D049BB133111EBull;
    x ^= x >> 31;
    return x;
}

// Order-dependent 64-bit checksum of the bit-packed panel (word value mixed
// with its index, summed): identifies the panel a stored index was built on.
__global__ void panel_checksum_kernel(const uint32_t* __restrict__ words, uint64_t n,
                                      unsigned long long* __restrict__ out) {
    unsigned long long acc = 0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        acc += mix_entry(words[i], (uint32_t)(i ^ (i >> 32)));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(out, acc);
}

constexpr int kSweepThreads = 1024;

// Sequential sweep over all markers in one CTA. Thread t owns the contiguous
// positions [t*E, t*E + E) of the current order. Per marker:
//   1. count zeros among the owned haplotypes' bits of the marker row,
//   2. block-exclusive scan of per-thread zero counts (warp shuffles, one
//      barrier, every warp rescans the 32 warp totals itself),
//   3. scatter into the next order: zeros keep their relative order at
//      [zeros-before), ones at [Z + ones-before) — the stable partition of
//      pbwt_index.cpp:176-207 — and emit the row's outputs.
// Two barriers per marker. perm arrays live in shared memory when they fit,
// otherwise in the global scratch (L2-resident at these sizes).
// Block b sweeps its own slice jobs[b] = {m0, len, head_off}: the order
// restarts from iota at m0 (a region swept on its own, as the reference does
// on a sliced panel). The whole-panel build is one job {0, M, 0}; only it may
// also write the full prefix rows and row hashes.
// kE > 0: each thread holds its (at most kE) entries and their bits in
// registers, loaded with independent shared-memory reads; kE = 0: any number
// of entries, re-read in the scatter pass.
template <bool kSmemPerm, int kE>
__global__ void __launch_bounds__(kSweepThreads, 1)
pbwt_sweep_kernel(const uint32_t* __restrict__ panel_all, const SweepJob* __restrict__ jobs, uint32_t N, uint32_t W,
                  uint32_t E, uint32_t* __restrict__ head_all, uint32_t* __restrict__ prefix,
                  unsigned long long* __restrict__ row_hash, uint32_t* __restrict__ gperm_all) {
    extern __shared__ __align__(16) uint32_t smem[];
    const SweepJob job = jobs[blockIdx.x];
    const uint32_t* panel = panel_all + (uint64_t)job.m0 * W;
    const uint32_t M = job.len;
    uint32_t* head = head_all + job.head_off;
    uint32_t* gperm = kSmemPerm ? nullptr : gperm_all + (uint64_t)blockIdx.x * 2 * N;
    uint32_t* rows = smem;                       // [2][W]
    uint32_t* wsum = rows + 2 * W;               // [2][32]
    uint32_t* perm_base = kSmemPerm ? (wsum + 64) : gperm;
    uint32_t* cur = perm_base;
    uint32_t* nxt = perm_base + N;

    const uint32_t t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const uint32_t nwarps = blockDim.x >> 5;
    const uint32_t beg = t * E;

    for (uint32_t i = t; i < N; i += blockDim.x) cur[i] = i;  // iota, pbwt_index.cpp:226
    for (uint32_t i = t; i < W; i += blockDim.x) rows[i] = panel[i];
    __syncthreads();

    // the next marker's row is loaded into registers at the top of a step and
    // written to the other shared buffer after the scatter, so the load's
    // latency overlaps the step instead of stalling it
    constexpr uint32_t kRowRegs = 4;
    for (uint32_t m = 0; m < M; ++m) {
        const uint32_t* row = rows + (m & 1) * W;
        uint32_t nxt_words[kRowRegs];
        if (m + 1 < M) {
#pragma unroll
            for (uint32_t r = 0; r < kRowRegs; ++r) {
                const uint32_t i = t + r * blockDim.x;
                nxt_words[r] = (i < W) ? __ldg(panel + (uint64_t)(m + 1) * W + i) : 0u;
            }
            for (uint32_t i = t + kRowRegs * blockDim.x; i < W; i += blockDim.x)  // rows wider than the registers
                rows[((m + 1) & 1) * W + i] = panel[(uint64_t)(m + 1) * W + i];
        }

        uint32_t n_own = 0;
        if (beg < N) n_own = min(E, N - beg);
        // pass 1: zero count of the owned entries
        uint32_t z = 0;
        uint32_t hv[kE > 0 ? kE : 1];
        uint32_t ones = 0;
        if (kE > 0) {
#pragma unroll
            for (int i = 0; i < kE; ++i) hv[i] = (uint32_t)i < n_own ? cur[beg + i] : 0u;
#pragma unroll
            for (int i = 0; i < kE; ++i)
                if ((uint32_t)i < n_own) ones |= ((row[hv[i] >> 5] >> (hv[i] & 31)) & 1u) << i;
            z = n_own - __popc(ones);
        } else {
            for (uint32_t i = 0; i < n_own; ++i) {
                const uint32_t v = cur[beg + i];
                z += ((row[v >> 5] >> (v & 31)) & 1u) ^ 1u;
            }
        }

        // warp inclusive scan of zero counts
        uint32_t incl = z;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= (uint32_t)o) incl += y;
        }
        uint32_t* ws = wsum + (m & 1) * 32;
        if (lane == 31) ws[warp] = incl;
        __syncthreads();
        // every warp scans the warp totals itself (no second barrier)
        uint32_t wt = (lane < nwarps) ? ws[lane] : 0u;
        uint32_t wincl = wt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, wincl, o);
            if (lane >= (uint32_t)o) wincl += y;
        }
        const uint32_t total_zeros = __shfl_sync(0xffffffffu, wincl, 31);
        const uint32_t warp_before = __shfl_sync(0xffffffffu, wincl - wt, warp);
        uint32_t zb = warp_before + incl - z;  // zeros before my first entry
        uint32_t ob = beg - zb;                // ones before my first entry

        unsigned long long hacc = 0;
        uint32_t* out_row = prefix ? prefix + (uint64_t)m * N : nullptr;
        uint32_t* head_row = head + (uint64_t)m * kHead;
        // pass 2: stable scatter
        if (kE > 0) {
#pragma unroll
            for (int i = 0; i < kE; ++i) {
                if ((uint32_t)i < n_own) {
                    const uint32_t v = hv[i];
                    const uint32_t pos = ((ones >> i) & 1u) ? (total_zeros + ob++) : zb++;
                    nxt[pos] = v;
                    if (out_row) out_row[pos] = v;
                    if (pos < kHead) head_row[pos] = v;
                    if (row_hash) hacc += mix_entry(v, pos);
                }
            }
        } else {
            for (uint32_t i = 0; i < n_own; ++i) {
                const uint32_t v = cur[beg + i];
                const uint32_t pos = ((row[v >> 5] >> (v & 31)) & 1u) ? (total_zeros + ob++) : zb++;
                nxt[pos] = v;
                if (out_row) out_row[pos] = v;
                if (pos < kHead) head_row[pos] = v;
                if (row_hash) hacc += mix_entry(v, pos);
            }
        }
        if (row_hash) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) hacc += __shfl_xor_sync(0xffffffffu, hacc, o);
            if (lane == 0) atomicAdd(row_hash + m, hacc);
        }
        if (m + 1 < M) {
#pragma unroll
            for (uint32_t r = 0; r < kRowRegs; ++r) {
                const uint32_t i = t + r * blockDim.x;
                if (i < W) rows[((m + 1) & 1) * W + i] = nxt_words[r];
            }
        }
        __syncthreads();
        uint32_t* tmp = cur; cur = nxt; nxt = tmp;
    }
}

}  // namespace

cudaError_t launch_pack_panel(const uint8_t* d_u8, uint32_t M, uint32_t N, uint32_t W, uint32_t* d_words,
                              cudaStream_t s) {
    const uint64_t threads = (uint64_t)M * W * 32;
    const uint32_t bs = 256;
    const uint64_t grid = (threads + bs - 1) / bs;
    if (grid > 0x7fffffffull) return cudaErrorInvalidConfiguration;
    pack_panel_kernel<<<(uint32_t)grid, bs, 0, s>>>(d_u8, M, N, W, d_words);
    return cudaGetLastError();
}

cudaError_t launch_panel_checksum(const uint32_t* d_words, uint64_t n, unsigned long long* d_out, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(d_out, 0, 8, s);
    if (e != cudaSuccess) return e;
    panel_checksum_kernel<<<148 * 8, 256, 0, s>>>(d_words, n, d_out);
    return cudaGetLastError();
}

size_t pbwt_sweep_smem_bytes(uint32_t N, uint32_t W) {
    return (size_t)(2 * W + 64) * 4 + (size_t)2 * N * 4;
}

// One CTA per job (device array d_jobs[n_jobs]); head must be zero-filled for
// rows shorter than kHead; d_perm_scratch holds 2 N words per job.
cudaError_t launch_pbwt_sweep(const uint32_t* d_panel, const SweepJob* d_jobs, uint32_t n_jobs, uint32_t N,
                              uint32_t W, uint32_t* d_head, uint32_t* d_prefix, unsigned long long* d_hash,
                              uint32_t* d_perm_scratch, cudaStream_t s) {
    uint32_t T = ((N + 4 * 32 - 1) / (4 * 32)) * 32;  // ~4 entries per thread, 128..1024 threads
    T = T < 128 ? 128 : (T > kSweepThreads ? kSweepThreads : T);
    const uint32_t E = (N + T - 1) / T;
    int dev = 0, max_optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    const size_t full = pbwt_sweep_smem_bytes(N, W);
    auto go = [&](auto kernel, size_t smem, uint32_t* gp) -> cudaError_t {
        cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        kernel<<<n_jobs, T, smem, s>>>(d_panel, d_jobs, N, W, E, d_head, d_prefix, d_hash, gp);
        return cudaSuccess;
    };
    cudaError_t e;
    if (full <= (size_t)max_optin) {
        e = E <= 4 ? go(pbwt_sweep_kernel<true, 4>, full, nullptr)
          : E <= 8 ? go(pbwt_sweep_kernel<true, 8>, full, nullptr)
          : E <= 16 ? go(pbwt_sweep_kernel<true, 16>, full, nullptr)
                    : go(pbwt_sweep_kernel<true, 0>, full, nullptr);
    } else {
        const size_t small = (size_t)(2 * W + 64) * 4;
        e = E <= 16 ? go(pbwt_sweep_kernel<false, 16>, small, d_perm_scratch)
                    : go(pbwt_sweep_kernel<false, 0>, small, d_perm_scratch);
    }
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

}  // namespace si
