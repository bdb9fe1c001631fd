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
// Block b sweeps its own slice jobs[b] = {m0, len, head_off, init_off}: the
// order restarts from iota at m0 (a region swept on its own, as the reference
// does on a sliced panel), or, for a segment of the whole-panel build, from
// the order before m0 that the segment composition computed. Only the
// whole-panel build writes prefix rows and row hashes (at absolute markers).
// kE > 0: each thread holds its (at most kE) entries and their bits in
// registers, loaded with independent shared-memory reads; kE = 0: any number
// of entries, re-read in the scatter pass.
template <bool kSmemPerm, int kE>
__global__ void __launch_bounds__(kSweepThreads, 1)
pbwt_sweep_kernel(const uint32_t* __restrict__ panel_all, const SweepJob* __restrict__ jobs, uint32_t N, uint32_t W,
                  uint32_t E, const uint32_t* __restrict__ init, uint32_t* __restrict__ head_all,
                  uint32_t* __restrict__ prefix, unsigned long long* __restrict__ row_hash,
                  uint32_t* __restrict__ gperm_all) {
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

    if (job.init_off == kIota) {
        for (uint32_t i = t; i < N; i += blockDim.x) cur[i] = i;  // iota, pbwt_index.cpp:226
    } else {
        for (uint32_t i = t; i < N; i += blockDim.x) cur[i] = init[job.init_off + i];  // a later segment's start
    }
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
#pragma unroll 8
            for (uint32_t i = 0; i < n_own; ++i) {  // unrolled: eight independent loads in flight
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
        uint32_t* out_row = prefix ? prefix + (uint64_t)(job.m0 + m) * N : nullptr;
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
#pragma unroll 8
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
            if (lane == 0) atomicAdd(row_hash + job.m0 + m, hacc);
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

// ---------------------------------------------------------------- segmented whole-panel build
//
// The sweep is sequential in the markers, but its order at the end of a
// segment [a, b) is the order before a, stably sorted by the haplotypes'
// alleles over [a, b) read as a key (marker b-1 most significant): the order
// swept from 0 .. N-1 over the segment alone ranks those keys, and the order
// before a breaks their ties. So the build runs in three passes:
//   groups   every segment but the last, on its own CTA: the sweep from
//            0 .. N-1 over its markers, carrying for each entry the index of
//            its group (haplotypes equal over the markers swept so far); the
//            final group index of each haplotype is the key rank above;
//   compose  for each segment in turn, one CTA: the order before the next
//            segment = this segment's start order stably sorted by group index
//            (an LSD radix sort, 8-bit digits);
//   sweep    every segment on its own CTA from its start order, writing its
//            rows (pbwt_sweep_kernel with init_off).
// The result is bit-identical to one sweep over all markers.

// Block-wide exclusive scans of per-thread values over kSweepThreads threads:
// a warp scan, one barrier, and every warp scanning the warp totals itself.
// buf: [K][32] totals for this call (distinct per call within a marker, and
// per marker parity, so no second barrier is needed). Returns the block total.
template <int K>
__device__ __forceinline__ void block_scan(uint32_t (&v)[K], const bool (&is_max)[K], uint32_t* buf,
                                           uint32_t (&total)[K]) {
    const uint32_t t = threadIdx.x, lane = t & 31, warp = t >> 5, nwarps = blockDim.x >> 5;
    uint32_t incl[K];
#pragma unroll
    for (int k = 0; k < K; ++k) incl[k] = v[k];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl[k], o);
            if (lane >= (uint32_t)o) incl[k] = is_max[k] ? max(incl[k], y) : incl[k] + y;
        }
    }
    if (lane == 31) {
#pragma unroll
        for (int k = 0; k < K; ++k) buf[k * 32 + warp] = incl[k];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < K; ++k) {
        const uint32_t wt = lane < nwarps ? buf[k * 32 + lane] : 0u;
        uint32_t w = wt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= (uint32_t)o) w = is_max[k] ? max(w, y) : w + y;
        }
        total[k] = __shfl_sync(0xffffffffu, w, 31);
        const uint32_t before = warp ? __shfl_sync(0xffffffffu, w, warp - 1) : 0u;  // warps before mine
        // exclusive value of this thread: warps before, then lanes before within the warp
        const uint32_t ex_lane = __shfl_up_sync(0xffffffffu, incl[k], 1);
        const uint32_t within = lane ? ex_lane : 0u;
        v[k] = is_max[k] ? max(before, within) : before + within;
    }
}

// Groups pass: jobs[b] = {m0, len, -, -} swept from 0 .. N-1 with group
// indices; gid_all[b][h] = the index of haplotype h's group at the end.
// Entries live in shared memory when 4 N words fit, else in scratch [b][4][N].
template <bool kSmem>
__global__ void __launch_bounds__(kSweepThreads, 1)
pbwt_group_kernel(const uint32_t* __restrict__ panel_all, const SweepJob* __restrict__ jobs, uint32_t N, uint32_t W,
                  uint32_t E, uint32_t* __restrict__ gid_all, uint32_t* __restrict__ scratch) {
    extern __shared__ __align__(16) uint32_t smem[];
    const SweepJob job = jobs[blockIdx.x];
    const uint32_t* panel = panel_all + (uint64_t)job.m0 * W;
    const uint32_t M = job.len;
    uint32_t* rows = smem;          // [2][W]
    uint32_t* sbuf = rows + 2 * W;  // [2 parities][5][32] scan totals
    uint32_t* base = kSmem ? (sbuf + 2 * 5 * 32) : scratch + (uint64_t)blockIdx.x * 4 * N;
    uint32_t* cur = base;           // haplotype at each position
    uint32_t* nxt = base + N;
    uint32_t* cg = base + 2 * N;    // its group index
    uint32_t* ng = base + 3 * N;
    const uint32_t t = threadIdx.x;
    const uint32_t beg = t * E;
    const uint32_t n_own = beg < N ? min(E, N - beg) : 0u;
    for (uint32_t i = t; i < N; i += blockDim.x) { cur[i] = i; cg[i] = 0u; }
    for (uint32_t i = t; i < W; i += blockDim.x) rows[i] = panel[i];
    __syncthreads();
    for (uint32_t m = 0; m < M; ++m) {
        const uint32_t* row = rows + (m & 1) * W;
        uint32_t* sb = sbuf + (m & 1) * 5 * 32;
        // 1: zeros, and the last zero's and last one's group (+1, 0 = none) among the owned entries
        uint32_t a[3] = {0u, 0u, 0u};
#pragma unroll 4
        for (uint32_t i = 0; i < n_own; ++i) {
            const uint32_t v = cur[beg + i], g1 = cg[beg + i] + 1u;
            if ((row[v >> 5] >> (v & 31)) & 1u) a[2] = g1;
            else { a[0] += 1u; a[1] = g1; }
        }
        const bool k1[3] = {false, true, true};
        uint32_t tot1[3];
        block_scan<3>(a, k1, sb, tot1);
        const uint32_t zb = a[0], Z = tot1[0], cz = a[1], co = a[2];
        // 2: group starts among the owned zeros and ones (an entry starts a group when the
        // previous entry of its side came from another group)
        uint32_t b[2] = {0u, 0u};
        {
            uint32_t pz = cz, po = co;
#pragma unroll 4
            for (uint32_t i = 0; i < n_own; ++i) {
                const uint32_t v = cur[beg + i], g1 = cg[beg + i] + 1u;
                if ((row[v >> 5] >> (v & 31)) & 1u) { b[1] += g1 != po; po = g1; }
                else { b[0] += g1 != pz; pz = g1; }
            }
        }
        const bool k2[2] = {false, false};
        uint32_t tot2[2];
        block_scan<2>(b, k2, sb + 3 * 32, tot2);
        // 3: stable scatter with the new group indices
        {
            uint32_t pz = cz, po = co, rz = b[0], ro = b[1], zpos = zb, opos = Z + (beg - zb);
            const uint32_t tzb = tot2[0];
#pragma unroll 4
            for (uint32_t i = 0; i < n_own; ++i) {
                const uint32_t v = cur[beg + i], g1 = cg[beg + i] + 1u;
                if ((row[v >> 5] >> (v & 31)) & 1u) {
                    ro += g1 != po;
                    po = g1;
                    nxt[opos] = v;
                    ng[opos] = tzb + ro - 1u;
                    ++opos;
                } else {
                    rz += g1 != pz;
                    pz = g1;
                    nxt[zpos] = v;
                    ng[zpos] = rz - 1u;
                    ++zpos;
                }
            }
        }
        if (m + 1 < M)
            for (uint32_t i = t; i < W; i += blockDim.x) rows[((m + 1) & 1) * W + i] = panel[(uint64_t)(m + 1) * W + i];
        __syncthreads();
        uint32_t* x = cur; cur = nxt; nxt = x;
        x = cg; cg = ng; ng = x;
    }
    uint32_t* gid = gid_all + (uint64_t)blockIdx.x * N;
    for (uint32_t i = t; i < N; i += blockDim.x) gid[cur[i]] = cg[i];
}

// Compose: next = order stably sorted by gid[order[r]]; one CTA of 1024
// threads, LSD radix sort with 8-bit digits over the bits of N - 1. Warp w
// owns the contiguous elements [w c, w c + c) of every pass, so ranks within a
// digit follow the input order: per-warp digit counts, their scan in (digit,
// warp) order, then each warp places its elements 32 at a time, lanes with
// equal digits ranked by lane (match_any). sortbuf: keys and values, twice.
constexpr uint32_t kComposeThreads = 1024;
__global__ void __launch_bounds__(kComposeThreads, 1)
pbwt_compose_kernel(const uint32_t* __restrict__ order, const uint32_t* __restrict__ gid, uint32_t* __restrict__ next,
                    uint32_t N, uint32_t bits, uint32_t* __restrict__ sortbuf) {
    __shared__ uint32_t cnt[256 * 32];  // [digit][warp]
    const uint32_t t = threadIdx.x, lane = t & 31, warp = t >> 5;
    constexpr uint32_t nw = kComposeThreads / 32;
    uint32_t* k0 = sortbuf;
    uint32_t* v0 = sortbuf + N;
    uint32_t* k1 = sortbuf + 2 * N;
    uint32_t* v1 = sortbuf + 3 * N;
    for (uint32_t i = t; i < N; i += blockDim.x) {
        const uint32_t h = order[i];
        k0[i] = gid[h];
        v0[i] = h;
    }
    __syncthreads();
    const uint32_t c = (N + nw - 1) / nw;
    const uint32_t e0 = min(N, warp * c), e1 = min(N, e0 + c);
    const uint32_t passes = (bits + 7) / 8;
    for (uint32_t p = 0; p < passes; ++p) {
        const uint32_t sh = 8 * p;
        const bool last = p + 1 == passes;
        uint32_t* kout = last ? nullptr : k1;
        uint32_t* vout = last ? next : v1;
        for (uint32_t i = t; i < 256 * nw; i += blockDim.x) cnt[i] = 0u;
        __syncthreads();
        for (uint32_t i = e0 + lane; i < e1; i += 32) atomicAdd(&cnt[((k0[i] >> sh) & 255u) * nw + warp], 1u);
        __syncthreads();
        // exclusive scan of cnt in (digit, warp) order: 8192 counts, 8 per thread
        uint32_t loc[8], sum = 0;
#pragma unroll
        for (int j = 0; j < 8; ++j) { loc[j] = cnt[t * 8 + j]; sum += loc[j]; }
        uint32_t incl = sum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= (uint32_t)o) incl += y;
        }
        __shared__ uint32_t wsum[32];
        if (lane == 31) wsum[warp] = incl;
        __syncthreads();
        uint32_t wt = lane < nw ? wsum[lane] : 0u, wi = wt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= (uint32_t)o) wi += y;
        }
        const uint32_t wbefore = __shfl_sync(0xffffffffu, wi - wt, warp);
        uint32_t run = wbefore + incl - sum;
#pragma unroll
        for (int j = 0; j < 8; ++j) { const uint32_t x = loc[j]; cnt[t * 8 + j] = run; run += x; }
        __syncthreads();
        // stable placement: warp-private counters, 32 elements at a time in order
        for (uint32_t b0 = e0; b0 < e1; b0 += 32) {
            const uint32_t i = b0 + lane;
            const bool ok = i < e1;
            const uint32_t key = ok ? k0[i] : 0u, val = ok ? v0[i] : 0u;
            const uint32_t d = ok ? ((key >> sh) & 255u) : 256u + lane;  // idle lanes match nobody
            const uint32_t peers = __match_any_sync(0xffffffffu, d);
            const uint32_t below = peers & ((1u << lane) - 1u);
            if (ok) {
                const uint32_t pos = cnt[d * nw + warp] + __popc(below);
                if (kout) kout[pos] = key;
                vout[pos] = val;
            }
            __syncwarp();
            if (ok && (peers >> lane) == 1u) cnt[d * nw + warp] += __popc(peers);  // the highest lane of the group
            __syncwarp();
        }
        __syncthreads();
        uint32_t* x = k0; k0 = k1; k1 = x;
        x = v0; v0 = v1; v1 = x;
    }
    if (passes == 0)
        for (uint32_t i = t; i < N; i += blockDim.x) next[i] = v0[i];
}

__global__ void iota_kernel(uint32_t* d, uint32_t N) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N) d[i] = i;
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
                              uint32_t W, const uint32_t* d_init, uint32_t* d_head, uint32_t* d_prefix,
                              unsigned long long* d_hash, uint32_t* d_perm_scratch, cudaStream_t s) {
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
        kernel<<<n_jobs, T, smem, s>>>(d_panel, d_jobs, N, W, E, d_init, d_head, d_prefix, d_hash, gp);
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

size_t pbwt_group_smem_bytes(uint32_t N, uint32_t W) { return (size_t)(2 * W + 2 * 5 * 32) * 4 + (size_t)4 * N * 4; }

cudaError_t launch_pbwt_groups(const uint32_t* d_panel, const SweepJob* d_jobs, uint32_t n_jobs, uint32_t N,
                               uint32_t W, uint32_t* d_gid, uint32_t* d_scratch, cudaStream_t s) {
    if (n_jobs == 0) return cudaSuccess;
    const uint32_t T = kSweepThreads;
    const uint32_t E = (N + T - 1) / T;
    int dev = 0, max_optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    const size_t full = pbwt_group_smem_bytes(N, W);
    cudaError_t e;
    if (full <= (size_t)max_optin) {
        e = cudaFuncSetAttribute(pbwt_group_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)full);
        if (e == cudaSuccess) pbwt_group_kernel<true><<<n_jobs, T, full, s>>>(d_panel, d_jobs, N, W, E, d_gid, nullptr);
    } else {
        const size_t small = (size_t)(2 * W + 2 * 5 * 32) * 4;
        e = cudaFuncSetAttribute(pbwt_group_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)small);
        if (e == cudaSuccess)
            pbwt_group_kernel<false><<<n_jobs, T, small, s>>>(d_panel, d_jobs, N, W, E, d_gid, d_scratch);
    }
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

cudaError_t launch_pbwt_compose(const uint32_t* d_order, const uint32_t* d_gid, uint32_t* d_next, uint32_t N,
                                uint32_t* d_sortbuf, cudaStream_t s) {
    const uint32_t bits = N > 1 ? 32u - (uint32_t)__builtin_clz(N - 1) : 0u;  // group indices are < N
    pbwt_compose_kernel<<<1, kComposeThreads, 0, s>>>(d_order, d_gid, d_next, N, bits, d_sortbuf);
    return cudaGetLastError();
}

cudaError_t launch_iota(uint32_t* d, uint32_t N, cudaStream_t s) {
    iota_kernel<<<(N + 255) / 256, 256, 0, s>>>(d, N);
    return cudaGetLastError();
}

}  // namespace si
