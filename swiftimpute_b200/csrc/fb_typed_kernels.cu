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
//   anchor_chain     one lane per sample and direction (all slots in
//                    registers): forward and backward over anchors; backward
//                    checkpoints every C anchors (a window), forward ones
//                    every K windows
//   anchor_posterior one lane per sample walks the markers of K windows:
//                    the window's backward records are rebuilt from its
//                    checkpoint, alpha is carried from anchor to anchor, and
//                    every marker's dosage, P(hap=1) and haplotypes are
//                    written through a shared-memory tile.
#include "fb_typed.hpp"
#include "philox.cuh"

namespace si {
namespace {

__device__ __forceinline__ int exp2_of(float x) { return ((__float_as_int(x) >> 23) & 0xff) - 127; }
__device__ __forceinline__ float pow2_neg(int e) { return __int_as_float((127 - e) << 23); }

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

// {Q[n], S[n]}: table entry, or the closed form past the table
__device__ __forceinline__ float2 tabQS(const Tabs& t, uint32_t n) {
    if (n < t.NT) return __ldg(t.QS + n);
    const float qn = exp2f((float)n * t.log2q);
    return make_float2(qn, (1.0f - qn) * t.invL);
}
__device__ __forceinline__ double tabG(const Tabs& t, uint32_t n) {
    if (n < t.NT) return __ldg(t.G + n);
    if (t.regime == 0) return -(double)n * t.lr + log1p(-exp((double)n * t.lr)) - t.lgc;
    if (t.regime == 1) return log(-expm1(-(double)n * t.lr)) - t.lgc;
    return log((double)n);
}

// asynchronous global -> shared copies (cp.async); a thread waits for its own copies
__device__ __forceinline__ void cp_async4(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait_group() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// ---------------------------------------------------------------- anchor lists

constexpr uint32_t kWarpsPerBlock = 8;

// 16 consecutive codes of a lane (bytes past len read as missing): one 128-bit
// load when the row is 16-byte aligned and the chunk lies inside it.
__device__ __forceinline__ uint4 load16(const uint8_t* g, uint32_t base, uint32_t len, bool vec) {
    if (base >= len) return make_uint4(0x03030303u, 0x03030303u, 0x03030303u, 0x03030303u);
    if (vec && base + 16 <= len) return *reinterpret_cast<const uint4*>(g + base);
    uint32_t w[4] = {0x03030303u, 0x03030303u, 0x03030303u, 0x03030303u};
#pragma unroll
    for (uint32_t j = 0; j < 16; ++j)  // unrolled: the word index is a constant, w stays in registers
        if (base + j < len)
            w[j >> 2] = (w[j >> 2] & ~(0xffu << (8 * (j & 3)))) | ((uint32_t)g[base + j] << (8 * (j & 3)));
    return make_uint4(w[0], w[1], w[2], w[3]);
}

// bit j set when code j of the chunk is below 3 (typed)
__device__ __forceinline__ uint32_t typed_bits(uint4 c) {
    const uint32_t ww[4] = {c.x, c.y, c.z, c.w};
    uint32_t bits = 0;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const uint32_t lt = __vcmpltu4(ww[q], 0x03030303u);  // 0xff in each byte below 3
#pragma unroll
        for (int b = 0; b < 4; ++b) bits |= ((lt >> (8 * b + 7)) & 1u) << (4 * q + b);
    }
    return bits;
}

// Per-sample anchor counts: a warp per sample, 16 codes per lane per chunk of
// 512, the next chunk's load in flight while the current one is counted; the
// count of every segment of kFillSeg markers goes to segc[s][segment] for the
// fill, the total (cut to a plan's capacity) to counts[s].
__global__ void anchor_count_kernel(TypedArgs A) {
    const uint32_t s = blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
    const uint32_t lane = threadIdx.x & 31;
    if (s >= A.B) return;
    const View v = view_of(A, s);
    const bool vec = (reinterpret_cast<uintptr_t>(v.geno) & 15u) == 0;
    uint32_t* segc = A.segc + (size_t)s * A.nseg;
    uint32_t n = 0, seg = 0;
    uint4 cur = load16(v.geno, lane * 16, v.len, vec);
    for (uint32_t b0 = 0; b0 < v.len; b0 += kFillSeg) {
        uint32_t c = 0;
        for (uint32_t base = b0 + lane * 16; base < min(b0 + kFillSeg, v.len); base += 512) {
            const uint4 nxt = load16(v.geno, base + 512, v.len, vec);
            uint32_t bits = typed_bits(cur);
            if (base == 0) bits |= 1u;  // marker 0 is always an anchor
            c += __popc(bits);
            cur = nxt;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
        if (lane == 0) segc[seg] = c;
        n += c;
        ++seg;
    }
    if (lane == 0) {
        if (A.cap && n > A.cap[s]) {
            atomicOr(A.err, 1u);  // the job is cut to its capacity; the host reports it
            n = A.cap[s];
        }
        A.counts[s] = n;
    }
}

// Exclusive scans over the 32-sample groups of the interleaved lists, in one
// CTA: a group takes 32 x its most anchors and 32 x its most windows
// (ceil(count / C)). Entry G holds the totals, also written with the most
// windows of any sample to host_totals[0..2] (mapped pinned host memory) when
// given: a copy would queue behind other device-to-host copies on the copy
// engine.
__global__ void __launch_bounds__(1024) anchor_scan_kernel(const uint32_t* __restrict__ counts, uint32_t B,
                                                           uint32_t C, unsigned long long* __restrict__ aoff,
                                                           unsigned long long* __restrict__ woff,
                                                           unsigned long long* __restrict__ host_totals) {
    __shared__ unsigned long long sa[32], sw[32];
    __shared__ uint32_t smax[32];
    const uint32_t t = threadIdx.x, T = blockDim.x, lane = t & 31, warp = t >> 5;
    const uint32_t G = (B + 31) / 32;
    const uint32_t per = (G + T - 1) / T;
    const uint32_t g0 = min(G, t * per), g1 = min(G, g0 + per);
    auto group_max = [&](uint32_t g) {
        uint32_t x = 0;
        for (uint32_t b = g * 32; b < min(B, g * 32 + 32); ++b) x = max(x, counts[b]);
        return x;
    };
    unsigned long long la = 0, lw = 0;
    uint32_t mx = 0;
    for (uint32_t g = g0; g < g1; ++g) {
        const uint32_t x = group_max(g);
        la += 32ull * x;
        lw += 32ull * ((x + C - 1) / C);
        mx = max(mx, x);
    }
    mx = __reduce_max_sync(0xffffffffu, mx);
    if (lane == 0) smax[warp] = mx;
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
        smax[lane] = __reduce_max_sync(0xffffffffu, lane < (T >> 5) ? smax[lane] : 0u);
    }
    __syncthreads();
    unsigned long long ra = sa[warp] + ia - la, rw = sw[warp] + iw - lw;
    for (uint32_t g = g0; g < g1; ++g) {
        aoff[g] = ra;
        woff[g] = rw;
        const uint32_t x = group_max(g);
        ra += 32ull * x;
        rw += 32ull * ((x + C - 1) / C);
    }
    if (t == T - 1) {
        aoff[G] = ra;
        woff[G] = rw;
        if (host_totals) {  // mapped host memory: the host reads the totals without a copy
            host_totals[0] = ra;
            host_totals[1] = rw;
            host_totals[2] = (smax[0] + C - 1) / C;
            __threadfence_system();
        }
    }
}

// Anchor lists: marker position (with the "no slot matches" flag, which
// scales every slot by e^-999, counted in beta's unit, in bit 31) and emission
// mask over the slots, in marker order; marker 0 is always an anchor. A warp
// (one CTA) fills one segment of kFillSeg markers of the 32 samples of a
// group, lane = sample: chunks of 32 rows x 256 codes (and, for a plain batch,
// the chunk's slot masks) come into shared memory by cp.async, the next chunk
// in flight while each lane scans its own row of the current one, and lanes
// that meet their anchors in step (shared typed positions) write whole
// 128-byte lines of the interleaved lists. A lane's first entry of the segment
// is the sum of its earlier segments' counts.
constexpr uint32_t kFillChunk = 256;                 // markers per staged chunk
constexpr uint32_t kFillRow = kFillChunk + 16;        // row stride in shared memory (bytes): conflict-free 128-bit reads
constexpr size_t kFillBuf = 32 * kFillRow + kFillChunk * sizeof(SlotMasks);  // codes of 32 rows, the chunk's slot masks
constexpr size_t kFillSmem = 2 * kFillBuf + 32 * 16;  // two chunk buffers and the row descriptors

__global__ void __launch_bounds__(32) anchor_fill_kernel(TypedArgs A) {
    extern __shared__ __align__(16) unsigned char fsm[];
    const uint32_t lane = threadIdx.x;
    const uint32_t G = (A.B + 31) / 32;
    const uint32_t g = blockIdx.x % G, seg = blockIdx.x / G;
    const uint32_t s = g * 32 + lane;
    uint4* rowd = reinterpret_cast<uint4*>(fsm + 2 * kFillBuf);  // [32] {ptr lo, ptr hi, len, 16-byte aligned}
    View v{};
    uint32_t len = 0, at = 0, lim = 0;
    if (s < A.B) {
        v = view_of(A, s);
        len = v.len;
        const uint32_t* segc = A.segc + (size_t)s * A.nseg;
        for (uint32_t j = 0; j < seg; ++j) at += segc[j];
        lim = A.counts[s];  // a plan's capacity cut, else every anchor
    }
    const uint32_t m0 = seg * kFillSeg;
    const uint32_t mlast = __reduce_max_sync(0xffffffffu, len);
    if (m0 >= mlast) return;  // whole warp: no row reaches this segment
    const unsigned long long gp = reinterpret_cast<unsigned long long>(v.geno);
    rowd[lane] = make_uint4((uint32_t)gp, (uint32_t)(gp >> 32), len, (gp & 15u) == 0 ? 1u : 0u);
    __syncwarp();
    const uint32_t lmask = lmask_of(v.r.L);
    const unsigned long long lb = A.aoff[g] + lane;
    // a plain batch shares one slot-mask table: its chunk is staged beside the codes
    const bool stage_masks = A.samples == nullptr;
    const SlotMasks* gmasks = A.reg0.masks;
    // chunk at c0 into buffer b: rows 2 it + lane / 16, bytes 16 (lane % 16) .. + 16, and the masks
    auto issue = [&](uint32_t c0, unsigned char* b) {
        const uint32_t mm = c0 + 16 * (lane & 15);
#pragma unroll 4
        for (uint32_t it = 0; it < 16; ++it) {
            const uint32_t r = 2 * it + (lane >> 4);
            const uint4 d = rowd[r];
            const uint8_t* gr = reinterpret_cast<const uint8_t*>(((unsigned long long)d.y << 32) | d.x);
            unsigned char* dst = b + r * kFillRow + 16 * (lane & 15);
            if (d.w && mm + 16 <= d.z) cp_async16(dst, gr + mm);
            else *reinterpret_cast<uint4*>(dst) = load16(gr, mm, d.z, d.w != 0);  // a ragged or unaligned row
        }
        if (stage_masks) {
            SlotMasks* sm = reinterpret_cast<SlotMasks*>(b + 32 * kFillRow);
            for (uint32_t i = lane; i < kFillChunk && c0 + i < A.M; i += 32) cp_async16(sm + i, gmasks + c0 + i);
        }
        cp_async_commit();
    };
    const uint32_t cend = min(m0 + kFillSeg, mlast);
    issue(m0, fsm);
    uint32_t bi = 0;
    for (uint32_t c0 = m0; c0 < cend; c0 += kFillChunk, bi ^= 1) {
        if (c0 + kFillChunk < cend) {
            issue(c0 + kFillChunk, fsm + (bi ^ 1) * kFillBuf);
            cp_async_wait_group<1>();  // this lane's copies of the current chunk have landed
        } else {
            cp_async_wait_group<0>();
        }
        __syncwarp();  // ... and every lane's
        if (c0 < len) {
            const unsigned char* buf = fsm + bi * kFillBuf;
            const unsigned char* row = buf + lane * kFillRow;
            const SlotMasks* sm = reinterpret_cast<const SlotMasks*>(buf + 32 * kFillRow);
            for (uint32_t q = 0; q < kFillChunk / 16; ++q) {
                const uint4 x = *reinterpret_cast<const uint4*>(row + 16 * q);
                uint32_t bits = typed_bits(x);
                const uint32_t base = c0 + 16 * q;
                if (base == 0) bits |= 1u;
                while (bits) {
                    const uint32_t j = __ffs(bits) - 1;
                    bits &= bits - 1;
                    const uint32_t m = base + j;
                    if (at < lim) {
                        uint32_t sh;
                        const uint32_t w = j < 8 ? (j < 4 ? x.x : x.y) : (j < 12 ? x.z : x.w);
                        const SlotMasks mk = stage_masks ? sm[m - c0] : v.r.masks[m];
                        const uint32_t em = emission_mask((w >> (8 * (j & 3))) & 0xffu, mk, lmask, &sh);
                        A.apos[lb + 32ull * at] = m | (sh ? kShiftBit : 0u);
                        A.aem[lb + 32ull * at] = em;
                    }
                    ++at;
                }
            }
        }
        __syncwarp();  // the buffer is read before it is refilled
    }
}

// ---------------------------------------------------------------- chain

template <int LM>
__device__ __forceinline__ float vsum(const float (&v)[LM]) {
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < LM; ++k) s += v[k];
    return s;
}

// Exact int -> double on the FP64 pipe: 2^52 + 2^31 + x has x + 2^31 in its
// low word, so one subtraction recovers x (a conversion instruction would use
// the special-function pipe, which the backward chain otherwise saturates).
__device__ __forceinline__ double i2d(int x) {
    return __hiloint2double(0x43300000, (int)((uint32_t)x ^ 0x80000000u)) - 4503601774854144.0;  // 2^52 + 2^31
}
__device__ __forceinline__ double u2d(uint32_t x) { return __hiloint2double(0x43300000, (int)x) - 4503599627370496.0; }

// sum over slot pairs, as a tree
template <uint32_t H>
__device__ __forceinline__ float vsum2(const float2 (&v)[H]) {
    float2 t[H];
#pragma unroll
    for (uint32_t h = 0; h < H; ++h) t[h] = v[h];
#pragma unroll
    for (uint32_t w = H / 2; w >= 1; w >>= 1)
#pragma unroll
        for (uint32_t h = 0; h < w; ++h) t[h] = __fadd2_rn(t[h], t[h + w]);
    return t[0].x + t[0].y;
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
    const float2 qs = tabQS(tb, n);
    const float Qn = qs.x, Sn = qs.y;
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
    const float2 qs = tabQS(tb, n);
    const float Qn = qs.x, Sn = qs.y;
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

constexpr uint32_t kChainBlock = 8;  // anchors per block of list entries

// One chain per lane with all LM slots in registers: even warps run forward
// chains, odd warps the backward chains of the same 32 samples. The warp
// steps in lockstep to the longest of its chains (a finished chain holds its
// state), in blocks of kChainBlock anchors. A block's list entries are loaded
// two blocks ahead and its run-table entries one block ahead, so a step's
// dependent path is its own arithmetic: the slot update, the sum over the
// slots and the power-of-two rescale (and, backward, the unit's log when
// beta's e^-999 floor matters). Checkpoints: backward vector and the log of
// its unit at anchors k % C == 0 (window starts); forward vector at anchors
// k % (K C) == 0.
template <int LM>
__global__ void __launch_bounds__(32) anchor_chain_kernel(TypedArgs A) {
    constexpr uint32_t KB = kChainBlock;
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t wg = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const bool forward = (wg & 1u) == 0;
    const uint32_t s = (wg >> 1) * 32 + lane;
    const bool live = s < A.B;
    // A lane past the batch's end takes the last sample's tables: its discarded
    // lookups (gap 0) then read the tables like its warp's live lanes instead of
    // evaluating the FP64 closed form past a table of zero entries every step.
    const View v = view_of(A, live ? s : A.B - 1);
    uint32_t NA = 0;
    unsigned long long base = 0, wb = 0;
    if (live) {
        base = A.aoff[s >> 5] + lane;
        wb = A.woff[s >> 5] + lane;
        NA = A.counts[s];
    }
    const uint32_t NAw = __reduce_max_sync(0xffffffffu, NA);
    if (NAw == 0) return;  // whole warp
    const Tabs& tb = v.r.tabs;
    const uint32_t* apos = A.apos + base;  // entry k at apos[32 k]
    const uint32_t* aemk = A.aem + base;
    auto pos = [&](uint32_t k) { return apos[32ull * k] & ~kShiftBit; };
    auto aem = [&](uint32_t k) { return aemk[32ull * k]; };
    const uint32_t C = A.C, K = A.K;
    auto ck = [&](uint32_t w) { return wb + 32ull * w; };  // window w's checkpoint entry
    constexpr uint32_t H = LM / 2;  // slot pairs
    auto store = [&](float* dst, const float2 (&x)[H]) {
#pragma unroll
        for (uint32_t q = 0; q < H / 2; ++q)
            reinterpret_cast<float4*>(dst)[q] = make_float4(x[2 * q].x, x[2 * q].y, x[2 * q + 1].x, x[2 * q + 1].y);
    };
    // a step's update of the slot pairs: em bit l ? g x_l + b : 0, its sum, and the power-of-two
    // rescale that brings the sum into [1, 2) (the scale's exponent is -e)
    auto update = [&](float2 (&x)[H], uint32_t em, float g, float b, float& sum, int& e) {
        const float2 G2 = make_float2(g, g), B2 = make_float2(b, b);
        float2 xn[H];
#pragma unroll
        for (uint32_t h = 0; h < H; ++h) {
            const float2 t = __ffma2_rn(G2, x[h], B2);
            xn[h] = make_float2(((em >> (2 * h)) & 1u) ? t.x : 0.f, ((em >> (2 * h + 1)) & 1u) ? t.y : 0.f);
        }
        const float s2 = vsum2<H>(xn);
        const int bits = __float_as_int(s2) & 0x7f800000;
        const float sc = __int_as_float(0x7f000000 - bits);
        const float2 S2 = make_float2(sc, sc);
#pragma unroll
        for (uint32_t h = 0; h < H; ++h) x[h] = __fmul2_rn(xn[h], S2);
        sum = s2 * sc;
        e = (bits >> 23) - 127;
    };
    if (forward) {
        // step k (anchor k = 1 .. NA - 1): the run from anchor k - 1, then anchor k's emission
        float2 a[H];
        uint32_t prev = 0;
#pragma unroll
        for (uint32_t h = 0; h < H; ++h) a[h] = make_float2(0.f, 0.f);
        float sa = 0.f;
        if (NA > 0) {
            int e;
            const uint32_t em = aem(0);
#pragma unroll
            for (uint32_t h = 0; h < H; ++h) a[h] = make_float2(1.f, 1.f);
            update(a, em, 0.f, 1.f, sa, e);  // the emission of anchor 0 over uniform slots
            prev = pos(0);
            store(A.ckptF + ck(0) * LM, a);
        }
        uint32_t cc = C, ci = 1;  // anchors to the next checkpoint, its window
        auto load = [&](uint32_t k0, uint32_t (&p)[KB], uint32_t (&e)[KB]) {
#pragma unroll
            for (uint32_t j = 0; j < KB; ++j) {
                const uint32_t k = k0 + j;
                p[j] = k < NA ? pos(k) : 0u;
                e[j] = k < NA ? aem(k) : 0u;
            }
        };
        auto tables = [&](uint32_t k0, const uint32_t (&p)[KB], uint32_t before, float2 (&q)[KB]) {
#pragma unroll
            for (uint32_t j = 0; j < KB; ++j) q[j] = tabQS(tb, k0 + j < NA ? p[j] - (j ? p[j - 1] : before) : 0u);
        };
        auto step = [&](uint32_t em, float2 q) {
            int e;
            update(a, em, q.x, sa * q.y, sa, e);
            if (--cc == 0) {
                if (ci % K == 0) store(A.ckptF + ck(ci) * LM, a);
                ++ci;
                cc = C;
            }
        };
        uint32_t p0[KB], e0[KB], p1[KB], e1[KB];
        float2 q0[KB];
        load(1, p0, e0);
        load(1 + KB, p1, e1);
        tables(1, p0, prev, q0);
        for (uint32_t k0 = 1; k0 < NAw; k0 += KB) {
            uint32_t p2[KB], e2[KB];
            float2 q1[KB];
            load(k0 + 2 * KB, p2, e2);           // two blocks ahead
            tables(k0 + KB, p1, p0[KB - 1], q1);  // one block ahead
            if (__all_sync(0xffffffffu, k0 + KB <= NA)) {
#pragma unroll
                for (uint32_t j = 0; j < KB; ++j) step(e0[j], q0[j]);
            } else {
#pragma unroll
                for (uint32_t j = 0; j < KB; ++j)
                    if (k0 + j < NA) step(e0[j], q0[j]);  // a finished chain holds its state
            }
#pragma unroll
            for (uint32_t j = 0; j < KB; ++j) {
                p0[j] = p1[j]; e0[j] = e1[j]; q0[j] = q1[j];
                p1[j] = p2[j]; e1[j] = e2[j];
            }
        }
    } else {
        // step t handles anchor k = NA - 2 - t (t = 0 .. NA - 2): the run to anchor k + 1
        float2 w[H];
        uint32_t nextp = 0;
        double logU = 0.0;
#pragma unroll
        for (uint32_t h = 0; h < H; ++h) w[h] = make_float2(0.f, 0.f);
        float sw = 0.f;
        if (NA > 0) {
            const uint32_t pl = apos[32ull * (NA - 1)];
            nextp = pl & ~kShiftBit;
            logU = chain_end_logU(tb, v.len - 1 - nextp) - ((pl & kShiftBit) ? 999.0 : 0.0);
            const uint32_t em = aem(NA - 1);
#pragma unroll
            for (uint32_t h = 0; h < H; ++h)
                w[h] = make_float2(((em >> (2 * h)) & 1u) ? 1.f : 0.f, ((em >> (2 * h + 1)) & 1u) ? 1.f : 0.f);
            sw = vsum2<H>(w);
            if ((NA - 1) % C == 0) {
                store(A.ckptB + ck((NA - 1) / C) * LM, w);
                A.ckptU[ck((NA - 1) / C)] = logU;
            }
        }
        uint32_t cc = NA >= 2 ? (NA - 2) % C + 1 : 0u;  // anchors to the next checkpoint (k % C == 0)
        uint32_t ci = NA >= 2 ? (NA - 2) / C : 0u;      // its window
        auto load = [&](uint32_t t0, uint32_t (&p)[KB], uint32_t (&e)[KB], uint32_t (&h)[KB]) {
#pragma unroll
            for (uint32_t j = 0; j < KB; ++j) {
                const uint32_t t = t0 + j;
                const bool ok = t + 2 <= NA;
                const uint32_t k = NA - 2 - t;
                const uint32_t pk = ok ? apos[32ull * k] : 0u;
                p[j] = pk & ~kShiftBit;
                e[j] = ok ? aem(k) : 0u;
                h[j] = pk >> 31;
            }
        };
        // per step: {Q, S} of the run, G(n) - 999 and the unit's change n log rho - 999 shift
        auto tables = [&](uint32_t t0, const uint32_t (&p)[KB], const uint32_t (&h)[KB], uint32_t after,
                          float2 (&q)[KB], double (&g)[KB], double (&c)[KB]) {
#pragma unroll
            for (uint32_t j = 0; j < KB; ++j) {
                const uint32_t n = t0 + j + 2 <= NA ? (j ? p[j - 1] : after) - p[j] : 0u;
                q[j] = tabQS(tb, n);
                g[j] = tabG(tb, n) - 999.0;
                c[j] = fma(u2d(n), tb.lr, h[j] ? -999.0 : 0.0);
            }
        };
        auto step = [&](uint32_t em, float2 q, double g, double c) {
            // the floor's log in units of U: fterm > 0, the floor dominates and the unit
            // becomes U rho^n e^fterm; fterm <= -104, it is negligible (the common case:
            // the carried terms alone, and the unit's bookkeeping stays off this step's path)
            const double fterm = g - logU;
            const bool big = fterm > 0.0;
            float xs = 1.f, F = 0.f;
            if (fterm > -104.0) {
                const float ex = expf(-(float)fmin(fabs(fterm), 104.0));
                xs = big ? ex : 1.f;  // scale of the carried terms
                F = big ? 1.f : ex;   // the floor term
            }
            int e;
            update(w, em, xs * q.x, fmaf(xs * sw, q.y, F), sw, e);
            logU = fma(i2d(e), 0.69314718055994530942, (big ? g : logU) + c);
            if (--cc == 0) {
                store(A.ckptB + ck(ci) * LM, w);
                A.ckptU[ck(ci)] = logU;
                --ci;
                cc = C;
            }
        };
        uint32_t p0[KB], e0[KB], h0[KB], p1[KB], e1[KB], h1[KB];
        float2 q0[KB];
        double g0[KB], c0[KB];
        load(0, p0, e0, h0);
        load(KB, p1, e1, h1);
        tables(0, p0, h0, nextp, q0, g0, c0);
        for (uint32_t t0 = 0; t0 + 1 < NAw; t0 += KB) {
            uint32_t p2[KB], e2[KB], h2[KB];
            float2 q1[KB];
            double g1[KB], c1[KB];
            load(t0 + 2 * KB, p2, e2, h2);
            tables(t0 + KB, p1, h1, p0[KB - 1], q1, g1, c1);
            if (__all_sync(0xffffffffu, t0 + KB + 1 <= NA)) {
#pragma unroll
                for (uint32_t j = 0; j < KB; ++j) step(e0[j], q0[j], g0[j], c0[j]);
            } else {
#pragma unroll
                for (uint32_t j = 0; j < KB; ++j)
                    if (t0 + j + 2 <= NA) step(e0[j], q0[j], g0[j], c0[j]);  // a finished chain holds its state
            }
#pragma unroll
            for (uint32_t j = 0; j < KB; ++j) {
                p0[j] = p1[j]; e0[j] = e1[j]; h0[j] = h1[j]; q0[j] = q1[j]; g0[j] = g1[j]; c0[j] = c1[j];
                p1[j] = p2[j]; e1[j] = e2[j]; h1[j] = h2[j];
            }
        }
    }
}

// ---------------------------------------------------------------- posterior
//
// One warp per (32 samples, group of K consecutive windows of C anchors); lane
// = sample (the warp's samples are one group of the interleaved lists). A lane
// walks its sample's markers of the group in tiles of 32 absolute markers:
//   group start: alpha from the forward checkpoint at the group's first anchor
//     (the chain writes one every K windows), and the first window's
//     backward records;
//   at an anchor (a typed marker, or marker 0): alpha steps over the run from
//     the previous anchor and takes the anchor's emission; the run starting
//     there takes its backward record, and at a window's first anchor the
//     window's records are rebuilt from the window's end checkpoint;
//   every marker: p_l = (Q[i] a'_l + S[i]) (X w'_l + Y), dosage, pick and
//     P(hap=1), two markers of a run per step.
// The backward record of the run [pos[k], pos[k+1]) holds
//   w'     the backward vector of anchor k+1 (E . beta), divided by its sum;
//   farg'  -999 - logU - ln(sum w), the log of beta's e^-999 floor in units of
//          w': -inf when the floor is negligible over the whole run, and the
//          run is "uniform" (w' = 0, beta constant) for the chain's last run
//          or where the floor dominates everywhere;
//   the run's end (pos[k+1], or the slice length) and anchor k+1's emission
//          mask, so an anchor step reads nothing from global memory.
// A window's inputs (its list entries and end checkpoint) are copied into a
// per-lane staging area with cp.async while the previous window is walked.
// With a' and w' of unit sum, a cell i markers after pos[k] and j = pos[k+1]
// - m before the next anchor has alpha_l ~ Q[i] a'_l + S[i] and beta_l ~
// Q[j] w'_l + S[j] (+ floor). Lanes whose samples share typed positions (an
// array's sites, every batch of the benchmark workloads) step through the
// same markers, so the per-marker slot data are warp-uniform loads; other
// lanes still work, with divergent anchor steps. Outputs are staged in a
// per-warp tile [32 samples][32 markers] in shared memory and leave as row
// segments of 32 consecutive markers.

// high word of farg' for a uniform run and for a negligible floor
constexpr uint32_t kInfHi = 0x7ff00000u;
constexpr uint32_t kNegInfHi = 0xfff00000u;

__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// three-input maximum (sm_100)
__device__ __forceinline__ float max3(float a, float b, float c) {
    float r;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

template <int LM>
__device__ __forceinline__ float vmax(const float (&p)[LM]) {
    float m = p[0];
#pragma unroll
    for (int l = 1; l + 1 < LM; l += 2) m = max3(m, p[l], p[l + 1]);
    if (LM % 2 == 0) m = fmaxf(m, p[LM - 1]);
    return m;
}


// Argmax picks of two cells: the first slot with p >= (1 - eps) max; the
// sign of p - thr marks the slots below the threshold.
template <int LM>
__device__ __forceinline__ void pick_pair(const float2 (&p2)[LM], float keep, uint32_t& k0, uint32_t& k1) {
    float px[LM], py[LM];
#pragma unroll
    for (int l = 0; l < LM; ++l) { px[l] = p2[l].x; py[l] = p2[l].y; }
    const float2 thr2 = __fmul2_rn(make_float2(vmax<LM>(px), vmax<LM>(py)), make_float2(-keep, -keep));
    uint32_t bx = 0u, by = 0u;  // bit LM-1-l: slot l below the threshold
#pragma unroll
    for (int l = 0; l < LM; ++l) {
        const float2 d = __fadd2_rn(p2[l], thr2);
        bx = __funnelshift_l(__float_as_uint(d.x), bx, 1);
        by = __funnelshift_l(__float_as_uint(d.y), by, 1);
    }
    constexpr uint32_t kLow = LM >= 32 ? 0xffffffffu : ((1u << LM) - 1u);
    k0 = (uint32_t)__clz(~bx & kLow) - (32u - LM);
    k1 = (uint32_t)__clz(~by & kLow) - (32u - LM);
}

// Shared memory of one warp: backward records [C][LM/4][32] float4 and
// [C][32] {farg' lo, farg' hi, run end, end emission}; the flush descriptors
// [2][32] uint4; the dosage tile [32][36] f32, the allele tile [64][36] u8
// (rows 2r and 2r + 1: the two haplotypes of lane r) and, for P(hap=1),
// [32][34] f32x2; the staging area of the next window: end checkpoint
// [LM/4][32] float4 and [32] f64, list entries [C+1][32] positions and
// [C+1][32] emission masks.
__host__ __device__ constexpr size_t post_warp_bytes(uint32_t LM, uint32_t C, bool hprob) {
    return (size_t)C * LM * 128 + (size_t)C * 512 + 1024 + 32 * 36 * 4 + 64 * 36 + (hprob ? 32 * 34 * 8 : 0) +
           (size_t)LM * 128 + 256 + 2 * ((size_t)C + 1) * 128;
}

struct Staging {
    float4* B;    // [LM/4][32] backward checkpoint at the window's end
    double* U;    // [32] its unit's log
    uint32_t* P;  // [C+1][32] list positions (with the shift bit) of anchors wC .. wC + C
    uint32_t* E;  // [C+1][32] their emission masks
};

// Issue the copies of window w's inputs into the lane's staging column.
template <int LM>
__device__ __forceinline__ void stage_window(const TypedArgs& A, const uint32_t* apos, const uint32_t* aem,
                                             unsigned long long wb, uint32_t NA, uint32_t w, const Staging& st,
                                             uint32_t lane) {
    const uint32_t C = A.C, k0 = w * C, k1 = min(k0 + C, NA);
    const uint32_t kl = min(k1, NA - 1);
    for (uint32_t k = k0; k <= kl; ++k) {
        cp_async4(st.P + (k - k0) * 32 + lane, apos + 32ull * k);
        cp_async4(st.E + (k - k0) * 32 + lane, aem + 32ull * k);
    }
    if (k1 < NA) {
        const unsigned long long e = wb + 32ull * (w + 1);
        const float4* src = reinterpret_cast<const float4*>(A.ckptB + e * LM);
#pragma unroll
        for (uint32_t q = 0; q < LM / 4; ++q) cp_async16(st.B + q * 32 + lane, src + q);
        cp_async8(st.U + lane, A.ckptU + e);
    }
    cp_async_commit();
}

// Backward records of window w (anchors [wC, min(wC + C, NA))) of one sample,
// rebuilt from the staged end checkpoint, into the lane's column of recW/recF.
template <int LM>
__device__ __forceinline__ void rebuild_window(const TypedArgs& A, const Tabs& tb, uint32_t NA, uint32_t len,
                                               uint32_t w, const Staging& st, float4* recW, uint4* recF,
                                               uint32_t lane) {
    constexpr uint32_t Q4 = LM / 4;
    cp_async_wait_all();
    const uint32_t C = A.C;
    const uint32_t k0 = w * C, k1 = min(k0 + C, NA);
    auto P = [&](uint32_t k) { return st.P[(k - k0) * 32 + lane]; };
    auto E = [&](uint32_t k) { return st.E[(k - k0) * 32 + lane]; };
    float bv[LM];
    double logU;
    uint32_t kstart;
    if (k1 < NA) {
#pragma unroll
        for (uint32_t q = 0; q < Q4; ++q) {
            const float4 x = st.B[q * 32 + lane];
            bv[4 * q] = x.x; bv[4 * q + 1] = x.y; bv[4 * q + 2] = x.z; bv[4 * q + 3] = x.w;
        }
        logU = st.U[lane];
        kstart = k1;
    } else {
        // the chain's last run: beta is uniform there
        const uint32_t pl = P(NA - 1);
        logU = chain_end_logU(tb, len - 1 - (pl & ~kShiftBit)) - ((pl & kShiftBit) ? 999.0 : 0.0);
        init_forward<LM>(bv, E(NA - 1));
        kstart = NA - 1;
        const uint32_t r = NA - 1 - k0;
#pragma unroll
        for (uint32_t q = 0; q < Q4; ++q) recW[(r * Q4 + q) * 32 + lane] = make_float4(0.f, 0.f, 0.f, 0.f);
        recF[r * 32 + lane] = make_uint4(0u, kInfHi, len, 0u);
    }
    for (uint32_t k = kstart; k > k0; --k) {
        const uint32_t pk = P(k) & ~kShiftBit, pb = P(k - 1);
        const uint32_t n = pk - (pb & ~kShiftBit);
        const float sw = vsum<LM>(bv);
        const double farg = -999.0 - logU;
        uint32_t lo = 0u, hi;
        if (farg + tabG(tb, n) < -104.0) hi = kNegInfHi;  // floor negligible over the run
        else if (farg + tabG(tb, 1) > 60.0) hi = kInfHi;  // floor dominates: beta uniform
        else {
            const double f = farg - (double)logf(sw);
            lo = (uint32_t)__double_as_longlong(f);
            hi = (uint32_t)((unsigned long long)__double_as_longlong(f) >> 32);
        }
        const uint32_t r = k - 1 - k0;
        const float inv = hi == kInfHi ? 0.f : rcp_approx(sw);
#pragma unroll
        for (uint32_t q = 0; q < Q4; ++q)
            recW[(r * Q4 + q) * 32 + lane] =
                make_float4(bv[4 * q] * inv, bv[4 * q + 1] * inv, bv[4 * q + 2] * inv, bv[4 * q + 3] * inv);
        recF[r * 32 + lane] = make_uint4(lo, hi, pk, E(k));
        if (k - 1 > k0) backward_step<LM>(tb, n, bv, logU, E(k - 1), pb >> 31, 0u);
    }
}

// kFull: every sample of the launch uses all LM slots (no active-slot masking).
// kFast: argmax picks, no P(hap=1). kPlain: every sample covers the whole
// panel with the launch's one region (read from the kernel parameters).
// kDos: dosage written (false only with kFast, for calls that return the
// phased alleles alone: no dosage sums and no g2 loads).
// A lane takes two consecutive cells of a run per step (an even marker and
// the next one) with f32x2 arithmetic across the two cells; a run's odd first
// marker or last marker takes a step alone (the second half is discarded).
// The next step's run coefficients are loaded while the current step runs.
// Tiles are aligned to absolute 32-marker columns, so a tile every lane of a
// warp fills completely (lanes that share typed positions) leaves as 128-bit
// row segments.
template <int LM, bool kFull, bool kFast, bool kPlain, bool kDos>
__global__ void __launch_bounds__(128, (LM <= 8 ? (kPlain ? 4 : 3) : 2))
    anchor_posterior_kernel(const __grid_constant__ TypedArgs A) {
    extern __shared__ __align__(16) unsigned char smem[];
    constexpr uint32_t Q4 = LM / 4;
    constexpr uint32_t kAll = 0xffffffffu;
    constexpr bool kBcast = LM <= 16;  // a', w' held as (x, x) pairs: no per-step pairing moves
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const uint32_t C = A.C, K = A.K;
    unsigned char* wbase = smem + (size_t)warp * post_warp_bytes(LM, C, !kFast);
    float4* recW = reinterpret_cast<float4*>(wbase);                     // [C][Q4][32]
    uint4* recF = reinterpret_cast<uint4*>(recW + (size_t)C * Q4 * 32);  // [C][32]
    uint4* meta = recF + (size_t)C * 32;                                 // [2][32]
    float* tD = reinterpret_cast<float*>(meta + 64);                     // [32][36]
    uint8_t* tH = reinterpret_cast<uint8_t*>(tD + 32 * 36);              // [64][36]
    float2* tP = reinterpret_cast<float2*>(tH + 64 * 36);                // [32][34] (P(hap=1) only)
    Staging st;
    st.B = reinterpret_cast<float4*>(reinterpret_cast<unsigned char*>(tP) + (kFast ? 0 : 32 * 34 * 8));
    st.U = reinterpret_cast<double*>(st.B + Q4 * 32);
    st.P = reinterpret_cast<uint32_t*>(st.U + 32);
    st.E = st.P + (C + 1) * 32;

    const uint32_t SG = (A.B + 31) / 32;
    const unsigned long long gw = (unsigned long long)blockIdx.x * nw + warp;
    const uint32_t g = (uint32_t)(gw % SG);
    const uint32_t s = g * 32 + lane;
    const unsigned long long grp = gw / SG;
    bool live = s < A.B && grp * K < A.max_windows;
    View v{};
    uint32_t NA = 0;
    if (live) {
        if (!kPlain) v = view_of(A, s);
        NA = A.counts[s];
    }
    const unsigned long long ab = A.aoff[g] + lane, wb = A.woff[g] + lane;
    const uint32_t NW = (NA + C - 1) / C;
    const uint32_t w0 = live ? (uint32_t)grp * K : 0u;
    const uint32_t wend = min(w0 + K, NW);
    live = live && w0 < wend;
    if (!__any_sync(kAll, live)) return;  // whole warp

    const TypedRegion& R = kPlain ? A.reg0 : v.r;
    const uint32_t len = kPlain ? A.M : v.len;
    const unsigned long long out = kPlain ? (unsigned long long)s * A.M : v.out;
    const Tabs& tb = R.tabs;
    const uint32_t Lr = R.L;
    const uint32_t* apos = A.apos + ab;  // entry k at [32 k]
    const uint32_t* aem = A.aem + ab;
    const bool w_dos = kDos && A.dosage != nullptr, w_hap = A.haps != nullptr;
    const bool w_hp = !kFast && A.hprob != nullptr;
    const bool argmax = kFast || A.sampling == SI_SAMPLE_ARGMAX;
    const float keep = 1.0f - A.tie_eps;

    float2 a2[kBcast ? LM : 1], w2[kBcast ? LM : 1];  // (a'_l, a'_l), (w'_l, w'_l)
    float ap[kBcast ? 1 : LM], wp[kBcast ? 1 : LM];
#pragma unroll
    for (int l = 0; l < LM; ++l) {
        if constexpr (kBcast) { a2[l] = make_float2(0.f, 0.f); w2[l] = make_float2(0.f, 0.f); }
        else { ap[l] = 0.f; wp[l] = 0.f; }
    }
    auto A2 = [&](int l) { if constexpr (kBcast) return a2[l]; else return make_float2(ap[l], ap[l]); };
    auto W2 = [&](int l) { if constexpr (kBcast) return w2[l]; else return make_float2(wp[l], wp[l]); };
    auto a_of = [&](int l) { if constexpr (kBcast) return a2[l].x; else return ap[l]; };
    auto set_a = [&](int l, float x) { if constexpr (kBcast) a2[l] = make_float2(x, x); else ap[l] = x; };
    auto set_w = [&](int l, float x) { if constexpr (kBcast) w2[l] = make_float2(x, x); else wp[l] = x; };
    uint4 fr = make_uint4(0u, kNegInfHi, 0u, 0u);  // the current run's record: farg' lo, hi, end, end emission
    float2 FH = make_float2(0.f, 0.f), FL = make_float2(0.f, 0.f);  // a floor run's farg' as float hi + lo
    uint32_t k = w0 * C, p0 = 0, p1 = 0, m = 0, mend = 0;
    auto load_record = [&](uint32_t r) {
#pragma unroll
        for (uint32_t q = 0; q < Q4; ++q) {
            const float4 x = recW[(r * Q4 + q) * 32 + lane];
            set_w(4 * q, x.x); set_w(4 * q + 1, x.y); set_w(4 * q + 2, x.z); set_w(4 * q + 3, x.w);
        }
        fr = recF[r * 32 + lane];
        if ((fr.y & kInfHi) != kInfHi) {
            const double fa = __hiloint2double((int)fr.y, (int)fr.x);
            const float h = (float)fa, l = (float)(fa - (double)h);
            FH = make_float2(h, h);
            FL = make_float2(l, l);
        }
    };
    if (live) {
        stage_window<LM>(A, apos, aem, wb, NA, w0, st, lane);
        const float4* src = reinterpret_cast<const float4*>(A.ckptF + (wb + 32ull * w0) * LM);
        float x[LM];
#pragma unroll
        for (uint32_t q = 0; q < Q4; ++q) {
            const float4 y = src[q];
            x[4 * q] = y.x; x[4 * q + 1] = y.y; x[4 * q + 2] = y.z; x[4 * q + 3] = y.w;
        }
        const float inv = rcp_approx(vsum<LM>(x));
#pragma unroll
        for (int l = 0; l < LM; ++l) set_a(l, x[l] * inv);
        p0 = apos[32ull * k] & ~kShiftBit;
        mend = wend * C < NA ? (apos[32ull * wend * C] & ~kShiftBit) : len;
        m = p0;
        rebuild_window<LM>(A, tb, NA, len, w0, st, recW, recF, lane);
        if (w0 + 1 < wend) stage_window<LM>(A, apos, aem, wb, NA, w0 + 1, st, lane);
        load_record(0);
        p1 = fr.z;
    }
    bool in_tab = p1 - p0 < tb.NT;  // every i, i+1, j, j-1 of the run index the pair tables

    const bool vec_ok = kPlain && (A.M & 3u) == 0 && !w_hp &&
                        (reinterpret_cast<uintptr_t>(A.dosage) & 15u) == 0 &&
                        (reinterpret_cast<uintptr_t>(A.haps) & 3u) == 0;
    // Write out the tile at absolute columns [tbase, tbase + 32): this lane
    // filled columns [tlo, thi).
    auto flush = [&](uint32_t tbase, uint32_t tlo, uint32_t thi, bool on) {
        __syncwarp();
        const bool has = on && thi > tlo;
        const uint32_t tb0 = __shfl_sync(kAll, tbase, 0);
        if (__all_sync(kAll, vec_ok && has && tlo == 0 && thi == 32 && tbase == tb0)) {
            // every lane filled the same whole tile: 128-bit rows of dosage, 32-bit rows of alleles
            const unsigned long long s0 = s - lane;
            if (w_dos) {
#pragma unroll 4
                for (uint32_t it = 0; it < 8; ++it) {
                    const uint32_t r = it * 4 + (lane >> 3), c = (lane & 7) * 4;
                    const float4 x = *reinterpret_cast<const float4*>(tD + r * 36 + c);
                    *reinterpret_cast<float4*>(A.dosage + (s0 + r) * A.M + tb0 + c) = x;
                }
            }
            if (w_hap) {
#pragma unroll 4
                for (uint32_t it = 0; it < 16; ++it) {
                    const uint32_t rr = it * 4 + (lane >> 3), c = (lane & 7) * 4;
                    const uint32_t x = *reinterpret_cast<const uint32_t*>(tH + rr * 36 + c);
                    *reinterpret_cast<uint32_t*>(A.haps + (2 * (s0 + (rr >> 1)) + (rr & 1)) * A.M + tb0 + c) = x;
                }
            }
        } else {
            const unsigned long long od = out + tbase, oh = 2ull * out + tbase;
            meta[lane] = make_uint4((uint32_t)od, (uint32_t)(od >> 32), (uint32_t)oh, (uint32_t)(oh >> 32));
            meta[32 + lane] = make_uint4(len, tlo, thi, has ? 1u : 0u);
            __syncwarp();
            for (uint32_t r = 0; r < 32; ++r) {
                const uint4 m1 = meta[32 + r];
                if (!m1.w) continue;  // same value in every lane
                const uint4 m0 = meta[r];
                if (lane >= m1.y && lane < m1.z) {
                    const unsigned long long rd = ((unsigned long long)m0.y << 32) | m0.x;
                    const unsigned long long rh = ((unsigned long long)m0.w << 32) | m0.z;
                    if (w_dos) A.dosage[rd + lane] = tD[r * 36 + lane];
                    if (w_hap) {
                        A.haps[rh + lane] = tH[(2 * r) * 36 + lane];
                        A.haps[rh + m1.x + lane] = tH[(2 * r + 1) * 36 + lane];
                    }
                    if (w_hp) reinterpret_cast<float2*>(A.hprob)[rd + lane] = tP[r * 34 + lane];
                }
            }
        }
        __syncwarp();
    };

    // run coefficients of cells (mm, mm + 1): {Q_i, Q_i+1, S_i, S_i+1}, {Q_j, Q_j-1, S_j, S_j-1}
    auto coeffs = [&](uint32_t mm, float4& qa, float4& qb) {
        const uint32_t i = mm - p0, j = p1 - mm;
        if (in_tab) {
            qa = __ldg(tb.QSup + i);
            qb = __ldg(tb.QSdn + j);
        } else {
            const float2 x0 = tabQS(tb, i), x1 = tabQS(tb, i + 1), y0 = tabQS(tb, j), y1 = tabQS(tb, j - 1);
            qa = make_float4(x0.x, x1.x, x0.y, x1.y);
            qb = make_float4(y0.x, y1.x, y0.y, y1.y);
        }
    };

    // cells m (and m + 1 when two) of the current run, into tile columns c0 (, c0 + 1)
    auto cells = [&](uint32_t mm, bool two, const float4 qa, const float4 qb, uint32_t c0) {
        const uint32_t j = p1 - mm;
        float2 XX = make_float2(qb.x, qb.y), YY = make_float2(qb.z, qb.w);
        if (fr.y == kInfHi) {
            YY = make_float2(1.f, 1.f);  // uniform run: w' = 0, beta = 1
        } else if ((fr.y & kInfHi) != kInfHi) {
            // floor e^ft beside Q w' + S, ft = farg' + G(j); when it dominates (ft > 0) scale both by e^-ft
            float2 ft2;
            if (in_tab) {
                // (hi + hi) + (lo + lo) in FP32: where the floor is within reach of the carried
                // terms the high parts nearly cancel, and their sum is exact
                const float4 g = __ldg(tb.Gdn + j);
                ft2 = __fadd2_rn(__fadd2_rn(FH, make_float2(g.x, g.y)), __fadd2_rn(FL, make_float2(g.z, g.w)));
            } else {
                const double fa = __hiloint2double((int)fr.y, (int)fr.x);
                ft2 = make_float2((float)(fa + tabG(tb, j)), (float)(fa + tabG(tb, j - 1)));
            }
            const float ft[2] = {ft2.x, ft2.y};
            float xx[2] = {XX.x, XX.y}, yy[2] = {YY.x, YY.y};
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                const float e = exp2f(fminf(fabsf(ft[c]), 104.f) * -1.44269504088896341f);  // e^-|ft|
                const bool big = ft[c] > 0.f;
                const float xs = big ? e : 1.f;
                const float F = big ? 1.f : (ft[c] > -104.f ? e : 0.f);
                yy[c] = fmaf(yy[c], xs, F);
                xx[c] *= xs;
            }
            XX = make_float2(xx[0], xx[1]);
            YY = make_float2(yy[0], yy[1]);
        }
        const float2 QQ = make_float2(qa.x, qa.y), SS = make_float2(qa.z, qa.w);
        const SlotMasks mkA = R.masks[mm];
        const SlotMasks mkB = two ? R.masks[mm + 1] : mkA;
        const float4* g4 = reinterpret_cast<const float4*>(R.g2 + (size_t)mm * R.gs);
        float2 p2[LM];
#pragma unroll
        for (int l = 0; l < LM; ++l) {
            p2[l] = __fmul2_rn(__ffma2_rn(QQ, A2(l), SS), __ffma2_rn(XX, W2(l), YY));
            if (!kFull && (uint32_t)l >= Lr) p2[l] = make_float2(0.f, 0.f);
        }
        float2 t2[LM / 2];
#pragma unroll
        for (int l = 0; l < LM / 2; ++l) t2[l] = __fadd2_rn(p2[2 * l], p2[2 * l + 1]);
#pragma unroll
        for (int h = LM / 4; h >= 1; h >>= 1)
#pragma unroll
            for (int l = 0; l < h; ++l) t2[l] = __fadd2_rn(t2[l], t2[l + h]);
        const float2 tot2 = t2[0];
        float2 d2 = make_float2(0.f, 0.f);
#pragma unroll
        for (int q = 0; q < LM / 2; ++q) {
            if (kDos && (kFull || (uint32_t)(2 * q) < R.gs)) {
                const float4 gv = __ldg(g4 + q);
                d2 = __ffma2_rn(p2[2 * q], make_float2(gv.x, gv.y), d2);
                d2 = __ffma2_rn(p2[2 * q + 1], make_float2(gv.z, gv.w), d2);
            }
        }
        uint32_t pk[2];
        if (argmax) {
            pick_pair<LM>(p2, keep, pk[0], pk[1]);
        } else {
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                float pc[LM];
#pragma unroll
                for (int l = 0; l < LM; ++l) pc[l] = c ? p2[l].y : p2[l].x;
                const float tot = c ? tot2.y : tot2.x;
                const float target = cell_uniform(A.seed, kPlain ? A.sid_base + s : v.sid,
                                                  (kPlain ? 0u : v.m0) + mm + c) * tot;
                float cum = 0.f;
                uint32_t last_nz = 0, pick = LM;
#pragma unroll
                for (int l = 0; l < LM; ++l) {
                    cum += pc[l];
                    if (pc[l] > 0.f) last_nz = (uint32_t)l;
                    if (pick == LM && target < cum) pick = (uint32_t)l;
                }
                pk[c] = pick == LM ? last_nz : pick;
            }
        }
        const float2 inv2 = make_float2(rcp_approx(tot2.x), rcp_approx(tot2.y));
        const float2 dos2 = __fmul2_rn(d2, inv2);
        const uint32_t hA = slot_alleles(mkA, R.raw, R.gs, mm, pk[0]);
        if (two) {
            const uint32_t hB = slot_alleles(mkB, R.raw, R.gs, mm + 1, pk[1]);
            if constexpr (kDos) *reinterpret_cast<float2*>(tD + lane * 36 + c0) = dos2;
            *reinterpret_cast<uint16_t*>(tH + (2 * lane) * 36 + c0) = (uint16_t)((hA & 0xffu) | ((hB & 0xffu) << 8));
            *reinterpret_cast<uint16_t*>(tH + (2 * lane + 1) * 36 + c0) = (uint16_t)((hA >> 8) | (hB & 0xff00u));
            if (w_hp) {
                float q0[2] = {0.f, 0.f}, q1[2] = {0.f, 0.f};
#pragma unroll
                for (int l = 0; l < LM; ++l) {
                    q0[0] += ((mkA.a0 >> l) & 1u) ? p2[l].x : 0.f;
                    q1[0] += ((mkA.a1 >> l) & 1u) ? p2[l].x : 0.f;
                    q0[1] += ((mkB.a0 >> l) & 1u) ? p2[l].y : 0.f;
                    q1[1] += ((mkB.a1 >> l) & 1u) ? p2[l].y : 0.f;
                }
                *reinterpret_cast<float4*>(tP + lane * 34 + c0) =
                    make_float4(q0[0] * inv2.x, q1[0] * inv2.x, q0[1] * inv2.y, q1[1] * inv2.y);
            }
        } else {
            if constexpr (kDos) tD[lane * 36 + c0] = dos2.x;
            tH[(2 * lane) * 36 + c0] = (uint8_t)(hA & 0xffu);
            tH[(2 * lane + 1) * 36 + c0] = (uint8_t)(hA >> 8);
            if (w_hp) {
                float q0 = 0.f, q1 = 0.f;
#pragma unroll
                for (int l = 0; l < LM; ++l) {
                    q0 += ((mkA.a0 >> l) & 1u) ? p2[l].x : 0.f;
                    q1 += ((mkA.a1 >> l) & 1u) ? p2[l].x : 0.f;
                }
                tP[lane * 34 + c0] = make_float2(q0 * inv2.x, q1 * inv2.x);
            }
        }
    };

    uint32_t tbase = m & ~31u;
    for (;;) {
        const bool on = live && m < mend;
        if (!__any_sync(kAll, on)) break;
        uint32_t tlo = 32, thi = 0;
        if (on) {
            const uint32_t tend = min(tbase + 32, mend);
            tlo = m - tbase;
            while (m < tend) {
                if (m == p1) {
                    // anchor k + 1: alpha steps over the run and takes its emission
                    const uint32_t kn = k + 1, n = p1 - p0, em = fr.w;
                    if (kn % C == 0) {
                        const uint32_t wn = kn / C;
                        rebuild_window<LM>(A, tb, NA, len, wn, st, recW, recF, lane);
                        if (wn + 1 < wend) stage_window<LM>(A, apos, aem, wb, NA, wn + 1, st, lane);
                    }
                    const float2 qs = tabQS(tb, n);
                    float x[LM];
#pragma unroll
                    for (int l = 0; l < LM; ++l) x[l] = a_of(l);
                    const float base = vsum<LM>(x) * qs.y;
#pragma unroll
                    for (int l = 0; l < LM; ++l) x[l] = ((em >> l) & 1u) ? fmaf(qs.x, x[l], base) : 0.f;
                    const float inv = rcp_approx(vsum<LM>(x));
#pragma unroll
                    for (int l = 0; l < LM; ++l) set_a(l, x[l] * inv);
                    load_record(kn % C);
                    k = kn;
                    p0 = p1;
                    p1 = fr.z;
                    in_tab = p1 - p0 < tb.NT;
                }
                // cells [m, e) of the run, two per step when they pair up
                const uint32_t e = min(p1, tend);
                float4 qa, qb;
                coeffs(m, qa, qb);
                while (m < e) {
                    const bool two = (m & 1u) == 0u && m + 1 < e;
                    const uint32_t mn = m + (two ? 2u : 1u);
                    float4 na = qa, nb = qb;
                    if (mn < e) coeffs(mn, na, nb);  // the next step's coefficients in flight
                    cells(m, two, qa, qb, m - tbase);
                    qa = na;
                    qb = nb;
                    m = mn;
                }
            }
            thi = m - tbase;
        }
        flush(tbase, tlo, thi, on);
        tbase += 32;
    }
}

template <int LM, bool kFull, bool kFast, bool kPlain, bool kDos = true>
cudaError_t launch_post_v(const TypedArgs& a, cudaStream_t s) {
    const uint32_t T = a.threads;
    const size_t sm = (size_t)(T / 32) * post_warp_bytes(LM, a.C, !kFast);
    // set outside stream capture only (a plan launches once before it is captured)
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaError_t e = cudaStreamIsCapturing(s, &cs);
    if (e != cudaSuccess) return e;
    if (cs == cudaStreamCaptureStatusNone) {
        e = cudaFuncSetAttribute(anchor_posterior_kernel<LM, kFull, kFast, kPlain, kDos>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e != cudaSuccess) return e;
    }
    const unsigned long long groups = ((unsigned long long)a.max_windows + a.K - 1) / a.K;
    const unsigned long long warps = (unsigned long long)((a.B + 31) / 32) * groups;
    const unsigned long long grid = (warps + T / 32 - 1) / (T / 32);
    if (grid == 0) return cudaSuccess;
    if (grid > 0x7fffffffull) return cudaErrorInvalidConfiguration;
    anchor_posterior_kernel<LM, kFull, kFast, kPlain, kDos><<<(uint32_t)grid, T, sm, s>>>(a);
    return cudaGetLastError();
}

template <int LM, bool kFull>
cudaError_t launch_post(const TypedArgs& a, cudaStream_t s) {
    const bool fast = !a.hprob && a.sampling == SI_SAMPLE_ARGMAX;
    if (fast && !a.dosage)
        return a.samples ? launch_post_v<LM, kFull, true, false, false>(a, s)
                         : launch_post_v<LM, kFull, true, true, false>(a, s);
    if (!a.samples)
        return fast ? launch_post_v<LM, kFull, true, true>(a, s) : launch_post_v<LM, kFull, false, true>(a, s);
    return fast ? launch_post_v<LM, kFull, true, false>(a, s) : launch_post_v<LM, kFull, false, false>(a, s);
}

template <int LM>
cudaError_t launch_typed_lm(const TypedArgs& a, bool full, cudaStream_t s) {
    // a lane per chain, forward and backward warps; one warp per CTA spreads the few warps evenly over the SMs
    const unsigned long long warps = 2ull * ((a.B + 31) / 32);
    anchor_chain_kernel<LM><<<(uint32_t)warps, 32, 0, s>>>(a);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (a.ev_chain_done && (e = cudaEventRecord(a.ev_chain_done, s)) != cudaSuccess) return e;
    return full ? launch_post<LM, true>(a, s) : launch_post<LM, false>(a, s);
}

}  // namespace

// The window (anchors rebuilt from one checkpoint) fixes where rounding
// restarts, so it must not depend on the batch: one value for every L. The
// CTA size changes nothing numerically.
uint32_t typed_default_window(uint32_t) { return 2u; }
uint32_t typed_default_threads(uint32_t lmax) { return lmax <= 16 ? 128u : 64u; }

size_t typed_post_smem_bytes(uint32_t L, uint32_t T, uint32_t C) {
    return (size_t)(T / 32) * post_warp_bytes(fb_lmax(L), C, true);
}

cudaError_t launch_anchor_lists_count(const TypedArgs& a, cudaStream_t s) {
    anchor_count_kernel<<<(a.B + kWarpsPerBlock - 1) / kWarpsPerBlock, kWarpsPerBlock * 32, 0, s>>>(a);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    anchor_scan_kernel<<<1, 1024, 0, s>>>(a.counts, a.B, a.C, a.aoff, a.woff, a.host_totals);
    return cudaGetLastError();
}

cudaError_t launch_anchor_count_only(const TypedArgs& a, cudaStream_t s) {
    anchor_count_kernel<<<(a.B + kWarpsPerBlock - 1) / kWarpsPerBlock, kWarpsPerBlock * 32, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_anchor_lists_fill(const TypedArgs& a, cudaStream_t s) {
    const unsigned long long grid = (unsigned long long)typed_groups(a.B) * a.nseg;  // a warp per CTA
    if (grid == 0) return cudaSuccess;
    if (grid > 0x7fffffffull) return cudaErrorInvalidConfiguration;
    anchor_fill_kernel<<<(uint32_t)grid, 32, kFillSmem, s>>>(a);
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
