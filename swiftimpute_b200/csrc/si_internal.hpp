// si_internal.hpp — device context shared by the C ABI translation units.
#pragma once

#include "../../include/swiftimpute_b200.h"

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <cstdint>
#include <map>
#include <tuple>
#include <string>
#include <utility>
#include <vector>

namespace si {

// A named host range for profiler timelines (NVTX, header-only); without an
// attached tool each push and pop is a few nanoseconds.
struct Range {
    explicit Range(const char* name) { nvtxRangePushA(name); }
    ~Range() { nvtxRangePop(); }
    Range(const Range&) = delete;
    Range& operator=(const Range&) = delete;
};

// Bit-packed panel row: ceil(N / 32) words, padded to a multiple of 4 so every
// row starts on a 16-byte boundary (128-bit loads, bulk copies).
inline uint32_t words_per_row_pad(uint32_t N) { return ((N + 31) / 32 + 3) & ~3u; }

// Number of prefix entries kept per marker for selection: the warp pattern
// reads positions 0, 32, 64, 96 and the insertion pattern positions 0..L-1
// (L <= 64), so the first 128 entries of each row cover every pattern.
constexpr uint32_t kHead = 128;
constexpr uint32_t kMaxMarkers = 0x80000000u;  // anchor lists keep a flag in bit 31 of a position

// Per-marker slot data consumed by the forward-backward kernels: for slot k,
// bit k of a0 / a1 is set when the pair's first / second haplotype carries a
// non-zero allele (the PBWT's "1" side), and bit k of x when either of its
// alleles is neither 0 nor 1 (missing, 255, or multi-allelic); such slots take
// their allele bytes from the selection's raw table.
struct alignas(16) SlotMasks {
    uint32_t a0;
    uint32_t a1;
    uint32_t x;
    uint32_t pad;
};

// Linear-space transition into a marker: T[i][j] = c + delta * [i == j], with
// c = exp(log10 switch) and c + delta = exp(log10 stay) as the reference's
// log10 values are consumed by natural-log recursions.
struct LinTrans {
    float c;
    float delta;
};

// A PBWT sweep over panel rows [m0, m0 + len), head rows written at head + head_off.
struct SweepJob {
    uint32_t m0;
    uint32_t len;
    uint64_t head_off;
    uint64_t init_off;  // the order before m0: init[init_off .. init_off + N), or kIota for 0 .. N-1
};
constexpr uint64_t kIota = ~0ull;

struct DeviceBuffer {
    void* ptr = nullptr;
    size_t bytes = 0;
};

struct SelectionCache {
    uint32_t L = 0;
    int kind = 0;
    DeviceBuffer pairs;  // [M][L][2] u32
    DeviceBuffer masks;  // [M] SlotMasks
    DeviceBuffer g2;     // [M][fb_lmax(L)] f32x2 non-zero alleles per slot at m and m + 1
    DeviceBuffer raw;    // [M][fb_lmax(L)][2] u8 allele bytes (panels with alleles other than 0/1 only)
};

}  // namespace si

struct si_ctx {
    int device = 0;
    uint64_t budget = 0;
    uint64_t used = 0;
    std::string err;
    cudaStream_t stream = nullptr;
    cudaStream_t copy_in = nullptr, copy_out = nullptr;  // host-buffer calls: copies beside the compute
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    cudaEvent_t kev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};  // per-kernel timing of the last call
    float kernel_ms[4] = {0.f, 0.f, 0.f, 0.f};
    bool kernel_pending = false;

    // panel
    uint32_t M = 0, N = 0, W = 0;
    si::DeviceBuffer panel;          // [M][W] u32 bit-packed (bit set: non-zero allele)
    // alleles other than 0 and 1, per marker sorted by haplotype: entry h << 8 | byte
    si::DeviceBuffer ex_off;         // [M + 1] u64 offsets into ex_ent
    si::DeviceBuffer ex_ent;         // [n_ex] u32
    uint64_t n_ex = 0;
    std::vector<double> morgans;     // genetic position per marker
    bool has_map = false;

    // PBWT
    bool has_index = false;
    uint32_t pbwt_flags = 0;
    si::DeviceBuffer head;           // [M][kHead] u32, first entries of each prefix row
    si::DeviceBuffer prefix;         // [M][N] u32 (SI_PBWT_STORE_INDEX)
    si::DeviceBuffer row_hash;       // [M] u64 (SI_PBWT_ROW_HASHES)
    si::DeviceBuffer rank_bits;      // [M][W] target-aware selection rank tables (built on first use)
    si::DeviceBuffer rank_zeros;     // [M][W+1]
    float pbwt_ms = 0.f;

    // selection, keyed by (L, kind)
    std::map<std::pair<uint32_t, int>, si::SelectionCache> sel;

    // imputation scratch, grown on demand
    si::DeviceBuffer trans;          // [M] LinTrans
    uint64_t trans_key = ~0ull;
    si::LinTrans trans0{1.f, 0.f};  // host copy of the first gap's transition
    si::DeviceBuffer ckpt;           // forward checkpoints (full-chain kernel)
    si::DeviceBuffer smasks;         // per-target slot masks [M][B] (target-aware selection)
    // typed-marker kernel scratch and tables
    si::DeviceBuffer t_counts, t_segc, t_aoff, t_woff, t_apos, t_aem, t_ckF, t_ckB, t_ckU;
    struct TableSet {
        si::DeviceBuffer QS, G;
        double consts[4] = {0, 0, 0, 0};  // log2q, lr, lgc, regime
    };
    std::map<uint64_t, TableSet> tables;  // closed-form run tables per (transition, L)
    // region-local selection tables (index restarted at the region start), per (m_begin, m_end, L, kind)
    struct RegionSel {
        si::DeviceBuffer masks;
        si::DeviceBuffer g2;
        si::DeviceBuffer raw;
    };
    std::map<std::tuple<uint32_t, uint32_t, uint32_t, int>, RegionSel> region_sel;
    si::DeviceBuffer job_regions, job_samples;  // uploaded descriptors of the last uneven batch
    unsigned long long* pinned_totals = nullptr;  // mapped [4]: written by the scan kernel
    unsigned long long* pinned_totals_dev = nullptr;
    cudaEvent_t totals_ev = nullptr;
    si::DeviceBuffer io_geno, io_dosage, io_hprob, io_haps;  // staging for host-buffer calls
    si::DeviceBuffer io_geno2, io_hbits;                     // compact host formats (2-bit codes, haplotype bits)
    float last_ms[3] = {0.f, 0.f, 0.f};
    bool timings_pending = false;
    void* noalloc_scratch = nullptr;  // device address of the allocation-free path's fixed array
};

namespace si {

// Allocation under the ctx's HBM budget.
si_status dev_alloc(si_ctx* ctx, DeviceBuffer& buf, size_t bytes);
void dev_free(si_ctx* ctx, DeviceBuffer& buf);
// Grow-only scratch: keep the buffer if it is already large enough; a regrown
// buffer takes 1.5x its old size when the budget allows.
si_status dev_reserve(si_ctx* ctx, DeviceBuffer& buf, size_t bytes);
si_status fail(si_ctx* ctx, si_status s, const std::string& msg);
si_status cuda_fail(si_ctx* ctx, cudaError_t e, const char* what);
// Whether the first-gap transition of markers [m_begin, m_end) has a switch
// weight the FP32 closed form can carry (false when the first two markers
// share a genetic position). Reads only the ctx's map and writes nothing, so
// threads other than the ctx's user may call it.
bool region_first_gap_ok(const si_ctx* ctx, const si_impute_params* p, uint32_t m_begin, uint32_t m_end);

// Kernel launchers (pbwt_kernels.cu, select_kernels.cu, fb_kernels.cu).
cudaError_t launch_pack_panel(const uint8_t* d_u8, uint32_t M, uint32_t N, uint32_t W, uint32_t* d_words,
                              cudaStream_t s);
// d_init: the orders jobs with init_off != kIota start from (may be null when none does)
cudaError_t launch_pbwt_sweep(const uint32_t* d_panel, const SweepJob* d_jobs, uint32_t n_jobs, uint32_t N,
                              uint32_t W, const uint32_t* d_init, uint32_t* d_head, uint32_t* d_prefix,
                              unsigned long long* d_hash, uint32_t* d_perm_scratch, cudaStream_t s);
size_t pbwt_sweep_smem_bytes(uint32_t N, uint32_t W);
size_t pbwt_group_smem_bytes(uint32_t N, uint32_t W);
// Segmented whole-panel sweep (pbwt_kernels.cu): per segment the groups of
// haplotypes equal over its markers, swept from 0 .. N-1 (d_gid [n_jobs][N],
// by haplotype; d_scratch 4 N words per job), and the composition of an order
// with one segment's groups (a stable sort by group; d_sortbuf 4 N words).
cudaError_t launch_pbwt_groups(const uint32_t* d_panel, const SweepJob* d_jobs, uint32_t n_jobs, uint32_t N,
                               uint32_t W, uint32_t* d_gid, uint32_t* d_scratch, cudaStream_t s);
cudaError_t launch_pbwt_compose(const uint32_t* d_order, const uint32_t* d_gid, uint32_t* d_next, uint32_t N,
                                uint32_t* d_sortbuf, cudaStream_t s);
cudaError_t launch_iota(uint32_t* d, uint32_t N, cudaStream_t s);
cudaError_t launch_panel_checksum(const uint32_t* d_words, uint64_t n, unsigned long long* d_out, cudaStream_t s);
// Selection over markers [0, M) of the given panel rows; ex_off/ex_ent (may be
// null) are the rows' exception lists, raw (may be null) receives allele bytes.
cudaError_t launch_select(const uint32_t* d_head, const uint32_t* d_panel, uint32_t M, uint32_t N, uint32_t W,
                          uint32_t L, int kind, const unsigned long long* d_ex_off, const uint32_t* d_ex_ent,
                          uint32_t* d_pairs, SlotMasks* d_masks, float2* d_g2, uint8_t* d_raw, uint32_t gs,
                          cudaStream_t s);

// Compact host formats (formats.cu): 2-bit codes [rows][ceil(M/4)] -> bytes
// [rows][M]; allele bytes [rows][M] -> bit words [rows][ceil(M/32)].
cudaError_t launch_unpack_codes(const uint8_t* d_in, uint64_t rows, uint32_t M, uint8_t* d_out, cudaStream_t s);
cudaError_t launch_pack_haps(const uint8_t* d_in, uint64_t rows, uint32_t M, uint32_t* d_out, cudaStream_t s);

struct FbLaunch {
    const uint8_t* geno;   // [B][M]
    const SlotMasks* masks;
    const SlotMasks* smasks;  // per-target masks [M][B] (target-aware selection), or null: masks per marker
    const uint8_t* raw;    // [M][fb_lmax(L)][2] allele bytes, or null (0/1 panel)
    const LinTrans* trans;
    uint32_t B, M, L, C;
    uint32_t threads;
    int sampling;
    float tie_eps;
    uint64_t seed, sample_id_base;
    float* ckpt;           // [B][nseg][Lmax]
    float* dosage;         // [B][M] or null
    float* hprob;          // [B][M][2] or null
    uint8_t* haps;         // [B][2][M] or null
};
cudaError_t launch_fb(const FbLaunch& a, cudaStream_t s);
// Target-aware selection (select_kernels.cu): rank tables [M][W] bits and
// [M][W+1] zero counts from the stored prefix rows, then per target the slot
// masks smasks[m][s] (and, if d_pairs, the pairs [s][m][L][2]).
cudaError_t launch_target_ranks(const uint32_t* d_prefix, const uint32_t* d_panel, uint32_t M, uint32_t N, uint32_t W,
                                uint32_t* d_bits, uint32_t* d_zeros, cudaStream_t s);
cudaError_t launch_target_select(const uint8_t* d_geno, uint32_t B, uint32_t M, uint32_t N, uint32_t W, uint32_t L,
                                 const uint32_t* d_prefix, const uint32_t* d_panel, const uint32_t* d_bits,
                                 const uint32_t* d_zeros, SlotMasks* d_smasks, uint32_t* d_pairs, cudaStream_t s);
size_t fb_ckpt_bytes(uint32_t B, uint32_t M, uint32_t L, uint32_t C);
// slots held per thread (and the stride of per-slot tables) for L slots
inline __host__ __device__ uint32_t fb_lmax(uint32_t L) { return L <= 4 ? 4 : L <= 8 ? 8 : L <= 16 ? 16 : 32; }
size_t fb_smem_bytes(uint32_t L, uint32_t T, uint32_t C);

}  // namespace si
