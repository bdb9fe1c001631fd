/*
 * swiftimpute_b200.h — C ABI of the B200 Li–Stephens imputation engine.
 *
 * Plain pointers and sizes only; every call returns an si_status and never
 * throws. Host pointers are read/written before the call returns unless a
 * function says otherwise. One si_ctx per device; a ctx is not thread-safe
 * except for the si_serve_* functions.
 *
 * Each entry point names the reference (tcBio/SwiftImpute) interface it
 * replaces, as path:line in the reference source tree.
 */
#ifndef SWIFTIMPUTE_B200_H
#define SWIFTIMPUTE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SI_ABI_VERSION 1

typedef enum {
    SI_OK = 0,
    SI_ERR_INVALID_ARG = 1,   /* bad pointer, size or enum */
    SI_ERR_CUDA = 2,          /* a CUDA runtime call failed; see si_last_error */
    SI_ERR_OUT_OF_MEMORY = 3, /* cudaMalloc failed */
    SI_ERR_UNSUPPORTED = 4,   /* shape or parameter outside what the kernels handle */
    SI_ERR_STATE = 5,         /* call order (e.g. impute before panel upload) */
    SI_ERR_TIMEOUT = 6,       /* a bounded device or host wait gave up */
    SI_ERR_BUDGET = 7,        /* request exceeds the context's HBM budget */
    SI_ERR_CANCELLED = 8      /* serving request cancelled */
} si_status;

typedef struct si_ctx si_ctx;

/* Selection kinds: which reference kernel's pattern to reproduce. AUTO picks
 * as launch_select_states does (pbwt_selector.cu:413-456). FIRST_PAIRS is the
 * reference Imputer's choice without an index or with PBWT selection off:
 * slot k = haplotypes (2k, 2k+1) at every marker (imputer.cpp:929-942); it
 * needs no index and N >= 2L. */
enum { SI_SEL_AUTO = 0, SI_SEL_WARP = 1, SI_SEL_INSERTION = 2, SI_SEL_FIRST_PAIRS = 3, SI_SEL_TARGET = 4 };
/* SI_SEL_TARGET (opt-in; changes results, so never the default): slots chosen
 * per target from the haplotypes that match it longest, the way Durbin's PBWT
 * follows an inserted sequence. It replaces the positional patterns of
 * PBWTIndex::select_states (pbwt_index.cpp:20-79), whose divergences all equal
 * m. The target's pseudo-haplotype carries 0 at code 0, 1 at code 2, and
 * elsewhere the allele of the panel haplotype at its position in the order;
 * its position p moves as z(p) (allele 0) or Z + p - z(p) (allele 1), with Z
 * the zeros at the marker and z(p) those among the first p entries of the
 * previous order (the target goes before equal keys). Slots: the L haplotypes
 * at positions clamp(p - L/2, 0, N - L) .. + L of the marker's order, paired
 * (h, (h + 1) % N). Needs the index built with SI_PBWT_STORE_INDEX and a panel
 * of 0/1 alleles; si_impute / si_impute_device run it through the full-chain
 * kernel with each target's own slots ([M][B] slot masks of scratch). */

/* Transition modes. MATRIX0 reproduces the reference, whose forward-backward
 * reads the first gap's matrix for every gap (forward_backward.cu:108,201,234,269).
 * PER_GAP uses each gap's own matrix. */
enum { SI_TRANS_MATRIX0 = 0, SI_TRANS_PER_GAP = 1 };

/* Haplotype output: argmax slot (sampling.cu:138-182 with a tie tolerance) or
 * a draw from the posterior with a counter-based Philox4x32-10 stream keyed by
 * (seed, sample id, marker), so a sample's draw never depends on its batch. */
enum { SI_SAMPLE_ARGMAX = 0, SI_SAMPLE_PHILOX = 1 };

/* si_pbwt_build flags */
enum {
    SI_PBWT_STORE_INDEX = 1u,  /* keep the full prefix array [M][N] u32 on the device */
    SI_PBWT_ROW_HASHES = 2u    /* keep a 64-bit hash of every prefix row */
};

/* si_impute_params.flags */
enum {
    SI_IMPUTE_RESELECT = 1u,    /* recompute the per-marker selection tables in this call (else cached per L) */
    SI_IMPUTE_FULL_CHAIN = 2u,  /* use the marker-by-marker kernel even where the typed-marker kernel applies */
    /* Compact host formats of si_impute (host-buffer call only): */
    SI_IMPUTE_CODES_2BIT = 4u,  /* geno is [B][ceil(M/4)] bytes, cell m at bits 2 (m % 4) of byte m / 4 */
    SI_IMPUTE_HAPS_BITS = 8u    /* haps is [B][2][ceil(M/32)] u32 words, allele of marker m at bit m % 32 of
                                   word m / 32 (set for a non-zero allele; 0/1 panels only) */
};

/* Genotype codes for si_impute: 0, 1, 2 = ALT allele count of a hard call,
 * 3 = missing (the reference's GL triple {0,0,0}, imputer.cpp:253-267). */
enum { SI_GENO_MISSING = 3 };

typedef struct {
    uint32_t num_states;          /* L, 1..32 (HMMParameters::num_states, core/types.hpp:81) */
    uint32_t ne;                  /* effective population size (HMMParameters::ne) */
    double rho_rate;              /* HMMParameters::rho_rate (default 4.0) */
    double theta;                 /* HMMParameters::theta (unused by the reference kernels) */
    int32_t transition_mode;      /* SI_TRANS_* */
    int32_t selection_kind;       /* SI_SEL_* */
    int32_t sampling;             /* SI_SAMPLE_* */
    uint32_t flags;               /* SI_IMPUTE_* */
    double tie_eps;               /* argmax picks the first slot with p >= (1 - tie_eps) * max p */
    uint64_t seed;                /* Philox key */
    uint64_t sample_id_base;      /* Philox counter: sample id of row 0 */
    uint32_t checkpoint_interval; /* full-chain kernel: markers per checkpoint segment; typed-marker
                                     kernel: typed markers per posterior window; 0 = default */
    uint32_t block_threads;       /* threads per CTA; 0 = default */
    uint64_t reserved[4];
} si_impute_params;

/* Library / context ------------------------------------------------------ */

int si_abi_version(void);
const char* si_status_string(si_status s);

/* Replaces Imputer::initialize_gpu (imputer.cpp:555-567). hbm_budget_bytes = 0
 * means "all free memory". */
si_status si_ctx_create(int device, uint64_t hbm_budget_bytes, si_ctx** out);
si_status si_ctx_destroy(si_ctx* ctx);
/* Message of the last failed call on this ctx (never NULL). */
const char* si_last_error(const si_ctx* ctx);
/* Replaces Imputer::device_memory_usage (imputer.cpp:1176-1212). */
si_status si_ctx_memory(const si_ctx* ctx, uint64_t* used_bytes, uint64_t* budget_bytes);

/* Panel ------------------------------------------------------------------ */

/* Upload a u8 panel [M][N] (ReferencePanel::haplotypes(), imputer.hpp:86).
 * Any byte is accepted, as the reference stores it (imputer.cpp:85-112):
 * ALLELE_MISSING = 255 for '.', the allele index for multi-allelic calls. The
 * device keeps one bit per allele (set for a non-zero byte, the side the
 * reference's PBWT sorts it to, pbwt_index.cpp:183) and, per marker, a list of
 * the bytes other than 0 and 1 (N < 2^24 when there are any). Emission classes
 * follow the byte sum (emission.cu:35-54), sampled haplotypes carry the panel
 * byte (sampling.cu:121-126), and dosage and P(hap=1) count non-zero alleles.
 * Replaces the panel copies of EmissionComputer::set_reference_panel
 * (emission.cu:189) and HaplotypeSampler::set_reference_panel (sampling.cu:219). */
si_status si_panel_upload_u8(si_ctx* ctx, const uint8_t* alleles, uint32_t M, uint32_t N);

/* Number of panel entries other than 0 and 1 in the uploaded panel. */
si_status si_panel_exception_count(const si_ctx* ctx, uint64_t* count);

/* Upload an already bit-packed panel [M][words_per_row] u32: bit i of word w
 * is haplotype 32 w + i (alleles 0 and 1 only). words_per_row >= ceil(N / 32). */
si_status si_panel_upload_packed(si_ctx* ctx, const uint32_t* words, uint32_t M, uint32_t N,
                                 uint32_t words_per_row);

/* Marker positions for the genetic map: Morgans = cM / 100 where cM > 0, else
 * pos / 1e8, as Imputer::initialize_gpu_kernels (imputer.cpp:596-604).
 * cM may be NULL. Replaces TransitionComputer::set_genetic_map (transition.cu:218). */
si_status si_panel_set_map(si_ctx* ctx, const uint64_t* pos, const double* cM);

/* PBWT ------------------------------------------------------------------- */

/* Run the PBWT prefix sweep on the device. Replaces Imputer::build_index
 * (imputer.cpp:706-728) -> PBWTIndex::build (pbwt_index.cpp:12) and
 * GPUStateSelector::transfer_index_to_device (pbwt_index.cpp:355). The
 * divergence array of the reference is m in every entry of row m
 * (pbwt_index.cpp:173-191), so it is implicit. */
si_status si_pbwt_build(si_ctx* ctx, uint32_t flags);

/* Copy prefix rows [m0, m0 + count) to host out [count][N]. Needs
 * SI_PBWT_STORE_INDEX. Replaces PBWTIndex::prefix() (pbwt_index.hpp:61). */
si_status si_pbwt_get_prefix_rows(si_ctx* ctx, uint32_t m0, uint32_t count, uint32_t* out);

/* Copy the per-row hashes [M] (needs SI_PBWT_ROW_HASHES). */
si_status si_pbwt_row_hashes(si_ctx* ctx, uint64_t* out);

/* Milliseconds of the last si_pbwt_build sweep (CUDA events). */
si_status si_pbwt_last_ms(const si_ctx* ctx, float* ms);

/* Stored index. Replace save_pbwt_index / load_pbwt_index (declared in
 * pbwt_index.hpp:257-258, never defined by the reference). The stored form is
 * the part of the index selection reads, the first 128 prefix entries of every
 * marker (M * 512 bytes plus a 32-byte header), with the panel's shape and a
 * checksum of its bits: si_pbwt_load refuses it for any other panel. */
si_status si_pbwt_stored_bytes(const si_ctx* ctx, uint64_t* bytes);
si_status si_pbwt_save(si_ctx* ctx, void* out, uint64_t bytes);
si_status si_pbwt_load(si_ctx* ctx, const void* in, uint64_t bytes);

/* Selection -------------------------------------------------------------- */

/* Slots of markers [m0, m1) as haplotype pairs out [m1-m0][L][2], the result
 * of launch_select_states (pbwt_selector.cu:400) followed by the host pair
 * expansion (h, (h + 1) % N) (imputer.cpp:863-874). The selection does not
 * depend on the target sample, so it is computed once per marker. */
si_status si_select_states(si_ctx* ctx, uint32_t L, int32_t kind, uint32_t m0, uint32_t m1,
                           uint32_t* out_pairs);

/* SI_SEL_TARGET slots of B targets: codes [B][M] (host), pairs out
 * [B][M][L][2] (host), L <= 32. No reference counterpart (the reference's
 * selection is the same for every target). */
si_status si_select_states_target(si_ctx* ctx, uint32_t L, const uint8_t* geno_codes, uint32_t B,
                                  uint32_t* out_pairs);

/* Imputation ------------------------------------------------------------- */

si_status si_impute_params_default(si_impute_params* p);

/* Impute B samples over all M markers from HOST buffers (copies inside).
 * geno [B][M] genotype codes (with SI_IMPUTE_CODES_2BIT: [B][ceil(M/4)] bytes,
 * four codes per byte). Outputs (each may be NULL):
 *   dosage   [B][M]     posterior ALT dosage
 *   hap_prob [B][M][2]  P(hap0 = 1), P(hap1 = 1) (ImputationResult::posteriors_, imputer.hpp:192)
 *   haps     [B][2][M]  phased alleles (ImputationResult::haplotypes_, imputer.hpp:191); with
 *                       SI_IMPUTE_HAPS_BITS: [B][2][ceil(M/32)] u32 words (cast the pointer)
 * The compact formats are converted on the device, so only their bytes cross
 * the host link (0.5 B per cell for codes in and haplotypes out).
 * Replaces Imputer::impute_batch (imputer.cpp:787-1042): selection, emission
 * (emission.cu:208), forward/backward (forward_backward.cu:321,356) and
 * HaplotypeSampler::sample (sampling.cu:269) run as one fused device pass. */
si_status si_impute(si_ctx* ctx, const si_impute_params* p, const uint8_t* geno, uint32_t B,
                    float* dosage, float* hap_prob, uint8_t* haps);

/* Same, from reference-layout genotype likelihoods gl [B][M][3] (log10,
 * TargetData::genotype_likelihoods(), imputer.hpp:125). Cells whose three
 * values are equal are missing; cells with one 0 and two -999 are hard calls;
 * any other triple is SI_ERR_UNSUPPORTED. */
si_status si_impute_gl(si_ctx* ctx, const si_impute_params* p, const float* gl, uint32_t B,
                       float* dosage, float* hap_prob, uint8_t* haps);

/* Device-pointer variant: all buffers are device memory owned by the caller,
 * work is queued on `stream` (a cudaStream_t, may be NULL). With the default
 * transition mode the call waits once on `stream` for a 16-byte count (the
 * size of the per-sample typed-marker lists) before queueing the rest, then
 * returns without a further synchronisation. Scratch memory comes from the ctx. */
si_status si_impute_device(si_ctx* ctx, const si_impute_params* p, const uint8_t* d_geno, uint32_t B,
                           float* d_dosage, float* d_hap_prob, uint8_t* d_haps, void* stream);

/* Allocation-free variant of si_impute_device. It has no counterpart in the
 * reference. It is for callers that cannot call cudaMalloc while they impute:
 * programs whose device memory belongs to another allocator (a framework's
 * pool that reserves the free memory and forbids raw allocations beside it),
 * and latency-bound programs that share the device with other streams, where
 * cudaMalloc/cudaFree may synchronise the device. The caller passes device
 * inputs and outputs; the forward checkpoints live in a fixed 16 MiB array
 * inside the library (held by every GPU that loads it, until exit).
 * It always runs the marker-by-marker (full-chain) recursion, whatever the
 * transition mode; flags other than SI_IMPUTE_FULL_CHAIN are refused. Results
 * agree with si_impute_device within the parity tolerance (1e-4 in dosage),
 * not bit for bit, where that call takes the typed-marker path.
 * Checkpoint bytes: max(ceil(M / C) - 1, 1) * Lmax * B * 4, with C =
 * checkpoint_interval or 32 markers (16 for L > 16) and Lmax = L rounded up to
 * 4/8/16/32; more than 16 MiB is refused with SI_ERR_UNSUPPORTED. The ctx must
 * hold the slot and transition tables for these parameters: make one
 * allocating call (si_impute or si_impute_device) with them first, and let it
 * complete. The first call on a ctx is its set-up: it looks up the array's
 * device address (with lazy module loading, that is also when the driver
 * commits the array's memory); make that call before any stream capture.
 * After a device reset, create a new ctx. Calls share the array, so calls
 * whose kernels overlap on the GPU race; serialise them on one stream.
 * si_last_timings / si_last_kernel_ms do not cover this entry point: after it
 * they still report the last allocating call. */
si_status si_impute_device_noalloc(si_ctx* ctx, const si_impute_params* p, const uint8_t* d_geno, uint32_t B,
                                   float* d_dosage, float* d_hap_prob, uint8_t* d_haps, void* stream);

/* Uneven batches ----------------------------------------------------------
 * One launch sequence over targets that cover different marker ranges
 * (regions) with different slot counts. A region is a contiguous panel slice
 * [m_begin, m_end) imputed with num_states slots. Its selection comes either
 * from the resident index (SI_INDEX_GLOBAL: the PBWT swept from marker 0, as
 * the serving loop uses it) or from a sweep restarted at m_begin
 * (SI_INDEX_REGION: what the reference computes when run on the sliced panel,
 * ReferencePanel::load_vcf(filename, region), imputer.cpp:27-44, including
 * the slice's own first-gap transition matrix). A GLOBAL region uses the
 * panel's first-gap matrix, like a full-panel imputation. Each job is one target of one region: its codes are the
 * (m_end - m_begin) bytes at geno + geno_offset; its outputs are packed at
 * out_offset: dosage[out_offset + i], hap_prob[2 (out_offset + i) + phase],
 * haps[2 out_offset + i] (hap0) and haps[2 out_offset + len + i] (hap1).
 * Philox draws are keyed by (seed, sample_id, absolute marker), so a job's
 * draws do not depend on the rest of the batch. */
enum { SI_INDEX_GLOBAL = 0, SI_INDEX_REGION = 1 };

typedef struct {
    uint32_t m_begin;
    uint32_t m_end;
    uint32_t num_states;   /* 1..32 */
    int32_t index_origin;  /* SI_INDEX_* */
} si_region;

typedef struct {
    uint32_t region;
    uint32_t reserved;
    uint64_t geno_offset;
    uint64_t out_offset;
    uint64_t sample_id;
} si_job;

/* Device buffers; regions and jobs are host arrays. params->num_states is
 * ignored (each region has its own); params->transition_mode must be
 * SI_TRANS_MATRIX0. */
si_status si_impute_jobs_device(si_ctx* ctx, const si_impute_params* p, const si_region* regions, uint32_t n_regions,
                                const si_job* jobs, uint32_t n_jobs, const uint8_t* d_geno, float* d_dosage,
                                float* d_hap_prob, uint8_t* d_haps, void* stream);

/* Milliseconds of the last si_impute* device work (CUDA events): [0] selection,
 * [1] forward-backward kernel, [2] whole call including copies (host-buffer
 * calls only). For si_impute_device this waits for the call's kernels. */
si_status si_last_timings(si_ctx* ctx, float* ms3);

/* Milliseconds of each kernel stage of the last si_impute* call (CUDA events on
 * its stream): [0] selection, [1] typed-marker lists, [2] anchor chain,
 * [3] posterior pass (or the whole full-chain kernel). Waits for the call. */
si_status si_last_kernel_ms(si_ctx* ctx, float* ms4);

/* ---- Plans: a fixed uneven batch launched with no host work in between.
 *
 * No counterpart in the reference, which sizes and launches each batch from
 * the host (imputer.cpp:787-1042). si_impute_jobs_device reads the number of
 * typed markers back from the device before it sizes its lists; a plan fixes
 * each job's anchor capacity up front (max_anchors = 0: the job's marker
 * count; else min(marker count, max_anchors), which must cover marker 0 plus
 * the typed markers, e.g. the typed sites of a genotyping array + 1), owns its
 * scratch, and holds the device pointers given here. si_plan_launch queues
 * four kernels with fixed arguments and no host synchronisation, so it can be
 * captured into a CUDA graph; si_plan_graph_launch captures it once and
 * replays the graph. Rewrite the codes in d_geno between launches. A plan
 * reads the ctx's panel, index and selection tables: it stays valid while they
 * are unchanged and no server runs on the ctx.
 * SI_PLAN_AUTOTUNE (with params checkpoint_interval and block_threads 0)
 * times the launch on this batch for each window size (anchors per
 * checkpoint) and posterior CTA size and keeps the fastest. */
typedef struct si_plan si_plan;
enum { SI_PLAN_AUTOTUNE = 1u };
si_status si_plan_create(si_ctx* ctx, const si_impute_params* params, const si_region* regions, uint32_t n_regions,
                         const si_job* jobs, uint32_t n_jobs, uint32_t max_anchors, const uint8_t* d_geno,
                         float* d_dosage, float* d_hap_prob, uint8_t* d_haps, uint32_t flags, si_plan** out);
si_status si_plan_launch(si_plan* plan, void* stream);
si_status si_plan_graph_launch(si_plan* plan, void* stream);
/* Wait for the device; SI_ERR_BUDGET if a job since the last check had more
 * anchors than its capacity (it was cut to it; nothing outside the plan's
 * buffers was touched). */
si_status si_plan_check(si_plan* plan);
si_status si_plan_info(const si_plan* plan, uint32_t* window, uint32_t* threads, float* tuned_ms);
si_status si_plan_destroy(si_plan* plan);

/* ---- Serving: requests of any size over a resident panel and index.
 *
 * The reference imputes one target set per Imputer::impute call
 * (imputer.cpp:787-1042, batches of max_batch_size over one panel) and has no
 * request queue. A server owns a ctx (panel, map and PBWT index already set
 * up) and one worker thread. Requests are queued from any thread; the worker
 * forms each launch from the queue in arrival order (continuous batching: a
 * request that arrives while a launch runs joins the next one), admits
 * requests while the launch stays within max_batch_cells and within the ctx's
 * HBM budget, and runs them as one uneven batch (si_impute_jobs_device), so a
 * request's results never depend on the requests beside it. While a server
 * runs, no other call may use its ctx. */
typedef struct si_server si_server;

typedef struct {
    uint64_t max_batch_cells;  /* samples x markers per launch; 0 = 2^25. Both staging slots
                                  (7 B per cell pinned and on the device) are allocated at start */
    uint32_t max_wait_us;      /* how long the oldest queued request waits for company; 0 = 200 */
    uint32_t max_queue;        /* queued requests before si_serve_submit refuses; 0 = 65536 */
    uint32_t max_batch_requests; /* requests per launch; 0 = no limit (1 = one request per launch) */
    uint32_t reserved;
} si_serve_config;

typedef struct {
    uint32_t m_begin, m_end;   /* panel markers [m_begin, m_end) */
    uint32_t num_states;       /* L, 1..32 */
    int32_t index_origin;      /* SI_INDEX_* (as si_region) */
    uint32_t n_samples;
    uint32_t reserved;
    uint64_t sample_id_base;   /* Philox id of the first sample; sample i uses base + i */
    const uint8_t* codes;      /* host [n_samples][m_end - m_begin] genotype codes */
    float* dosage;             /* host [n_samples][len], or NULL */
    uint8_t* haps;             /* host [n_samples][2][len], or NULL */
    float* hap_prob;           /* host [n_samples][len][2], or NULL */
} si_request;

typedef struct {
    uint64_t submitted, completed, failed, cancelled, batches, cells;
    double latency_p50_ms, latency_p99_ms, latency_max_ms;  /* submit -> finished, completed requests */
    double busy_ms;            /* worker time inside launches (copies included) */
    double wall_ms;            /* since si_serve_start */
} si_serve_statistics;

/* Start a server on ctx with fixed imputation parameters (num_states is taken
 * from each request). params->transition_mode must be SI_TRANS_MATRIX0. */
si_status si_serve_start(si_ctx* ctx, const si_impute_params* params, const si_serve_config* cfg, si_server** out);
/* Queue a request. Its host buffers must stay valid until it finishes. A
 * request larger than max_batch_cells, or than the HBM budget allows alone,
 * is refused here with SI_ERR_BUDGET. Thread-safe. */
si_status si_serve_submit(si_server* srv, const si_request* req, uint64_t* ticket);
/* *finished = 1 once the request has finished; *result is then its status
 * and the ticket is released. Thread-safe, never blocks on the device. */
si_status si_serve_poll(si_server* srv, uint64_t ticket, int* finished, si_status* result);
/* Wait up to timeout_ms (0 = no limit) for the request; SI_ERR_TIMEOUT if it
 * is still running (the ticket stays valid). Thread-safe. */
si_status si_serve_wait(si_server* srv, uint64_t ticket, uint32_t timeout_ms, si_status* result);
/* Cancel a queued request (it finishes as SI_ERR_CANCELLED, outputs untouched);
 * SI_ERR_STATE if it is already in a launch or finished. Thread-safe. */
si_status si_serve_cancel(si_server* srv, uint64_t ticket);
si_status si_serve_stats(si_server* srv, si_serve_statistics* out);
/* Cancel queued requests, finish the running launch, join the worker, free the
 * server's buffers. The ctx is usable again afterwards. */
si_status si_serve_stop(si_server* srv);

#ifdef __cplusplus
}
#endif
#endif
