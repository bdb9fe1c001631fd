// noalloc.cu — imputation entry point that performs no device allocation.
//
// For callers that cannot call cudaMalloc at the point where they impute: a
// host program whose device memory is owned by another allocator (a
// framework's memory pool that reserves the free memory up front and forbids
// raw allocations beside it), and latency-bound callers that share the device
// with other streams (cudaMalloc and cudaFree may synchronise the device, which
// stalls the other streams' work). The caller allocates inputs and outputs;
// the forward checkpoints, the only scratch this path needs, live in a fixed
// array compiled into the library.
//
// The array below is a file-scope __device__ variable: every GPU that loads
// this library holds kNoAllocScratchBytes of it until the process exits. In
// host code its name is only a host-side stand-in, so its device address is
// looked up with cudaGetSymbolAddress (with the ctx's device current) by the
// first call on a ctx, and kept in the ctx. A ctx lives in one CUDA context:
// after a device reset the caller creates a new ctx, whose first call looks
// the address up again. All calls share the array: a call leaves its
// checkpoints there, and calls whose kernels overlap on the GPU (different
// streams, or different host threads) race on it. Checkpoints are written
// before they are read within a call, so nothing needs clearing.
#include "si_internal.hpp"

#include <cstring>
#include <string>

namespace si {
namespace {

constexpr size_t kNoAllocScratchBytes = 16u << 20;  // 16 MiB of forward checkpoints

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Device address of the scratch array, looked up by the ctx's first call (its
// device is current) and kept in the ctx.
cudaError_t scratch_address(si_ctx* ctx, void** out) {
    if (!ctx->noalloc_scratch) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        ctx->noalloc_scratch = p;
    }
    *out = ctx->noalloc_scratch;
    return cudaSuccess;
}

// Same key as the transition table cache of the allocating entry points.
uint64_t trans_key_of(const si_impute_params* p) {
    uint64_t key = (uint64_t)p->transition_mode * 0x9E3779B97F4A7C15ull;
    double pr[2] = {(double)p->ne, p->rho_rate};
    uint64_t bits[2];
    std::memcpy(bits, pr, sizeof bits);
    return key ^ (bits[0] * 0xBF58476D1CE4E5B9ull ^ bits[1] * 0x94D049BB133111EBull);
}

}  // namespace
}  // namespace si

using namespace si;

extern "C" si_status si_impute_device_noalloc(si_ctx* ctx, const si_impute_params* p, const uint8_t* d_geno,
                                              uint32_t B, float* d_dosage, float* d_hap_prob, uint8_t* d_haps,
                                              void* stream) {
    if (!ctx) return SI_ERR_INVALID_ARG;
    if (!p || !d_geno || B == 0) return fail(ctx, SI_ERR_INVALID_ARG, "params or geno is NULL, or B == 0");
    if (p->num_states == 0 || p->num_states > 32)
        return fail(ctx, SI_ERR_UNSUPPORTED, "num_states must be 1..32");
    if (p->sampling != SI_SAMPLE_ARGMAX && p->sampling != SI_SAMPLE_PHILOX)
        return fail(ctx, SI_ERR_INVALID_ARG, "bad sampling mode");
    if (!(p->tie_eps >= 0.0 && p->tie_eps < 1.0)) return fail(ctx, SI_ERR_INVALID_ARG, "tie_eps must be in [0, 1)");
    if (p->flags & SI_IMPUTE_RESELECT)
        return fail(ctx, SI_ERR_INVALID_ARG, "SI_IMPUTE_RESELECT is not available without allocation");
    // this entry point always runs the full-chain recursion; SI_IMPUTE_FULL_CHAIN is accepted
    if (p->flags & ~(uint32_t)SI_IMPUTE_FULL_CHAIN) return fail(ctx, SI_ERR_INVALID_ARG, "unknown flag bits");
    // set-up state must already exist: an earlier allocating call with the same
    // parameters built the slot table and the transition table
    if (p->selection_kind == SI_SEL_TARGET)
        return fail(ctx, SI_ERR_UNSUPPORTED, "target-aware selection needs per-target scratch: use si_impute_device");
    const uint32_t L = p->num_states;
    int kind = p->selection_kind;
    if (kind == SI_SEL_AUTO) kind = (L <= 32 && ctx->N <= 10000) ? SI_SEL_WARP : SI_SEL_INSERTION;
    auto it = ctx->sel.find({L, kind});
    if (it == ctx->sel.end() || !it->second.masks.ptr || !ctx->trans.ptr || ctx->trans_key != trans_key_of(p))
        return fail(ctx, SI_ERR_STATE,
                    "set-up missing: run si_impute or si_impute_device once with the same parameters first "
                    "(that call allocates the slot and transition tables)");
    const uint32_t lm = fb_lmax(L);
    const uint32_t C = p->checkpoint_interval ? p->checkpoint_interval : (lm >= 32 ? 16u : 32u);
    const uint32_t T = p->block_threads ? p->block_threads : (lm <= 8 ? 64u : 32u);
    if (C > 32 || T % 32 || T > 128) return fail(ctx, SI_ERR_UNSUPPORTED, "bad tile parameters");
    if (fb_smem_bytes(L, T, C) > 227u * 1024u) return fail(ctx, SI_ERR_UNSUPPORTED, "tile exceeds shared memory");
    const size_t need = fb_ckpt_bytes(B, ctx->M, L, C);
    if (need > kNoAllocScratchBytes)
        return fail(ctx, SI_ERR_UNSUPPORTED,
                    "needs " + std::to_string(need) + " bytes of checkpoint scratch; the allocation-free entry point "
                    "holds " + std::to_string(kNoAllocScratchBytes) + " (use fewer samples per call or "
                    "si_impute_device)");
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaSetDevice");
    void* scratch = nullptr;
    e = scratch_address(ctx, &scratch);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaGetSymbolAddress");
    FbLaunch l;
    l.geno = d_geno;
    l.masks = (const SlotMasks*)it->second.masks.ptr;
    l.smasks = nullptr;
    l.raw = (const uint8_t*)it->second.raw.ptr;
    l.trans = (const LinTrans*)ctx->trans.ptr;
    l.B = B; l.M = ctx->M; l.L = L; l.C = C; l.threads = T;
    l.sampling = p->sampling; l.tie_eps = (float)p->tie_eps; l.seed = p->seed; l.sample_id_base = p->sample_id_base;
    l.ckpt = (float*)scratch;
    l.dosage = d_dosage; l.hprob = d_hap_prob; l.haps = d_haps;
    e = launch_fb(l, stream ? (cudaStream_t)stream : ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "forward-backward kernel");
    return SI_OK;
}
