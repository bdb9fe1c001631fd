// plan.cpp — a fixed uneven batch whose launch sequence needs no host work.
//
// si_impute_jobs_device sizes its anchor lists from the codes: it counts the
// typed markers, reads the totals back and then allocates, so every call
// waits on the host in the middle. A plan instead fixes each job's anchor
// capacity in advance (its marker count, or a bound the caller knows, such as
// the number of typed sites of a genotyping array, plus one), lays out all
// lists and window checkpoints by those capacities, and uploads the job and
// region descriptors once. Its launch is then four kernels with fixed
// arguments (count, fill, chain, posterior) that can be captured into a CUDA
// graph and replayed after the caller rewrites the codes in place. A job with
// more anchors than its capacity is cut to it and flagged on the device;
// si_plan_check reports it.
//
// The autotuner times the launch on the plan's own batch for each candidate
// window size (anchors per checkpoint) and posterior CTA size and keeps the
// fastest. The window size moves where rounding restarts, so a tuned plan's
// results can differ from the untuned path's in the last bits (within the
// 1e-4 dosage bar; the tile test bounds it at 2e-5).
#include "fb_typed.hpp"

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

struct si_plan {
    si_ctx* ctx = nullptr;
    si::TypedArgs a{};
    uint32_t lmax = 4;
    bool all_full = true;
    uint32_t B = 0;
    std::vector<uint32_t> cap;             // anchor capacity per job (launch order)
    std::vector<unsigned long long> gcap;  // per 32-job group of the interleaved lists: its jobs' largest capacity
    si::DeviceBuffer regions, samples, counts, segc, jcap, aoff, woff, apos, aem, ckF, ckB, ckU, err;
    uint32_t C = 2, T = 128;
    float best_ms = 0.f;
    cudaStream_t capture_stream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

namespace {

using si::DeviceBuffer;

void free_plan(si_plan* P) {
    si_ctx* c = P->ctx;
    if (P->exec) cudaGraphExecDestroy(P->exec);
    if (P->graph) cudaGraphDestroy(P->graph);
    if (P->capture_stream) cudaStreamDestroy(P->capture_stream);
    for (DeviceBuffer* b : {&P->regions, &P->samples, &P->counts, &P->segc, &P->jcap, &P->aoff, &P->woff, &P->apos, &P->aem,
                            &P->ckF, &P->ckB, &P->ckU, &P->err})
        si::dev_free(c, *b);
    delete P;
}

// Group offsets of the interleaved lists (32 entries per anchor of a group's
// capacity) or, with C > 0, of its window checkpoints (32 per window).
std::vector<unsigned long long> group_offsets(const std::vector<unsigned long long>& gcap, uint32_t C) {
    std::vector<unsigned long long> o(gcap.size() + 1, 0);
    for (size_t g = 0; g < gcap.size(); ++g) o[g + 1] = o[g] + 32ull * (C ? (gcap[g] + C - 1) / C : gcap[g]);
    return o;
}

cudaError_t enqueue(si_plan* P, cudaStream_t s) {
    cudaError_t e = si::launch_anchor_count_only(P->a, s);
    if (e == cudaSuccess) e = si::launch_anchor_lists_fill(P->a, s);
    if (e == cudaSuccess) e = si::launch_typed_fb(P->a, P->lmax, P->all_full, s);
    return e;
}

// Use window size C and CTA size T: upload the window offsets, set the args.
si_status use_tiles(si_plan* P, uint32_t C, uint32_t T, cudaStream_t s) {
    const auto w = group_offsets(P->gcap, C);
    const cudaError_t e = cudaMemcpyAsync(P->woff.ptr, w.data(), w.size() * 8, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) {
        const cudaError_t f = cudaStreamSynchronize(s);  // the host vector dies here
        if (f != cudaSuccess) return si::cuda_fail(P->ctx, f, "plan window offsets");
    } else {
        return si::cuda_fail(P->ctx, e, "plan window offsets");
    }
    unsigned long long most = 0;
    for (unsigned long long c : P->gcap) most = std::max(most, (c + C - 1) / C);
    P->a.C = C;
    P->a.threads = T;
    P->a.K = si::kPostGroup;
    P->a.max_windows = (uint32_t)most;
    P->a.total_windows = w.back();
    P->C = C;
    P->T = T;
    return SI_OK;
}

}  // namespace

extern "C" {

si_status si_plan_create(si_ctx* ctx, const si_impute_params* p, const si_region* regions, uint32_t n_regions,
                         const si_job* jobs, uint32_t n_jobs, uint32_t max_anchors, const uint8_t* d_geno,
                         float* d_dosage, float* d_hap_prob, uint8_t* d_haps, uint32_t flags, si_plan** out) {
    si::Range range("si_plan_create");
    if (!ctx || !out) return SI_ERR_INVALID_ARG;
    si_status st = si::check_jobs_args(ctx, p, regions, n_regions, jobs, n_jobs);
    if (st != SI_OK) return st;
    if (!d_geno) return si::fail(ctx, SI_ERR_INVALID_ARG, "NULL genotype buffer");
    if (flags & ~(uint32_t)SI_PLAN_AUTOTUNE) return si::fail(ctx, SI_ERR_INVALID_ARG, "unknown plan flags");
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) return si::cuda_fail(ctx, e, "cudaSetDevice");
    cudaStream_t s = ctx->stream;
    auto* P = new si_plan();
    P->ctx = ctx;
    P->B = n_jobs;
    std::vector<si::TypedRegion> tr;
    std::vector<si::TypedSample> ts;
    st = si::prepare_jobs(ctx, p, regions, n_regions, jobs, n_jobs, s, tr, ts, P->lmax, P->all_full);
    if (st != SI_OK) {
        free_plan(P);
        return st;
    }
    // capacities: marker 0 and the typed markers, at most the job's length
    const uint32_t G = si::typed_groups(n_jobs);
    P->cap.resize(n_jobs);
    P->gcap.assign(G, 0);
    for (uint32_t j = 0; j < n_jobs; ++j) {
        const uint32_t len = ts[j].len;
        P->cap[j] = max_anchors ? std::min(len, max_anchors) : len;
        P->gcap[j / 32] = std::max<unsigned long long>(P->gcap[j / 32], P->cap[j]);
    }
    const std::vector<unsigned long long> aoff = group_offsets(P->gcap, 0);
    const unsigned long long NA = aoff.back();
    const uint32_t Cmin = p->checkpoint_interval ? p->checkpoint_interval : 1;
    const unsigned long long NWmax = group_offsets(P->gcap, Cmin).back();
    const uint32_t lm = P->lmax;
    auto alloc = [&](DeviceBuffer& b, size_t bytes) { return st == SI_OK ? (st = si::dev_alloc(ctx, b, bytes)) : st; };
    alloc(P->regions, tr.size() * sizeof(si::TypedRegion));
    alloc(P->samples, ts.size() * sizeof(si::TypedSample));
    const uint32_t max_len = ts.empty() ? 0u : ts.front().len;  // jobs are ordered longest first
    alloc(P->counts, (size_t)n_jobs * 4);
    alloc(P->segc, (size_t)n_jobs * si::typed_nseg(max_len) * 4);
    alloc(P->jcap, (size_t)n_jobs * 4);
    alloc(P->aoff, ((size_t)G + 1) * 8);
    alloc(P->woff, ((size_t)G + 1) * 8);
    alloc(P->apos, (size_t)NA * 4);
    alloc(P->aem, (size_t)NA * 4);
    alloc(P->ckF, (size_t)NWmax * lm * 4);
    alloc(P->ckB, (size_t)NWmax * lm * 4);
    alloc(P->ckU, (size_t)NWmax * 8);
    alloc(P->err, 4);
    if (st != SI_OK) {
        free_plan(P);
        return st;
    }
    e = cudaMemcpyAsync(P->regions.ptr, tr.data(), tr.size() * sizeof(si::TypedRegion), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(P->samples.ptr, ts.data(), ts.size() * sizeof(si::TypedSample), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(P->aoff.ptr, aoff.data(), aoff.size() * 8, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(P->jcap.ptr, P->cap.data(), (size_t)n_jobs * 4, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(P->err.ptr, 0, 4, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        free_plan(P);
        return si::cuda_fail(ctx, e, "plan upload");
    }
    si::TypedArgs& a = P->a;
    a.geno = d_geno;
    a.B = n_jobs;
    a.M = 0;
    a.sampling = p->sampling;
    a.tie_eps = (float)p->tie_eps;
    a.seed = p->seed;
    a.sid_base = 0;
    a.regions = (const si::TypedRegion*)P->regions.ptr;
    a.samples = (const si::TypedSample*)P->samples.ptr;
    a.counts = (uint32_t*)P->counts.ptr;
    a.max_len = max_len;
    a.nseg = si::typed_nseg(max_len);
    a.segc = (uint32_t*)P->segc.ptr;
    a.aoff = (unsigned long long*)P->aoff.ptr;
    a.woff = (unsigned long long*)P->woff.ptr;
    a.cap = (const uint32_t*)P->jcap.ptr;
    a.err = (uint32_t*)P->err.ptr;
    a.apos = (uint32_t*)P->apos.ptr;
    a.aem = (uint32_t*)P->aem.ptr;
    a.ckptF = (float*)P->ckF.ptr;
    a.ckptB = (float*)P->ckB.ptr;
    a.ckptU = (double*)P->ckU.ptr;
    a.dosage = d_dosage;
    a.hprob = d_hap_prob;
    a.haps = d_haps;
    a.ev_chain_done = nullptr;
    uint32_t C = p->checkpoint_interval ? p->checkpoint_interval : si::typed_default_window(lm);
    uint32_t T = p->block_threads ? p->block_threads : si::typed_default_threads(lm);
    if ((flags & SI_PLAN_AUTOTUNE) && !p->checkpoint_interval && !p->block_threads) {
        // candidates: window size x posterior CTA size, each timed on this batch
        std::vector<uint32_t> Cs = {1, 2, 4};
        std::vector<uint32_t> Ts = lm <= 16 ? std::vector<uint32_t>{64, 128} : std::vector<uint32_t>{32, 64};
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        float best = 1e30f;
        for (uint32_t c : Cs) {
            for (uint32_t t : Ts) {
                if (si::typed_post_smem_bytes(lm, t, c) > 227u * 1024u) continue;
                if ((st = use_tiles(P, c, t, s)) != SI_OK) break;
                e = enqueue(P, s);  // warm-up (and shared-memory attributes)
                if (e == cudaSuccess) e = cudaEventRecord(e0, s);
                for (int k = 0; k < 3 && e == cudaSuccess; ++k) e = enqueue(P, s);
                if (e == cudaSuccess) e = cudaEventRecord(e1, s);
                if (e == cudaSuccess) e = cudaEventSynchronize(e1);
                float ms = 0.f;
                if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
                if (e != cudaSuccess) break;
                if (ms < best) {
                    best = ms;
                    C = c;
                    T = t;
                }
            }
            if (st != SI_OK || e != cudaSuccess) break;
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (st != SI_OK || e != cudaSuccess) {
            free_plan(P);
            return st != SI_OK ? st : si::cuda_fail(ctx, e, "plan autotune");
        }
        P->best_ms = best / 3.f;
    }
    if (si::typed_post_smem_bytes(lm, T, C) > 227u * 1024u) {
        free_plan(P);
        return si::fail(ctx, SI_ERR_UNSUPPORTED, "posterior tile needs more than 227 KB of shared memory");
    }
    if ((st = use_tiles(P, C, T, s)) != SI_OK) {
        free_plan(P);
        return st;
    }
    // one launch outside any capture: sets the posterior's shared-memory attribute
    e = enqueue(P, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(P->err.ptr, 0, 4, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        free_plan(P);
        return si::cuda_fail(ctx, e, "plan first launch");
    }
    *out = P;
    return SI_OK;
}

si_status si_plan_launch(si_plan* P, void* stream) {
    si::Range range("si_plan_launch");
    if (!P) return SI_ERR_INVALID_ARG;
    cudaError_t e = cudaSetDevice(P->ctx->device);
    if (e == cudaSuccess) e = enqueue(P, stream ? (cudaStream_t)stream : P->ctx->stream);
    return e == cudaSuccess ? SI_OK : si::cuda_fail(P->ctx, e, "plan launch");
}

si_status si_plan_graph_launch(si_plan* P, void* stream) {
    si::Range range("si_plan_graph_launch");
    if (!P) return SI_ERR_INVALID_ARG;
    cudaError_t e = cudaSetDevice(P->ctx->device);
    if (e != cudaSuccess) return si::cuda_fail(P->ctx, e, "cudaSetDevice");
    if (!P->exec) {
        if (!P->capture_stream) {
            e = cudaStreamCreateWithFlags(&P->capture_stream, cudaStreamNonBlocking);
            if (e != cudaSuccess) return si::cuda_fail(P->ctx, e, "capture stream");
        }
        e = cudaStreamBeginCapture(P->capture_stream, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) return si::cuda_fail(P->ctx, e, "begin capture");
        const cudaError_t le = enqueue(P, P->capture_stream);
        cudaGraph_t g = nullptr;
        e = cudaStreamEndCapture(P->capture_stream, &g);
        if (le != cudaSuccess || e != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            return si::cuda_fail(P->ctx, le != cudaSuccess ? le : e, "capture plan launch");
        }
        e = cudaGraphInstantiate(&P->exec, g, 0);
        if (e != cudaSuccess) {
            cudaGraphDestroy(g);
            P->exec = nullptr;
            return si::cuda_fail(P->ctx, e, "instantiate plan graph");
        }
        P->graph = g;
    }
    e = cudaGraphLaunch(P->exec, stream ? (cudaStream_t)stream : P->ctx->stream);
    return e == cudaSuccess ? SI_OK : si::cuda_fail(P->ctx, e, "graph launch");
}

si_status si_plan_check(si_plan* P) {
    if (!P) return SI_ERR_INVALID_ARG;
    cudaError_t e = cudaSetDevice(P->ctx->device);
    uint32_t flag = 0;
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(&flag, P->err.ptr, 4, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemset(P->err.ptr, 0, 4);
    if (e != cudaSuccess) return si::cuda_fail(P->ctx, e, "plan check");
    if (flag)
        return si::fail(P->ctx, SI_ERR_BUDGET, "a job had more typed markers than its anchor capacity; "
                                               "its results were cut (create the plan with a larger bound)");
    return SI_OK;
}

si_status si_plan_info(const si_plan* P, uint32_t* window, uint32_t* threads, float* tuned_ms) {
    if (!P) return SI_ERR_INVALID_ARG;
    if (window) *window = P->C;
    if (threads) *threads = P->T;
    if (tuned_ms) *tuned_ms = P->best_ms;
    return SI_OK;
}

si_status si_plan_destroy(si_plan* P) {
    if (!P) return SI_ERR_INVALID_ARG;
    cudaSetDevice(P->ctx->device);
    cudaDeviceSynchronize();
    free_plan(P);
    return SI_OK;
}

}  // extern "C"
