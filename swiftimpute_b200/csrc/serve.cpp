// serve.cpp — request queue and continuous batching over the uneven-batch path.
//
// The worker thread is the only user of the server's ctx. Each launch is a
// list of queued requests taken in arrival order: every request becomes one
// region (its marker slice, slot count and index origin; equal regions are
// shared) and one job per sample, and the whole launch runs through
// si_impute_jobs_device. Codes are gathered into one pinned buffer, copied to
// the device once, and the outputs come back with one copy per array. Two
// staging slots alternate: while the worker runs launch k+1 on the device, a
// completion thread waits for launch k's copies and scatters its outputs into
// the requests' own buffers.
#include "fb_typed.hpp"
#include "si_internal.hpp"

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <tuple>
#include <unordered_map>
#include <vector>

namespace {

using Clock = std::chrono::steady_clock;

struct Pending {
    uint64_t ticket = 0;
    si_request req{};
    Clock::time_point t_submit;
    enum State { QUEUED, RUNNING, FINISHED } state = QUEUED;
    si_status status = SI_OK;
};

struct Pinned {
    void* ptr = nullptr;
    size_t bytes = 0;
};

uint64_t cells_of(const si_request& q) { return (uint64_t)q.n_samples * (q.m_end - q.m_begin); }

double ms_between(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

// Device bytes one launch may need beyond what the ctx keeps between calls,
// an upper bound: inputs and outputs, anchor lists (every marker typed at
// worst), window checkpoints (two anchors per window), job descriptors, and
// the temporary index sweep of a region-local slice not cached yet. The lists
// of a 32-job group take 32 x its longest job; with jobs ordered longest
// first, the groups' first jobs sum to at most the cells plus one longest job
// per lane, hence cells + 32 max_len.
struct Need {
    uint64_t cells = 0, jobs = 0, sweep = 0;
    uint32_t lmax = 4, max_len = 0;
    bool hap_prob = false;
    uint64_t bytes() const {
        const uint64_t io = cells * (1 + 4 + 2) + (hap_prob ? cells * 8 : 0);
        const uint64_t slots = cells + 32ull * max_len;
        const uint64_t lists = slots * 8 + jobs * (4 + 4 + 8 + 8 + 64) + jobs * 4ull * si::typed_nseg(max_len);
        const uint64_t windows = slots / 2 + jobs + 32;
        const uint64_t ckpt = windows * (2ull * lmax * 4 + 8 + 4);
        return io + lists + ckpt + sweep + (1ull << 20);
    }
};

uint32_t lmax_of(uint32_t L) { return L <= 4 ? 4 : L <= 8 ? 8 : L <= 16 ? 16 : 32; }

}  // namespace

struct si_server {
    si_ctx* ctx = nullptr;
    si_impute_params params{};
    uint64_t max_cells = 0;
    uint32_t max_wait_us = 0;
    uint32_t max_queue = 0;
    uint32_t max_requests = 0;  // per launch; 0 = no limit

    std::mutex mu;
    std::condition_variable cv_work;  // the worker waits for requests
    std::condition_variable cv_done;  // callers wait for finished requests
    std::deque<std::shared_ptr<Pending>> queue;
    std::unordered_map<uint64_t, std::shared_ptr<Pending>> live;  // tickets not yet collected
    uint64_t next_ticket = 1;
    uint64_t queued_cells = 0;
    uint32_t waiters = 0;  // callers inside si_serve_wait (si_serve_stop lets them leave first)
    bool stopping = false;
    std::thread worker;

    si_serve_statistics st{};
    std::vector<double> latency_ms;
    Clock::time_point t_start;

    // staging slots: the worker fills one while the completion thread drains the other
    struct Slot {
        si::DeviceBuffer d_geno, d_dos, d_haps, d_hp;
        Pinned h_geno, h_dos, h_haps, h_hp;
        cudaEvent_t copied = nullptr;  // the launch's output copies are done
        std::vector<std::shared_ptr<Pending>> batch;
        std::vector<uint64_t> first;   // cell offset of each request
        si_status status = SI_OK;
        bool busy = false;             // handed to the completion thread
        Clock::time_point t_launch;
    } slot[2];
    std::condition_variable cv_slot;   // slot handed over / released
    std::thread completer;
    bool worker_done = false;          // the worker has left its loop (set under mu)
};

namespace {

// Run body(i) for i in [0, n) on up to 8 threads, split so that each thread
// gets about the same number of bytes (weight(i)).
template <class W, class F>
void par_requests(size_t n, W weight, F body) {
    uint64_t total = 0;
    for (size_t i = 0; i < n; ++i) total += weight(i);
    const unsigned hw = std::max(2u, std::thread::hardware_concurrency());
    const unsigned T = (unsigned)std::min<uint64_t>(std::min(8u, hw / 2), total / (4u << 20) + 1);
    if (T <= 1 || n < 2) {
        for (size_t i = 0; i < n; ++i) body(i);
        return;
    }
    std::vector<size_t> cut{0};
    uint64_t acc = 0;
    for (size_t i = 0; i < n; ++i) {
        acc += weight(i);
        if (acc * T >= total * cut.size() && cut.size() < T) cut.push_back(i + 1);
    }
    cut.push_back(n);
    std::vector<std::thread> th;
    for (size_t t = 1; t + 1 < cut.size(); ++t)
        th.emplace_back([&, a = cut[t], b = cut[t + 1]] {
            for (size_t i = a; i < b; ++i) body(i);
        });
    for (size_t i = cut[0]; i < cut[1]; ++i) body(i);
    for (auto& x : th) x.join();
}

// Grow-only pinned staging (sized once for max_batch_cells at start; only
// P(hap=1) staging is allocated on first use).
si_status pinned_reserve(Pinned& b, size_t bytes) {
    if (b.ptr && b.bytes >= bytes) return SI_OK;
    if (b.ptr) cudaFreeHost(b.ptr);
    b.ptr = nullptr;
    b.bytes = 0;
    void* p = nullptr;
    if (cudaMallocHost(&p, bytes ? bytes : 16) != cudaSuccess) {
        cudaGetLastError();
        return SI_ERR_OUT_OF_MEMORY;
    }
    b.ptr = p;
    b.bytes = bytes;
    return SI_OK;
}

// Bytes of ctx memory the next launch can reuse or regrow (per-call scratch).
uint64_t reclaimable(const si_server* S, int k) {
    const si_ctx* c = S->ctx;
    const auto& z = S->slot[k];
    uint64_t b = 0;
    for (const si::DeviceBuffer* x : {&c->t_counts, &c->t_segc, &c->t_aoff, &c->t_woff, &c->t_apos, &c->t_aem,
                                      &c->t_ckF, &c->t_ckB, &c->t_ckU, &c->job_regions,
                                      &c->job_samples, &z.d_geno, &z.d_dos, &z.d_haps, &z.d_hp})
        b += x->bytes;
    return b;
}

// Device bytes a launch into slot k may use: the budget less everything the
// ctx holds that this launch cannot reuse (the other slot's staging included).
uint64_t headroom(const si_server* S, int k) {
    const si_ctx* c = S->ctx;
    const uint64_t fixed = c->used - std::min<uint64_t>(c->used, reclaimable(S, k));
    return c->budget > fixed ? c->budget - fixed : 0;
}

void add_need(const si_server* S, Need& n, const si_request& q) {
    n.cells += cells_of(q);
    n.jobs += q.n_samples;
    n.max_len = std::max(n.max_len, q.m_end - q.m_begin);
    n.lmax = std::max(n.lmax, lmax_of(q.num_states));
    n.hap_prob |= q.hap_prob != nullptr;
    if (q.index_origin == SI_INDEX_REGION) {
        const uint32_t L = q.num_states;
        const int kind = (L <= 32 && S->ctx->N <= 10000) ? SI_SEL_WARP : SI_SEL_INSERTION;
        if (!S->ctx->region_sel.count(std::make_tuple(q.m_begin, q.m_end, L, kind)))
            n.sweep += (uint64_t)(q.m_end - q.m_begin) * (si::kHead * 4 + 8) + 8ull * S->ctx->N;
    }
}

// Region-local selection tables accumulate one entry per distinct slice;
// drop them all once they hold more than an eighth of the budget.
void trim_region_cache(si_server* S) {
    si_ctx* c = S->ctx;
    uint64_t b = 0;
    for (auto& kv : c->region_sel) b += kv.second.masks.bytes + kv.second.g2.bytes + kv.second.raw.bytes;
    if (b <= c->budget / 8) return;
    for (auto& kv : c->region_sel) {
        si::dev_free(c, kv.second.masks);
        si::dev_free(c, kv.second.g2);
        si::dev_free(c, kv.second.raw);
    }
    c->region_sel.clear();
}

// Device stage of a launch into slot k: gather codes, copy in, impute, queue
// the output copies and the event that marks them done.
si_status launch_batch(si_server* S, int k) {
    si::Range range("serve launch");
    si_ctx* ctx = S->ctx;
    auto& z = S->slot[k];
    const auto& batch = z.batch;
    std::vector<si_region> regions;
    std::map<std::tuple<uint32_t, uint32_t, uint32_t, int32_t>, uint32_t> region_id;
    std::vector<si_job> jobs;
    z.first.assign(batch.size(), 0);
    uint64_t off = 0;
    bool any_hp = false;
    for (size_t b = 0; b < batch.size(); ++b) {
        const si_request& q = batch[b]->req;
        const uint32_t len = q.m_end - q.m_begin;
        auto key = std::make_tuple(q.m_begin, q.m_end, q.num_states, q.index_origin);
        auto it = region_id.find(key);
        uint32_t r;
        if (it == region_id.end()) {
            r = (uint32_t)regions.size();
            region_id.emplace(key, r);
            regions.push_back(si_region{q.m_begin, q.m_end, q.num_states, q.index_origin});
        } else {
            r = it->second;
        }
        z.first[b] = off;
        for (uint32_t i = 0; i < q.n_samples; ++i) {
            const uint64_t o = off + (uint64_t)i * len;
            jobs.push_back(si_job{r, 0u, o, o, q.sample_id_base + i});
        }
        off += (uint64_t)q.n_samples * len;
        any_hp |= q.hap_prob != nullptr;
    }
    const uint64_t cells = off;
    si_status st = pinned_reserve(z.h_geno, cells);
    if (st == SI_OK) st = pinned_reserve(z.h_dos, cells * 4);
    if (st == SI_OK) st = pinned_reserve(z.h_haps, cells * 2);
    if (st == SI_OK && any_hp) st = pinned_reserve(z.h_hp, cells * 8);
    if (st != SI_OK) return si::fail(ctx, st, "pinned staging for a serving launch");
    if ((st = si::dev_reserve(ctx, z.d_geno, cells)) != SI_OK) return st;
    if ((st = si::dev_reserve(ctx, z.d_dos, cells * 4)) != SI_OK) return st;
    if ((st = si::dev_reserve(ctx, z.d_haps, cells * 2)) != SI_OK) return st;
    if (any_hp && (st = si::dev_reserve(ctx, z.d_hp, cells * 8)) != SI_OK) return st;
    par_requests(
        batch.size(), [&](size_t b) { return cells_of(batch[b]->req); },
        [&](size_t b) { std::memcpy((uint8_t*)z.h_geno.ptr + z.first[b], batch[b]->req.codes, cells_of(batch[b]->req)); });
    cudaStream_t s = ctx->stream;
    cudaError_t e = cudaMemcpyAsync(z.d_geno.ptr, z.h_geno.ptr, cells, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return si::cuda_fail(ctx, e, "serving input copy");
    st = si_impute_jobs_device(ctx, &S->params, regions.data(), (uint32_t)regions.size(), jobs.data(),
                               (uint32_t)jobs.size(), (const uint8_t*)z.d_geno.ptr, (float*)z.d_dos.ptr,
                               any_hp ? (float*)z.d_hp.ptr : nullptr, (uint8_t*)z.d_haps.ptr, s);
    if (st != SI_OK) return st;
    e = cudaMemcpyAsync(z.h_dos.ptr, z.d_dos.ptr, cells * 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(z.h_haps.ptr, z.d_haps.ptr, cells * 2, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && any_hp)
        e = cudaMemcpyAsync(z.h_hp.ptr, z.d_hp.ptr, cells * 8, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaEventRecord(z.copied, s);
    if (e != cudaSuccess) return si::cuda_fail(ctx, e, "serving output copy");
    trim_region_cache(S);
    return SI_OK;
}

// Host stage: wait for slot k's copies, scatter into the requests' buffers (a
// request's jobs are consecutive, so each output is one contiguous block).
si_status complete_batch(si_server* S, int k) {
    si::Range range("serve complete");
    auto& z = S->slot[k];
    if (z.status != SI_OK) return z.status;
    const cudaError_t e = cudaEventSynchronize(z.copied);
    if (e != cudaSuccess) return SI_ERR_CUDA;
    par_requests(
        z.batch.size(), [&](size_t b) { return cells_of(z.batch[b]->req); },
        [&](size_t b) {
            const si_request& q = z.batch[b]->req;
            const uint64_t n = cells_of(q), f = z.first[b];
            if (q.dosage) std::memcpy(q.dosage, (const float*)z.h_dos.ptr + f, n * 4);
            if (q.haps) std::memcpy(q.haps, (const uint8_t*)z.h_haps.ptr + 2 * f, n * 2);
            if (q.hap_prob) std::memcpy(q.hap_prob, (const float*)z.h_hp.ptr + 2 * f, n * 8);
        });
    return SI_OK;
}

void finish(si_server* S, Pending& p, si_status status, Clock::time_point t) {
    p.state = Pending::FINISHED;
    p.status = status;
    if (status == SI_OK) {
        S->st.completed++;
        S->st.cells += cells_of(p.req);
        S->latency_ms.push_back(ms_between(p.t_submit, t));
    } else if (status == SI_ERR_CANCELLED) {
        S->st.cancelled++;
    } else {
        S->st.failed++;
    }
}

void worker_main(si_server* S) {
    cudaSetDevice(S->ctx->device);
    std::unique_lock<std::mutex> lk(S->mu);
    int k = 0;
    for (;;) {
        S->cv_work.wait(lk, [&] { return S->stopping || !S->queue.empty(); });
        if (S->stopping) break;
        // let the oldest request wait up to max_wait_us for company, unless a launch is full already
        const auto deadline = S->queue.front()->t_submit + std::chrono::microseconds(S->max_wait_us);
        while (!S->stopping && !S->queue.empty() && S->queued_cells < S->max_cells && S->max_requests != 1 &&
               Clock::now() < deadline)
            S->cv_work.wait_until(lk, deadline);
        if (S->stopping) break;
        // the slot must be drained by the completion thread before it is refilled
        S->cv_slot.wait(lk, [&] { return !S->slot[k].busy; });
        if (S->queue.empty()) continue;  // everything queued was cancelled meanwhile
        const uint64_t room = headroom(S, k);
        auto& z = S->slot[k];
        z.batch.clear();
        Need need;
        uint64_t cells = 0;
        while (!S->queue.empty()) {
            if (S->max_requests && z.batch.size() >= S->max_requests) break;
            std::shared_ptr<Pending> p = S->queue.front();
            const uint64_t c = cells_of(p->req);
            if (cells + c > S->max_cells) break;
            Need next = need;
            add_need(S, next, p->req);
            if (next.bytes() > room) {
                if (!z.batch.empty()) break;
                // alone it does not fit what the budget leaves: refuse it, keep serving
                S->queue.pop_front();
                S->queued_cells -= c;
                finish(S, *p, SI_ERR_BUDGET, Clock::now());
                S->cv_done.notify_all();
                continue;
            }
            S->queue.pop_front();
            S->queued_cells -= c;
            p->state = Pending::RUNNING;
            z.batch.push_back(p);
            need = next;
            cells += c;
        }
        if (z.batch.empty()) continue;
        lk.unlock();
        z.t_launch = Clock::now();
        z.status = launch_batch(S, k);
        const auto t1 = Clock::now();
        lk.lock();
        S->st.busy_ms += ms_between(z.t_launch, t1);
        S->st.batches++;
        z.busy = true;
        S->cv_slot.notify_all();
        k ^= 1;
    }
}

// Drains slots in launch order: their copies, the scatter, the requests' status.
void completer_main(si_server* S) {
    cudaSetDevice(S->ctx->device);
    std::unique_lock<std::mutex> lk(S->mu);
    int k = 0;
    for (;;) {
        S->cv_slot.wait(lk, [&] { return S->slot[k].busy || (S->stopping && S->worker_done); });
        if (!S->slot[k].busy) break;
        lk.unlock();
        const si_status rs = complete_batch(S, k);
        const auto t = Clock::now();
        lk.lock();
        for (auto& p : S->slot[k].batch) finish(S, *p, rs, t);
        S->slot[k].batch.clear();
        S->slot[k].busy = false;
        S->cv_done.notify_all();
        S->cv_slot.notify_all();
        k ^= 1;
    }
}

}  // namespace

extern "C" {

si_status si_serve_start(si_ctx* ctx, const si_impute_params* params, const si_serve_config* cfg, si_server** out) {
    if (!ctx || !params || !out) return SI_ERR_INVALID_ARG;
    if (params->transition_mode != SI_TRANS_MATRIX0)
        return si::fail(ctx, SI_ERR_UNSUPPORTED, "serving uses the first-gap transition (SI_TRANS_MATRIX0)");
    if (!ctx->panel.ptr || !ctx->has_map) return si::fail(ctx, SI_ERR_STATE, "panel and map must be set first");
    auto* S = new si_server();
    S->ctx = ctx;
    S->params = *params;
    S->max_cells = cfg && cfg->max_batch_cells ? cfg->max_batch_cells : (1ull << 25);
    S->max_wait_us = cfg && cfg->max_wait_us ? cfg->max_wait_us : 200u;
    S->max_queue = cfg && cfg->max_queue ? cfg->max_queue : 65536u;
    S->max_requests = cfg ? cfg->max_batch_requests : 0u;
    S->t_start = Clock::now();
    for (auto& z : S->slot) {
        if (cudaSetDevice(ctx->device) != cudaSuccess ||
            cudaEventCreateWithFlags(&z.copied, cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            for (auto& y : S->slot)
                if (y.copied) cudaEventDestroy(y.copied);
            delete S;
            return si::fail(ctx, SI_ERR_CUDA, "serving events");
        }
    }
    // staging for a full launch in both slots, allocated once: growing pinned
    // memory or device buffers between launches stalls the device
    for (auto& z : S->slot) {
        const uint64_t c = S->max_cells;
        si_status st = pinned_reserve(z.h_geno, c);
        if (st == SI_OK) st = pinned_reserve(z.h_dos, c * 4);
        if (st == SI_OK) st = pinned_reserve(z.h_haps, c * 2);
        if (st == SI_OK) st = si::dev_reserve(ctx, z.d_geno, c);
        if (st == SI_OK) st = si::dev_reserve(ctx, z.d_dos, c * 4);
        if (st == SI_OK) st = si::dev_reserve(ctx, z.d_haps, c * 2);
        if (st != SI_OK) {
            for (auto& y : S->slot) {
                si::dev_free(ctx, y.d_geno);
                si::dev_free(ctx, y.d_dos);
                si::dev_free(ctx, y.d_haps);
                for (Pinned* b : {&y.h_geno, &y.h_dos, &y.h_haps})
                    if (b->ptr) cudaFreeHost(b->ptr);
                if (y.copied) cudaEventDestroy(y.copied);
            }
            delete S;
            return si::fail(ctx, st, "serving staging for max_batch_cells");
        }
    }
    S->worker = std::thread([S] {
        worker_main(S);
        std::lock_guard<std::mutex> lk(S->mu);
        S->worker_done = true;
        S->cv_slot.notify_all();
    });
    S->completer = std::thread(completer_main, S);
    *out = S;
    return SI_OK;
}

si_status si_serve_submit(si_server* S, const si_request* q, uint64_t* ticket) {
    if (!S || !q || !ticket) return SI_ERR_INVALID_ARG;
    const si_ctx* c = S->ctx;
    if (q->m_begin >= q->m_end || q->m_end > c->M || q->n_samples == 0 || !q->codes ||
        q->num_states == 0 || q->num_states > 32 ||
        (q->index_origin != SI_INDEX_GLOBAL && q->index_origin != SI_INDEX_REGION) ||
        (!q->dosage && !q->haps && !q->hap_prob))
        return SI_ERR_INVALID_ARG;
    // what the launch would refuse for this request alone is refused here, so
    // that it cannot fail the requests it would share a launch with
    if (q->index_origin == SI_INDEX_GLOBAL) {
        if (S->params.selection_kind == SI_SEL_FIRST_PAIRS) {
            if ((uint64_t)2 * q->num_states > c->N) return SI_ERR_UNSUPPORTED;
        } else if (!c->has_index) {
            return SI_ERR_STATE;  // the global index is not built
        }
        if (!si::region_first_gap_ok(c, &S->params, 0, c->M)) return SI_ERR_UNSUPPORTED;
    } else if (!si::region_first_gap_ok(c, &S->params, q->m_begin, q->m_end)) {
        return SI_ERR_UNSUPPORTED;
    }
    auto p = std::make_shared<Pending>();
    p->req = *q;
    const uint64_t cells = cells_of(*q);
    std::lock_guard<std::mutex> lk(S->mu);
    if (S->stopping) return SI_ERR_STATE;
    if (cells > S->max_cells) return SI_ERR_BUDGET;
    if (S->queue.size() >= S->max_queue) return SI_ERR_BUDGET;
    Need alone;
    alone.cells = cells;
    alone.jobs = q->n_samples;
    alone.lmax = lmax_of(q->num_states);
    alone.hap_prob = q->hap_prob != nullptr;
    if (alone.bytes() > c->budget) return SI_ERR_BUDGET;
    p->ticket = S->next_ticket++;
    p->t_submit = Clock::now();
    S->queue.push_back(p);
    S->live.emplace(p->ticket, p);
    S->queued_cells += cells;
    S->st.submitted++;
    *ticket = p->ticket;
    S->cv_work.notify_one();
    return SI_OK;
}

si_status si_serve_poll(si_server* S, uint64_t ticket, int* finished, si_status* result) {
    if (!S || !finished) return SI_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->live.find(ticket);
    if (it == S->live.end()) return SI_ERR_INVALID_ARG;
    *finished = it->second->state == Pending::FINISHED;
    if (*finished) {
        if (result) *result = it->second->status;
        S->live.erase(it);
    }
    return SI_OK;
}

si_status si_serve_wait(si_server* S, uint64_t ticket, uint32_t timeout_ms, si_status* result) {
    if (!S) return SI_ERR_INVALID_ARG;
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->live.find(ticket);
    if (it == S->live.end()) return SI_ERR_INVALID_ARG;
    std::shared_ptr<Pending> p = it->second;
    auto done = [&] { return p->state == Pending::FINISHED; };
    S->waiters++;
    bool ok = true;
    if (timeout_ms) ok = S->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), done);
    else S->cv_done.wait(lk, done);
    S->waiters--;
    if (S->waiters == 0) S->cv_done.notify_all();
    if (!ok) return SI_ERR_TIMEOUT;
    if (result) *result = p->status;
    S->live.erase(ticket);
    return SI_OK;
}

si_status si_serve_cancel(si_server* S, uint64_t ticket) {
    if (!S) return SI_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->live.find(ticket);
    if (it == S->live.end()) return SI_ERR_INVALID_ARG;
    if (it->second->state != Pending::QUEUED) return SI_ERR_STATE;
    auto q = std::find(S->queue.begin(), S->queue.end(), it->second);
    if (q != S->queue.end()) S->queue.erase(q);
    S->queued_cells -= cells_of(it->second->req);
    finish(S, *it->second, SI_ERR_CANCELLED, Clock::now());
    S->cv_done.notify_all();
    return SI_OK;
}

si_status si_serve_stats(si_server* S, si_serve_statistics* out) {
    if (!S || !out) return SI_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(S->mu);
    *out = S->st;
    out->wall_ms = ms_between(S->t_start, Clock::now());
    if (!S->latency_ms.empty()) {
        std::vector<double> v = S->latency_ms;
        auto q = [&](double f) {
            const size_t k = std::min(v.size() - 1, (size_t)(f * (double)(v.size() - 1) + 0.5));
            std::nth_element(v.begin(), v.begin() + k, v.end());
            return v[k];
        };
        out->latency_p50_ms = q(0.50);
        out->latency_p99_ms = q(0.99);
        out->latency_max_ms = *std::max_element(v.begin(), v.end());
    }
    return SI_OK;
}

si_status si_serve_stop(si_server* S) {
    if (!S) return SI_ERR_INVALID_ARG;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stopping = true;
        const auto t = Clock::now();
        for (auto& p : S->queue) finish(S, *p, SI_ERR_CANCELLED, t);
        S->queue.clear();
        S->queued_cells = 0;
        S->cv_work.notify_all();
        S->cv_done.notify_all();
    }
    if (S->worker.joinable()) S->worker.join();
    if (S->completer.joinable()) S->completer.join();
    {
        // every request has finished: let callers still inside si_serve_wait return first
        std::unique_lock<std::mutex> lk(S->mu);
        S->cv_done.wait(lk, [&] { return S->waiters == 0; });
    }
    si_ctx* c = S->ctx;
    for (auto& z : S->slot) {
        si::dev_free(c, z.d_geno);
        si::dev_free(c, z.d_dos);
        si::dev_free(c, z.d_haps);
        si::dev_free(c, z.d_hp);
        for (Pinned* b : {&z.h_geno, &z.h_dos, &z.h_haps, &z.h_hp})
            if (b->ptr) cudaFreeHost(b->ptr);
        if (z.copied) cudaEventDestroy(z.copied);
    }
    delete S;
    return SI_OK;
}

}  // extern "C"
