// ref_gpu_driver.cu — TEST INFRASTRUCTURE.
//
// Drives the reference's own hot-path code (tcBio/SwiftImpute), compiled from
// its unmodified sources for sm_100a, through the same steps as
// Imputer::impute_batch with window_size = 0 (src/api/imputer.cpp:787-1042):
//   PBWTIndex::build (CPU)            pbwt_index.cpp:12
//   GPUStateSelector::select_on_device pbwt_index.cpp:373 -> pbwt_selector.cu:400
//   pair expansion (h, (h+1) % N)     imputer.cpp:863-874
//   EmissionComputer::compute          emission.cu:208
//   TransitionComputer::compute        transition.cu:242 (map = pos / 1e8, imputer.cpp:596-604)
//   launch_forward_pass/backward_pass  forward_backward.cu:321,356 (C = (uint32)sqrtf(M), imputer.cpp:975)
//   HaplotypeSampler::sample(..., deterministic = true)  sampling.cu:269
// It is used on the GPU box to pin the CPU oracle (golden fixtures) and to
// time the reference's plain per-sample log-space path. Nothing in the
// product links it.
//
// The caller must stay inside the reference's valid range: N >= 128 (smaller
// panels put the warp selector's full-mask shuffles outside convergence),
// M <= 65535 (emission grid.y), M * N < 2^32 (32-bit row offset in the
// emission kernel), L <= 32 (sampler local arrays). The driver refuses
// anything else rather than launching it.
#include "core/types.hpp"
#include "kernels/emission.hpp"
#include "kernels/forward_backward.cuh"
#include "kernels/sampling.hpp"
#include "kernels/transition.hpp"
#include "pbwt/pbwt_index.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

using namespace swiftimpute;

namespace {
struct DevBuf {
    void* p = nullptr;
    ~DevBuf() { if (p) cudaFree(p); }
    template <typename T> T* as() { return static_cast<T*>(p); }
};
#define RCK(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) return 100 + (int)e_; } while (0)
}  // namespace

// Returns 0 on success, 1 on refused shape, 2 on exception, 100+cudaError on CUDA failure.
// Outputs (each may be NULL):
//   slots      [M][L]       haplotype chosen for each slot (same for every sample)
//   logpost    [B][M][L]    normalised log posterior as the reference computes it
//   haps       [B][2][M]    deterministic (argmax) haplotypes
//   stage_ms   [4]          selection, emission, forward+backward, sampling (ms, CUDA events, last iteration)
extern "C" int ref_gpu_impute(const uint8_t* panel, uint32_t M, uint32_t N, const uint64_t* pos,
                              const float* gl, uint32_t B, uint32_t L, uint32_t ne, float rho_rate,
                              int iters, uint32_t* slots, float* logpost, uint8_t* haps,
                              float* stage_ms) {
    if (N < 128 || M > 65535 || M < 2 || (uint64_t)M * N >= (1ull << 32) || L == 0 || L > 32 || B == 0)
        return 1;
    try {
        Logger::instance().set_level(Logger::ERROR);
        auto index = pbwt::PBWTIndex::build(panel, M, N);
        pbwt::GPUStateSelector selector(*index, L, 0);
        selector.transfer_index_to_device();

        const size_t cells = (size_t)B * M;
        DevBuf d_gl, d_tmp, d_states, d_emis, d_post, d_ckpt, d_scale, d_out;
        const uint32_t C = std::max(1u, (uint32_t)std::sqrt((float)M));
        const uint32_t n_ckpt = (M + C - 1) / C;
        RCK(cudaMalloc(&d_gl.p, cells * sizeof(GenotypeLikelihoods)));
        RCK(cudaMalloc(&d_tmp.p, cells * L * sizeof(uint32_t)));
        RCK(cudaMalloc(&d_states.p, cells * L * 2 * sizeof(uint32_t)));
        RCK(cudaMalloc(&d_emis.p, cells * L * sizeof(float)));
        RCK(cudaMalloc(&d_post.p, cells * L * sizeof(float)));
        RCK(cudaMalloc(&d_ckpt.p, (size_t)B * n_ckpt * L * sizeof(float)));
        RCK(cudaMalloc(&d_scale.p, cells * sizeof(float)));
        RCK(cudaMalloc(&d_out.p, cells * 2));
        RCK(cudaMemcpy(d_gl.p, gl, cells * sizeof(GenotypeLikelihoods), cudaMemcpyHostToDevice));

        kernels::EmissionComputer emis(M, N, L, 0);
        emis.set_reference_panel(panel);
        kernels::TransitionComputer trans(M, L, 0);
        std::vector<double> gd(M);
        for (uint32_t m = 0; m < M; ++m) gd[m] = (double)pos[m] / 1e8;
        trans.set_genetic_map(gd.data());
        kernels::HMMParameters hp;
        hp.ne = ne;
        hp.rho_rate = rho_rate;
        hp.theta = 0.001;
        trans.set_parameters(hp);
        trans.compute();
        kernels::HaplotypeSampler sampler(M, N, L, 0);
        sampler.set_reference_panel(panel);

        cudaEvent_t ev[5];
        for (auto& e : ev) RCK(cudaEventCreate(&e));
        std::vector<uint32_t> h_tmp(cells * L), h_states(cells * L * 2);
        for (int it = 0; it < (iters < 1 ? 1 : iters); ++it) {
            RCK(cudaEventRecord(ev[0], 0));
            selector.select_on_device(nullptr, B, M, d_tmp.as<uint32_t>(), 0);
            RCK(cudaMemcpy(h_tmp.data(), d_tmp.p, cells * L * sizeof(uint32_t), cudaMemcpyDeviceToHost));
            for (size_t c = 0; c < cells * L; ++c) {
                h_states[2 * c] = h_tmp[c];
                h_states[2 * c + 1] = (h_tmp[c] + 1) % N;
            }
            RCK(cudaMemcpy(d_states.p, h_states.data(), cells * L * 2 * sizeof(uint32_t), cudaMemcpyHostToDevice));
            RCK(cudaEventRecord(ev[1], 0));
            emis.compute(d_gl.as<GenotypeLikelihoods>(), d_states.as<uint32_t>(), d_emis.as<float>(), B, true);
            RCK(cudaEventRecord(ev[2], 0));
            kernels::launch_forward_pass(d_emis.as<float>(), trans.get_transition_matrices(),
                                         d_states.as<uint32_t>(), B, M, L, C, d_ckpt.as<float>(),
                                         d_scale.as<float>(), 0);
            kernels::launch_backward_pass(d_emis.as<float>(), trans.get_transition_matrices(),
                                          d_states.as<uint32_t>(), d_ckpt.as<float>(), d_scale.as<float>(),
                                          B, M, L, C, d_post.as<float>(), 0);
            RCK(cudaEventRecord(ev[3], 0));
            sampler.sample(d_post.as<float>(), d_states.as<uint32_t>(), d_out.as<uint8_t>(), B, true);
            RCK(cudaEventRecord(ev[4], 0));
            RCK(cudaDeviceSynchronize());
        }
        if (stage_ms)
            for (int s = 0; s < 4; ++s) RCK(cudaEventElapsedTime(&stage_ms[s], ev[s], ev[s + 1]));
        for (auto& e : ev) cudaEventDestroy(e);
        if (slots)
            for (uint32_t m = 0; m < M; ++m)
                for (uint32_t k = 0; k < L; ++k) slots[(size_t)m * L + k] = h_tmp[(size_t)m * L + k];
        if (logpost) RCK(cudaMemcpy(logpost, d_post.p, cells * L * sizeof(float), cudaMemcpyDeviceToHost));
        if (haps) RCK(cudaMemcpy(haps, d_out.p, cells * 2, cudaMemcpyDeviceToHost));
        return 0;
    } catch (...) {
        return 2;
    }
}

// Times the reference's plain per-sample log-space path without its selection
// kernel: EmissionComputer::compute, launch_forward_pass + launch_backward_pass
// (C = (uint32)sqrtf(M)) and the deterministic HaplotypeSampler, over B
// samples that share the given slot table slots [M][L] (expanded to pairs
// (h, (h+1) % N) and replicated per sample as the reference's layout wants).
// stage_ms[3]: emission, forward+backward, sampling (last iteration).
extern "C" int ref_gpu_fb_timing(const uint8_t* panel, uint32_t M, uint32_t N, const uint64_t* pos,
                                 const float* gl, uint32_t B, uint32_t L, uint32_t ne, float rho_rate,
                                 const uint32_t* slots, int iters, float* stage_ms) {
    if (N < 2 || M > 65535 || M < 2 || (uint64_t)M * N >= (1ull << 32) || L == 0 || L > 32 || B == 0) return 1;
    try {
        Logger::instance().set_level(Logger::ERROR);
        const size_t cells = (size_t)B * M;
        DevBuf d_gl, d_states, d_emis, d_post, d_ckpt, d_scale, d_out;
        const uint32_t C = std::max(1u, (uint32_t)std::sqrt((float)M));
        const uint32_t n_ckpt = (M + C - 1) / C;
        RCK(cudaMalloc(&d_gl.p, cells * sizeof(GenotypeLikelihoods)));
        RCK(cudaMalloc(&d_states.p, cells * L * 2 * sizeof(uint32_t)));
        RCK(cudaMalloc(&d_emis.p, cells * L * sizeof(float)));
        RCK(cudaMalloc(&d_post.p, cells * L * sizeof(float)));
        RCK(cudaMalloc(&d_ckpt.p, (size_t)B * n_ckpt * L * sizeof(float)));
        RCK(cudaMalloc(&d_scale.p, cells * sizeof(float)));
        RCK(cudaMalloc(&d_out.p, cells * 2));
        RCK(cudaMemcpy(d_gl.p, gl, cells * sizeof(GenotypeLikelihoods), cudaMemcpyHostToDevice));
        std::vector<uint32_t> one((size_t)M * L * 2);
        for (size_t c = 0; c < (size_t)M * L; ++c) { one[2 * c] = slots[c]; one[2 * c + 1] = (slots[c] + 1) % N; }
        for (uint32_t b = 0; b < B; ++b)
            RCK(cudaMemcpy(d_states.as<uint32_t>() + (size_t)b * M * L * 2, one.data(), one.size() * 4,
                           cudaMemcpyHostToDevice));
        kernels::EmissionComputer emis(M, N, L, 0);
        emis.set_reference_panel(panel);
        kernels::TransitionComputer trans(M, L, 0);
        std::vector<double> gd(M);
        for (uint32_t m = 0; m < M; ++m) gd[m] = (double)pos[m] / 1e8;
        trans.set_genetic_map(gd.data());
        kernels::HMMParameters hp;
        hp.ne = ne;
        hp.rho_rate = rho_rate;
        hp.theta = 0.001;
        trans.set_parameters(hp);
        trans.compute();
        kernels::HaplotypeSampler sampler(M, N, L, 0);
        sampler.set_reference_panel(panel);
        cudaEvent_t ev[4];
        for (auto& e : ev) RCK(cudaEventCreate(&e));
        for (int it = 0; it < (iters < 1 ? 1 : iters); ++it) {
            RCK(cudaEventRecord(ev[0], 0));
            emis.compute(d_gl.as<GenotypeLikelihoods>(), d_states.as<uint32_t>(), d_emis.as<float>(), B, true);
            RCK(cudaEventRecord(ev[1], 0));
            kernels::launch_forward_pass(d_emis.as<float>(), trans.get_transition_matrices(),
                                         d_states.as<uint32_t>(), B, M, L, C, d_ckpt.as<float>(),
                                         d_scale.as<float>(), 0);
            kernels::launch_backward_pass(d_emis.as<float>(), trans.get_transition_matrices(),
                                          d_states.as<uint32_t>(), d_ckpt.as<float>(), d_scale.as<float>(),
                                          B, M, L, C, d_post.as<float>(), 0);
            RCK(cudaEventRecord(ev[2], 0));
            sampler.sample(d_post.as<float>(), d_states.as<uint32_t>(), d_out.as<uint8_t>(), B, true);
            RCK(cudaEventRecord(ev[3], 0));
            RCK(cudaDeviceSynchronize());
        }
        if (stage_ms)
            for (int s = 0; s < 3; ++s) RCK(cudaEventElapsedTime(&stage_ms[s], ev[s], ev[s + 1]));
        for (auto& e : ev) cudaEventDestroy(e);
        return 0;
    } catch (...) {
        return 2;
    }
}
