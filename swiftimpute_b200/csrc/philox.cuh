// philox.cuh — Philox4x32-10 counter-based generator (Salmon, Moraes, Dror,
// Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC'11), written from
// the published round function. Only the first output word is used.
#pragma once
#include <cstdint>

namespace si {

__host__ __device__ __forceinline__ uint32_t philox4x32_10_w0(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                                             uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        if (r) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
#ifdef __CUDA_ARCH__
        const uint32_t hi0 = __umulhi(0xD2511F53u, c0), lo0 = 0xD2511F53u * c0;
        const uint32_t hi1 = __umulhi(0xCD9E8D57u, c2), lo1 = 0xCD9E8D57u * c2;
#else
        const uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
        const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
#endif
        const uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
    }
    return c0;
}

// Uniform in [0, 1) with 24 random bits for cell (sample_id, marker).
__host__ __device__ __forceinline__ float cell_uniform(uint64_t seed, uint64_t sample_id, uint32_t marker) {
    const uint32_t x = philox4x32_10_w0(marker, (uint32_t)sample_id, (uint32_t)(sample_id >> 32), 0u,
                                        (uint32_t)seed, (uint32_t)(seed >> 32));
    return (float)(x >> 8) * (1.0f / 16777216.0f);
}

}  // namespace si
