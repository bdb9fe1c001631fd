// formats.cu — compact host formats of si_impute, converted on the device.
//
// Codes in: 2 bits per cell, four cells per byte (cell m at bits 2 (m % 4) of
// byte m / 4 of its sample's row), a quarter of the one-byte codes. Haplotypes
// out: one bit per allele (bit m % 32 of word m / 32 of the haplotype's row,
// set for a non-zero allele), an eighth of the byte layout. The conversions
// run on the device beside the imputation, so only the compact bytes cross
// the host link.
#include "si_internal.hpp"

namespace si {
namespace {

// [rows][Mb] 2-bit codes -> [rows][M] bytes; one thread per packed byte.
__global__ void unpack_codes_kernel(const uint8_t* __restrict__ in, uint64_t rows, uint32_t M, uint32_t Mb,
                                    uint8_t* __restrict__ out) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= rows * Mb) return;
    const uint64_t r = i / Mb;
    const uint32_t j = (uint32_t)(i % Mb);
    const uint32_t v = in[i];
    uint8_t* o = out + r * M + 4ull * j;
#pragma unroll
    for (uint32_t t = 0; t < 4; ++t)
        if (4 * j + t < M) o[t] = (uint8_t)((v >> (2 * t)) & 3u);
}

// [rows][M] allele bytes -> [rows][Mw] bit words; one warp per word: lane =
// marker, a ballot of the non-zero bytes.
__global__ void pack_haps_kernel(const uint8_t* __restrict__ in, uint64_t rows, uint32_t M, uint32_t Mw,
                                 uint32_t* __restrict__ out) {
    const uint64_t wg = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31;
    if (wg >= rows * Mw) return;  // whole warps (blockDim a multiple of 32)
    const uint64_t r = wg / Mw;
    const uint32_t w = (uint32_t)(wg % Mw);
    const uint32_t m = 32 * w + lane;
    const bool one = m < M && in[r * M + m] != 0;
    const uint32_t bits = __ballot_sync(0xffffffffu, one);
    if (lane == 0) out[wg] = bits;
}

}  // namespace

cudaError_t launch_unpack_codes(const uint8_t* d_in, uint64_t rows, uint32_t M, uint8_t* d_out, cudaStream_t s) {
    const uint32_t Mb = (M + 3) / 4;
    const uint64_t n = rows * Mb;
    if (n == 0) return cudaSuccess;
    const uint64_t grid = (n + 255) / 256;
    if (grid > 0x7fffffffull) return cudaErrorInvalidConfiguration;
    unpack_codes_kernel<<<(uint32_t)grid, 256, 0, s>>>(d_in, rows, M, Mb, d_out);
    return cudaGetLastError();
}

cudaError_t launch_pack_haps(const uint8_t* d_in, uint64_t rows, uint32_t M, uint32_t* d_out, cudaStream_t s) {
    const uint32_t Mw = (M + 31) / 32;
    const uint64_t threads = rows * Mw * 32;
    if (threads == 0) return cudaSuccess;
    const uint64_t grid = (threads + 255) / 256;
    if (grid > 0x7fffffffull) return cudaErrorInvalidConfiguration;
    pack_haps_kernel<<<(uint32_t)grid, 256, 0, s>>>(d_in, rows, M, Mw, d_out);
    return cudaGetLastError();
}

}  // namespace si
