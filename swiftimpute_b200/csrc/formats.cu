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
    if ((M & 3u) == 0) {  // 4-byte aligned rows: the four codes as one word
        *reinterpret_cast<uint32_t*>(o) = (v & 3u) | ((v << 6) & 0x300u) | ((v << 12) & 0x30000u) | ((v << 18) & 0x3000000u);
        return;
    }
#pragma unroll
    for (uint32_t t = 0; t < 4; ++t)
        if (4 * j + t < M) o[t] = (uint8_t)((v >> (2 * t)) & 3u);
}

// 16 bytes -> 16 bits, bit j set for a non-zero byte j
__device__ __forceinline__ uint32_t nonzero16(uint4 x) {
    const uint32_t w[4] = {x.x, x.y, x.z, x.w};
    uint32_t bits = 0;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const uint32_t b = __vcmpne4(w[q], 0u);  // 0xff in each non-zero byte
        bits |= (((b >> 7) & 1u) | ((b >> 14) & 2u) | ((b >> 21) & 4u) | ((b >> 28) & 8u)) << (4 * q);
    }
    return bits;
}

// [rows][M] allele bytes -> [rows][Mw] bit words; two threads per word, each
// reading its 16 bytes in one 128-bit load when the rows are 16-byte aligned.
__global__ void pack_haps_kernel(const uint8_t* __restrict__ in, uint64_t rows, uint32_t M, uint32_t Mw,
                                 uint32_t* __restrict__ out) {
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = t < rows * Mw * 2;
    uint32_t bits = 0;
    uint64_t r = 0;
    uint32_t w = 0, h = 0;
    if (valid) {
        r = t / (2ull * Mw);
        const uint32_t q = (uint32_t)(t % (2ull * Mw));
        w = q >> 1;
        h = q & 1u;
        const uint32_t m0 = 32 * w + 16 * h;
        const uint8_t* row = in + r * M;
        if ((M & 15u) == 0 && (reinterpret_cast<uintptr_t>(in) & 15u) == 0 && m0 + 16 <= M) {
            bits = nonzero16(*reinterpret_cast<const uint4*>(row + m0));
        } else {
            for (uint32_t j = 0; j < 16 && m0 + j < M; ++j) bits |= (row[m0 + j] != 0 ? 1u : 0u) << j;
        }
    }
    const uint32_t other = __shfl_xor_sync(0xffffffffu, bits, 1);  // the word's other half
    if (valid && h == 0) out[r * Mw + w] = bits | (other << 16);
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
    const uint64_t threads = rows * Mw * 2;
    if (threads == 0) return cudaSuccess;
    const uint64_t grid = (threads + 255) / 256;
    if (grid > 0x7fffffffull) return cudaErrorInvalidConfiguration;
    pack_haps_kernel<<<(uint32_t)grid, 256, 0, s>>>(d_in, rows, M, Mw, d_out);
    return cudaGetLastError();
}

}  // namespace si
