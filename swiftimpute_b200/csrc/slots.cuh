// slots.cuh — per-marker slot data as the forward-backward kernels read it.
#pragma once
#include "si_internal.hpp"

namespace si {

// Emission mask of the slots whose pair matches genotype code g. The
// reference picks the GL entry by the sum of the pair's two allele bytes
// (emission.cu:35-54): 0 -> ll_00, 1 -> ll_01, anything else -> ll_11, so a
// missing (255) or multi-allelic panel allele puts its pair in the ll_11 class
// unless the other allele makes the sum exactly 1, which needs alleles 0 and 1.
// Codes above 2 are missing calls: every slot, *shift = 0. A call no slot
// matches: every slot, *shift = 1 (the reference scales every slot by e^-999).
__device__ __forceinline__ uint32_t emission_mask(uint32_t g, const SlotMasks& mk, uint32_t lmask, uint32_t* shift) {
    const uint32_t het = (mk.a0 ^ mk.a1) & ~mk.x;  // byte sum exactly 1
    uint32_t mg;
    if (g == 0) mg = ~(mk.a0 | mk.a1);
    else if (g == 1) mg = het;
    else if (g == 2) mg = (mk.a0 | mk.a1) & ~het;
    else {
        *shift = 0;
        return lmask;
    }
    mg &= lmask;
    *shift = mg ? 0u : 1u;
    return mg ? mg : lmask;
}

// Allele bytes of slot k at marker m, the pair's first haplotype in the low
// byte: the panel bits for 0/1 alleles, the raw table [marker][gs][2] where
// the slot holds another allele (the reference's sampler copies the panel
// byte, sampling.cu:121-126).
__device__ __forceinline__ uint32_t slot_alleles(const SlotMasks& mk, const uint8_t* raw, uint32_t gs, uint32_t m,
                                                 uint32_t k) {
    if ((mk.x >> k) & 1u) {
        const uint8_t* r = raw + ((size_t)m * gs + k) * 2;
        return (uint32_t)r[0] | ((uint32_t)r[1] << 8);
    }
    return ((mk.a0 >> k) & 1u) | (((mk.a1 >> k) & 1u) << 8);
}

}  // namespace si
