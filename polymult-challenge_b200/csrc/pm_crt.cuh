// pm_crt.cuh -- the last step of every CRT kernel: z (zl little-endian limbs in memory) to
// z mod q, for q = 2^W - delta (0 < delta < 2^63, so 2^W == delta mod q).
//
// The host bounds the CRT value: z < Plan::crt_bound < 2^(W+64), and from that bound derives
// P.fold_count, the number of folds
//     z -> (z mod 2^W) + h delta,   h = the 64 bits of z from bit W up,
// after which every admissible z is below 2q (one fold at every point with W a few bits above
// 64 + bits(delta); a few more only for W of a few dozen bits).  Below 2q, z >= q exactly when
// z + delta reaches 2^W, and then z - q = (z + delta) mod 2^W: so the last step adds delta and
// keeps the sum (minus 2^W) when bit W is set, else takes delta back off.  There is no
// data-dependent loop count (only carry ripples past the fourth limb, which almost never run);
// bits beyond the bound flag DEV_ERR_FOLD.
#pragma once

#include "pm_device.cuh"

namespace pm {

// z[0..3] += lo + hi 2^64 with the hardware carry chain; returns the carry out of limb 3
__device__ __forceinline__ uint32_t crt_add128(uint32_t* z, uint64_t lo, uint64_t hi) {
    uint32_t z0 = z[0], z1 = z[1], z2 = z[2], z3 = z[3], c;
    asm("add.cc.u32 %0, %0, %5;\n\t"
        "addc.cc.u32 %1, %1, %6;\n\t"
        "addc.cc.u32 %2, %2, %7;\n\t"
        "addc.cc.u32 %3, %3, %8;\n\t"
        "addc.u32 %4, 0, 0;"
        : "+r"(z0), "+r"(z1), "+r"(z2), "+r"(z3), "=r"(c)
        : "r"((uint32_t)lo), "r"((uint32_t)(lo >> 32)), "r"((uint32_t)hi), "r"((uint32_t)(hi >> 32)));
    z[0] = z0;
    z[1] = z1;
    z[2] = z2;
    z[3] = z3;
    return c;
}

// z[0..1] -= v; returns the borrow out of limb 1
__device__ __forceinline__ uint32_t crt_sub64(uint32_t* z, uint64_t v) {
    uint32_t z0 = z[0], z1 = z[1], b;
    asm("sub.cc.u32 %0, %0, %3;\n\t"
        "subc.cc.u32 %1, %1, %4;\n\t"
        "subc.u32 %2, 0, 0;"
        : "+r"(z0), "+r"(z1), "=r"(b)
        : "r"((uint32_t)v), "r"((uint32_t)(v >> 32)));
    z[0] = z0;
    z[1] = z1;
    return b & 1u;
}

__device__ __forceinline__ void crt_reduce_mod_q(uint32_t* z, int zl, const DevPlan& P) {
    const int wl = P.W >> 5, wb = P.W & 31;
    const uint32_t keep = wb ? (1u << wb) - 1u : 0u;  // bits of limb wl below bit W
    // bits from W + 64 up lie outside every bound the host derived
    uint32_t outside = wb ? (z[wl + 2] >> wb) : z[wl + 2];
    for (int l = wl + 3; l < zl; ++l) outside |= z[l];
    for (int f = 0; f < P.fold_count; ++f) {
        const uint64_t h = ((uint64_t)__funnelshift_r(z[wl + 1], z[wl + 2], wb) << 32) | __funnelshift_r(z[wl], z[wl + 1], wb);
        z[wl] &= keep;
        for (int l = wl + 1; l < zl; ++l) z[l] = 0;
        uint32_t c = crt_add128(z, h * P.delta, __umul64hi(h, P.delta));
        for (int l = 4; c && l < zl; ++l) c = ++z[l] == 0u;
    }
    // now z < 2q: bits from W + 1 up are zero
    outside |= wb < 31 ? z[wl] >> (wb + 1) : 0u;
    for (int l = wl + 1; l < zl; ++l) outside |= z[l];
    if (outside) flag_error(P.status, DEV_ERR_FOLD);
    // z >= q  <=>  z + delta >= 2^W
    uint32_t c = crt_add128(z, P.delta, 0);
    for (int l = 4; c && l < zl; ++l) c = ++z[l] == 0u;
    if ((z[wl] >> wb) & 1u) {
        z[wl] &= keep;  // z + delta - 2^W = z - q
    } else {
        uint32_t b = crt_sub64(z, P.delta);
        for (int l = 2; b && l < zl; ++l) b = z[l]-- == 0u;
    }
}

}  // namespace pm
