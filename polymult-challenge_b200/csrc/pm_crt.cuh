// pm_crt.cuh -- the last step of the CRT, shared by the plain and the tensor-core kernels:
// reduce z = sum_j y_j [(M/p_j) mod q] + [(-vM) mod q] (z < 2^(W+64), zl limbs) to z mod q.
// Uses 2^W == delta (mod q) with delta = 2^W - q < 2^63: while z >= 2^W, z = (z mod 2^W) +
// (z >> W) delta; then one conditional subtraction of q (z < 2^W = q + delta < 2q).
// Same reduction as the reference's CRT tail (solve.cu:462-493); the loop here is bounded
// and reports non-convergence in the device status word instead of spinning.
#pragma once

#include "pm_device.cuh"

namespace pm {

__device__ __forceinline__ void crt_reduce_mod_q(uint32_t* z, int zl, const DevPlan& P) {
    const int wl = P.W >> 5, wb = P.W & 31, L = P.L;
    bool done = false;
    for (int iter = 0; iter < 64 && !done; ++iter) {
        uint64_t hi;
        if (wb == 0) hi = (uint64_t)z[wl] | ((uint64_t)z[wl + 1] << 32);
        else
            hi = ((uint64_t)z[wl] >> wb) | ((uint64_t)z[wl + 1] << (32 - wb)) | ((uint64_t)z[wl + 2] << (64 - wb));
        if (hi == 0) {
            done = true;
            break;
        }
        z[wl] = wb ? (z[wl] & ((1u << wb) - 1u)) : 0u;
        for (int l = wl + 1; l < zl; ++l) z[l] = 0;
        const uint64_t lo64 = hi * P.delta, hi64 = __umul64hi(hi, P.delta);
        const uint32_t add4[4] = {(uint32_t)lo64, (uint32_t)(lo64 >> 32), (uint32_t)hi64, (uint32_t)(hi64 >> 32)};
        uint64_t c = 0;
        for (int l = 0; l < zl; ++l) {
            const uint64_t s = (uint64_t)z[l] + (l < 4 ? add4[l] : 0u) + c;
            z[l] = (uint32_t)s;
            c = s >> 32;
            if (l >= 3 && c == 0) break;
        }
    }
    if (!done) flag_error(P.status, DEV_ERR_FOLD);
    bool ge = true;
    for (int l = L - 1; l >= 0; --l) {
        const uint32_t ql = P.q[l];
        if (z[l] != ql) {
            ge = z[l] > ql;
            break;
        }
    }
    if (ge) {
        uint64_t br = 0;
        for (int l = 0; l < L; ++l) {
            const uint64_t d = (uint64_t)z[l] - P.q[l] - br;
            z[l] = (uint32_t)d;
            br = (d >> 63) & 1u;
        }
    }
}

}  // namespace pm
