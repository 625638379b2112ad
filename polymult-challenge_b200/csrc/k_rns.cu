// k_rns.cu -- the plain (CUDA-core int32) forms of the two dense integer contractions:
//   RNS decomposition  R[j][n] = a_n mod p_j                       (solve.cu:147-202)
//   CRT straight to mod q  c_n = sum_j y_j Q_j + T_v  (mod q)      (solve.cu:380-501)
// These are the comparator for the tensor-core forms in k_tc.cu and the path for shapes
// the tensor-core kernels do not cover.
//
// Decomposition: a_n = sum_h half_h 2^(16h) over the 2L 16-bit halves of its limbs.  With
// dec16[h][j] = 2^(16h) R mod p_j the 64-bit dot product stays < 2L 2^16 p < p 2^32, so one
// REDC returns a_n mod p_j.  Each thread owns a 4-coefficient x 4-prime tile.
#include "pm_crt.cuh"
#include "pm_kernels.cuh"

namespace pm {

__global__ void __launch_bounds__(256) k_rns_plain(DevPlan P, const uint32_t* __restrict__ src, ChunkMap C,
                                                   uint32_t npos, uint32_t* __restrict__ R, int tab_in_smem) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int L = P.L, H = 2 * L, KP = P.KP;
    uint32_t* tab_s = reinterpret_cast<uint32_t*>(smem_raw);                                  // [2L][KP]
    uint16_t* hs = reinterpret_cast<uint16_t*>(tab_s + (tab_in_smem ? (size_t)H * KP : 0));  // [2L][DEC_TM]
    const uint32_t b = blockIdx.z;
    const uint32_t pos0 = blockIdx.x * DEC_TM;
    const int cnt = (int)min((uint32_t)DEC_TM, npos - pos0);
    const uint32_t* s = src + ((size_t)b * npos + pos0) * L;
    uint32_t* Rb = R + (size_t)b * P.K * P.N;
    pdl_trigger();
    pdl_wait();

    for (int idx = threadIdx.x; idx < L * DEC_TM; idx += blockDim.x) {
        const int l = idx / DEC_TM, m = idx - l * DEC_TM;
        const uint32_t v = m < cnt ? __ldg(s + (size_t)m * L + l) : 0u;
        hs[(2 * l) * DEC_TM + m] = (uint16_t)(v & 0xFFFFu);
        hs[(2 * l + 1) * DEC_TM + m] = (uint16_t)(v >> 16);
    }
    if (tab_in_smem)
        for (int idx = threadIdx.x; idx < H * KP / 4; idx += blockDim.x)
            reinterpret_cast<uint4*>(tab_s)[idx] = reinterpret_cast<const uint4*>(P.dec16)[idx];
    __syncthreads();

    const uint4* tab = reinterpret_cast<const uint4*>(tab_in_smem ? tab_s : P.dec16);
    constexpr int MG = DEC_TM / 4;
    for (int task = threadIdx.x; task < MG * (KP / 4); task += blockDim.x) {
        const int mg = task % MG, jg = task / MG;
        uint64_t acc[4][4];
#pragma unroll
        for (int x = 0; x < 4; ++x)
#pragma unroll
            for (int y = 0; y < 4; ++y) acc[x][y] = 0;
        for (int h = 0; h < H; ++h) {
            const uint2 a4 = *reinterpret_cast<const uint2*>(hs + h * DEC_TM + 4 * mg);
            const uint4 c4 = tab[h * (KP / 4) + jg];
            const uint32_t av[4] = {a4.x & 0xFFFFu, a4.x >> 16, a4.y & 0xFFFFu, a4.y >> 16};
            const uint32_t cv[4] = {c4.x, c4.y, c4.z, c4.w};
#pragma unroll
            for (int x = 0; x < 4; ++x)
#pragma unroll
                for (int y = 0; y < 4; ++y) acc[x][y] += (uint64_t)av[x] * cv[y];
        }
#pragma unroll
        for (int y = 0; y < 4; ++y) {
            const int j = 4 * jg + y;
            if (j >= P.K) continue;
            const uint32_t p = P.p[j], pinv = P.pinv[j];
#pragma unroll
            for (int x = 0; x < 4; ++x) {
                const int m = 4 * mg + x;
                if (m >= cnt) continue;
                Rb[(size_t)j * P.N + chunk_pos_to_n(P, C, pos0 + m)] = red_once(redc64(acc[x][y], p, pinv), p);
            }
        }
    }
}

// CRT of CRT_TM positions.  y_j = r_j crt_c_j 2^-32 = x_j (M/p_j)^-1 mod p_j (the N^-1 of the
// inverse NTT and the 2^-32 of the pointwise product are folded into crt_c).
// v = round(sum_j y_j / p_j) in fp32: the true sum is within 1/8 of v because |x| < M/8, so a
// distance above 1/4 flags DEV_ERR_CRT_BOUND.  acc[m][h] = sum_j y_j Qh[j][h] over the 16-bit
// halves of Q_j = (M/p_j) mod q, then carries, + T_v, and the delta-fold reduction.
__global__ void __launch_bounds__(128) k_crt_plain(DevPlan P, const uint32_t* __restrict__ R, ChunkMap C,
                                                   uint32_t npos, uint32_t* __restrict__ out) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int K = P.K, KP = P.KP, L = P.L, HP = P.HP;
    const int zl = crt_zl(L), zs = crt_zstride(L);
    uint64_t* acc_s = reinterpret_cast<uint64_t*>(smem_raw);                  // [CRT_TM][HP]
    uint32_t* y_s = reinterpret_cast<uint32_t*>(acc_s + (size_t)CRT_TM * HP);  // [KP][CRT_TM]
    uint32_t* z_s = y_s + (size_t)KP * CRT_TM;                                 // [CRT_TM][zs]
    int* v_s = reinterpret_cast<int*>(z_s + (size_t)CRT_TM * zs);              // [CRT_TM]
    const uint32_t b = blockIdx.z;
    const uint32_t pos0 = blockIdx.x * CRT_TM;
    const int cnt = (int)min((uint32_t)CRT_TM, npos - pos0);
    const uint32_t* Rb = R + (size_t)b * K * P.N;
    pdl_trigger();
    pdl_wait();

    for (int idx = threadIdx.x; idx < KP * CRT_TM; idx += blockDim.x) {
        const int j = idx / CRT_TM, m = idx - j * CRT_TM;
        uint32_t y = 0;
        if (j < K && m < cnt) {
            const uint32_t p = P.p[j];
            const uint32_t r = Rb[(size_t)j * P.N + chunk_pos_to_n(P, C, pos0 + m)];
            y = red_once(mul_ms(r, P.crt_c[j], P.crt_cc[j], p), p);
        }
        y_s[idx] = y;
    }
    __syncthreads();
    for (int m = threadIdx.x; m < CRT_TM; m += blockDim.x) {
        float s = 0.f;
        for (int j = 0; j < K; ++j) s = fmaf((float)y_s[j * CRT_TM + m], P.rcp[j], s);
        const float v = rintf(s);
        if (m < cnt && fabsf(s - v) > 0.25f) flag_error(P.status, DEV_ERR_CRT_BOUND);
        v_s[m] = min(max((int)v, 0), K);
    }
    constexpr int MG = CRT_TM / 4;
    for (int task = threadIdx.x; task < MG * (HP / 4); task += blockDim.x) {
        const int mg = task % MG, hg = task / MG;
        uint64_t acc[4][4];
#pragma unroll
        for (int x = 0; x < 4; ++x)
#pragma unroll
            for (int y = 0; y < 4; ++y) acc[x][y] = 0;
        const uint2* qtab = reinterpret_cast<const uint2*>(P.qh16);
        for (int j = 0; j < K; ++j) {
            const uint4 y4 = *reinterpret_cast<const uint4*>(y_s + j * CRT_TM + 4 * mg);
            const uint2 q4 = __ldg(qtab + j * (HP / 4) + hg);
            const uint32_t yv[4] = {y4.x, y4.y, y4.z, y4.w};
            const uint32_t qv[4] = {q4.x & 0xFFFFu, q4.x >> 16, q4.y & 0xFFFFu, q4.y >> 16};
#pragma unroll
            for (int x = 0; x < 4; ++x)
#pragma unroll
                for (int y = 0; y < 4; ++y) acc[x][y] += (uint64_t)yv[x] * qv[y];
        }
#pragma unroll
        for (int x = 0; x < 4; ++x)
#pragma unroll
            for (int y = 0; y < 4; ++y) acc_s[(4 * mg + x) * HP + 4 * hg + y] = acc[x][y];
    }
    __syncthreads();

    for (int m = threadIdx.x; m < cnt; m += blockDim.x) {
        uint32_t* z = z_s + (size_t)m * zs;
        const uint64_t* a = acc_s + (size_t)m * HP;
        const uint32_t* T = P.tneg + (size_t)v_s[m] * L;
        uint64_t carry = 0;
        for (int l = 0; l < zl; ++l) {
            const uint64_t t0 = 2 * l < HP ? a[2 * l] : 0, t1 = 2 * l + 1 < HP ? a[2 * l + 1] : 0;
            const uint64_t t = carry + t0 + ((t1 & 0xFFFFull) << 16) + (l < L ? T[l] : 0u);
            z[l] = (uint32_t)t;
            carry = (t >> 32) + (t1 >> 16);
        }
        crt_reduce_mod_q(z, zl, P);
    }
    __syncthreads();
    uint32_t* o = out + ((size_t)b * npos + pos0) * L;
    for (int idx = threadIdx.x; idx < cnt * L; idx += blockDim.x) {
        const int m = idx / L, l = idx - m * L;
        o[idx] = z_s[(size_t)m * zs + l];
    }
}

size_t rns_plain_smem(const DevPlan& P, bool tab_in_smem) {
    return (tab_in_smem ? (size_t)2 * P.L * P.KP * 4 : 0) + (size_t)2 * P.L * DEC_TM * 2;
}

size_t crt_plain_smem(const DevPlan& P) {
    return (size_t)CRT_TM * P.HP * 8 + (size_t)P.KP * CRT_TM * 4 + (size_t)CRT_TM * crt_zstride(P.L) * 4 +
           CRT_TM * 4;
}

}  // namespace pm
