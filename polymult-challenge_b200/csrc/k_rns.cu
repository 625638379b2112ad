// k_rns.cu -- the plain (CUDA-core int32) forms of the two dense integer contractions: the
// comparator of the tensor-core forms in k_tc.cu and the path for shapes those do not cover.
//   RNS decomposition  R[j][n] = a_n mod p_j                       (reference: solve.cu:147-202)
//   CRT straight to mod q  c_n = sum_j y_j Q_j + v T_1  (mod q)    (reference: solve.cu:380-501)
//
// Both run on 24-bit digits: a W-bit value is sum_d x_d 2^(24 d), d < D = ceil(W / 24), and four
// digits come from three 32-bit limbs.  A 30-bit factor times a digit is below 2^54, so every
// dot product here (at most 1023 terms) accumulates exactly in 64 bits with one wide
// multiply-add per term, over D digit rows instead of the 2L rows that 16-bit halves need
// (73 against 110 at W = 1747).
//
// Decomposition: t = sum_d a_d (2^(24 d) R mod p) < D 2^24 p < p 2^32, so one REDC gives
// a mod p in (0, 2p) (the forward transform takes inputs below 4p).  Each thread owns a tile of
// 4 coefficients x 4 primes.
//
// CRT: y_j = r_j crt_c_j 2^-32 mod p_j (the N^-1 of the inverse transform and the 2^-32 of the
// pointwise product are folded into crt_c); v = round(sum_j y_j / p_j) in fp32 (|x| < M/8 puts
// the true sum within 1/8 of v, so a distance above 1/4 flags DEV_ERR_CRT_BOUND) becomes row K
// of the y matrix against the digits of T_1 = (-M) mod q, so the GEMM itself adds v T_1; then
// S[m][d] = sum_j y_j[m] digit_d(Q_j) are carried into 32-bit limbs and reduced mod q
// (pm_crt.cuh).  Each thread owns a tile of 4 coefficients x 4 digits.
#include "pm_crt.cuh"
#include "pm_kernels.cuh"
#include "pm_plan.h"

namespace pm {
namespace {

// the four 24-bit digits held by limbs 3g .. 3g + 2 (limbs past the last read as zero)
__device__ __forceinline__ uint4 digits_of_three(uint32_t l0, uint32_t l1, uint32_t l2) {
    return make_uint4(l0 & 0xFFFFFFu, __funnelshift_r(l0, l1, 24) & 0xFFFFFFu, __funnelshift_r(l1, l2, 16) & 0xFFFFFFu,
                      l2 >> 8);
}

// Digit rows dig[d][m] (row stride TM) of the cnt coefficients staged row-major in raw[m][L];
// positions past cnt get zero digits.  m runs fastest over the threads, so that the strided
// reads of raw (L odd or even) and the row writes of dig stay spread over the banks.
template <int TM>
__device__ __forceinline__ void stage_digits(const uint32_t* raw, uint32_t* dig, int L, int DP, int cnt) {
    const int groups = DP / 4;
    for (int idx = threadIdx.x; idx < groups * TM; idx += blockDim.x) {
        const int g = idx / TM, m = idx - g * TM;
        uint4 d4 = make_uint4(0, 0, 0, 0);
        if (m < cnt) {
            const uint32_t* r = raw + m * L;
            const int l = 3 * g;
            d4 = digits_of_three(l < L ? r[l] : 0u, l + 1 < L ? r[l + 1] : 0u, l + 2 < L ? r[l + 2] : 0u);
        }
        dig[(4 * g) * TM + m] = d4.x;
        dig[(4 * g + 1) * TM + m] = d4.y;
        dig[(4 * g + 2) * TM + m] = d4.z;
        dig[(4 * g + 3) * TM + m] = d4.w;
    }
}

// acc[x][y] += a[x] * b[y], 64-bit accumulators
__device__ __forceinline__ void mac4x4(uint64_t (&acc)[4][4], uint4 a, uint4 b) {
    const uint32_t av[4] = {a.x, a.y, a.z, a.w}, bv[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
    for (int x = 0; x < 4; ++x)
#pragma unroll
        for (int y = 0; y < 4; ++y) acc[x][y] += (uint64_t)av[x] * bv[y];
}

}  // namespace

// smem: [raw TM x L][digits DP x TM][table DP x KP if tab_in_smem]
__global__ void __launch_bounds__(256) k_rns_plain(DevPlan P, const uint32_t* __restrict__ src, ChunkMap C,
                                                   uint32_t npos, uint32_t* __restrict__ R, int tab_in_smem) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int TM = DEC_TM;
    const int L = P.L, DP = P.DP, KP = P.KP;
    uint32_t* raw = reinterpret_cast<uint32_t*>(smem_raw);
    uint32_t* dig = raw + ((TM * L + 3) & ~3);
    uint32_t* tab_s = dig + DP * TM;
    const uint32_t pos0 = blockIdx.x * TM;
    const int cnt = (int)min((uint32_t)TM, npos - pos0);
    const uint32_t* s = src + ((size_t)blockIdx.z * npos + pos0) * L;
    uint32_t* Rb = R + (size_t)blockIdx.z * P.Kr * P.N;
    if (tab_in_smem)  // a constant table: before the dependency wait
        for (int idx = threadIdx.x; idx < DP * KP / 4; idx += blockDim.x)
            reinterpret_cast<uint4*>(tab_s)[idx] = __ldg(reinterpret_cast<const uint4*>(P.dec24) + idx);
    pdl_trigger();
    pdl_wait();
    for (int w = threadIdx.x; w < cnt * L; w += blockDim.x) raw[w] = __ldg(s + w);  // contiguous
    __syncthreads();
    stage_digits<TM>(raw, dig, L, DP, cnt);
    __syncthreads();

    const uint4* tab = reinterpret_cast<const uint4*>(tab_in_smem ? tab_s : P.dec24);
    constexpr int MT = TM / 4;
    for (int task = threadIdx.x; task < MT * (KP / 4); task += blockDim.x) {
        const int mt = task % MT, jt = task / MT;
        uint64_t acc[4][4] = {};
        for (int d = 0; d < P.D; ++d)
            mac4x4(acc, *reinterpret_cast<const uint4*>(dig + d * TM + 4 * mt), tab[d * (KP / 4) + jt]);
#pragma unroll
        for (int y = 0; y < 4; ++y) {
            const int j = 4 * jt + y;
            if (j >= P.K) break;
            const uint32_t p = P.p[j], pinv = P.pinv[j];
            uint32_t* row = Rb + (size_t)j * P.N;
#pragma unroll
            for (int x = 0; x < 4; ++x) {
                const int m = 4 * mt + x;
                if (m < cnt) row[chunk_pos_to_n(P, C, pos0 + m)] = redc64(acc[x][y], p, pinv);
            }
        }
    }
}

// smem: [y (K+1) x TM][S TM x DP (u64)][z TM x zs][table (K+1) x DP if tab_in_smem]
__global__ void __launch_bounds__(256) k_crt_plain(DevPlan P, const uint32_t* __restrict__ R, ChunkMap C,
                                                   uint32_t npos, uint32_t* __restrict__ out, int tab_in_smem) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int TM = CRT_TM;
    const int K = P.K, L = P.L, DP = P.DP;
    const int zl = crt_zl(L), zs = crt_zstride(L);
    uint32_t* y = reinterpret_cast<uint32_t*>(smem_raw);                          // [K + 1][TM]
    uint64_t* S = reinterpret_cast<uint64_t*>(y + (((K + 1) * TM + 3) & ~3));      // [TM][DP]
    uint32_t* z = reinterpret_cast<uint32_t*>(S + (size_t)TM * DP);                // [TM][zs]
    uint32_t* tab_s = z + ((TM * zs + 3) & ~3);                                    // [K + 1][DP]
    const uint32_t pos0 = blockIdx.x * TM;
    const int cnt = (int)min((uint32_t)TM, npos - pos0);
    const uint32_t* Rb = R + (size_t)blockIdx.z * P.Kr * P.N;
    if (tab_in_smem)
        for (int idx = threadIdx.x; idx < (K + 1) * DP / 4; idx += blockDim.x)
            reinterpret_cast<uint4*>(tab_s)[idx] = __ldg(reinterpret_cast<const uint4*>(P.crt24) + idx);
    pdl_trigger();
    pdl_wait();

    // y_j in [0, p_j); positions past cnt repeat the first one (their rows are never stored)
    for (int idx = threadIdx.x; idx < K * TM; idx += blockDim.x) {
        const int j = idx / TM, m = idx - j * TM;
        const uint32_t p = P.p[j];
        const uint32_t r = Rb[(size_t)j * P.N + chunk_pos_to_n(P, C, pos0 + (m < cnt ? m : 0))];
        y[idx] = red_once(mul_ms(r, P.crt_c[j], P.crt_cc[j], p), p);
    }
    __syncthreads();
    // v: four threads per coefficient, each over every fourth prime, then a shuffle sum
    static_assert(TM * 4 == 256, "four threads per coefficient");
    {
        const int m = threadIdx.x >> 2, part = threadIdx.x & 3;
        float s = 0.f;
        for (int j = part; j < K; j += 4) s = fmaf((float)y[j * TM + m], P.rcp[j], s);
        s += __shfl_xor_sync(0xffffffffu, s, 1);
        s += __shfl_xor_sync(0xffffffffu, s, 2);
        if (part == 0) {
            const float v = rintf(s);
            if (m < cnt && fabsf(s - v) > 0.25f) flag_error(P.status, DEV_ERR_CRT_BOUND);
            y[K * TM + m] = (uint32_t)min(max((int)v, 0), K);
        }
    }
    __syncthreads();

    // S[m][d] = sum_{j <= K} y_j[m] digit_d(row j), every sum < (K + 1) 2^54 < 2^64
    const uint4* tab = reinterpret_cast<const uint4*>(tab_in_smem ? tab_s : P.crt24);
    constexpr int MT = TM / 4;
    for (int task = threadIdx.x; task < MT * (DP / 4); task += blockDim.x) {
        const int mt = task % MT, dt = task / MT;
        uint64_t acc[4][4] = {};
        for (int j = 0; j <= K; ++j)
            mac4x4(acc, *reinterpret_cast<const uint4*>(y + j * TM + 4 * mt), tab[j * (DP / 4) + dt]);
#pragma unroll
        for (int x = 0; x < 4; ++x)
#pragma unroll
            for (int d = 0; d < 4; ++d) S[(size_t)(4 * mt + x) * DP + 4 * dt + d] = acc[x][d];
    }
    __syncthreads();

    // z = sum_d S[m][d] 2^(24 d) into zl limbs (the value is below the plan's CRT bound, so every
    // limb past zl is zero), then mod q
    for (int m = threadIdx.x; m < cnt; m += blockDim.x) {
        uint32_t* zm = z + (size_t)m * zs;
        const uint64_t* sm = S + (size_t)m * DP;
        unsigned __int128 acc = 0;
        int e = 0;  // limbs emitted: acc holds the value's bits from 32 e up
        for (int d = 0; d < DP; ++d) {
            acc += (unsigned __int128)sm[d] << (kDigitBits * d - 32 * e);
            for (; kDigitBits * (d + 1) - 32 * e >= 32; ++e, acc >>= 32)
                if (e < zl) zm[e] = (uint32_t)acc;
        }
        for (; e < zl; ++e, acc >>= 32) zm[e] = (uint32_t)acc;
        crt_reduce_mod_q(zm, zl, P);
    }
    __syncthreads();
    uint32_t* o = out + ((size_t)blockIdx.z * npos + pos0) * L;
    for (int w = threadIdx.x; w < cnt * L; w += blockDim.x) {
        const int m = w / L;
        o[w] = z[(size_t)m * zs + (w - m * L)];
    }
}

size_t rns_plain_smem(const DevPlan& P, bool tab_in_smem) {
    return (size_t)((DEC_TM * P.L + 3) & ~3) * 4 + (size_t)P.DP * DEC_TM * 4 + (tab_in_smem ? (size_t)P.DP * P.KP * 4 : 0);
}

size_t crt_plain_smem(const DevPlan& P, bool tab_in_smem) {
    return (size_t)(((P.K + 1) * CRT_TM + 3) & ~3) * 4 + (size_t)CRT_TM * P.DP * 8 +
           (size_t)((CRT_TM * crt_zstride(P.L) + 3) & ~3) * 4 + (tab_in_smem ? (size_t)(P.K + 1) * P.DP * 4 : 0);
}

}  // namespace pm
