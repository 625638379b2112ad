// k_ntt.cu -- the negacyclic NTT per RNS prime, 4-step split into a column pass and a row
// pass over the residue arrays R[batch][prime][n], n = row * ncols + col.
//
// Same transform as the reference (psi-merged Cooley-Tukey forward, natural order in and
// bit-reversed out; Gentleman-Sande inverse with the mirrored-twiddle identity
// psi^-bitrev(2^s+i) = -psi^bitrev(2^s+2^s-1-i); solve.cu:204-378), organised differently:
//   * every stage uses Harvey lazy butterflies with Shoup twiddle products (pm_device.cuh), so
//     no butterfly reduces to [0, p);
//   * twiddles come from one table tw[j][k] = {psi_j^bitrev(k), floor(psi_j^bitrev(k) 2^32 / p_j)},
//     read directly in 16-byte runs (row pass: a stage's 2^t twiddles of a thread are
//     consecutive) or staged once per CTA (column pass: the first nrows entries), instead of
//     forming trow * tsmall with a Montgomery product at every butterfly (solve.cu:286-338);
//   * a line of 2^NB elements is transformed in PHASES of up to RB = 4 stages.  In a phase a
//     thread holds 16 elements of the line in registers -- the 16 values of the 4 index bits
//     [b0, b0 + 4) that the phase's stages pair up -- and runs a radix-16 butterfly network on
//     them with compile-time indexing.  Between phases the elements are exchanged through
//     shared memory once (a 256-point row: load -> 4 stages -> exchange -> 4 stages -> store),
//     where the previous design went through shared memory at every radix-8 pass.
//
// Phase k of an NB-bit line covers stage bits NB-1-4k down to b0_k = max(0, NB - 4(k+1));
// its registers hold index bits [b0_k, b0_k + 4) and the thread's position supplies the
// rest (low bits below b0_k, high bits above).  The last phase of a line whose length is
// not a power of 16 re-uses bits [0, 4) and skips the stages an earlier phase has done.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <cstdlib>
#include <type_traits>

#include "pm_async.cuh"
#include "pm_kernels.cuh"

namespace pm {
namespace {

template <int NB>
struct LineCfg {
    static constexpr int RB = NB < 4 ? NB : 4;      // index bits held in registers
    static constexpr int E = 1 << RB;               // elements per thread
    static constexpr int NPH = RB == 0 ? 0 : (NB + RB - 1) / RB;  // phases (none for a 1-point line)
    __host__ __device__ static constexpr int b0(int k) { return NB - RB * (k + 1) > 0 ? NB - RB * (k + 1) : 0; }
    // first local stage of phase k (local stage t pairs register bit RB-1-t)
    __host__ __device__ static constexpr int t0(int k) { return b0(k) + RB - 1 - (NB - 1 - RB * k); }
    // global stage index of local stage t of phase k: ls = NB - 1 - (b0 + RB - 1 - t)
    __host__ __device__ static constexpr int ls(int k, int t) { return NB - b0(k) - RB + t; }
};

// Forward (CT) radix network on v[] over local stages t0..RB-1 of one phase.  stw(t) returns
// the stage's twiddle source: w[m] is the Shoup-form Tw2 {w, floor(w 2^32 / p)} of group m
// (gi = (hi << t) | m; hi is folded in by stw).
template <int RB, int T0, class StwF>
__device__ __forceinline__ void radix_fwd(uint32_t (&v)[1 << RB], const StwF& stw, uint32_t p) {
#pragma unroll
    for (int t = T0; t < RB; ++t) {
        const int h = (1 << RB) >> (t + 1);
        const auto w = stw(t);
#pragma unroll
        for (int m = 0; m < (1 << t); ++m) {
            const Tw2 wm = w[m];
#pragma unroll
            for (int i = 0; i < h; ++i) {
                bfly_ct_sh(v[m * 2 * h + i], v[m * 2 * h + i + h], wm, p);
            }
        }
    }
}

// The forward network on two operands' lines that share their twiddles (the same prime and
// row): each twiddle is read once for both butterflies.
template <int RB, int T0, class StwF>
__device__ __forceinline__ void radix_fwd2(uint32_t (&v)[1 << RB], uint32_t (&u)[1 << RB], const StwF& stw,
                                           uint32_t p) {
#pragma unroll
    for (int t = T0; t < RB; ++t) {
        const int h = (1 << RB) >> (t + 1);
        const auto w = stw(t);
#pragma unroll
        for (int m = 0; m < (1 << t); ++m) {
            const Tw2 wm = w[m];
#pragma unroll
            for (int i = 0; i < h; ++i) {
                bfly_ct_sh(v[m * 2 * h + i], v[m * 2 * h + i + h], wm, p);
                bfly_ct_sh(u[m * 2 * h + i], u[m * 2 * h + i + h], wm, p);
            }
        }
    }
}

// Inverse (GS) network, local stages RB-1 down to T0, mirrored twiddles from stw(t).
template <int RB, int T0, class StwF>
__device__ __forceinline__ void radix_inv(uint32_t (&v)[1 << RB], const StwF& stw, uint32_t p) {
#pragma unroll
    for (int t = RB - 1; t >= T0; --t) {
        const int h = (1 << RB) >> (t + 1);
        const auto w = stw(t);
#pragma unroll
        for (int m = 0; m < (1 << t); ++m) {
            const Tw2 wm = w[m];
#pragma unroll
            for (int i = 0; i < h; ++i) {
                bfly_gs_sh(v[m * 2 * h + i], v[m * 2 * h + i + h], wm, p);
            }
        }
    }
}

// The inverse network on two lines that share their twiddles.
template <int RB, int T0, class StwF>
__device__ __forceinline__ void radix_inv2(uint32_t (&v)[1 << RB], uint32_t (&u)[1 << RB], const StwF& stw,
                                           uint32_t p) {
#pragma unroll
    for (int t = RB - 1; t >= T0; --t) {
        const int h = (1 << RB) >> (t + 1);
        const auto w = stw(t);
#pragma unroll
        for (int m = 0; m < (1 << t); ++m) {
            const Tw2 wm = w[m];
#pragma unroll
            for (int i = 0; i < h; ++i) {
                bfly_gs_sh(v[m * 2 * h + i], v[m * 2 * h + i + h], wm, p);
                bfly_gs_sh(u[m * 2 * h + i], u[m * 2 * h + i + h], wm, p);
            }
        }
    }
}

// A stage's run of 2^t consecutive Shoup-form twiddles {w, floor(w 2^32 / p)} starting at
// `src`, aligned to 2^t entries.  w[m] is entry m (REV: entry 2^t - 1 - m), read at use as
// half of a 16-byte pair (the two entries of a pair come from one load), so that no more of
// the run than the current butterflies need is held in registers.
template <bool REV>
struct RunTw {
    const uint2* src;
    int n;
    __device__ __forceinline__ Tw2 operator[](int m) const {
        const int e = REV ? n - 1 - m : m;
        if (n == 1) {
            const uint2 u = __ldg(src);
            return Tw2{u.x, u.y};
        }
        const uint4 u = __ldg(reinterpret_cast<const uint4*>(src) + (e >> 1));
        return (e & 1) ? Tw2{u.z, u.w} : Tw2{u.x, u.y};
    }
};

// A column stage's run of 2^t Shoup twiddles in shared memory, starting at `start` (aligned to
// 2^t entries): w[m] is entry m (REV: entry 2^t - 1 - m), read as half of a 16-byte pair.
template <bool REV>
struct SmemRun {
    const Tw2* start;
    int n;
    __device__ __forceinline__ Tw2 operator[](int m) const {
        const int e = REV ? n - 1 - m : m;
        if (n == 1) return start[0];
        const uint4 u = reinterpret_cast<const uint4*>(start)[e >> 1];
        return (e & 1) ? Tw2{u.z, u.w} : Tw2{u.x, u.y};
    }
};

// ---------------------------------------------------------------------------------------
// Row pass layout.  LPR = 2^(NB-RB) threads share a row; a shared-memory region serves
// GRP = max(32, LPR) threads (one warp, or the two warps of a 1024-point row) and holds
// RPG = GRP / LPR rows.  Inside a region an element has the index X = (row << NB) | x; it
// is stored at X ^ G(X >> 5), an XOR swizzle chosen (by exhaustive search over linear maps)
// so that every exchange of the phase layouts below is free of bank conflicts -- with
// 16-byte vector access in the last phase for NB = 6, 7, 8.
// ---------------------------------------------------------------------------------------
template <int NB>
struct RowCfg : LineCfg<NB> {
    using B = LineCfg<NB>;
    static constexpr int LPR = 1 << (NB - B::RB);
    static constexpr int GRP = LPR > 32 ? LPR : 32;
    static constexpr int RPG = GRP / LPR;             // rows per shared-memory region
    static constexpr int ROWS_PER_CTA = 128 / LPR;   // 128 threads per CTA
    static constexpr bool VEC = NB >= 6 && NB <= 8;   // swizzle keeps runs of 4 contiguous
    static constexpr int REGION = GRP * B::E;         // words per region
    __host__ __device__ static constexpr uint32_t g(int i) {
        // G(input bit i of X >> 5) for each NB; NB <= 4 has a single phase and no exchange
        return NB == 5 || NB == 9 ? (i == 0 ? 2u : i == 1 ? 4u : i == 2 ? 8u : i == 3 ? 17u : 0u)
             : NB == 6           ? (i == 0 ? 4u : i == 1 ? 8u : i == 2 ? 4u : i == 3 ? 16u : 0u)
             : NB == 7           ? (i == 0 ? 4u : i == 1 ? 8u : i == 2 ? 8u : i == 3 ? 16u : 0u)
             : NB == 8           ? (i == 0 ? 4u : i == 1 ? 8u : i == 2 ? 0u : i == 3 ? 16u : 0u)
             : NB == 10          ? (i == 0 ? 1u : i == 1 ? 18u : i == 2 ? 4u : i == 3 ? 8u : 0u)
                                 : 0u;
    }
    // X ^ G(X >> 5) is linear over XOR: swz(a ^ b) = swz(a) ^ swz(b), so an element's address
    // is the thread's swizzled base XOR a compile-time constant
    __host__ __device__ static constexpr int swz(int X) {
        return X ^ (((X >> 5) & 1 ? (int)g(0) : 0) ^ ((X >> 5) & 2 ? (int)g(1) : 0) ^ ((X >> 5) & 4 ? (int)g(2) : 0) ^
                    ((X >> 5) & 8 ? (int)g(3) : 0) ^ ((X >> 5) & 16 ? (int)g(4) : 0));
    }
};

template <int NB>
__device__ __forceinline__ void region_sync() {
    if constexpr (RowCfg<NB>::LPR > 32) __syncthreads();
    else __syncwarp();
}

// Element index x (within the row) of register e in phase K for row-lane r.
template <int NB, int K>
__device__ __forceinline__ int row_x(int r, int e) {
    using C = RowCfg<NB>;
    constexpr int b0 = C::b0(K);
    return ((r >> b0) << (b0 + C::RB)) | (e << b0) | (r & ((1 << b0) - 1));
}

// Writes (TO_SMEM) or reads the thread's registers in the layout of phase K.
template <int NB, int K, bool TO_SMEM>
__device__ __forceinline__ void row_xchg(uint32_t (&v)[RowCfg<NB>::E], uint32_t* region, int rho, int r) {
    using C = RowCfg<NB>;
    constexpr int b0 = C::b0(K);
    // the register bits of X are zero in the base: X(e) = base ^ (e << b0)
    const int sbase = C::swz((rho << NB) | row_x<NB, K>(r, 0));
    if constexpr (C::VEC && b0 == 0) {
#pragma unroll
        for (int q = 0; q < C::E / 4; ++q) {
            uint4* a = reinterpret_cast<uint4*>(region + (sbase ^ C::swz(4 * q)));
            if (TO_SMEM) *a = make_uint4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
            else {
                const uint4 u = *a;
                v[4 * q] = u.x;
                v[4 * q + 1] = u.y;
                v[4 * q + 2] = u.z;
                v[4 * q + 3] = u.w;
            }
        }
    } else {
#pragma unroll
        for (int e = 0; e < C::E; ++e) {
            uint32_t* a = region + (sbase ^ C::swz(e << b0));
            if (TO_SMEM) *a = v[e];
            else v[e] = *a;
        }
    }
}

// global <-> registers in the layout of phase K (rows of nc consecutive words)
template <int NB, int K, bool LOAD>
__device__ __forceinline__ void row_global(uint32_t (&v)[RowCfg<NB>::E], uint32_t* row, int r, bool active) {
    using C = RowCfg<NB>;
    if (!active) {
        if (LOAD)
#pragma unroll
            for (int e = 0; e < C::E; ++e) v[e] = 0;
        return;
    }
    if constexpr (C::b0(K) == 0 && C::E >= 4) {  // E consecutive words, 16-byte aligned
        uint4* g = reinterpret_cast<uint4*>(row + row_x<NB, K>(r, 0));
#pragma unroll
        for (int q = 0; q < C::E / 4; ++q) {
            if (LOAD) {
                const uint4 u = g[q];
                v[4 * q] = u.x;
                v[4 * q + 1] = u.y;
                v[4 * q + 2] = u.z;
                v[4 * q + 3] = u.w;
            } else {
                g[q] = make_uint4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
            }
        }
    } else {
#pragma unroll
        for (int e = 0; e < C::E; ++e) {
            if (LOAD) v[e] = row[row_x<NB, K>(r, e)];
            else row[row_x<NB, K>(r, e)] = v[e];
        }
    }
}

// Forward phases K..NPH-1 of a row (registers in the layout of phase K on entry, of phase
// NPH-1 on exit).  Stage ls of row hi, group gi uses tw[2^(w1+ls) + hi 2^ls + gi].
template <int NB, int K>
__device__ __forceinline__ void row_forward(uint32_t (&v)[RowCfg<NB>::E], uint32_t* region, int rho, int r,
                                            const uint2* twj, int w1, uint32_t hi, uint32_t p) {
    using C = RowCfg<NB>;
    if constexpr (K < C::NPH) {
        constexpr int b0 = C::b0(K);
        const uint32_t hip = (uint32_t)(r >> b0);  // index bits above the registers
        // per local stage t: the row's run of twiddles, tw[2^(w1+ls) + hi 2^ls + (hip << t) + m],
        // m < 2^t: 2^t consecutive words aligned to 2^t (ls >= t)
        auto stw = [&](int t) {
            const int ls = C::ls(K, t);
            return RunTw<false>{twj + (1u << (w1 + ls)) + (hi << ls) + (hip << t), 1 << t};
        };
        radix_fwd<C::RB, C::t0(K)>(v, stw, p);
        if constexpr (K + 1 < C::NPH) {
            row_xchg<NB, K, true>(v, region, rho, r);
            region_sync<NB>();
            row_xchg<NB, K + 1, false>(v, region, rho, r);
            region_sync<NB>();
            row_forward<NB, K + 1>(v, region, rho, r, twj, w1, hi, p);
        }
    }
}

// row_forward on two operands' rows of the same prime and row index (b in v, a in u), each in
// its own shared-memory region for the exchanges.
template <int NB, int K>
__device__ __forceinline__ void row_forward2(uint32_t (&v)[RowCfg<NB>::E], uint32_t (&u)[RowCfg<NB>::E],
                                             uint32_t* region, uint32_t* region_u, int rho, int r, const uint2* twj,
                                             int w1, uint32_t hi, uint32_t p) {
    using C = RowCfg<NB>;
    if constexpr (K < C::NPH) {
        constexpr int b0 = C::b0(K);
        const uint32_t hip = (uint32_t)(r >> b0);
        auto stw = [&](int t) {
            const int ls = C::ls(K, t);
            return RunTw<false>{twj + (1u << (w1 + ls)) + (hi << ls) + (hip << t), 1 << t};
        };
        radix_fwd2<C::RB, C::t0(K)>(v, u, stw, p);
        if constexpr (K + 1 < C::NPH) {
            row_xchg<NB, K, true>(v, region, rho, r);
            row_xchg<NB, K, true>(u, region_u, rho, r);
            region_sync<NB>();
            row_xchg<NB, K + 1, false>(v, region, rho, r);
            row_xchg<NB, K + 1, false>(u, region_u, rho, r);
            region_sync<NB>();
            row_forward2<NB, K + 1>(v, u, region, region_u, rho, r, twj, w1, hi, p);
        }
    }
}

// Inverse phases K down to 0 (registers in the layout of phase K on entry, phase 0 on exit).
// The inverse twiddle of (ls, hi, gi) is the forward entry of the mirrored row nrows-1-hi at
// 2^ls - 1 - gi.
template <int NB, int K>
__device__ __forceinline__ void row_inverse(uint32_t (&v)[RowCfg<NB>::E], uint32_t* region, int rho, int r,
                                            const uint2* twj, int w1, uint32_t hi_m, uint32_t p) {
    using C = RowCfg<NB>;
    if constexpr (K >= 0) {
        constexpr int b0 = C::b0(K);
        const uint32_t hip = (uint32_t)(r >> b0);
        // tw[2^(w1+ls) + hi_m 2^ls + 2^ls - 1 - ((hip << t) + m)], m < 2^t: the aligned run of 2^t
        // words ending there, read in reverse
        auto stw = [&](int t) {
            const int ls = C::ls(K, t);
            return RunTw<true>{twj + (1u << (w1 + ls)) + (hi_m << ls) + (1u << ls) - ((hip + 1u) << t), 1 << t};
        };
        radix_inv<C::RB, C::t0(K)>(v, stw, p);
        if constexpr (K > 0) {
            row_xchg<NB, K, true>(v, region, rho, r);
            region_sync<NB>();
            row_xchg<NB, K - 1, false>(v, region, rho, r);
            region_sync<NB>();
            row_inverse<NB, K - 1>(v, region, rho, r, twj, w1, hi_m, p);
        }
    }
}

}  // namespace

// Row pass over ROWS_PER_CTA consecutive rows of one prime and batch entry, 128 threads.
//   ROWS_FWD  : forward row stages (operand a).
//   ROWS_FUSED: forward row stages of b, pointwise product with the finished transform of a
//               (RA), inverse row stages.  Batch z pairs with transform ra_sel[z] of RA when
//               ra_sel is given (a server's resident operands), else with transform z.
//   ROWS_BOTH : forward row stages of b and of a (RA, after its column pass) side by side,
//               each twiddle read once for both, then the pointwise product and the inverse
//               stages of b; RA is read and not written.
// The Montgomery pointwise product leaves a factor 2^-32 that the CRT constant crt_c
// compensates.  Blocks per SM: the most at which the variants do not spill (64 registers at 8,
// 80 at 6, 128 at 4); the fused kernels hold the other operand's row and more twiddle runs.
// The two-operand form at 6 (80 registers) ran its pass in 34.2 us per multiply against 36.1 at
// 5 (96) and 37.4 at 4 (117) (N=65536, W=1747, launches of 8); since the 64-bit product forms it
// fits 7 (72 registers, no spill): 31.4 -> 31.0 us in launches of 32; at 8 (64) it spills.  The
// fused form (host pipeline, server) keeps a 4-byte stack slot at 7 (8 bytes at 6).
enum : int { ROWS_FWD = 0, ROWS_FUSED = 1, ROWS_BOTH = 2 };
__host__ __device__ constexpr int rows_min_blocks(int nb, int mode) {
    return nb >= 9 ? (mode == ROWS_FWD ? 5 : 4) : (mode == ROWS_FWD ? 8 : 7);
}
// POLYMULT_ROW_STATIC: the row kernels take the column-stage count w1 (and with it nrows and N)
// as a template constant for the common splits, and a grid ordered (batch, row block, prime) so
// that the block's indices need no division (row pass of both operands at N=65536, W=1747:
// 34.2 -> 32.8 us per multiply, N=32768, W=868: 9.47 -> 9.03); otherwise w1 from the plan and a
// (row block, prime, batch) grid linearised batch entry fastest.
#ifndef POLYMULT_ROW_STATIC
#define POLYMULT_ROW_STATIC 1
#endif
template <int NB, int MODE, int W1>
__global__ void __launch_bounds__(128, rows_min_blocks(NB, MODE)) k_ntt_rows(DevPlan P, uint32_t* __restrict__ R,
                                                                           const uint32_t* __restrict__ RA,
                                                                           const uint32_t* __restrict__ ra_sel) {
    using C = RowCfg<NB>;
    const int w1 = W1 >= 0 ? W1 : P.w1;
    const uint32_t nrows = W1 >= 0 ? (1u << (W1 >= 0 ? W1 : 0)) : P.nrows;
    const uint32_t Nn = W1 >= 0 ? (1u << ((W1 >= 0 ? W1 : 0) + NB)) : P.N;  // N <= 2^20
    constexpr int REGION_WORDS = C::NPH > 1 ? (128 / C::GRP) * C::REGION : 4;  // one operand's regions
    __shared__ __align__(16) uint32_t sh[MODE == ROWS_BOTH ? 2 * REGION_WORDS : REGION_WORDS];
    const int tid = threadIdx.x;
    const int li = tid % C::GRP;                 // thread within the shared-memory region
    const int rho = li / C::LPR, r = li % C::LPR;
    uint32_t* region = sh + (tid / C::GRP) * C::REGION;
    // blocks run batch entry fastest in launch order, so the nb blocks of one (row block, prime),
    // which read the same twiddles, run side by side and share them in L2
    uint32_t zb, xb;
    int j;
    if (POLYMULT_ROW_STATIC) {  // grid (batch, row blocks, primes)
        zb = blockIdx.x;
        xb = blockIdx.y;
        j = (int)blockIdx.z;
    } else {  // grid (row blocks, primes, batch), linearised
        const uint32_t lin = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
        zb = lin % gridDim.z;
        const uint32_t rest = lin / gridDim.z;
        xb = rest % gridDim.x;
        j = (int)(rest / gridDim.x);
    }
    const uint32_t hi = xb * C::ROWS_PER_CTA + (uint32_t)(tid / C::LPR);
    const bool active = hi < nrows;
    const uint32_t hic = active ? hi : nrows - 1;  // keeps twiddle reads in range
    const uint32_t p = P.p[j], pinv = P.pinv[j];
    const size_t off = ((size_t)zb * P.K + j) * Nn + (size_t)hic * (1u << NB);
    uint32_t* row = R + off;
    const uint2* twj = P.tw + (size_t)j * Nn;

    uint32_t v[C::E];
    pdl_trigger();
    pdl_wait();
    row_global<NB, 0, true>(v, row, r, active);
    if constexpr (MODE == ROWS_BOTH) {
        uint32_t a[C::E];
        row_global<NB, 0, true>(a, const_cast<uint32_t*>(RA + off), r, active);
        row_forward2<NB, 0>(v, a, region, region + REGION_WORDS, rho, r, twj, w1, hic, p);
#pragma unroll
        for (int e = 0; e < C::E; ++e) v[e] = mont_mul(red_once(red_once(a[e], 2 * p), p), v[e], p, pinv);
        row_inverse<NB, C::NPH - 1>(v, region, rho, r, twj, w1, nrows - 1 - hic, p);
        row_global<NB, 0, false>(v, row, r, active);
    } else if constexpr (MODE == ROWS_FUSED) {
        row_forward<NB, 0>(v, region, rho, r, twj, w1, hic, p);
        uint32_t a[C::E];
        const size_t za = ra_sel ? (size_t)__ldg(ra_sel + zb) : (size_t)zb;
        const size_t offa = (za * P.K + j) * Nn + (size_t)hic * (1u << NB);
        row_global<NB, (C::NPH > 0 ? C::NPH - 1 : 0), true>(a, const_cast<uint32_t*>(RA + offa), r, active);
#pragma unroll
        for (int e = 0; e < C::E; ++e) v[e] = mont_mul(red_once(red_once(a[e], 2 * p), p), v[e], p, pinv);
        row_inverse<NB, C::NPH - 1>(v, region, rho, r, twj, w1, nrows - 1 - hic, p);
        row_global<NB, 0, false>(v, row, r, active);
    } else {
        row_forward<NB, 0>(v, region, rho, r, twj, w1, hic, p);
        row_global<NB, (C::NPH > 0 ? C::NPH - 1 : 0), false>(v, row, r, active);
    }
}

// ---------------------------------------------------------------------------------------
// Column pass: the first w1 = NB stages on a tile of 2^NB rows x TC = 2^ltc columns of prime
// blockIdx.y, batch blockIdx.z, 256 threads.  Thread t owns column t % TC and, in each phase,
// the element groups t / TC + i (256 / TC): a group is the 16 rows that differ in the phase's
// register bits.  Phase 0 (forward) reads its groups straight from global memory and the last
// phase writes straight back; the tile in shared memory ([row][TC], a warp touching 32
// consecutive columns of one row) carries the values between phases.  Column stage s, group
// i uses tw[2^s + i] (forward) or tw[2^(s+1) - 1 - i] (inverse), staged once per CTA.
// ---------------------------------------------------------------------------------------
namespace {

// LTC >= 0: the tile width 2^LTC at compile time (shared-memory offsets become immediates);
// -1: the runtime ltc (narrow column chunks of the host pipeline)
template <int NB, bool INV, int K, int LTC>
__device__ __forceinline__ void col_phase(uint32_t* tile, const Tw2* tws, uint32_t* gbase, size_t gstride, int ltc_rt,
                                          uint32_t p) {
    using C = LineCfg<NB>;
    constexpr int b0 = C::b0(K);
    constexpr int NGRP = (1 << NB) / C::E;  // groups per column
    constexpr bool FIRST = INV ? K == C::NPH - 1 : K == 0;
    constexpr bool LAST = INV ? K == 0 : K == C::NPH - 1;
    const int ltc = LTC >= 0 ? LTC : ltc_rt;
    const int tc = 1 << ltc;
    const int c = threadIdx.x & (tc - 1);
    const int slots = blockDim.x >> ltc;
    for (int gidx = threadIdx.x >> ltc; gidx < NGRP; gidx += slots) {
        const int lo = gidx & ((1 << b0) - 1), hip = gidx >> b0;
        const int xb = (hip << (b0 + C::RB)) | lo;
        // element e is row xb + (e << b0): global offset gb + e (gstride << b0), tile offset sb + e (tc << b0)
        uint32_t* gb = gbase + (size_t)xb * gstride + c;
        uint32_t* sb = tile + (xb << ltc) + c;
        const size_t gstep = gstride << b0;
        const int sstep = 1 << (b0 + ltc);
        uint32_t v[C::E];
#pragma unroll
        for (int e = 0; e < C::E; ++e) v[e] = FIRST ? gb[e * gstep] : sb[e * sstep];
        int tb[C::RB];
#pragma unroll
        for (int t = 0; t < C::RB; ++t)
            tb[t] = INV ? (2 << C::ls(K, t)) - 1 - (hip << t) : (1 << C::ls(K, t)) + (hip << t);
        // stage t's 2^t twiddles: tws[tb[t] + m] (forward) or tws[tb[t] - m] (inverse), runs
        // aligned to 2^t entries
        if (!INV) {
            auto stw = [&](int t) { return SmemRun<false>{tws + tb[t], 1 << t}; };
            radix_fwd<C::RB, C::t0(K)>(v, stw, p);
        } else {
            auto stw = [&](int t) { return SmemRun<true>{tws + tb[t] - ((1 << t) - 1), 1 << t}; };
            radix_inv<C::RB, C::t0(K)>(v, stw, p);
        }
#pragma unroll
        for (int e = 0; e < C::E; ++e) {
            if (LAST) gb[e * gstep] = v[e];
            else sb[e * sstep] = v[e];
        }
    }
}

template <int NB, bool INV, int I, int LTC>
__device__ __forceinline__ void col_phases(uint32_t* tile, const Tw2* tws, uint32_t* gbase, size_t gstride, int ltc,
                                           uint32_t p) {
    using C = LineCfg<NB>;
    if constexpr (I < C::NPH) {
        constexpr int K = INV ? C::NPH - 1 - I : I;
        col_phase<NB, INV, K, LTC>(tile, tws, gbase, gstride, ltc, p);
        if constexpr (I + 1 < C::NPH) {
            __syncthreads();
            col_phases<NB, INV, I + 1, LTC>(tile, tws, gbase, gstride, ltc, p);
        }
    }
}

}  // namespace

// Two-column form (lines of 128 or 256 rows, tiles of 64 columns: 33 / 66 KB of shared memory,
// three CTAs per SM at 256 rows; longer lines keep the one-column form): thread t owns columns
// 2 (t % 32) and 2 (t % 32) + 1 and, in each phase, the groups t / 32 + 8 i.  Every global and
// shared access moves both columns' elements in one 8-byte word, and each twiddle read serves
// both columns' butterflies (radix_fwd2 / radix_inv2): per butterfly half the memory and twiddle
// instructions of the one-column form.  GL >= 0: log2 of the row pitch ncols at compile time, so
// that an element's global address is its group's base plus an immediate.
constexpr int COL2_TC = 64;

template <int NB, bool INV, int K, int GL>
__device__ __forceinline__ void col2_phase(uint32_t* tile, const Tw2* tws, uint32_t* gbase, uint32_t ncols_rt,
                                           uint32_t p) {
    using C = LineCfg<NB>;
    constexpr int b0 = C::b0(K);
    constexpr int NGRP = (1 << NB) / C::E;  // groups per column
    constexpr bool FIRST = INV ? K == C::NPH - 1 : K == 0;
    constexpr bool LAST = INV ? K == 0 : K == C::NPH - 1;
    const uint32_t ncols = GL >= 0 ? (1u << (GL >= 0 ? GL : 0)) : ncols_rt;
    const int c2 = 2 * (int)(threadIdx.x & 31);
    static_assert(NGRP % 8 == 0, "every warp takes whole groups");
#pragma unroll 1
    for (int gidx = (int)(threadIdx.x >> 5); gidx < NGRP; gidx += 8) {
        const int lo = gidx & ((1 << b0) - 1), hip = gidx >> b0;
        const int xb = (hip << (b0 + C::RB)) | lo;
        // element e of the group is row xb + (e << b0)
        uint2* gb = reinterpret_cast<uint2*>(gbase + (size_t)xb * ncols + c2);
        uint2* sb = reinterpret_cast<uint2*>(tile + xb * COL2_TC + c2);
        const size_t gstep = ((size_t)ncols << b0) / 2;  // in 8-byte words
        constexpr int sstep = (COL2_TC << b0) / 2;
        uint32_t v[C::E], u[C::E];
#pragma unroll
        for (int e = 0; e < C::E; ++e) {
            const uint2 w = FIRST ? gb[e * gstep] : sb[e * sstep];
            v[e] = w.x;
            u[e] = w.y;
        }
        int tb[C::RB];
#pragma unroll
        for (int t = 0; t < C::RB; ++t)
            tb[t] = INV ? (2 << C::ls(K, t)) - 1 - (hip << t) : (1 << C::ls(K, t)) + (hip << t);
        if (!INV) {
            auto stw = [&](int t) { return SmemRun<false>{tws + tb[t], 1 << t}; };
            radix_fwd2<C::RB, C::t0(K)>(v, u, stw, p);
        } else {
            auto stw = [&](int t) { return SmemRun<true>{tws + tb[t] - ((1 << t) - 1), 1 << t}; };
            radix_inv2<C::RB, C::t0(K)>(v, u, stw, p);
        }
#pragma unroll
        for (int e = 0; e < C::E; ++e) {
            if (LAST) gb[e * gstep] = make_uint2(v[e], u[e]);
            else sb[e * sstep] = make_uint2(v[e], u[e]);
        }
    }
}

template <int NB, bool INV, int I, int GL>
__device__ __forceinline__ void col2_phases(uint32_t* tile, const Tw2* tws, uint32_t* gbase, uint32_t ncols,
                                            uint32_t p) {
    using C = LineCfg<NB>;
    if constexpr (I < C::NPH) {
        constexpr int K = INV ? C::NPH - 1 - I : I;
        col2_phase<NB, INV, K, GL>(tile, tws, gbase, ncols, p);
        if constexpr (I + 1 < C::NPH) {
            __syncthreads();
            col2_phases<NB, INV, I + 1, GL>(tile, tws, gbase, ncols, p);
        }
    }
}

template <int NB, bool INV, int GL>
__global__ void __launch_bounds__(256, 3) k_ntt_cols2(DevPlan P, uint32_t* __restrict__ R, uint32_t col0) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int NR = 1 << NB;
    Tw2* tws = reinterpret_cast<Tw2*>(smem_raw);            // [NR]
    uint32_t* tile = reinterpret_cast<uint32_t*>(tws + NR);  // [NR][64]
    const int j = (int)blockIdx.y;
    const uint32_t p = P.p[j];
    uint32_t* base = R + ((size_t)blockIdx.z * P.K + j) * P.N + col0 + (blockIdx.x * COL2_TC);
    const uint2* tw = P.tw + (size_t)j * P.N;
    pdl_trigger();
    for (int k = threadIdx.x; k < NR; k += blockDim.x) {
        const uint2 w = __ldg(tw + k);
        tws[k] = Tw2{w.x, w.y};
    }
    pdl_wait();
    __syncthreads();
    col2_phases<NB, INV, 0, GL>(tile, tws, base, P.ncols, p);
}

// ---------------------------------------------------------------------------------------
// TMA column pass (lines of 256 rows, 64-column tiles).  A persistent kernel, one CTA
// per SM, whose producer warp streams tiles of [2^NB rows][64
// columns] -- a TMA box of R viewed as a [batch * K * nrows][ncols] matrix -- together with the
// tile's prime's first 2^NB Shoup twiddles (a bulk copy) into a ring of shared-
// memory slots (G::STAGES), while the consumer warps transform earlier tiles: 16-row element
// groups and two columns per thread as in k_ntt_cols2, phase 0 from the slot and back in
// place, the last phase from the slot straight to global memory.  The loads of the next tiles thus
// overlap this tile's butterflies, which a one-tile-per-CTA kernel leaves to the other CTAs
// of the SM.  The consumers form two groups of 8 warps, each on every other tile of the CTA
// with its own barriers, so that one group's phase barrier is covered by the other's work.
// All waits are bounded (the plan's wait_clocks); a wait that gives up makes the group leave
// together (one barrier-OR per tile) and the other group and the producer see the abort flag;
// the producer waits for the copies it issued, and the kernel reports DEV_ERR_WAIT.
// ---------------------------------------------------------------------------------------
template <int NB>
struct ColtCfg {
    static constexpr int NR = 1 << NB;
    static constexpr int TC = 64;                     // tile columns (64 or 32)
    static constexpr int LPR = TC / 2;                // lanes per tile row (two columns each)
    static constexpr int GPW = 32 / LPR;              // element groups a warp covers at once
    static constexpr int GROUPS = 2;                  // consumer groups, each on its own tiles
    static constexpr int GROUP_WARPS = 8;
    static constexpr int GROUP_THREADS = 32 * GROUP_WARPS;
    static constexpr int THREADS = GROUPS * GROUP_THREADS + 32;
    static constexpr int TILE_BYTES = NR * TC * 4;
    static constexpr int SLOT_BYTES = TILE_BYTES + NR * 8;  // tile, then the prime's twiddles
    static constexpr int STAGES = TC == 64 ? 3 : 6;   // slots: 198 / 204 KB
    static constexpr size_t SMEM = 128 + (size_t)STAGES * SLOT_BYTES;  // barriers, then the slots
    static constexpr int MIN_BLOCKS = 1;
    static_assert(SLOT_BYTES % 128 == 0, "slots stay 128-byte aligned");
};

template <int NB, bool INV, int K, int GL>
__device__ __forceinline__ void colt_phase(uint32_t* tile, const Tw2* tws, uint32_t* gout, uint32_t ncols_rt, uint32_t p,
                                           int gw) {
    const uint32_t ncols = GL >= 0 ? (1u << (GL >= 0 ? GL : 0)) : ncols_rt;
    using C = LineCfg<NB>;
    constexpr int b0 = C::b0(K);
    constexpr int NGRP = (1 << NB) / C::E;  // element groups per column
    constexpr bool LAST = INV ? K == 0 : K == C::NPH - 1;
    using G = ColtCfg<NB>;
    const int lane = (int)(threadIdx.x & 31);
    const int c2 = 2 * (lane % G::LPR);
    static_assert(NGRP % (G::GROUP_WARPS * G::GPW) == 0, "every warp takes whole element groups");
#pragma unroll 1
    for (int gidx = gw * G::GPW + lane / G::LPR; gidx < NGRP; gidx += G::GROUP_WARPS * G::GPW) {
        const int lo = gidx & ((1 << b0) - 1), hip = gidx >> b0;
        const int xb = (hip << (b0 + C::RB)) | lo;
        // element e of the group is row xb + (e << b0)
        uint2* sb = reinterpret_cast<uint2*>(tile + xb * G::TC + c2);
        constexpr int sstep = (G::TC << b0) / 2;
        uint32_t v[C::E], u[C::E];
#pragma unroll
        for (int e = 0; e < C::E; ++e) {
            const uint2 w = sb[e * sstep];
            v[e] = w.x;
            u[e] = w.y;
        }
        int tb[C::RB];
#pragma unroll
        for (int t = 0; t < C::RB; ++t)
            tb[t] = INV ? (2 << C::ls(K, t)) - 1 - (hip << t) : (1 << C::ls(K, t)) + (hip << t);
        if (!INV) {
            auto stw = [&](int t) { return SmemRun<false>{tws + tb[t], 1 << t}; };
            radix_fwd2<C::RB, C::t0(K)>(v, u, stw, p);
        } else {
            auto stw = [&](int t) { return SmemRun<true>{tws + tb[t] - ((1 << t) - 1), 1 << t}; };
            radix_inv2<C::RB, C::t0(K)>(v, u, stw, p);
        }
        if (LAST) {
            uint2* gb = reinterpret_cast<uint2*>(gout + (size_t)xb * ncols + c2);
            const size_t gstep = ((size_t)ncols << b0) / 2;  // in 8-byte words
#pragma unroll
            for (int e = 0; e < C::E; ++e) gb[e * gstep] = make_uint2(v[e], u[e]);
        } else {
#pragma unroll
            for (int e = 0; e < C::E; ++e) sb[e * sstep] = make_uint2(v[e], u[e]);
        }
    }
}

template <int NB, bool INV, int I, int GL>
__device__ __forceinline__ void colt_phases(uint32_t* tile, const Tw2* tws, uint32_t* gout, uint32_t ncols, uint32_t p,
                                            int grp, int gw) {
    using C = LineCfg<NB>;
    if constexpr (I < C::NPH) {
        constexpr int K = INV ? C::NPH - 1 - I : I;
        colt_phase<NB, INV, K, GL>(tile, tws, gout, ncols, p, gw);
        if constexpr (I + 1 < C::NPH) {
            named_sync(1 + grp, ColtCfg<NB>::GROUP_THREADS);
            colt_phases<NB, INV, I + 1, GL>(tile, tws, gout, ncols, p, grp, gw);
        }
    }
}

// tile t: columns col0 + TC (t mod tiles_x) .., line (batch entry, prime) unit = t / tiles_x.
// GL >= 0: log2 of the row pitch ncols at compile time (the last phase's stores then address
// their rows with immediates); -1: the pitch at run time.
template <int NB, bool INV, int GL>
__global__ void __launch_bounds__(ColtCfg<NB>::THREADS, ColtCfg<NB>::MIN_BLOCKS)
    k_ntt_cols_tma(const __grid_constant__ CUtensorMap tmap, DevPlan P, uint32_t* __restrict__ R, uint32_t col0,
                   uint32_t tiles_x, uint32_t ntiles) {
    using G = ColtCfg<NB>;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw);
    uint64_t* empty = full + G::STAGES;
    volatile int* abort_f = reinterpret_cast<volatile int*>(smem_raw + 64);
    const int warp = (int)(threadIdx.x >> 5);
    if (threadIdx.x == 0) {
        for (int s = 0; s < G::STAGES; ++s) {
            mbar_init(full + s, 1);
            mbar_init(empty + s, G::GROUP_WARPS);
        }
        *abort_f = 0;
    }
    __syncthreads();
    pdl_trigger();
    pdl_wait();
    if (warp == G::GROUPS * G::GROUP_WARPS) {
        // producer: one lane issues every copy of this CTA's tiles
        if ((threadIdx.x & 31) == 0) {
            uint32_t k = 0;
            for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x, ++k) {
                const uint32_t s = k % G::STAGES, use = k / G::STAGES;
                if (use > 0 && !wait_or_abort(empty + s, (use - 1) & 1, abort_f, P.wait_clocks)) break;
                const uint32_t unit = t / tiles_x, tx = t - unit * tiles_x, j = unit % P.K;
                unsigned char* slot = smem_raw + 128 + (size_t)s * G::SLOT_BYTES;
                mbar_arrive_expect_tx(full + s, G::SLOT_BYTES);
                tma_load_2d(slot, &tmap, (int)(col0 + tx * G::TC), (int)(unit << NB), full + s);
                bulk_g2s(slot + G::TILE_BYTES, P.tw + (size_t)j * P.N, G::NR * 8, full + s);
            }
            // every copy issued into a slot lands before the CTA exits (the latest per slot)
            for (uint32_t q = k > G::STAGES ? k - G::STAGES : 0; q < k; ++q)
                mbar_wait_bounded(full + q % G::STAGES, (q / G::STAGES) & 1, P.wait_clocks);
        }
        __syncwarp();
    } else {
        // consumer group grp takes this CTA's tiles k = grp, grp + GROUPS, ...
        const int grp = warp / G::GROUP_WARPS, gw = warp % G::GROUP_WARPS;
        uint32_t k = (uint32_t)grp;
        for (uint32_t t = blockIdx.x + grp * gridDim.x; t < ntiles; t += G::GROUPS * gridDim.x, k += G::GROUPS) {
            const uint32_t s = k % G::STAGES;
            const bool ok = wait_or_abort(full + s, (k / G::STAGES) & 1, abort_f, P.wait_clocks);
            if (named_sync_or(1 + G::GROUPS + grp, G::GROUP_THREADS, !ok)) break;  // the group leaves together
            const uint32_t unit = t / tiles_x, tx = t - unit * tiles_x, j = unit % P.K;
            unsigned char* slot = smem_raw + 128 + (size_t)s * G::SLOT_BYTES;
            colt_phases<NB, INV, 0, GL>(reinterpret_cast<uint32_t*>(slot), reinterpret_cast<const Tw2*>(slot + G::TILE_BYTES),
                                    R + (size_t)unit * P.N + col0 + tx * G::TC, P.ncols, P.p[j], grp, gw);
            fence_smem_to_async();  // the in-place phase-0 writes, before the slot's next TMA load
            __syncwarp();
            if ((threadIdx.x & 31) == 0) mbar_arrive(empty + s);
        }
    }
    __syncthreads();
    if (threadIdx.x == 0 && *abort_f) flag_error(P.status, DEV_ERR_WAIT);
}

template <int NB, bool INV>
__global__ void __launch_bounds__(256, NB >= 5 ? 4 : 1) k_ntt_cols(DevPlan P, uint32_t* __restrict__ R, uint32_t col0, int ltc) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int NR = 1 << NB;
    Tw2* tws = reinterpret_cast<Tw2*>(smem_raw);            // [NR]
    uint32_t* tile = reinterpret_cast<uint32_t*>(tws + NR);  // [NR][TC]
    const int j = (int)blockIdx.y;
    const uint32_t p = P.p[j];
    uint32_t* base = R + ((size_t)blockIdx.z * P.K + j) * P.N + col0 + ((uint32_t)blockIdx.x << ltc);
    const uint2* tw = P.tw + (size_t)j * P.N;
    pdl_trigger();
    for (int k = threadIdx.x; k < NR; k += blockDim.x) {
        const uint2 u = __ldg(tw + k);
        tws[k] = Tw2{u.x, u.y};
    }
    pdl_wait();
    __syncthreads();
    if (ltc == 5) col_phases<NB, INV, 0, 5>(tile, tws, base, P.ncols, ltc, p);  // the common 32-column tile
    else col_phases<NB, INV, 0, -1>(tile, tws, base, P.ncols, ltc, p);
}

namespace {

#ifndef POLYMULT_COL2
#define POLYMULT_COL2 1
#endif
// the two-column kernel for a line length 2^NB, row pitch 2^w2 (GL: the pitch at compile time
// for the splits the tuner tries, w2 in [NB - 1, NB + 1]; else at run time)
template <int NB, bool INV>
auto col2_kernel(int w2) {
    if constexpr (NB >= 7 && NB <= 8) {
        if (w2 == NB) return k_ntt_cols2<NB, INV, NB>;
        if (w2 == NB + 1) return k_ntt_cols2<NB, INV, NB + 1>;
        if (w2 == NB - 1) return k_ntt_cols2<NB, INV, NB - 1>;
        return k_ntt_cols2<NB, INV, -1>;
    } else {
        return k_ntt_cols2<7, INV, -1>;  // not used (col2_applies)
    }
}

// the TMA column kernel for row pitch 2^w2 (compile-time pitch for w2 = 6 .. 9: N = 2^14 .. 2^17
// at w1 = 8)
template <bool INV>
auto colt_kernel(int w2) {
    if (w2 == 8) return k_ntt_cols_tma<8, INV, 8>;
    if (w2 == 7) return k_ntt_cols_tma<8, INV, 7>;
    if (w2 == 9) return k_ntt_cols_tma<8, INV, 9>;
    if (w2 == 6) return k_ntt_cols_tma<8, INV, 6>;
    return k_ntt_cols_tma<8, INV, -1>;
}

// cuTensorMapEncodeTiled from the driver (no link against libcuda); null if unavailable
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            f = nullptr;
        }
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
    }();
    return fn;
}

// The TMA column pass over grid.x << (ltc - 6) tiles of 64 columns from col0 (a multiple of
// 64) of every line (grid.y primes x grid.z batch entries); false where it does not apply.
template <int NB>
bool launch_cols_tma(bool inv, dim3 grid, cudaStream_t s, const DevPlan& P, uint32_t* R, uint32_t col0, int ltc,
                     bool pdl) {
    // lines of 256 rows only: at 128 rows (N = 32768) the one-tile-per-CTA kernel, three CTAs per
    // SM, measured faster (3.33 against 3.39 us per pass at W = 868)
    if constexpr (NB == 8) {
        using G = ColtCfg<NB>;
        const uint32_t cw = grid.x << ltc;
        if (!P.col_tma || cw % G::TC != 0 || col0 % G::TC != 0 || P.nrows != (1u << NB)) return false;
        const auto enc = tensor_map_encoder();
        if (!enc) return false;
        const uint32_t tiles_x = cw / G::TC;
        const uint64_t lines = (uint64_t)grid.y * grid.z;
        const uint64_t ntiles = tiles_x * lines;
        if (ntiles == 0) return true;
        // R as a [lines * nrows][ncols] matrix of u32, boxes of [2^NB rows][TC columns]
        CUtensorMap m;
        const cuuint64_t dims[2] = {P.ncols, lines * P.nrows};
        const cuuint64_t strides[1] = {(cuuint64_t)P.ncols * 4};
        const cuuint32_t box[2] = {(cuuint32_t)G::TC, (cuuint32_t)G::NR};
        const cuuint32_t es[2] = {1, 1};
        if (ntiles > 0xFFFFFFFFull || lines * P.nrows > 0x7FFFFFFFull ||
            enc(&m, CU_TENSOR_MAP_DATA_TYPE_UINT32, 2, R, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return false;
        int dev = 0, sms = 148;
        if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) !=
                                                      cudaSuccess)
            throw_cuda(cudaGetLastError(), "device attributes");
        const uint32_t g = (uint32_t)std::min<uint64_t>(ntiles, (uint64_t)sms * G::MIN_BLOCKS);
        const cudaError_t e = launch_kernel(inv ? colt_kernel<true>(P.w2) : colt_kernel<false>(P.w2), dim3(g),
                                            dim3(G::THREADS), G::SMEM, s, pdl, m, P, R, col0, tiles_x, (uint32_t)ntiles);
        if (e != cudaSuccess) throw_cuda(e, inv ? "launch k_ntt_cols_tma<inverse>" : "launch k_ntt_cols_tma<forward>");
        return true;
    } else {
        (void)inv, (void)grid, (void)s, (void)P, (void)R, (void)col0, (void)ltc, (void)pdl;
        return false;
    }
}

template <int NB>
void launch_cols_nb(bool inv, dim3 grid, size_t smem, cudaStream_t s, const DevPlan& P, uint32_t* R, uint32_t col0,
                    int ltc, bool pdl) {
    if (launch_cols_tma<NB>(inv, grid, s, P, R, col0, ltc, pdl)) return;
    if (POLYMULT_COL2 && NB >= 7 && NB <= 8 && ltc >= 6) {
        // 2^ltc columns as 2^(ltc - 6) tiles of 64
        const dim3 g2(grid.x << (ltc - 6), grid.y, grid.z);
        const size_t sm2 = ((size_t)8 + 4 * COL2_TC) << NB;
        const cudaError_t e = launch_kernel(inv ? col2_kernel<NB, true>(P.w2) : col2_kernel<NB, false>(P.w2), g2,
                                            dim3(256), sm2, s, pdl, P, R, col0);
        if (e != cudaSuccess) throw_cuda(e, inv ? "launch k_ntt_cols2<inverse>" : "launch k_ntt_cols2<forward>");
        return;
    }
    const cudaError_t e = launch_kernel(inv ? k_ntt_cols<NB, true> : k_ntt_cols<NB, false>, grid, dim3(256), smem, s,
                                        pdl, P, R, col0, ltc);
    if (e != cudaSuccess) throw_cuda(e, inv ? "launch k_ntt_cols<inverse>" : "launch k_ntt_cols<forward>");
}

// the row kernel of a mode for line length 2^NB and the plan's w1: a compile-time w1 for the
// splits of N = 4096 .. 65536 that the batches and the engine use, else w1 from the plan
template <int NB, int MODE>
auto row_kernel(int w1) {
    if constexpr (POLYMULT_ROW_STATIC && NB >= 6 && NB <= 8) {
        if (w1 == NB) return k_ntt_rows<NB, MODE, NB>;
        if (w1 == NB - 1) return k_ntt_rows<NB, MODE, NB - 1>;
    }
    (void)w1;
    return k_ntt_rows<NB, MODE, -1>;
}

template <int NB>
void launch_rows_nb(int mode, dim3 grid, cudaStream_t s, const DevPlan& P, uint32_t* R, const uint32_t* RA,
                    const uint32_t* ra_sel, bool pdl) {
    // grid comes as (row blocks, primes, batch); the static form takes it as (batch, row blocks, primes)
    const dim3 g = POLYMULT_ROW_STATIC ? dim3(grid.z, grid.x, grid.y) : grid;
    const cudaError_t e = launch_kernel(mode == ROWS_BOTH    ? row_kernel<NB, ROWS_BOTH>(P.w1)
                                        : mode == ROWS_FUSED ? row_kernel<NB, ROWS_FUSED>(P.w1)
                                                             : row_kernel<NB, ROWS_FWD>(P.w1),
                                        g, dim3(128), 0, s, pdl, P, R, RA, ra_sel);
    if (e != cudaSuccess)
        throw_cuda(e, mode == ROWS_BOTH    ? "launch k_ntt_rows<both operands>"
                      : mode == ROWS_FUSED ? "launch k_ntt_rows<fused>"
                                           : "launch k_ntt_rows<forward>");
}

// Applies F<NB>::run(...) for the line length 2^nb, nb in [0, 10].
template <template <int> class F, class... A>
void dispatch_nb(int nb, A&&... a) {
    switch (nb) {
        case 0: F<0>::run(a...); break;
        case 1: F<1>::run(a...); break;
        case 2: F<2>::run(a...); break;
        case 3: F<3>::run(a...); break;
        case 4: F<4>::run(a...); break;
        case 5: F<5>::run(a...); break;
        case 6: F<6>::run(a...); break;
        case 7: F<7>::run(a...); break;
        case 8: F<8>::run(a...); break;
        case 9: F<9>::run(a...); break;
        case 10: F<10>::run(a...); break;
        default: throw_cuda(cudaErrorInvalidValue, "NTT line length above 2^10");
    }
}

template <int NB>
struct ColsF {
    template <class... A>
    static void run(A&&... a) { launch_cols_nb<NB>(a...); }
};
template <int NB>
struct RowsF {
    template <class... A>
    static void run(A&&... a) { launch_rows_nb<NB>(a...); }
};
template <int NB>
struct ColAttrF {
    static void run(int bytes, int w2) {
        const void* fns[2] = {(const void*)k_ntt_cols<NB, false>, (const void*)k_ntt_cols<NB, true>};
        for (const void* f : fns) {
            const cudaError_t e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
            if (e != cudaSuccess) throw_cuda(e, "NTT kernel attribute");
        }
        if constexpr (NB >= 7 && NB <= 8) {
            const void* f2[2] = {(const void*)col2_kernel<NB, false>(w2), (const void*)col2_kernel<NB, true>(w2)};
            for (const void* f : f2) {
                const cudaError_t e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
                if (e != cudaSuccess) throw_cuda(e, "NTT kernel attribute");
            }
        }
        if constexpr (NB == 8) {
            const void* ft[2] = {(const void*)colt_kernel<false>(w2), (const void*)colt_kernel<true>(w2)};
            for (const void* f : ft) {
                const cudaError_t e =
                    cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ColtCfg<NB>::SMEM);
                if (e != cudaSuccess) throw_cuda(e, "NTT kernel attribute");
            }
        }
    }
};
template <int NB>
struct ColProbeF {
    static void run(int w2) {
        const void* fns[2] = {(const void*)k_ntt_cols<NB, false>, (const void*)k_ntt_cols<NB, true>};
        for (const void* f : fns) {
            cudaFuncAttributes fa{};
            const cudaError_t e = cudaFuncGetAttributes(&fa, f);
            if (e != cudaSuccess) throw_cuda(e, "NTT kernel image");
        }
        if constexpr (NB >= 7 && NB <= 8) {
            const void* f2[4] = {(const void*)col2_kernel<NB, false>(w2), (const void*)col2_kernel<NB, true>(w2),
                                 NB == 8 ? (const void*)colt_kernel<false>(w2) : nullptr,
                                 NB == 8 ? (const void*)colt_kernel<true>(w2) : nullptr};
            for (const void* f : f2) {
                if (!f) continue;
                cudaFuncAttributes fa{};
                const cudaError_t e = cudaFuncGetAttributes(&fa, f);
                if (e != cudaSuccess) throw_cuda(e, "NTT kernel image");
            }
        }
    }
};
template <int NB>
struct RowProbeF {
    static void run() {
        const void* fns[3] = {(const void*)k_ntt_rows<NB, ROWS_FWD, -1>, (const void*)k_ntt_rows<NB, ROWS_FUSED, -1>,
                              (const void*)k_ntt_rows<NB, ROWS_BOTH, -1>};
        for (const void* f : fns) {
            cudaFuncAttributes fa{};
            const cudaError_t e = cudaFuncGetAttributes(&fa, f);
            if (e != cudaSuccess) throw_cuda(e, "NTT kernel image");
        }
    }
};
template <int NB>
struct RowsPerCtaF {
    static void run(int* out) { *out = RowCfg<NB>::ROWS_PER_CTA; }
};

}  // namespace

void launch_ntt_cols(bool inv, dim3 grid, size_t smem, cudaStream_t s, const DevPlan& P, uint32_t* R, uint32_t col0,
                     int ltc, bool pdl) {
    dispatch_nb<ColsF>(P.w1, inv, grid, smem, s, P, R, col0, ltc, pdl);
}

void launch_ntt_rows(int mode, dim3 grid, cudaStream_t s, const DevPlan& P, uint32_t* R, const uint32_t* RA,
                     const uint32_t* ra_sel, bool pdl) {
    dispatch_nb<RowsF>(P.w2, mode, grid, s, P, R, RA, ra_sel, pdl);
}

int ntt_rows_per_cta(int w2) {
    int r = 0;
    dispatch_nb<RowsPerCtaF>(w2, &r);
    return r;
}

void ntt_set_smem_limit(int bytes, int w1, int w2) {
    // (the row kernels use static shared memory only)
    if (w1 > 0) dispatch_nb<ColAttrF>(w1, bytes, w2);
}

void ntt_probe_images(int w1, int w2) {
    if (w1 > 0) dispatch_nb<ColProbeF>(w1, w2);
    dispatch_nb<RowProbeF>(w2);
}

size_t ntt_cols_smem(const DevPlan& P, int ltc) {
    if (POLYMULT_COL2 && P.w1 >= 7 && P.w1 <= 8 && ltc >= 6) return ((size_t)8 + 4 * COL2_TC) << P.w1;
    return (size_t)P.nrows * sizeof(Tw2) + ((size_t)P.nrows << ltc) * 4;
}

}  // namespace pm
