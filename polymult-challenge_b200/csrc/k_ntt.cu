// k_ntt.cu -- the negacyclic NTT per RNS prime, 4-step split into a column pass and a row
// pass over the residue arrays R[batch][prime][n], n = row * ncols + col.
//
// Same transform as the reference (psi-merged Cooley-Tukey forward, natural order in and
// bit-reversed out; Gentleman-Sande inverse with the mirrored-twiddle identity
// psi^-bitrev(2^s+i) = -psi^bitrev(2^s+2^s-1-i); solve.cu:204-378), organised differently:
//   * every stage uses Harvey lazy butterflies and Montgomery-Shoup twiddle products
//     (pm_device.cuh), so no butterfly reduces to [0, p);
//   * twiddles come from one table tw[j][k] = psi_j^bitrev(k) R (mod p_j); a row-pass CTA
//     stages the forward and mirrored twiddles of its rows in shared memory with their
//     Shoup companions, instead of forming trow * tsmall with a Montgomery product at every
//     butterfly (solve.cu:286-338);
//   * column tiles are 32 columns wide (128-byte row segments) so that a warp reads whole
//     lines and its 32 lanes hit 32 different banks.
#include <type_traits>

#include "pm_kernels.cuh"

namespace pm {
namespace {

// Radix-2^RAD group g of the pass that starts at local stage LS0 of a line of 2^NB elements
// at element stride es (all shapes compile-time except the stride).  The group's elements are
// idx_e = (hi << (NB - LS0)) | (e << SUB) | lo with SUB = NB - LS0 - RAD, lo = g mod 2^SUB,
// hi = g >> SUB.  Local stage LS0 + k pairs e and e + 2^(RAD-1-k); the twiddle argument (the
// stage's group index within the line) is (hi << k) | (e >> (RAD - k)).  twf(ls, gi) returns
// the twiddle (for INV, already the mirrored one).
template <int NB, int LS0, int RAD, bool INV, class TwF>
__device__ __forceinline__ void radix_group(uint32_t* line, int es, int g, const TwF& twf, uint32_t p) {
    constexpr int G = 1 << RAD;
    constexpr int SUB = NB - LS0 - RAD;
    const int lo = g & ((1 << SUB) - 1), hi = g >> SUB;
    uint32_t* b = line + ((hi << (NB - LS0)) | lo) * es;
    const int step = es << SUB;
    uint32_t v[G];
#pragma unroll
    for (int e = 0; e < G; ++e) v[e] = b[e * step];
    if (!INV) {
#pragma unroll
        for (int k = 0; k < RAD; ++k) {
            const int h = G >> (k + 1);
#pragma unroll
            for (int m = 0; m < (1 << k); ++m) {
                const Tw2 w = twf(LS0 + k, (hi << k) | m);
#pragma unroll
                for (int i = 0; i < h; ++i) bfly_ct(v[m * 2 * h + i], v[m * 2 * h + i + h], w, p);
            }
        }
    } else {
#pragma unroll
        for (int k = RAD - 1; k >= 0; --k) {
            const int h = G >> (k + 1);
#pragma unroll
            for (int m = 0; m < (1 << k); ++m) {
                const Tw2 w = twf(LS0 + k, (hi << k) | m);
#pragma unroll
                for (int i = 0; i < h; ++i) bfly_gs(v[m * 2 * h + i], v[m * 2 * h + i + h], w, p);
            }
        }
    }
#pragma unroll
    for (int e = 0; e < G; ++e) b[e * step] = v[e];
}

// Row tiles live in shared memory swizzled within each row: element x of a row sits at
// swz(x) = x ^ (((x >> 5) & 7) << 2).  The XOR only touches bits 2-4, so aligned runs of 4
// stay contiguous (16-byte vector access), and with the thread mapping of k_ntt_rows every
// radix pass of a 256-point row is free of bank conflicts: the pass at stage 3 (elements 4
// apart) spreads its 8 high index values over the bank bits 2-4, and the pass at stage 6
// (4 contiguous elements per thread) uses 16-byte loads.
__device__ __forceinline__ int swz(int x) { return x ^ (((x >> 5) & 7) << 2); }

template <int RAD, int LS0, bool INV, class TwF>
__device__ __forceinline__ void radix_butterflies(uint32_t (&v)[1 << RAD], int hi, const TwF& twf, uint32_t p) {
    constexpr int G = 1 << RAD;
    if (!INV) {
#pragma unroll
        for (int k = 0; k < RAD; ++k) {
            const int h = G >> (k + 1);
#pragma unroll
            for (int m = 0; m < (1 << k); ++m) {
                const Tw2 w = twf(LS0 + k, (hi << k) | m);
#pragma unroll
                for (int i = 0; i < h; ++i) bfly_ct(v[m * 2 * h + i], v[m * 2 * h + i + h], w, p);
            }
        }
    } else {
#pragma unroll
        for (int k = RAD - 1; k >= 0; --k) {
            const int h = G >> (k + 1);
#pragma unroll
            for (int m = 0; m < (1 << k); ++m) {
                const Tw2 w = twf(LS0 + k, (hi << k) | m);
#pragma unroll
                for (int i = 0; i < h; ++i) bfly_gs(v[m * 2 * h + i], v[m * 2 * h + i + h], w, p);
            }
        }
    }
}

// radix_group for one swizzled row (element stride 1).
template <int NB, int LS0, int RAD, bool INV, class TwF>
__device__ __forceinline__ void radix_group_row(uint32_t* row, int g, const TwF& twf, uint32_t p) {
    constexpr int G = 1 << RAD;
    constexpr int SUB = NB - LS0 - RAD;
    const int lo = g & ((1 << SUB) - 1), hi = g >> SUB;
    const int x0 = (hi << (NB - LS0)) | lo;
    uint32_t v[G];
    if constexpr (SUB == 0 && RAD >= 2) {
#pragma unroll
        for (int q = 0; q < G / 4; ++q) {
            const uint4 u = *reinterpret_cast<const uint4*>(row + swz(x0 + 4 * q));
            v[4 * q] = u.x;
            v[4 * q + 1] = u.y;
            v[4 * q + 2] = u.z;
            v[4 * q + 3] = u.w;
        }
    } else if constexpr (SUB == 0 && RAD == 1) {
        const uint2 u = *reinterpret_cast<const uint2*>(row + swz(x0));
        v[0] = u.x;
        v[1] = u.y;
    } else {
#pragma unroll
        for (int e = 0; e < G; ++e) v[e] = row[swz(x0 + (e << SUB))];
    }
    radix_butterflies<RAD, LS0, INV>(v, hi, twf, p);
    if constexpr (SUB == 0 && RAD >= 2) {
#pragma unroll
        for (int q = 0; q < G / 4; ++q)
            *reinterpret_cast<uint4*>(row + swz(x0 + 4 * q)) = make_uint4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
    } else if constexpr (SUB == 0 && RAD == 1) {
        *reinterpret_cast<uint2*>(row + swz(x0)) = make_uint2(v[0], v[1]);
    } else {
#pragma unroll
        for (int e = 0; e < G; ++e) row[swz(x0 + (e << SUB))] = v[e];
    }
}

// rows [0, rpb) x 2^NB words between global (contiguous) and shared (swizzled rows),
// 16-byte vectors, eight in flight per thread.  Requires 2^NB >= 4.
template <int NB, bool TO_SMEM>
__device__ __forceinline__ void move_rows(uint32_t* sh, uint32_t* g, int rpb) {
    constexpr int Q = (1 << NB) / 4;  // vectors per row
    const int total = rpb * Q;
    for (int b0 = threadIdx.x; b0 < total; b0 += 8 * blockDim.x) {
        uint4 v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int q = b0 + u * blockDim.x;
            if (q < total) {
                const int rr = q / Q, x = 4 * (q % Q);
                v[u] = TO_SMEM ? *reinterpret_cast<const uint4*>(g + 4 * (size_t)q)
                               : *reinterpret_cast<const uint4*>(sh + (rr << NB) + swz(x));
            }
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int q = b0 + u * blockDim.x;
            if (q < total) {
                const int rr = q / Q, x = 4 * (q % Q);
                if (TO_SMEM) *reinterpret_cast<uint4*>(sh + (rr << NB) + swz(x)) = v[u];
                else *reinterpret_cast<uint4*>(g + 4 * (size_t)q) = v[u];
            }
        }
    }
}

template <int V>
using IntC = std::integral_constant<int, V>;

// Runs body(IntC<LS0>, IntC<RAD>) for every radix-8 pass of a 2^NB-point line transform
// (forward: LS0 = 0, 3, 6, ...; inverse: the same passes in reverse), one barrier after each.
template <int NB, int PI, bool INV, class Body>
__device__ __forceinline__ void for_each_pass(const Body& body) {
    constexpr int NPASS = (NB + 2) / 3;
    if constexpr (PI < NPASS) {
        constexpr int IDX = INV ? NPASS - 1 - PI : PI;
        constexpr int LS0 = 3 * IDX;
        constexpr int RAD = (NB - LS0) < 3 ? (NB - LS0) : 3;
        body(IntC<LS0>{}, IntC<RAD>{});
        __syncthreads();
        for_each_pass<NB, PI + 1, INV>(body);
    }
}

// Copies a tile of `rows` x `tc` words between global (row stride gstride) and shared
// (dense [rows][tc]); with 16-byte vectors, eight loads in flight per thread before any store.
template <bool TO_SMEM>
__device__ __forceinline__ void move_tile(uint32_t* sh, uint32_t* g, int rows, int tc, size_t gstride) {
    const bool vec = ((tc & 3) == 0) && (((uintptr_t)g & 15) == 0) && ((gstride & 3) == 0);
    if (vec) {
        const int q4 = tc >> 2, lq = 31 - __clz(q4);
        const int total = rows * q4;
        for (int b0 = threadIdx.x; b0 < total; b0 += 8 * blockDim.x) {
            uint4 v[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int idx = b0 + u * blockDim.x;
                if (idx < total) {
                    const int r = idx >> lq, c = (idx & (q4 - 1)) << 2;
                    v[u] = TO_SMEM ? *reinterpret_cast<const uint4*>(g + (size_t)r * gstride + c)
                                   : reinterpret_cast<const uint4*>(sh)[idx];
                }
            }
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int idx = b0 + u * blockDim.x;
                if (idx < total) {
                    const int r = idx >> lq, c = (idx & (q4 - 1)) << 2;
                    if (TO_SMEM) reinterpret_cast<uint4*>(sh)[idx] = v[u];
                    else *reinterpret_cast<uint4*>(g + (size_t)r * gstride + c) = v[u];
                }
            }
        }
    } else {
        for (int idx = threadIdx.x; idx < rows * tc; idx += blockDim.x) {
            uint32_t* gp = g + (size_t)(idx / tc) * gstride + (idx % tc);
            if (TO_SMEM) sh[idx] = *gp;
            else *gp = sh[idx];
        }
    }
}

// Stages the twiddles of row stages 0..w2-1 for rows [hi0, hi0 + rpb) as Tw2 pairs:
// twf[rpb (2^ls - 1) + t] = tw[2^(w1+ls) + hi0 2^ls + t]; with MIRROR, the entries of the
// mirrored rows in reverse: tw[2^(w1+ls) + (nrows - hi0) 2^ls - 1 - t].
template <bool MIRROR>
__device__ __forceinline__ void stage_row_twiddles(Tw2* out, const uint32_t* tw, int rpb, int w1, int w2,
                                                   uint32_t nrows, uint32_t hi0, uint32_t pinv) {
    if ((rpb & 3) == 0 && w1 + 0 >= 2) {
        const int total4 = rpb * ((1 << w2) - 1) / 4;  // groups of 4 entries, stage blocks are multiples of 4
        for (int g0 = threadIdx.x; g0 < total4; g0 += 4 * blockDim.x) {
            uint4 v[4];
            int dst[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int g = g0 + u * blockDim.x;
                dst[u] = -1;
                if (g < total4) {
                    const int ls = 31 - __clz(4 * g / rpb + 1);
                    const int o = rpb * ((1 << ls) - 1), t = 4 * g - o;
                    const uint32_t s0 = 1u << (w1 + ls);
                    const uint32_t src = MIRROR ? s0 + ((nrows - hi0) << ls) - 4 - t : s0 + (hi0 << ls) + t;
                    v[u] = *reinterpret_cast<const uint4*>(tw + src);
                    dst[u] = o + t;
                }
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                if (dst[u] < 0) continue;
                uint32_t w[4] = {v[u].x, v[u].y, v[u].z, v[u].w};
                if (MIRROR) {
                    const uint32_t t0 = w[0], t1 = w[1];
                    w[0] = w[3];
                    w[1] = w[2];
                    w[2] = t1;
                    w[3] = t0;
                }
                uint4* o4 = reinterpret_cast<uint4*>(out + dst[u]);
                o4[0] = make_uint4(w[0], w[0] * pinv, w[1], w[1] * pinv);
                o4[1] = make_uint4(w[2], w[2] * pinv, w[3], w[3] * pinv);
            }
        }
    } else {
        for (int ls = 0; ls < w2; ++ls) {
            const int o = rpb * ((1 << ls) - 1), cnt = rpb << ls;
            const uint32_t s0 = 1u << (w1 + ls);
            for (int t = threadIdx.x; t < cnt; t += blockDim.x)
                out[o + t] = make_tw(tw[MIRROR ? s0 + ((nrows - hi0) << ls) - 1 - t : s0 + (hi0 << ls) + t], pinv);
        }
    }
}

}  // namespace

// Column pass: the first w1 = NB stages on a tile of 2^ltc columns x 2^NB rows of prime
// blockIdx.y, batch blockIdx.z.  Column stage s, group i uses tw[2^s + i] (forward) or
// tw[2^(s+1) - 1 - i] (inverse); all of them index below nrows.  Consecutive threads take
// consecutive columns, so a warp's 32 lanes hit 32 banks and share one twiddle.
template <int NB, bool INV>
__global__ void __launch_bounds__(256) k_ntt_cols(DevPlan P, uint32_t* __restrict__ R, uint32_t col0, int ltc) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int NR = 1 << NB;
    const int tc = 1 << ltc;
    Tw2* tws = reinterpret_cast<Tw2*>(smem_raw);            // [NR]
    uint32_t* sh = reinterpret_cast<uint32_t*>(tws + NR);   // [NR][tc]
    const int j = (int)blockIdx.y;
    const uint32_t p = P.p[j], pinv = P.pinv[j];
    uint32_t* base = R + ((size_t)blockIdx.z * P.K + j) * P.N + col0 + ((uint32_t)blockIdx.x << ltc);
    const uint32_t* tw = P.tw + (size_t)j * P.N;

    move_tile<true>(sh, base, NR, tc, P.ncols);
    for (int k = threadIdx.x; k < NR; k += blockDim.x) tws[k] = make_tw(__ldg(tw + k), pinv);
    __syncthreads();

    auto twf = [&](int ls, int gi) { return INV ? tws[(2 << ls) - 1 - gi] : tws[(1 << ls) + gi]; };
    for_each_pass<NB, 0, INV>([&](auto l0, auto rd) {
        constexpr int LS0 = decltype(l0)::value, RAD = decltype(rd)::value;
        for (int t = threadIdx.x; t < ((NR >> RAD) << ltc); t += blockDim.x)
            radix_group<NB, LS0, RAD, INV>(sh + (t & (tc - 1)), tc, t >> ltc, twf, p);
    });
    move_tile<false>(sh, base, NR, tc, P.ncols);
}

// Row pass over `rpb` consecutive rows of prime blockIdx.y, batch blockIdx.z.
//   FUSED = false: forward row stages (operand a).
//   FUSED = true : forward row stages of b, pointwise product with the finished transform of
//                  a (RA), inverse row stages.  The Montgomery pointwise product leaves a
//                  factor 2^-32 that the CRT constant crt_c compensates.
// Row stage ls of row hi, group gi uses tw[2^(w1+ls) + hi 2^ls + gi]; for a block of rows
// [hi0, hi0 + rpb) those entries are one contiguous run per stage, staged in shared memory
// as twf[rpb (2^ls - 1) + rr 2^ls + gi].  The inverse twiddle of (hi, gi) is the forward
// entry of the mirrored row nrows-1-hi at 2^ls-1-gi, staged as twi with the same indexing.
template <int NB, bool FUSED>
__global__ void __launch_bounds__(128) k_ntt_rows(DevPlan P, uint32_t* __restrict__ R, const uint32_t* __restrict__ RA,
                                                  int rpb) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int w2 = NB, nc = 1 << NB;
    const int w1 = P.w1;
    const int ntw = ntt_row_twiddle_slots(rpb, nc);
    Tw2* twf_s = reinterpret_cast<Tw2*>(smem_raw);
    Tw2* twi_s = twf_s + ntw;
    uint32_t* sh = reinterpret_cast<uint32_t*>(twi_s + (FUSED ? ntw : 0));
    const int j = (int)blockIdx.y;
    const uint32_t p = P.p[j], pinv = P.pinv[j];
    const uint32_t hi0 = blockIdx.x * (uint32_t)rpb;
    const size_t off = ((size_t)blockIdx.z * P.K + j) * P.N + (size_t)hi0 * nc;
    uint32_t* rows = R + off;
    const uint32_t* tw = P.tw + (size_t)j * P.N;
    constexpr bool VEC = nc >= 4;

    if constexpr (VEC) move_rows<NB, true>(sh, rows, rpb);
    else
        for (int idx = threadIdx.x; idx < rpb * nc; idx += blockDim.x) sh[idx] = rows[idx];
    stage_row_twiddles<false>(twf_s, tw, rpb, w1, w2, P.nrows, hi0, pinv);
    if (FUSED) stage_row_twiddles<true>(twi_s, tw, rpb, w1, w2, P.nrows, hi0, pinv);
    __syncthreads();

    for_each_pass<NB, 0, false>([&](auto l0, auto rd) {
        constexpr int LS0 = decltype(l0)::value, RAD = decltype(rd)::value, LG = NB - RAD;
        for (int t = threadIdx.x; t < (rpb << LG); t += blockDim.x) {
            const int rr = t >> LG;
            auto twf = [&](int ls, int gi) { return twf_s[rpb * ((1 << ls) - 1) + (rr << ls) + gi]; };
            radix_group_row<NB, LS0, RAD, false>(sh + (rr << NB), t & ((1 << LG) - 1), twf, p);
        }
    });
    if (FUSED) {
        const uint32_t* arows = RA + off;
        if constexpr (VEC) {
            for (int q = threadIdx.x; q < rpb * nc / 4; q += blockDim.x) {
                const int rr = q / (nc / 4), x = 4 * (q % (nc / 4));
                const uint4 a4 = *reinterpret_cast<const uint4*>(arows + 4 * (size_t)q);
                uint4* s4 = reinterpret_cast<uint4*>(sh + (rr << NB) + swz(x));
                uint4 b4 = *s4;
                // a in [0, 4p) -> [0, p); Montgomery product (0, 2p)
                b4.x = mont_mul(red_once(red_once(a4.x, 2 * p), p), b4.x, p, pinv);
                b4.y = mont_mul(red_once(red_once(a4.y, 2 * p), p), b4.y, p, pinv);
                b4.z = mont_mul(red_once(red_once(a4.z, 2 * p), p), b4.z, p, pinv);
                b4.w = mont_mul(red_once(red_once(a4.w, 2 * p), p), b4.w, p, pinv);
                *s4 = b4;
            }
        } else {
            for (int idx = threadIdx.x; idx < rpb * nc; idx += blockDim.x) {
                const uint32_t a = red_once(red_once(arows[idx], 2 * p), p);
                sh[idx] = mont_mul(a, sh[idx], p, pinv);
            }
        }
        __syncthreads();
        for_each_pass<NB, 0, true>([&](auto l0, auto rd) {
            constexpr int LS0 = decltype(l0)::value, RAD = decltype(rd)::value, LG = NB - RAD;
            for (int t = threadIdx.x; t < (rpb << LG); t += blockDim.x) {
                const int rr = t >> LG;
                auto twf = [&](int ls, int gi) { return twi_s[rpb * ((1 << ls) - 1) + (rr << ls) + gi]; };
                radix_group_row<NB, LS0, RAD, true>(sh + (rr << NB), t & ((1 << LG) - 1), twf, p);
            }
        });
    }
    if constexpr (VEC) move_rows<NB, false>(sh, rows, rpb);
    else
        for (int idx = threadIdx.x; idx < rpb * nc; idx += blockDim.x) rows[idx] = sh[idx];
}

namespace {

template <int NB>
void launch_cols_nb(bool inv, dim3 grid, size_t smem, cudaStream_t s, const DevPlan& P, uint32_t* R, uint32_t col0,
                    int ltc) {
    if (inv) k_ntt_cols<NB, true><<<grid, 256, smem, s>>>(P, R, col0, ltc);
    else k_ntt_cols<NB, false><<<grid, 256, smem, s>>>(P, R, col0, ltc);
}

template <int NB>
void launch_rows_nb(bool fused, dim3 grid, size_t smem, cudaStream_t s, const DevPlan& P, uint32_t* R,
                    const uint32_t* RA, int rpb) {
    if (fused) k_ntt_rows<NB, true><<<grid, 128, smem, s>>>(P, R, RA, rpb);
    else k_ntt_rows<NB, false><<<grid, 128, smem, s>>>(P, R, RA, rpb);
}

// Applies f<NB>() for the line length nb in [0, PM_MAX_LINE_LOG].
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
struct AttrF {
    static void run(int bytes) {
        const void* fns[4] = {(const void*)k_ntt_cols<NB, false>, (const void*)k_ntt_cols<NB, true>,
                              (const void*)k_ntt_rows<NB, false>, (const void*)k_ntt_rows<NB, true>};
        for (const void* f : fns) {
            const cudaError_t e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
            if (e != cudaSuccess) throw_cuda(e, "NTT kernel attribute");
        }
    }
};
template <int NB>
struct ProbeF {
    static void run() {
        const void* fns[4] = {(const void*)k_ntt_cols<NB, false>, (const void*)k_ntt_cols<NB, true>,
                              (const void*)k_ntt_rows<NB, false>, (const void*)k_ntt_rows<NB, true>};
        for (const void* f : fns) {
            cudaFuncAttributes fa{};
            const cudaError_t e = cudaFuncGetAttributes(&fa, f);
            if (e != cudaSuccess) throw_cuda(e, "NTT kernel image");
        }
    }
};

}  // namespace

void launch_ntt_cols(bool inv, dim3 grid, size_t smem, cudaStream_t s, const DevPlan& P, uint32_t* R, uint32_t col0,
                     int ltc) {
    dispatch_nb<ColsF>(P.w1, inv, grid, smem, s, P, R, col0, ltc);
}

void launch_ntt_rows(bool fused, dim3 grid, size_t smem, cudaStream_t s, const DevPlan& P, uint32_t* R,
                     const uint32_t* RA, int rpb) {
    dispatch_nb<RowsF>(P.w2, fused, grid, smem, s, P, R, RA, rpb);
}

void ntt_set_smem_limit(int bytes, int w1, int w2) {
    dispatch_nb<AttrF>(w1, bytes);
    if (w2 != w1) dispatch_nb<AttrF>(w2, bytes);
}

void ntt_probe_images(int w1, int w2) {
    dispatch_nb<ProbeF>(w1);
    if (w2 != w1) dispatch_nb<ProbeF>(w2);
}

size_t ntt_cols_smem(const DevPlan& P, int ltc) {
    return (size_t)P.nrows * sizeof(Tw2) + ((size_t)P.nrows << ltc) * 4;
}

size_t ntt_rows_smem(const DevPlan& P, int rpb, bool fused) {
    const size_t ntw = (size_t)ntt_row_twiddle_slots(rpb, (int)P.ncols);
    return ntw * sizeof(Tw2) * (fused ? 2 : 1) + (size_t)rpb * P.ncols * 4;
}

}  // namespace pm
