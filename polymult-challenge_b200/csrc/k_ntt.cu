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
#include "pm_kernels.cuh"

namespace pm {
namespace {

// Radix-2^RAD group g of a pass starting at local stage ls0 on a line of 2^nb elements at
// element stride es.  Its elements are idx_e = (hi << (nb - ls0)) | (e << sub) | lo with
// sub = nb - ls0 - RAD, lo = g mod 2^sub, hi = g >> sub.  Local stage ls0 + k pairs e and
// e + 2^(RAD-1-k); the twiddle argument (the stage's group index within the line) is
// (hi << k) | (e >> (RAD - k)).  twf(ls, gi) returns the (already mirrored, for INV) twiddle.
template <int RAD, bool INV, class TwF>
__device__ __forceinline__ void radix_group(uint32_t* line, int es, int nb, int ls0, int g, const TwF& twf,
                                            uint32_t p) {
    constexpr int G = 1 << RAD;
    const int sub = nb - ls0 - RAD;
    const int lo = g & ((1 << sub) - 1), hi = g >> sub;
    uint32_t* b = line + (size_t)((hi << (nb - ls0)) | lo) * es;
    const int step = es << sub;
    uint32_t v[G];
#pragma unroll
    for (int e = 0; e < G; ++e) v[e] = b[e * step];
    if (!INV) {
#pragma unroll
        for (int k = 0; k < RAD; ++k) {
            const int h = G >> (k + 1);
#pragma unroll
            for (int m = 0; m < (1 << k); ++m) {
                const Tw2 w = twf(ls0 + k, (hi << k) | m);
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
                const Tw2 w = twf(ls0 + k, (hi << k) | m);
#pragma unroll
                for (int i = 0; i < h; ++i) bfly_gs(v[m * 2 * h + i], v[m * 2 * h + i + h], w, p);
            }
        }
    }
#pragma unroll
    for (int e = 0; e < G; ++e) b[e * step] = v[e];
}

template <bool INV, class TwF>
__device__ __forceinline__ void radix_group_r(int r, uint32_t* line, int es, int nb, int ls0, int g, const TwF& twf,
                                              uint32_t p) {
    if (r == 3) radix_group<3, INV>(line, es, nb, ls0, g, twf, p);
    else if (r == 2) radix_group<2, INV>(line, es, nb, ls0, g, twf, p);
    else radix_group<1, INV>(line, es, nb, ls0, g, twf, p);
}

}  // namespace

// Column pass: the first w1 stages on a tile of 2^ltc columns x nrows rows of prime
// blockIdx.y, batch blockIdx.z.  Column stage s, group i uses tw[2^s + i] (forward) or
// tw[2^(s+1) - 1 - i] (inverse); all of them index below nrows.
template <bool INV>
__global__ void __launch_bounds__(256) k_ntt_cols(DevPlan P, uint32_t* __restrict__ R, uint32_t col0, int ltc) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int nr = (int)P.nrows, w1 = P.w1, tc = 1 << ltc;
    Tw2* tws = reinterpret_cast<Tw2*>(smem_raw);            // [nrows]
    uint32_t* sh = reinterpret_cast<uint32_t*>(tws + nr);   // [nrows][tc]
    const int j = (int)blockIdx.y;
    const uint32_t p = P.p[j], pinv = P.pinv[j];
    uint32_t* base = R + ((size_t)blockIdx.z * P.K + j) * P.N + col0 + ((uint32_t)blockIdx.x << ltc);
    const uint32_t* tw = P.tw + (size_t)j * P.N;

    for (int k = threadIdx.x; k < nr; k += blockDim.x) tws[k] = make_tw(tw[k], pinv);
    for (int idx = threadIdx.x; idx < (nr << ltc); idx += blockDim.x)
        sh[idx] = base[(size_t)(idx >> ltc) * P.ncols + (idx & (tc - 1))];
    __syncthreads();

    auto twf = [&](int ls, int gi) { return INV ? tws[(2 << ls) - 1 - gi] : tws[(1 << ls) + gi]; };
    const int npass = (w1 + 2) / 3;
    for (int pi = 0; pi < npass; ++pi) {
        const int ls0 = 3 * (INV ? npass - 1 - pi : pi), r = min(3, w1 - ls0);
        for (int t = threadIdx.x; t < ((nr >> r) << ltc); t += blockDim.x)
            radix_group_r<INV>(r, sh + (t & (tc - 1)), tc, w1, ls0, t >> ltc, twf, p);
        __syncthreads();
    }
    for (int idx = threadIdx.x; idx < (nr << ltc); idx += blockDim.x)
        base[(size_t)(idx >> ltc) * P.ncols + (idx & (tc - 1))] = sh[idx];
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
template <bool FUSED>
__global__ void __launch_bounds__(128) k_ntt_rows(DevPlan P, uint32_t* __restrict__ R, const uint32_t* __restrict__ RA,
                                                  int rpb) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int w1 = P.w1, w2 = P.w2, nc = (int)P.ncols;
    const int ntw = rpb * (nc - 1);
    Tw2* twf_s = reinterpret_cast<Tw2*>(smem_raw);
    Tw2* twi_s = twf_s + (ntw > 0 ? ntw : 1);
    uint32_t* sh = reinterpret_cast<uint32_t*>(twi_s + (FUSED ? (ntw > 0 ? ntw : 1) : 0));
    const int j = (int)blockIdx.y;
    const uint32_t p = P.p[j], pinv = P.pinv[j];
    const uint32_t hi0 = blockIdx.x * (uint32_t)rpb;
    const size_t off = ((size_t)blockIdx.z * P.K + j) * P.N + (size_t)hi0 * nc;
    uint32_t* rows = R + off;
    const uint32_t* tw = P.tw + (size_t)j * P.N;

    for (int idx = threadIdx.x; idx < rpb * nc; idx += blockDim.x) sh[idx] = rows[idx];
    for (int ls = 0; ls < w2; ++ls) {
        const int o = rpb * ((1 << ls) - 1), cnt = rpb << ls;
        const uint32_t s0 = 1u << (w1 + ls);
        for (int t = threadIdx.x; t < cnt; t += blockDim.x) {
            twf_s[o + t] = make_tw(tw[s0 + (hi0 << ls) + t], pinv);
            if (FUSED) twi_s[o + t] = make_tw(tw[s0 + ((P.nrows - hi0) << ls) - 1 - t], pinv);
        }
    }
    __syncthreads();

    const int npass = (w2 + 2) / 3;
    for (int pi = 0; pi < npass; ++pi) {
        const int ls0 = 3 * pi, r = min(3, w2 - ls0), lg = w2 - r;
        for (int t = threadIdx.x; t < (rpb << lg); t += blockDim.x) {
            const int rr = t >> lg;
            auto twf = [&](int ls, int gi) { return twf_s[rpb * ((1 << ls) - 1) + (rr << ls) + gi]; };
            radix_group_r<false>(r, sh + rr * nc, 1, w2, ls0, t & ((1 << lg) - 1), twf, p);
        }
        __syncthreads();
    }
    if (FUSED) {
        const uint32_t* arows = RA + off;
        for (int idx = threadIdx.x; idx < rpb * nc; idx += blockDim.x) {
            const uint32_t a = red_once(red_once(arows[idx], 2 * p), p);   // [0, 4p) -> [0, p)
            sh[idx] = mont_mul(a, sh[idx], p, pinv);                        // (0, 2p)
        }
        __syncthreads();
        for (int pi = npass - 1; pi >= 0; --pi) {
            const int ls0 = 3 * pi, r = min(3, w2 - ls0), lg = w2 - r;
            for (int t = threadIdx.x; t < (rpb << lg); t += blockDim.x) {
                const int rr = t >> lg;
                auto twf = [&](int ls, int gi) { return twi_s[rpb * ((1 << ls) - 1) + (rr << ls) + gi]; };
                radix_group_r<true>(r, sh + rr * nc, 1, w2, ls0, t & ((1 << lg) - 1), twf, p);
            }
            __syncthreads();
        }
    }
    for (int idx = threadIdx.x; idx < rpb * nc; idx += blockDim.x) rows[idx] = sh[idx];
}

void launch_ntt_cols(bool inv, dim3 grid, size_t smem, cudaStream_t s, const DevPlan& P, uint32_t* R, uint32_t col0,
                     int ltc) {
    if (inv) k_ntt_cols<true><<<grid, 256, smem, s>>>(P, R, col0, ltc);
    else k_ntt_cols<false><<<grid, 256, smem, s>>>(P, R, col0, ltc);
}

void launch_ntt_rows(bool fused, dim3 grid, size_t smem, cudaStream_t s, const DevPlan& P, uint32_t* R,
                     const uint32_t* RA, int rpb) {
    if (fused) k_ntt_rows<true><<<grid, 128, smem, s>>>(P, R, RA, rpb);
    else k_ntt_rows<false><<<grid, 128, smem, s>>>(P, R, RA, rpb);
}

namespace {
struct NttKernel {
    const void* fn;
    const char* name;
};
const NttKernel kNttKernels[] = {{(const void*)k_ntt_cols<false>, "k_ntt_cols<forward>"},
                                 {(const void*)k_ntt_cols<true>, "k_ntt_cols<inverse>"},
                                 {(const void*)k_ntt_rows<false>, "k_ntt_rows<forward>"},
                                 {(const void*)k_ntt_rows<true>, "k_ntt_rows<fused>"}};
}  // namespace

void ntt_set_smem_limit(int bytes) {
    for (const NttKernel& k : kNttKernels) {
        const cudaError_t e = cudaFuncSetAttribute(k.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
        if (e != cudaSuccess) throw_cuda(e, k.name);
    }
}

void ntt_probe_images() {
    for (const NttKernel& k : kNttKernels) {
        cudaFuncAttributes fa{};
        const cudaError_t e = cudaFuncGetAttributes(&fa, k.fn);
        if (e != cudaSuccess) throw_cuda(e, k.name);
    }
}

size_t ntt_cols_smem(const DevPlan& P, int ltc) {
    return (size_t)P.nrows * sizeof(Tw2) + ((size_t)P.nrows << ltc) * 4;
}

size_t ntt_rows_smem(const DevPlan& P, int rpb, bool fused) {
    const size_t ntw = std::max<size_t>(1, (size_t)rpb * (P.ncols - 1));
    return ntw * sizeof(Tw2) * (fused ? 2 : 1) + (size_t)rpb * P.ncols * 4;
}

}  // namespace pm
