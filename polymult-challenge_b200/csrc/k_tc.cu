// k_tc.cu -- the RNS decomposition and the CRT as exact tcgen05 kind::i8 tensor-core GEMMs.
//
// Both contractions of the reference (solve.cu:147-202 and 380-501, u16 x u32 -> u64 on
// CUDA cores) are recast with every operand split into unsigned bytes, accumulated exactly
// in s32 in tensor memory, and recombined in the epilogue:
//
// Decomposition, per tile of 128 coefficients (A = coefficient bytes, K-dim = 4L bytes):
//   D[m][4j+t] = sum_s byte_s(a_m) * byte_t(2^(8s) R mod p_j)      (< 4L 255^2 < 2^25)
//   x = sum_t D[m][4j+t] 2^(8t)  (< 2^49 < p 2^32)  ->  REDC(x) = a_m mod p_j
// CRT, per tile of 128 coefficients (A = bytes of y_j, K-dim = 4K bytes):
//   D[m][v] = sum_{j,t} byte_t(y_j) * byte_(v-t)(Q_j)               (< 4K 255^2 < 2^31)
//   z = sum_v D[m][v] 2^(8v) + T_v  ->  carries into limbs, delta-fold, - q
//
// Operands live in shared memory in the UMMA K-major no-swizzle canonical layout (core
// matrices of 8 rows x 16 bytes; LBO = 128 B between K-adjacent core matrices, SBO =
// 8 * k_bytes between 8-row groups).  The B operand (a per-point constant table, built on
// the host in exactly that layout) is copied into shared memory once per persistent CTA;
// the A tile is re-laid-out from global memory by the CTA's 128 threads.  One elected thread
// issues the MMAs (M = 128, N <= 256 per instruction, K = 32 bytes) into TMEM and commits
// them to an mbarrier; each warp then reads its 32 TMEM lanes (one coefficient per thread)
// with tcgen05.ld for the epilogue.  Every mbarrier wait is bounded by a clock limit and
// reports DEV_ERR_WAIT instead of hanging.
#include "pm_crt.cuh"
#include "pm_kernels.cuh"

namespace pm {
namespace {

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, P1;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Waits for phase `parity` of `bar`; false after about one second of clocks.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity))
        if (clock64() - t0 > 2000000000ll) return false;
    return true;
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_smem_to_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// whole warp
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// D[tmem] (+)= A[smem] * B[smem]^T, unsigned bytes, s32 accumulate; one thread.
__device__ __forceinline__ void umma_u8(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                        uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar))
                 : "memory");
}

// 32 TMEM lanes (this warp's) x 16 consecutive 32-bit columns.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Shared-memory matrix descriptor, K-major, no swizzle (layout type 0), Blackwell version 1.
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor, kind::i8: D = s32, A = B = u8, both K-major, M = 128.
__device__ __forceinline__ uint32_t idesc_u8(int n) {
    return (2u << 4) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(TC_M >> 4) << 24);
}

// Issues D[:, col0 : col0 + nn) = A * B[row0 : row0 + nn, :]^T into TMEM column col0.
__device__ __forceinline__ void issue_gemm_rows(uint32_t tmem_col, uint32_t a_base, uint32_t b_base, int row0, int nn,
                                                int kbytes) {
    const uint32_t sbo = 8u * (uint32_t)kbytes;
    const uint32_t idesc = idesc_u8(nn);
    for (int kk = 0; kk < kbytes / 32; ++kk) {
        const uint64_t ad = sdesc(a_base + 256u * kk, 128u, sbo);
        const uint64_t bd = sdesc(b_base + (uint32_t)(row0 >> 3) * sbo + 256u * kk, 128u, sbo);
        umma_u8(tmem_col, ad, bd, idesc, kk > 0 ? 1u : 0u);
    }
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

// TMA-engine bulk copy global -> shared (16-byte aligned addresses, size a multiple of 16),
// completing `bytes` transactions on `bar`.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

// One thread: expect and issue a copy of `bytes` (multiple of 16) in pieces of <= 32 KB.
__device__ __forceinline__ void bulk_g2s_all(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    mbar_arrive_expect_tx(bar, bytes);
    for (uint32_t off = 0; off < bytes; off += 32768u) {
        const uint32_t n = min(32768u, bytes - off);
        bulk_g2s(static_cast<unsigned char*>(dst) + off, static_cast<const unsigned char*>(src) + off, n, bar);
    }
}

}  // namespace

// ----------------------------------------------------------------------------------------
// Decomposition.  Persistent: grid <= #SMs, tiles of 128 positions over (batch, npos).
// 256 threads = 8 epilogue warps; warp w reads TMEM lanes 32 (w % 4) of column half w / 4.
// Per tile: the raw coefficients (contiguous cnt*L words) arrive by one bulk copy into a
// double-buffered ring, prefetched two tiles ahead; all warps re-lay them out as the K-major
// A operand; thread 0 issues the MMAs of the two prime halves with one commit each, so the
// epilogue of half 0 overlaps the MMA of half 1.
// smem: [B image][A tile][raw ring 2 x 128*L words][bars: B, raw0, raw1, mma0, mma1][slot]
// ----------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256, 1) k_rns_tc(DevPlan P, const uint32_t* __restrict__ src, ChunkMap C,
                                                   uint32_t npos, uint32_t nbatch, uint32_t* __restrict__ R,
                                                   int use_bulk) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int L = P.L, kb = P.dec_kbytes, nrows_b = P.dec_nrows;
    const int KH = dec_half_primes(P.KP);                 // primes of half 0
    const int n0 = 4 * KH, n1 = nrows_b - n0;              // MMA N of the halves
    const uint32_t col1 = dec_half1_col(n0);               // TMEM column of half 1
    unsigned char* b_s = smem_raw;
    unsigned char* a_s = b_s + (size_t)nrows_b * kb;
    uint32_t* raw_s = reinterpret_cast<uint32_t*>(a_s + (size_t)TC_M * kb);
    const size_t raw_words = (size_t)TC_M * L;
    uint64_t* bars = reinterpret_cast<uint64_t*>(raw_s + 2 * raw_words);
    uint64_t *bar_b = bars, *bar_raw = bars + 1, *bar_mma = bars + 3;
    uint32_t* slot = reinterpret_cast<uint32_t*>(bars + 5);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t ncols = tmem_cols_for((int)col1 + n1);

    const uint32_t tiles_per_batch = (npos + TC_M - 1) / TC_M;
    const uint32_t ntiles = tiles_per_batch * nbatch;
    auto tile_src = [&](uint32_t tile, int* cnt) {
        const uint32_t b = tile / tiles_per_batch;
        const uint32_t pos0 = (tile - b * tiles_per_batch) * TC_M;
        *cnt = (int)min((uint32_t)TC_M, npos - pos0);
        return src + ((size_t)b * npos + pos0) * L;
    };

    if (threadIdx.x == 0) {
        for (int i = 0; i < 5; ++i) mbar_init(bars + i, 1);
        bulk_g2s_all(b_s, P.dec_b, (uint32_t)((size_t)nrows_b * kb), bar_b);
        if (use_bulk)
            for (int k = 0; k < 2; ++k) {
                const uint32_t t = blockIdx.x + k * gridDim.x;
                if (t < ntiles) {
                    int cnt;
                    const uint32_t* s = tile_src(t, &cnt);
                    bulk_g2s_all(raw_s + k * raw_words, s, (uint32_t)cnt * L * 4, bar_raw + k);
                }
            }
    }
    if (warp == 0) tmem_alloc(slot, ncols);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *slot;
    bool ok = mbar_wait_bounded(bar_b, 0);

    const uint32_t sbo = 8u * (uint32_t)kb;
    const int groups = kb / 16;
    const int half = warp >> 2, m = (warp & 3) * 32 + lane;
    uint32_t i = 0;
    for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++i) {
        const int buf = (int)(i & 1);
        int cnt;
        const uint32_t* s = tile_src(tile, &cnt);
        uint32_t* raw = raw_s + buf * raw_words;
        if (use_bulk) {
            ok = ok && mbar_wait_bounded(bar_raw + buf, (i >> 1) & 1);
        } else {
            for (int w = threadIdx.x; w < cnt * L; w += blockDim.x) raw[w] = __ldg(s + w);
        }
        if (__syncthreads_or(!ok)) break;
        // re-layout: row mm, 16-byte group g = limbs 4g..4g+3 (zero past L or past cnt)
        for (int w = threadIdx.x; w < TC_M * groups; w += blockDim.x) {
            const int mm = w & (TC_M - 1), g = w >> 7;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (mm < cnt) {
                const uint32_t* row = raw + mm * L;
                const int l0 = 4 * g;
                v.x = l0 < L ? row[l0] : 0u;
                v.y = l0 + 1 < L ? row[l0 + 1] : 0u;
                v.z = l0 + 2 < L ? row[l0 + 2] : 0u;
                v.w = l0 + 3 < L ? row[l0 + 3] : 0u;
            }
            *reinterpret_cast<uint4*>(a_s + (size_t)(mm >> 3) * sbo + (size_t)g * 128 + (mm & 7) * 16) = v;
        }
        fence_smem_to_async();
        __syncthreads();
        if (threadIdx.x == 0) {
            const uint32_t nxt = tile + 2 * gridDim.x;
            if (use_bulk && nxt < ntiles) {  // the ring slot was just consumed
                int c2;
                const uint32_t* s2 = tile_src(nxt, &c2);
                bulk_g2s_all(raw, s2, (uint32_t)c2 * L * 4, bar_raw + buf);
            }
            tc_fence_after();
            issue_gemm_rows(tmem, smem_addr(a_s), smem_addr(b_s), 0, n0, kb);
            umma_commit(bar_mma);
            if (n1 > 0) {
                issue_gemm_rows(tmem + col1, smem_addr(a_s), smem_addr(b_s), n0, n1, kb);
                umma_commit(bar_mma + 1);
            }
        }
        if (half == 0 || n1 > 0) {
            const bool got = mbar_wait_bounded(bar_mma + half, i & 1);
            if (!got) flag_error(P.status, DEV_ERR_WAIT);
            tc_fence_after();
            const uint32_t b = tile / tiles_per_batch;
            const uint32_t pos0 = (tile - b * tiles_per_batch) * TC_M;
            const uint32_t n = m < cnt ? chunk_pos_to_n(P, C, pos0 + m) : 0;
            uint32_t* Rb = R + (size_t)b * P.K * P.N + n;
            const int j0 = half ? KH : 0;
            const int cols = half ? n1 : n0;
            const uint32_t tcol = tmem + (half ? col1 : 0) + ((uint32_t)((warp & 3) * 32) << 16);
            for (int c16 = 0; c16 < cols / 16 && got; ++c16) {
                uint32_t r[16];
                tmem_ld16(tcol + (uint32_t)(16 * c16), r);
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int j = j0 + 4 * c16 + q;
                    if (j < P.K && m < cnt) {
                        const uint64_t x = (uint64_t)r[4 * q] + ((uint64_t)r[4 * q + 1] << 8) +
                                           ((uint64_t)r[4 * q + 2] << 16) + ((uint64_t)r[4 * q + 3] << 24);
                        const uint32_t p = __ldg(P.p + j);
                        Rb[(size_t)j * P.N] = red_once(redc64(x, p, __ldg(P.pinv + j)), p);
                    }
                }
            }
            ok = ok && got;
        }
        tc_fence_before();
        if (__syncthreads_or(!ok)) break;
    }
    if (!ok && threadIdx.x == 0) flag_error(P.status, DEV_ERR_WAIT);
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, ncols);
}

// ----------------------------------------------------------------------------------------
// CRT.  Persistent; 256 threads, two per coefficient: warp w serves TMEM lane quarter w % 4
// (coefficient m = 32 (w % 4) + lane) and half h = w / 4 of the work -- half of the prime
// groups in the prologue, half of the result limbs in the epilogue (each half runs its own
// carry chain; half 0's carry-out is then added into half 1's limbs).  The residues of the
// next tile arrive by bulk copies into one staging tile while this tile's MMA and epilogue run.
// smem: [B image][A tile (z rows after the MMA)][R tile K x 128][per-prime constants]
//       [partial sums 2 x 128][bars][slot]
// ----------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256, 1) k_crt_tc(DevPlan P, const uint32_t* __restrict__ R, ChunkMap C,
                                                   uint32_t npos, uint32_t nbatch, uint32_t* __restrict__ out,
                                                   int gather) {
    const bool use_bulk = gather == CRT_GATHER_BULK;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int K = P.K, KP = P.KP, L = P.L, kb = P.crt_kbytes, nrows_b = P.crt_nrows;
    const int zl = crt_zl(L), zs = crt_zstride(L);
    unsigned char* b_s = smem_raw;
    unsigned char* a_s = b_s + (size_t)nrows_b * kb;
    uint32_t* z_s = reinterpret_cast<uint32_t*>(a_s);            // after the MMA has consumed A
    uint32_t* rt = reinterpret_cast<uint32_t*>(a_s + crt_a_bytes(P));  // [K][128] (rows >= K never read)
    uint32_t* cp = rt + (size_t)K * TC_M;                         // p_j
    uint32_t* cc = cp + KP;                                       // crt_c_j
    uint32_t* ccc = cc + KP;                                      // crt_cc_j
    float* crc = reinterpret_cast<float*>(ccc + KP);              // 1 / p_j
    float* spart = crc + KP;                                      // [2][128]
    uint64_t* bars = reinterpret_cast<uint64_t*>(spart + 2 * TC_M);
    uint64_t *bar_b = bars, *bar_r = bars + 1, *bar_mma = bars + 2;
    uint32_t* slot = reinterpret_cast<uint32_t*>(bars + 3);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int hf = warp >> 2, m = (warp & 3) * 32 + lane;
    const uint32_t ncols = tmem_cols_for(nrows_b);
    const uint32_t tiles_per_batch = (npos + TC_M - 1) / TC_M;
    const uint32_t ntiles = tiles_per_batch * nbatch;
    const uint32_t seg = min(C.cw, (uint32_t)TC_M);  // positions per contiguous segment
    const int kgroups = kb / 16;
    const int gh = (kgroups + 1) / 2;                 // prime groups of half 0
    const int nl = nrows_b / 4;                       // limbs covered by the accumulator columns
    const int lh = ((nl + 1) / 2 + 3) / 4 * 4;        // limbs of half 0 (multiple of 4: 16 columns)

    // warp 0: bulk copies of tile `t`'s residues into rt
    auto issue_r = [&](uint32_t t) {
        const uint32_t b = t / tiles_per_batch;
        const uint32_t pos0 = (t - b * tiles_per_batch) * TC_M;
        const uint32_t cnt = min((uint32_t)TC_M, npos - pos0);
        const uint32_t nseg = (cnt + seg - 1) / seg;
        if (lane == 0) mbar_arrive_expect_tx(bar_r, (uint32_t)K * cnt * 4u);
        __syncwarp();
        const uint32_t* Rb = R + (size_t)b * K * P.N;
        for (uint32_t c = lane; c < (uint32_t)K * nseg; c += 32) {
            const uint32_t j = c / nseg, sg = c - j * nseg;
            const uint32_t p0 = pos0 + sg * seg;
            const uint32_t len = min(seg, pos0 + cnt - p0);
            bulk_g2s(rt + (size_t)j * TC_M + sg * seg, Rb + (size_t)j * P.N + chunk_pos_to_n(P, C, p0), len * 4, bar_r);
        }
    };

    if (threadIdx.x == 0) {
        for (int k = 0; k < 3; ++k) mbar_init(bars + k, 1);
        bulk_g2s_all(b_s, P.crt_b, (uint32_t)((size_t)nrows_b * kb), bar_b);
    }
    for (int j = threadIdx.x; j < KP; j += blockDim.x) {
        cp[j] = P.p[j];
        cc[j] = P.crt_c[j];
        ccc[j] = P.crt_cc[j];
        crc[j] = P.rcp[j];
    }
    __syncthreads();
    if (warp == 0) {
        if (use_bulk && blockIdx.x < ntiles) issue_r(blockIdx.x);
        tmem_alloc(slot, ncols);
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *slot;
    bool ok = mbar_wait_bounded(bar_b, 0);

    const uint32_t sbo = 8u * (uint32_t)kb;
    const uint32_t tlane = tmem + ((uint32_t)((warp & 3) * 32) << 16);
    uint32_t i = 0;
    for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++i) {
        const uint32_t b = tile / tiles_per_batch;
        const uint32_t pos0 = (tile - b * tiles_per_batch) * TC_M;
        const int cnt = (int)min((uint32_t)TC_M, npos - pos0);
        const bool valid = m < cnt;
        if (use_bulk) {
            ok = ok && mbar_wait_bounded(bar_r, i & 1);
        } else if (gather == CRT_GATHER_VEC) {
            // runs of 4 positions are 4 consecutive residues (cw, col0 multiples of 4): one
            // 16-byte load per prime and run, spread over all 256 threads
            const uint32_t* Rb = R + (size_t)b * K * P.N;
            for (int idx = threadIdx.x; idx < K * (TC_M / 4); idx += blockDim.x) {
                const int j = idx / (TC_M / 4), q4 = 4 * (idx % (TC_M / 4));
                uint4 v = make_uint4(0, 0, 0, 0);
                if (q4 < cnt) v = *reinterpret_cast<const uint4*>(Rb + (size_t)j * P.N + chunk_pos_to_n(P, C, pos0 + q4));
                *reinterpret_cast<uint4*>(rt + (size_t)j * TC_M + q4) = v;
            }
        } else if (hf == 0) {
            const uint32_t* Rb = R + (size_t)b * K * P.N;
            const uint32_t n = valid ? chunk_pos_to_n(P, C, pos0 + m) : 0;
            for (int j = 0; j < K; ++j) rt[(size_t)j * TC_M + m] = valid ? Rb[(size_t)j * P.N + n] : 0u;
        }
        if (__syncthreads_or(!ok)) break;

        // prologue: y_j for 4 primes -> one 16-byte core-matrix row; partial fp32 sums in 4 chains
        float s4[4] = {0.f, 0.f, 0.f, 0.f};
        const int g0 = hf ? gh : 0, g1 = hf ? kgroups : gh;
        for (int g = g0; g < g1; ++g) {
            uint32_t y[4] = {0, 0, 0, 0};
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int j = 4 * g + q;
                if (j < K) {
                    const uint32_t p = cp[j];
                    y[q] = red_once(mul_ms(rt[(size_t)j * TC_M + m], cc[j], ccc[j], p), p);
                    s4[q] = fmaf((float)y[q], crc[j], s4[q]);
                }
            }
            *reinterpret_cast<uint4*>(a_s + (size_t)(m >> 3) * sbo + (size_t)g * 128 + (m & 7) * 16) =
                make_uint4(y[0], y[1], y[2], y[3]);
        }
        spart[hf * TC_M + m] = (s4[0] + s4[1]) + (s4[2] + s4[3]);
        fence_smem_to_async();
        __syncthreads();
        const float s = spart[m] + spart[TC_M + m];
        const float vf = rintf(s);
        if (hf == 0 && valid && fabsf(s - vf) > 0.25f) flag_error(P.status, DEV_ERR_CRT_BOUND);
        const int v = min(max((int)vf, 0), K);
        if (warp == 0) {
            const uint32_t nxt = tile + gridDim.x;
            if (use_bulk && nxt < ntiles) issue_r(nxt);  // rt was consumed before the barrier
            if (lane == 0) {
                tc_fence_after();
                issue_gemm_rows(tmem, smem_addr(a_s), smem_addr(b_s), 0, min(nrows_b, 256), kb);
                if (nrows_b > 256) issue_gemm_rows(tmem + 256, smem_addr(a_s), smem_addr(b_s), 256, nrows_b - 256, kb);
                umma_commit(bar_mma);
            }
            __syncwarp();
        }
        const bool got = mbar_wait_bounded(bar_mma, i & 1);
        if (__syncthreads_or(!got)) {
            ok = false;
            break;
        }
        tc_fence_after();

        // epilogue: accumulator bytes -> limbs with carries, + T_v; half h owns limbs
        // [0, lh) or [lh, zl) of this coefficient's staging row
        uint32_t* z = z_s + (size_t)m * zs;
        const uint32_t* T = P.tneg + (size_t)v * L;
        uint64_t carry = 0;
        const int c0 = hf ? lh / 4 : 0, c1 = hf ? nl / 4 : lh / 4;
        int l = 4 * c0;
        for (int c16 = c0; c16 < c1; ++c16) {
            uint32_t r[16];
            tmem_ld16(tlane + (uint32_t)(16 * c16), r);
#pragma unroll
            for (int q = 0; q < 4; ++q, ++l) {
                const uint64_t t = carry + (uint64_t)r[4 * q] + ((uint64_t)r[4 * q + 1] << 8) +
                                   ((uint64_t)r[4 * q + 2] << 16) + ((uint64_t)r[4 * q + 3] << 24) +
                                   (l < L ? __ldg(T + l) : 0u);
                if (l < zl) z[l] = (uint32_t)t;
                carry = t >> 32;
            }
        }
        if (hf) {
            for (; l < zl; ++l) {
                z[l] = (uint32_t)carry;
                carry >>= 32;
            }
        }
        __syncthreads();
        if (hf == 0 && valid) {
            for (int k = lh; carry && k < zl; ++k) {  // half 0's carry-out into half 1's limbs
                const uint64_t t = (uint64_t)z[k] + carry;
                z[k] = (uint32_t)t;
                carry = t >> 32;
            }
            crt_reduce_mod_q(z, zl, P);
        }
        __syncthreads();
        uint32_t* o = out + ((size_t)b * npos + pos0) * L;
        for (int mm = warp; mm < cnt; mm += 8)
            for (int ll = lane; ll < L; ll += 32) o[(size_t)mm * L + ll] = z_s[(size_t)mm * zs + ll];
        tc_fence_before();
        __syncthreads();
    }
    if (!ok && threadIdx.x == 0) flag_error(P.status, DEV_ERR_WAIT);
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, ncols);
}

size_t rns_tc_smem(const DevPlan& P) {
    return (size_t)P.dec_nrows * P.dec_kbytes + (size_t)TC_M * P.dec_kbytes + 2 * (size_t)TC_M * P.L * 4 + 64;
}

size_t crt_tc_smem(const DevPlan& P) {
    return (size_t)P.crt_nrows * P.crt_kbytes + crt_a_bytes(P) + (size_t)P.K * TC_M * 4 + (size_t)P.KP * 16 +
           2 * TC_M * 4 + 64;
}

}  // namespace pm
