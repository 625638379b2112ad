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

// Issues D[:, 0:n_rows) = A(128 x kbytes) * B(n_rows x kbytes)^T, N split into <= 256 chunks.
__device__ __forceinline__ void issue_gemm(uint32_t tmem, uint32_t a_base, uint32_t b_base, int n_rows, int kbytes) {
    const uint32_t sbo = 8u * (uint32_t)kbytes;
    for (int n0 = 0; n0 < n_rows; n0 += 256) {
        const int nn = min(256, n_rows - n0);
        const uint32_t idesc = idesc_u8(nn);
        for (int kk = 0; kk < kbytes / 32; ++kk) {
            const uint64_t ad = sdesc(a_base + 256u * kk, 128u, sbo);
            const uint64_t bd = sdesc(b_base + (uint32_t)(n0 >> 3) * sbo + 256u * kk, 128u, sbo);
            umma_u8(tmem + (uint32_t)n0, ad, bd, idesc, kk > 0 ? 1u : 0u);
        }
    }
}

__device__ __forceinline__ void copy_to_smem(void* dst, const void* src, size_t bytes) {
    uint4* d = reinterpret_cast<uint4*>(dst);
    const uint4* s = reinterpret_cast<const uint4*>(src);
    for (size_t i = threadIdx.x; i < bytes / 16; i += blockDim.x) d[i] = __ldg(s + i);
}

}  // namespace

// ----------------------------------------------------------------------------------------
// Decomposition.  Persistent: grid <= #SMs, tiles of 128 positions over (batch, npos).
// smem: [B image][A tile 128 x kb][raw tile 128 x L words][mbar][tmem slot]
// ----------------------------------------------------------------------------------------
__global__ void __launch_bounds__(128, 1) k_rns_tc(DevPlan P, const uint32_t* __restrict__ src, ChunkMap C,
                                                   uint32_t npos, uint32_t nbatch, uint32_t* __restrict__ R) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int L = P.L, kb = P.dec_kbytes, nrows_b = P.dec_nrows;
    unsigned char* b_s = smem_raw;
    unsigned char* a_s = b_s + (size_t)nrows_b * kb;
    uint32_t* raw_s = reinterpret_cast<uint32_t*>(a_s + (size_t)TC_M * kb);
    uint64_t* bar = reinterpret_cast<uint64_t*>(raw_s + (size_t)TC_M * L + 4);
    uint32_t* slot = reinterpret_cast<uint32_t*>(bar + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t ncols = tmem_cols_for(nrows_b);

    copy_to_smem(b_s, P.dec_b, (size_t)nrows_b * kb);
    if (threadIdx.x == 0) mbar_init(bar, 1);
    if (warp == 0) tmem_alloc(slot, ncols);
    fence_smem_to_async();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *slot;

    const uint32_t tiles_per_batch = (npos + TC_M - 1) / TC_M;
    const uint32_t ntiles = tiles_per_batch * nbatch;
    const uint32_t sbo = 8u * (uint32_t)kb;
    const int groups = kb / 16;  // 16-byte core-matrix columns per row
    uint32_t phase = 0;
    for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const uint32_t b = tile / tiles_per_batch;
        const uint32_t pos0 = (tile - b * tiles_per_batch) * TC_M;
        const int cnt = (int)min((uint32_t)TC_M, npos - pos0);
        const uint32_t* s = src + ((size_t)b * npos + pos0) * L;
        // raw tile (contiguous cnt*L words), coalesced
        for (int i = threadIdx.x; i < cnt * L; i += blockDim.x) raw_s[i] = __ldg(s + i);
        __syncthreads();
        // re-layout: row m, 16-byte group g = limbs 4g..4g+3 (zero past L or past cnt)
        for (int i = threadIdx.x; i < TC_M * groups; i += blockDim.x) {
            const int m = i & (TC_M - 1), g = i >> 7;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (m < cnt) {
                const uint32_t* row = raw_s + m * L;
                const int l0 = 4 * g;
                v.x = l0 < L ? row[l0] : 0u;
                v.y = l0 + 1 < L ? row[l0 + 1] : 0u;
                v.z = l0 + 2 < L ? row[l0 + 2] : 0u;
                v.w = l0 + 3 < L ? row[l0 + 3] : 0u;
            }
            *reinterpret_cast<uint4*>(a_s + (size_t)(m >> 3) * sbo + (size_t)g * 128 + (m & 7) * 16) = v;
        }
        fence_smem_to_async();
        __syncthreads();
        if (threadIdx.x == 0) {
            tc_fence_after();
            issue_gemm(tmem, smem_addr(a_s), smem_addr(b_s), nrows_b, kb);
            umma_commit(bar);
        }
        const bool ok = mbar_wait_bounded(bar, phase);
        phase ^= 1u;
        if (__syncthreads_or(!ok)) {
            if (threadIdx.x == 0) flag_error(P.status, DEV_ERR_WAIT);
            break;
        }
        tc_fence_after();

        // epilogue: thread <-> row m = 32 warp + lane; 16 columns = 4 primes per TMEM load
        const int m = warp * 32 + lane;
        const uint32_t n = m < cnt ? chunk_pos_to_n(P, C, pos0 + m) : 0;
        uint32_t* Rb = R + (size_t)b * P.K * P.N + n;
        for (int c16 = 0; c16 < nrows_b / 16; ++c16) {
            uint32_t r[16];
            tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(16 * c16), r);
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int j = 4 * c16 + i;
                if (j < P.K && m < cnt) {
                    const uint64_t x = (uint64_t)r[4 * i] + ((uint64_t)r[4 * i + 1] << 8) +
                                       ((uint64_t)r[4 * i + 2] << 16) + ((uint64_t)r[4 * i + 3] << 24);
                    const uint32_t p = P.p[j];
                    Rb[(size_t)j * P.N] = red_once(redc64(x, p, P.pinv[j]), p);
                }
            }
        }
        tc_fence_before();
        __syncthreads();
    }
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, ncols);
}

// ----------------------------------------------------------------------------------------
// CRT.  Persistent like the decomposition.
// smem: [B image][A tile 128 x kb (aliased by the z staging rows after the MMA)][mbar][slot]
// ----------------------------------------------------------------------------------------
__global__ void __launch_bounds__(128, 1) k_crt_tc(DevPlan P, const uint32_t* __restrict__ R, ChunkMap C,
                                                   uint32_t npos, uint32_t nbatch, uint32_t* __restrict__ out) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int K = P.K, L = P.L, kb = P.crt_kbytes, nrows_b = P.crt_nrows;
    const int zl = crt_zl(L), zs = crt_zstride(L);
    unsigned char* b_s = smem_raw;
    unsigned char* a_s = b_s + (size_t)nrows_b * kb;
    const size_t a_mma = (size_t)TC_M * kb, a_z = (size_t)TC_M * zs * 4;
    const size_t a_bytes = a_mma > a_z ? a_mma : a_z;
    uint32_t* z_s = reinterpret_cast<uint32_t*>(a_s);  // after the MMA has consumed A
    uint64_t* bar = reinterpret_cast<uint64_t*>(a_s + a_bytes);
    uint32_t* slot = reinterpret_cast<uint32_t*>(bar + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t ncols = tmem_cols_for(nrows_b);

    copy_to_smem(b_s, P.crt_b, (size_t)nrows_b * kb);
    if (threadIdx.x == 0) mbar_init(bar, 1);
    if (warp == 0) tmem_alloc(slot, ncols);
    fence_smem_to_async();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *slot;

    const uint32_t tiles_per_batch = (npos + TC_M - 1) / TC_M;
    const uint32_t ntiles = tiles_per_batch * nbatch;
    const uint32_t sbo = 8u * (uint32_t)kb;
    const int kgroups = kb / 16;
    const int m = warp * 32 + lane;
    uint32_t phase = 0;
    for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const uint32_t b = tile / tiles_per_batch;
        const uint32_t pos0 = (tile - b * tiles_per_batch) * TC_M;
        const int cnt = (int)min((uint32_t)TC_M, npos - pos0);
        const bool valid = m < cnt;
        const uint32_t n = valid ? chunk_pos_to_n(P, C, pos0 + m) : 0;
        const uint32_t* Rb = R + (size_t)b * K * P.N + n;

        // prologue: y_j for 4 primes at a time -> one 16-byte core-matrix row; fp32 estimate
        float s = 0.f;
        for (int g = 0; g < kgroups; ++g) {
            uint32_t y[4] = {0, 0, 0, 0};
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int j = 4 * g + i;
                if (j < K && valid) {
                    const uint32_t p = P.p[j];
                    y[i] = red_once(mul_ms(Rb[(size_t)j * P.N], P.crt_c[j], P.crt_cc[j], p), p);
                    s = fmaf((float)y[i], P.rcp[j], s);
                }
            }
            *reinterpret_cast<uint4*>(a_s + (size_t)(m >> 3) * sbo + (size_t)g * 128 + (m & 7) * 16) =
                make_uint4(y[0], y[1], y[2], y[3]);
        }
        const float vf = rintf(s);
        if (valid && fabsf(s - vf) > 0.25f) flag_error(P.status, DEV_ERR_CRT_BOUND);
        const int v = min(max((int)vf, 0), K);

        fence_smem_to_async();
        __syncthreads();
        if (threadIdx.x == 0) {
            tc_fence_after();
            issue_gemm(tmem, smem_addr(a_s), smem_addr(b_s), nrows_b, kb);
            umma_commit(bar);
        }
        const bool ok = mbar_wait_bounded(bar, phase);
        phase ^= 1u;
        if (__syncthreads_or(!ok)) {
            if (threadIdx.x == 0) flag_error(P.status, DEV_ERR_WAIT);
            break;
        }
        tc_fence_after();

        // epilogue: bytes -> limbs with carries, + T_v, into this thread's staging row
        uint32_t* z = z_s + (size_t)m * zs;
        const uint32_t* T = P.tneg + (size_t)v * L;
        uint64_t carry = 0;
        int l = 0;
        for (int c16 = 0; c16 < nrows_b / 16; ++c16) {
            uint32_t r[16];
            tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(16 * c16), r);
#pragma unroll
            for (int i = 0; i < 4; ++i, ++l) {
                const uint64_t t = carry + (uint64_t)r[4 * i] + ((uint64_t)r[4 * i + 1] << 8) +
                                   ((uint64_t)r[4 * i + 2] << 16) + ((uint64_t)r[4 * i + 3] << 24) +
                                   (l < L ? __ldg(T + l) : 0u);
                if (l < zl) z[l] = (uint32_t)t;
                carry = t >> 32;
            }
        }
        for (; l < zl; ++l) {
            z[l] = (uint32_t)carry;
            carry >>= 32;
        }
        if (valid) crt_reduce_mod_q(z, zl, P);
        __syncthreads();
        uint32_t* o = out + ((size_t)b * npos + pos0) * L;
        for (int i = threadIdx.x; i < cnt * L; i += blockDim.x) {
            const int mm = i / L, ll = i - mm * L;
            o[i] = z_s[(size_t)mm * zs + ll];
        }
        tc_fence_before();
        __syncthreads();
    }
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, ncols);
}

size_t rns_tc_smem(const DevPlan& P) {
    return (size_t)P.dec_nrows * P.dec_kbytes + (size_t)TC_M * P.dec_kbytes + ((size_t)TC_M * P.L + 4) * 4 + 16;
}

size_t crt_tc_smem(const DevPlan& P) {
    const size_t a_bytes = std::max<size_t>((size_t)TC_M * P.crt_kbytes, (size_t)TC_M * crt_zstride(P.L) * 4);
    return (size_t)P.crt_nrows * P.crt_kbytes + a_bytes + 16;
}

}  // namespace pm
