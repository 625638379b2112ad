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
#include "pm_async.cuh"
#include "pm_crt.cuh"
#include "pm_kernels.cuh"

namespace pm {
namespace {





__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

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

// D[tmem] (+)= A[tmem] * B[smem]^T, unsigned bytes, s32 accumulate; one thread.  A in tensor
// memory is K-major: lane m holds row m, and each 32-bit column holds 4 consecutive K bytes.
__device__ __forceinline__ void umma_u8_ts(uint32_t d_tmem, uint32_t a_tmem, uint64_t bdesc, uint32_t idesc,
                                           uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], [%1], %2, %3, p;\n\t}" ::"r"(d_tmem),
        "r"(a_tmem), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

// This warp's 32 TMEM lanes x 8 consecutive 32-bit columns from registers (asynchronous: visible
// to the tensor core after tmem_wait_st and a before-thread-sync fence).
__device__ __forceinline__ void tmem_st8(uint32_t taddr, const uint32_t (&r)[8]) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"r"(taddr), "r"(r[0]),
                 "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7])
                 : "memory");
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// 16-byte asynchronous global -> shared copy, L2 only (both addresses 16-byte aligned)
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar))
                 : "memory");
}

// 32 TMEM lanes (this warp's) x 16 consecutive 32-bit columns, without waiting: the registers
// are valid after tmem_wait_ld().  Issuing several before one wait overlaps their latency.
__device__ __forceinline__ void tmem_ld16_async(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

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
// acc: the first MMA adds to the accumulator too (a further block of the K dimension)
__device__ __forceinline__ void issue_gemm_rows(uint32_t tmem_col, uint32_t a_base, uint32_t b_base, int row0, int nn,
                                                int kbytes, bool acc = false) {
    const uint32_t sbo = 8u * (uint32_t)kbytes;
    const uint32_t idesc = idesc_u8(nn);
    for (int kk = 0; kk < kbytes / 32; ++kk) {
        const uint64_t ad = sdesc(a_base + 256u * kk, 128u, sbo);
        const uint64_t bd = sdesc(b_base + (uint32_t)(row0 >> 3) * sbo + 256u * kk, 128u, sbo);
        umma_u8(tmem_col, ad, bd, idesc, (kk > 0 || acc) ? 1u : 0u);
    }
}


// 4-byte asynchronous global -> shared copy (no register staging); cp_async_wait_all waits for
// all of this thread's.
__device__ __forceinline__ void cp_async4(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }


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
// Decomposition.  Persistent, warp-specialised, 640 threads; tiles of 128 positions over
// (batch, npos).
//   loader group (warps 0-3): thread 0 keeps a ring of raw coefficient tiles filled by
//     bulk copies (contiguous cnt*L words each, prefetched two tiles ahead); the group
//     re-lays the tile out as the K-major A operand once the previous tile's MMAs have read
//     A; thread 0 then issues the MMAs of the two prime halves -- half h once the epilogue
//     has released TMEM half h -- with one commit per half (mma_done[h]);
//   epilogue group (warps 4-19): warp w reads TMEM lane quarter w % 4, the 16-column chunks
//     congruent to (w - 4) / 4 mod 4, of prime half 0 and then of half 1, and turns four byte
//     columns into one sum, one REDC and a residue store; all 512 threads arrive on
//     acc_empty[h] once they have read half h, so the next tile's half-0 MMA runs while they
//     read half 1.
// So tile i's epilogue (the long phase) overlaps tile i+1's copy, relayout and MMAs.  Bounded
// waits with a shared abort flag as in the CRT kernel.
// smem: [B image][A tile][raw ring 2 x 128*L words][bars: B, raw 2, mma_done 2, acc_empty 2]
//       [slot][abort][{p, p^-1 mod 2^32} x KP]
// ----------------------------------------------------------------------------------------
constexpr int DEC_LOAD_THREADS = 128;
constexpr int DEC_EPI_THREADS = RNS_TC_THREADS - DEC_LOAD_THREADS;
constexpr int DEC_SUBS = DEC_EPI_THREADS / TC_M;  // epilogue warps per TMEM lane quarter
static_assert(DEC_EPI_THREADS % TC_M == 0, "whole warps per lane quarter");

__global__ void __launch_bounds__(RNS_TC_THREADS, 1) k_rns_tc(DevPlan P, const uint32_t* __restrict__ src, ChunkMap C,
                                                              uint32_t npos, uint32_t nbatch, uint32_t* __restrict__ R,
                                                              int use_bulk, int ring) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int L = P.L, kb = P.dec_kbytes, nrows_b = P.dec_nrows;
    // ring: raw tiles in flight (1 .. DEC_MAX_RING: each slot is refilled with the tile `ring`
    // tiles ahead once its tile is relaid; 1 frees shared memory for wider prime blocks)
    const int KH = dec_half_primes(P.KP);                 // primes of half 0
    const int n0 = 4 * KH, n1 = nrows_b - n0;              // MMA N of the halves
    const uint32_t col1 = dec_half1_col(n0);               // TMEM column of half 1
    unsigned char* b_s = smem_raw;
    unsigned char* a_s = b_s + (size_t)nrows_b * kb;
    uint32_t* raw_s = reinterpret_cast<uint32_t*>(a_s + (size_t)TC_M * kb);
    const size_t raw_words = (size_t)TC_M * L;
    uint64_t* bars = reinterpret_cast<uint64_t*>(raw_s + ring * raw_words);
    uint64_t *bar_b = bars, *bar_raw = bars + 1, *mma_done = bars + 1 + DEC_MAX_RING, *acc_empty = mma_done + 2;
    uint32_t* slot = reinterpret_cast<uint32_t*>(acc_empty + 2);
    volatile int* abort_f = reinterpret_cast<volatile int*>(slot + 1);
    uint2* pc_s = reinterpret_cast<uint2*>(slot + 2);  // [KP] {p, p^-1 mod 2^32}
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t ncols = tmem_cols_for((int)col1 + n1);
    const int nhalves = n1 > 0 ? 2 : 1;

    const uint32_t tiles_per_batch = (npos + TC_M - 1) / TC_M;
    const uint32_t ntiles = tiles_per_batch * nbatch;
    auto tile_src = [&](uint32_t tile, int* cnt) {
        const uint32_t b = tile / tiles_per_batch;
        const uint32_t pos0 = (tile - b * tiles_per_batch) * TC_M;
        *cnt = (int)min((uint32_t)TC_M, npos - pos0);
        return src + ((size_t)b * npos + pos0) * L;
    };

    if (threadIdx.x == 0) {
        mbar_init(bar_b, 1);
        for (int k = 0; k < DEC_MAX_RING; ++k) mbar_init(bar_raw + k, 1);
        for (int k = 0; k < 2; ++k) {
            mbar_init(mma_done + k, 1);
            mbar_init(acc_empty + k, DEC_EPI_THREADS);
        }
        *abort_f = 0;
        bulk_g2s_all(b_s, P.dec_b, (uint32_t)((size_t)nrows_b * kb), bar_b);
    }
    for (int j = threadIdx.x; j < P.KP; j += blockDim.x) pc_s[j] = make_uint2(P.p[j], P.pinv[j]);
    if (warp == 0) tmem_alloc(slot, ncols);
    // the prologue above reads only the plan's constant tables; the operand and R come after
    // the previous kernel in the stream
    pdl_wait();
    if (threadIdx.x == 0 && use_bulk)
        for (int k = 0; k < ring; ++k) {
            const uint32_t t = blockIdx.x + k * gridDim.x;
            if (t < ntiles) {
                int cnt;
                const uint32_t* s = tile_src(t, &cnt);
                bulk_g2s_all(raw_s + k * raw_words, s, (uint32_t)cnt * L * 4, bar_raw + k);
            }
        }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    pdl_trigger();  // after this block's TMEM allocation
    const uint32_t tmem = *slot;
    // thread 0's record of what is in flight, for the abort path: the last commit (barrier and
    // phase parity) and, per ring slot, a bulk copy nobody has waited for (and its parity)
    int last_commit = -1;
    uint32_t last_commit_par = 0;
    bool b_seen = false;
    uint32_t raw_pending = 0, raw_par = 0;
    if (threadIdx.x == 0 && use_bulk)
        for (int k = 0; k < ring; ++k)
            if (blockIdx.x + k * gridDim.x < ntiles) raw_pending |= 1u << k;  // parity 0

    if (threadIdx.x < DEC_LOAD_THREADS) {
        // ---------------- loader / relayout / MMA issue ----------------
        const uint32_t sbo = 8u * (uint32_t)kb;
        const int groups = kb / 16;
        uint32_t i = 0;
        for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++i) {
            if (named_sync_or(1, DEC_LOAD_THREADS, *abort_f != 0)) break;
            const int buf = (int)(i % (uint32_t)ring);  // raw ring slot
            int cnt;
            const uint32_t* s = tile_src(tile, &cnt);
            uint32_t* raw = raw_s + buf * raw_words;
            if (use_bulk) {
                if (wait_or_abort(bar_raw + buf, (i / (uint32_t)ring) & 1, abort_f, P.wait_clocks) && threadIdx.x == 0)
                    raw_pending &= ~(1u << buf);
            } else {
                for (int w = threadIdx.x; w < cnt * L; w += DEC_LOAD_THREADS) raw[w] = __ldg(s + w);
            }
            // the previous tile's MMAs must have read A (mma_done of its last half)
            if (i > 0) wait_or_abort(mma_done + (nhalves - 1), (i - 1) & 1, abort_f, P.wait_clocks);
            named_sync(1, DEC_LOAD_THREADS);  // raw tile visible to the whole group
            // re-layout: thread = row mm; 16-byte group g = limbs 4g..4g+3 (zero past L or past
            // cnt).  The full groups unpredicated and unrolled, so that several groups' loads are
            // in flight at once (a latency chain per group otherwise: this group of 4 warps
            // shares the SM with the 16 epilogue warps)
            {
                static_assert(DEC_LOAD_THREADS == TC_M, "one loader thread per tile row");
                const int mm = threadIdx.x;
                const uint32_t* row = raw + mm * L;
                unsigned char* dst = a_s + (size_t)(mm >> 3) * sbo + (mm & 7) * 16;
                const int gfull = mm < cnt ? L / 4 : 0;
                int g = 0;
#pragma unroll 4
                for (; g < gfull; ++g)
                    *reinterpret_cast<uint4*>(dst + (size_t)g * 128) =
                        make_uint4(row[4 * g], row[4 * g + 1], row[4 * g + 2], row[4 * g + 3]);
                for (; g < groups; ++g) {
                    const int l0 = 4 * g;
                    uint4 v = make_uint4(0, 0, 0, 0);
                    if (mm < cnt) {
                        v.x = l0 < L ? row[l0] : 0u;
                        v.y = l0 + 1 < L ? row[l0 + 1] : 0u;
                        v.z = l0 + 2 < L ? row[l0 + 2] : 0u;
                        v.w = l0 + 3 < L ? row[l0 + 3] : 0u;
                    }
                    *reinterpret_cast<uint4*>(dst + (size_t)g * 128) = v;
                }
            }
            fence_smem_to_async();
            named_sync(1, DEC_LOAD_THREADS);
            if (threadIdx.x == 0) {
                const uint32_t nxt = tile + (uint32_t)ring * gridDim.x;
                if (use_bulk && nxt < ntiles) {  // the ring slot was just consumed
                    int c2;
                    const uint32_t* s2 = tile_src(nxt, &c2);
                    bulk_g2s_all(raw, s2, (uint32_t)c2 * L * 4, bar_raw + buf);
                    raw_pending |= 1u << buf;
                    const uint32_t use = (i + (uint32_t)ring) / (uint32_t)ring;  // the slot's next use
                    raw_par = (raw_par & ~(1u << buf)) | ((use & 1u) << buf);
                }
                bool ok = *abort_f == 0;
                if (ok && !b_seen) ok = b_seen = wait_or_abort(bar_b, 0, abort_f, P.wait_clocks);
                for (int h = 0; h < nhalves && ok; ++h) {
                    if (i > 0) ok = wait_or_abort(acc_empty + h, (i - 1) & 1, abort_f, P.wait_clocks);
                    if (!ok) break;
                    tc_fence_after();
                    if (h == 0) issue_gemm_rows(tmem, smem_addr(a_s), smem_addr(b_s), 0, n0, kb);
                    else issue_gemm_rows(tmem + col1, smem_addr(a_s), smem_addr(b_s), n0, n1, kb);
                    umma_commit(mma_done + h);
                    last_commit = h;
                    last_commit_par = i & 1;
                }
            }
        }
    } else {
        // ---------------- epilogue ----------------
        // every byte-column sum is < 255 * 255 * kb; with kb <= 256 the two-byte partial sums
        // r0 + r1 2^8 and r2 + r3 2^8 stay below 2^32 and x is formed in 32-bit halves
        const bool small_k = kb <= 256;
        const int we = warp - DEC_LOAD_THREADS / 32;
        const int sub = we >> 2, m = (warp & 3) * 32 + lane;  // sub < DEC_SUBS: chunk residue mod DEC_SUBS
        uint32_t i = 0;
        for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++i) {
            if (named_sync_or(2, DEC_EPI_THREADS, *abort_f != 0)) break;
            int cnt;
            (void)tile_src(tile, &cnt);
            const uint32_t b = tile / tiles_per_batch;
            const uint32_t pos0 = (tile - b * tiles_per_batch) * TC_M;
            const uint32_t n = m < cnt ? chunk_pos_to_n(P, C, pos0 + m) : 0;
            uint32_t* Rb = R + (size_t)b * P.Kr * P.N + n;
            const bool st = m < cnt;
            // every epilogue warp takes half 0, then half 1: the next tile's half-0 MMA runs while
            // half 1 is read out
            for (int half = 0; half < nhalves; ++half) {
                // warp-uniform: tcgen05.ld is executed by all lanes of a warp or by none
                const bool got = __all_sync(0xffffffffu, wait_or_abort(mma_done + half, i & 1, abort_f, P.wait_clocks));
                tc_fence_after();
                const int j0 = half ? KH : 0;
                const int cols = half ? n1 : n0;
                const uint32_t tcol = tmem + (half ? col1 : 0) + ((uint32_t)((warp & 3) * 32) << 16);
                // this thread's 16-column chunks c16 = sub, sub + DEC_SUBS, ...: two TMEM loads in
                // flight per wait (c16 and c16 + DEC_SUBS), the chunks' prime constants read from
                // shared memory while they are in flight
                const int nch = cols / 16;
                for (int c16 = sub; c16 < nch && got; c16 += 2 * DEC_SUBS) {
                    uint32_t r[2][16];
                    uint2 pc[2][4];
                    const bool two = c16 + DEC_SUBS < nch;
                    // (the second chunk's constants only if it exists: past the last chunk of half 1
                    // the index would leave the table)
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        pc[0][q] = pc_s[j0 + 4 * c16 + q];
                        pc[1][q] = two ? pc_s[j0 + 4 * (c16 + DEC_SUBS) + q] : make_uint2(0u, 0u);
                    }
                    tmem_ld16_async(tcol + (uint32_t)(16 * c16), r[0]);
                    if (two) tmem_ld16_async(tcol + (uint32_t)(16 * (c16 + DEC_SUBS)), r[1]);
                    tmem_wait_ld();
#pragma unroll
                    for (int u = 0; u < 2; ++u) {
                        if (u == 1 && !two) break;
                        const int jb = j0 + 4 * (c16 + DEC_SUBS * u);
                        uint32_t* out = Rb + (size_t)jb * P.N;
#pragma unroll
                        for (int q = 0; q < 4; ++q, out += P.N) {
                            const uint32_t p = pc[u][q].x, pinv = pc[u][q].y;
                            const uint32_t* rq = &r[u][4 * q];
                            uint32_t y;
                            // residue = REDC(x) in (0, 2p), stored unreduced: it only feeds the forward transform,
                            // whose Harvey butterflies take inputs below 4p
                            if (small_k) {
                                // x = t0 + t1 2^16 (one wide multiply-add) with t0 = r0 + r1 2^8 and t1 = r2 + r3 2^8
                                // below 2^32
                                const uint32_t t0 = rq[0] + (rq[1] << 8), t1 = rq[2] + (rq[3] << 8);
                                y = redc64(((uint64_t)t1 << 16) + t0, p, pinv);
                            } else {
                                const uint64_t x = (uint64_t)rq[0] + ((uint64_t)rq[1] << 8) + ((uint64_t)rq[2] << 16) +
                                                   ((uint64_t)rq[3] << 24);
                                y = redc64(x, p, pinv);
                            }
                            if (st && jb + q < P.K) *out = y;
                        }
                    }
                }
                tc_fence_before();
                mbar_arrive(acc_empty + half);  // this thread has read TMEM half `half` of tile i
            }
        }
    }
    __syncthreads();
    if (threadIdx.x == 0 && *abort_f) {
        flag_error(P.status, DEV_ERR_WAIT);
        // copies and MMAs still in flight must land before this CTA's memory goes away
        if (!b_seen) mbar_wait_bounded(bar_b, 0, P.wait_clocks);
        for (int k = 0; k < ring; ++k)
            if (raw_pending & (1u << k)) mbar_wait_bounded(bar_raw + k, (raw_par >> k) & 1u, P.wait_clocks);
        if (last_commit >= 0) mbar_wait_bounded(mma_done + last_commit, last_commit_par, P.wait_clocks);
    }
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, ncols);
}

namespace {

constexpr int CRT_PROD_THREADS = 256;
constexpr int CRT_EPI_THREADS = 256;

struct CrtSmem {
    unsigned char* b;
    unsigned char* a;
    uint32_t* z;
    float* rcp;
    float* spart;
    uint64_t* bars;
    uint32_t* slot;
    volatile int* abort;
};

__host__ __device__ inline size_t crt_z_bytes(const DevPlan& P) { return (size_t)TC_M * crt_zstride(P.L) * 4; }

__device__ __forceinline__ CrtSmem crt_smem(unsigned char* base, const DevPlan& P) {
    CrtSmem m;
    m.b = base;
    m.a = m.b + (size_t)P.crt_nrows * P.crt_kbytes;
    m.z = reinterpret_cast<uint32_t*>(m.a + (size_t)TC_M * P.crt_kbytes);
    m.rcp = reinterpret_cast<float*>(reinterpret_cast<unsigned char*>(m.z) + crt_z_bytes(P));
    m.spart = m.rcp + P.KP;
    m.bars = reinterpret_cast<uint64_t*>(m.spart + 4 * TC_M);
    m.slot = reinterpret_cast<uint32_t*>(m.bars + 8);  // bars: B, mma_done 2, acc_empty 2, v_ready 2, ab_free
    m.abort = reinterpret_cast<volatile int*>(m.slot + 1);
    return m;
}

}  // namespace

__global__ void __launch_bounds__(CRT_TC_THREADS, 1) k_crt_tc(DevPlan P, const uint32_t* __restrict__ R, ChunkMap C,
                                                              uint32_t npos, uint32_t nbatch,
                                                              uint32_t* __restrict__ out, CrtPartial part,
                                                              CrtPrimeBlocks pbs) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const CrtSmem S = crt_smem(smem_raw, P);
    // partial modes: the block's integer (and, if add_s, its share of sum y_j / p_j) goes into
    // the per-coefficient partial buffers instead of the output; zp_s stages a tile of them
    uint32_t* zp_s = S.slot + 8;  // after [slot][abort] and padding: 32 bytes past the barriers
    const int zlt = crt_zl(P.L);
    uint64_t *bar_b = S.bars, *mma_done = S.bars + 1, *acc_empty = S.bars + 3, *v_ready = S.bars + 5;
    const int K = P.K, KP = P.KP, L = P.L, kb = P.crt_kbytes, nrows_b = P.crt_nrows;
    const int zl = crt_zl(L), zs = crt_zstride(L);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t AS = tmem_cols_for(nrows_b);     // columns per accumulator (<= 512)
    // accumulators: two (tile i in i & 1, so that its epilogue overlaps tile i + 1's MMAs), or
    // one wide one (more than 256 result bytes); buffer of tile i and how often it was used before
    const int nbuf = 2 * AS <= 512 ? 2 : 1;
    auto buf_of = [&](uint32_t t) { return nbuf == 2 ? (int)(t & 1) : 0; };
    auto use_of = [&](uint32_t t) { return nbuf == 2 ? t >> 1 : t; };
    const uint32_t tiles_per_batch = (npos + TC_M - 1) / TC_M;
    const uint32_t ntiles = tiles_per_batch * nbatch;
    const uint32_t sbo = 8u * (uint32_t)kb;

    if (threadIdx.x == 0) {
        mbar_init(bar_b, 1);
        for (int k = 0; k < 2; ++k) {
            mbar_init(mma_done + k, 1);
            mbar_init(acc_empty + k, CRT_EPI_THREADS);
            mbar_init(v_ready + k, 1);
        }
        mbar_init(S.bars + 7, 1);  // ab_free: a prime block's MMAs have read A and B
        *S.abort = 0;
        if (pbs.n == 0) bulk_g2s_all(S.b, P.crt_b, (uint32_t)((size_t)nrows_b * kb), bar_b);  // else per block
    }
    for (int j = threadIdx.x; j < KP; j += blockDim.x) S.rcp[j] = P.rcp[j];
    if (warp == 0) tmem_alloc(S.slot, nbuf * AS);
    // the prologue above reads only the plan's constant tables; R, the partial buffers and the
    // output come after the previous kernel in the stream
    pdl_wait();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    pdl_trigger();  // after this block's TMEM allocation
    const uint32_t tmem = *S.slot;
    uint32_t issued = 0;         // tiles whose MMAs thread 0 issued
    bool b_seen = pbs.n != 0;    // thread 0 has seen the (one) B image land
    uint64_t* ab_free = S.bars + 7;
    uint32_t ab_commits = 0;     // thread 0: prime-block MMA groups committed to ab_free
    bool b_pend = false;         // thread 0: a per-block B copy nobody has waited for (parity b_par)
    uint32_t b_par = 0;

    if (threadIdx.x < CRT_PROD_THREADS) {
        // ---------------- producers ----------------
        // thread (m, h): position m of the tile, groups [g0, g0 + ng) of 4 primes (half h of
        // the G = KP / 4 groups).  The residues arrive as y_j itself (times a multiple of p_j):
        // the operand whose transform the fused row pass reads was decomposed with every
        // constant times gamma_j = crt_c_j 2^-32, the CRT's per-prime factor.  They stay
        // unreduced in [0, 2p_j): with y'_j = y_j + d_j p_j, sum y'_j M/p_j and
        // v' = round(sum y'_j / p_j) both grow by (sum d_j) M, so z = sum y'_j Q_j + v' T_1 is
        // the same residue mod q, v' <= 2K - 1 still fits A's v byte (K <= 128; the prime-block
        // form gives v' a second byte), and the fractional
        // part of the sum, which the exactness check reads, is unchanged.  The padding primes
        // K..KP-1 meet zero B columns (but for A's v column, written after them) and 1/p = 0.
        // With prime blocks (pbs.n > 0) a tile runs the blocks in turn: each block's residues into
        // A and (thread 0) its B image into S.b once the previous block's MMAs have read them
        // (ab_free), its MMAs accumulating into the tile's accumulator; the sums of y'_j / p_j run
        // over all blocks.
        const int m = threadIdx.x & (TC_M - 1), h = threadIdx.x >> 7;
        const size_t N = P.N;
        const int npb = pbs.n > 0 ? pbs.n : 1;
        uint32_t i = 0, seq = 0;  // seq: prime-block MMA groups so far (npb per tile)
        for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++i) {
            if (named_sync_or(1, CRT_PROD_THREADS, *S.abort != 0)) break;
            const int b = buf_of(i);
            const uint32_t bt = tile / tiles_per_batch;
            const uint32_t pos0 = (tile - bt * tiles_per_batch) * TC_M;
            // positions past the end of the batch repeat the tile's first one: their A rows and
            // partial sums only feed accumulator rows the epilogue does not store
            const uint32_t pm = (uint32_t)m < npos - pos0 ? pos0 + m : pos0;
            const uint32_t* rtile = R + (size_t)bt * P.Kr * N + chunk_pos_to_n(P, C, pm);
            float s4[4] = {0.f, 0.f, 0.f, 0.f};
            for (int pb = 0; pb < npb; ++pb, ++seq) {
                const int j0b = pbs.n ? pbs.j0[pb] : 0, Kb = pbs.n ? pbs.k[pb] : K;
                const int KPb = pbs.n ? pbs.kp[pb] : KP, kbb = pbs.n ? pbs.kb[pb] : kb;
                const int G = KPb / 4;
                const int gh = (G + 1) / 2;
                const int g0 = h ? gh : 0, ng = (h ? G : gh) - g0;
                unsigned char* arow = S.a + (size_t)(m >> 3) * (8 * kbb) + (m & 7) * 16;
                const uint32_t* rp = rtile + (size_t)(j0b + 4 * g0) * N;
                // the previous MMA group must have read A (and B) before they are overwritten
                if (pbs.n) {
                    if (seq > 0) wait_or_abort(ab_free, (seq - 1) & 1, S.abort, P.wait_clocks);
                    if (threadIdx.x == 0) {
                        bulk_g2s_all(S.b, pbs.b[pb], (uint32_t)((size_t)nrows_b * kbb), bar_b);
                        b_pend = true;
                        b_par = seq & 1;
                    }
                } else if (i > 0) {
                    wait_or_abort(mma_done + buf_of(i - 1), use_of(i - 1) & 1, S.abort, P.wait_clocks);
                }
                // every residue of this thread's primes straight into its A row with 4-byte async
                // copies: no register staging, the whole tile in flight at once (register batches
                // held ~24 KB per SM in flight and left the loads latency-bound); prime slots past
                // the block's last prime re-read it
                // The 4 bytes of prime 4g + k land in bank (m & 7) * 4 + k of the row's core matrix
                // (rows 8 apart are 8 kb bytes apart, a multiple of 128): taken in the order
                // k = (i + (m >> 3)) & 3, the four rows of a warp that share m & 7 write different
                // banks at every copy instruction (in the plain order they all hit the same one).
                // The global side is unchanged: each copy instruction still reads 8-word runs.
                const int rot = (m >> 3) & 3;
#pragma unroll 2
                for (int gg = 0; gg < ng; ++gg) {
                    const int g = g0 + gg;
#pragma unroll
                    for (int i = 0; i < 4; ++i) {
                        const int k = (i + rot) & 3;
                        cp_async4(arow + (size_t)g * 128 + 4 * k, rp + (size_t)(min(4 * g + k, Kb - 1) - 4 * g0) * N);
                    }
                }
                cp_async_wait_all();
                // sum y'_j / p_j over this thread's primes, read back from its A row
#pragma unroll 4
                for (int gg = 0; gg < ng; ++gg) {
                    const int g = g0 + gg;
                    const uint4 x = *reinterpret_cast<const uint4*>(arow + (size_t)g * 128);
                    const float4 r = *reinterpret_cast<const float4*>(S.rcp + j0b + 4 * g);
                    s4[0] = fmaf((float)x.x, r.x, s4[0]);
                    s4[1] = fmaf((float)x.y, r.y, s4[1]);
                    s4[2] = fmaf((float)x.z, r.z, s4[2]);
                    s4[3] = fmaf((float)x.w, r.w, s4[3]);
                }
                const bool last = pb + 1 == npb;
                if (last) {
                    // the epilogue of tile i - 2 must have read partial sums [b] (it arrives on
                    // acc_empty[b] after that)
                    if (use_of(i) > 0) wait_or_abort(acc_empty + b, (use_of(i) - 1) & 1, S.abort, P.wait_clocks);
                    S.spart[(b * 2 + h) * TC_M + m] = (s4[0] + s4[1]) + (s4[2] + s4[3]);
                    if (part.mode == CRT_FULL) {
                        // v = round(sum y_j / p_j) (|x| < M/8 keeps the sum within 1/8 of an integer;
                        // further than 1/4 is a failed check) into A's v column: the MMA adds v T_1
                        named_sync(1, CRT_PROD_THREADS);
                        if (h == 0) {
                            const float sum = S.spart[(b * 2) * TC_M + m] + S.spart[(b * 2 + 1) * TC_M + m];
                            const float vf = rintf(sum);
                            if ((uint32_t)m < npos - pos0 && fabsf(sum - vf) > 0.25f)
                                flag_error(P.status, DEV_ERR_CRT_BOUND);
                            // the v column, in the last prime block's K bytes; with prime blocks
                            // (K > 128) v may pass 255 and takes a second column: v / 256 against
                            // 256 T_1
                            const int v = min(max((int)vf, 0), 2 * K - 1);
                            const int kvl = P.crt_kv - (pbs.n ? 4 * pbs.j0[npb - 1] : 0);
                            arow[(size_t)(kvl >> 4) * 128 + (kvl & 15)] = (unsigned char)(v & 255);
                            if (pbs.n) arow[(size_t)((kvl + 1) >> 4) * 128 + ((kvl + 1) & 15)] = (unsigned char)(v >> 8);
                        }
                    }
                }
                fence_smem_to_async();
                named_sync(1, CRT_PROD_THREADS);
                if (threadIdx.x == 0) {
                    bool ok = *S.abort == 0;
                    if (ok && !b_seen) ok = b_seen = wait_or_abort(bar_b, 0, S.abort, P.wait_clocks);
                    if (ok && pbs.n) {
                        ok = wait_or_abort(bar_b, seq & 1, S.abort, P.wait_clocks);
                        if (ok) b_pend = false;
                        // the block's first MMA starts the accumulator afresh: tile i - 2's
                        // epilogue must have read it
                        if (ok && pb == 0 && use_of(i) > 0)
                            ok = wait_or_abort(acc_empty + b, (use_of(i) - 1) & 1, S.abort, P.wait_clocks);
                    }
                    if (ok) {
                        tc_fence_after();
                        const uint32_t acc = tmem + (uint32_t)b * AS;
                        // MMA N is at most 256: a wider accumulator takes two row ranges of B
                        const int n_lo = min(nrows_b, 256);
                        issue_gemm_rows(acc, smem_addr(S.a), smem_addr(S.b), 0, n_lo, kbb, pb > 0);
                        if (nrows_b > 256)
                            issue_gemm_rows(acc + 256, smem_addr(S.a), smem_addr(S.b), 256, nrows_b - 256, kbb, pb > 0);
                        if (pbs.n) {
                            umma_commit(ab_free);
                            ++ab_commits;
                        }
                        if (last) {
                            umma_commit(mma_done + b);
                            ++issued;
                        }
                    }
                    if (last) mbar_arrive(v_ready + b);  // releases this tile's partial sums
                }
            }
        }
    } else {
        // ---------------- epilogue ----------------
        const int et = threadIdx.x - CRT_PROD_THREADS;
        const int hf = et >> 7, m = (warp & 3) * 32 + lane;
        const int nl = nrows_b / 4;                 // limbs covered by the accumulator columns
        const int lh = ((nl + 1) / 2 + 3) / 4 * 4;  // limbs of half 0 (multiple of 4: 16 columns)
        uint32_t* z = S.z + (size_t)m * zs;
        uint32_t i = 0;
        for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++i) {
            if (named_sync_or(2, CRT_EPI_THREADS, *S.abort != 0)) break;
            const int b = buf_of(i);
            const uint32_t bt = tile / tiles_per_batch;
            const uint32_t pos0 = (tile - bt * tiles_per_batch) * TC_M;
            const int cnt = (int)min((uint32_t)TC_M, npos - pos0);
            const bool valid = m < cnt;
            // warp-uniform: tcgen05.ld is executed by all lanes of a warp or by none
            const bool got = __all_sync(0xffffffffu, wait_or_abort(v_ready + b, use_of(i) & 1, S.abort, P.wait_clocks) &&
                                                         wait_or_abort(mma_done + b, use_of(i) & 1, S.abort, P.wait_clocks));
            tc_fence_after();
            const size_t gpos = (size_t)bt * npos + pos0;  // first coefficient of the tile in the partial buffers
            if (part.mode != CRT_FULL && part.add_s && hf == 0 && valid) {
                const float sum = S.spart[(b * 2) * TC_M + m] + S.spart[(b * 2 + 1) * TC_M + m];
                part.sp[gpos + m] = (part.mode == CRT_PARTIAL_FIRST ? 0.f : part.sp[gpos + m]) + sum;
            }
            // accumulator bytes -> limbs with carries (the MMA already added v T_1: T_1 = (-M) mod q,
            // v T_1 == T_v mod q, < 2^(W+7), and the fold below reduces it); half hf owns limbs
            // [0, lh) or [lh, zl).  Byte sums are < 2^25: r0 + r1 2^8 and r2 + r3 2^8 each take one
            // wide multiply-add.
            const uint32_t tacc = tmem + (uint32_t)b * AS + ((uint32_t)((warp & 3) * 32) << 16);
            uint64_t carry = 0;
            const int c0 = hf ? lh / 4 : 0, c1 = hf ? nl / 4 : lh / 4;
            int l = 4 * c0;
            for (int c16 = c0; c16 < c1; c16 += 2) {
                // two TMEM loads in flight per wait
                uint32_t r[2][16];
                const bool two = c16 + 1 < c1;
                if (got) {
                    tmem_ld16_async(tacc + (uint32_t)(16 * c16), r[0]);
                    if (two) tmem_ld16_async(tacc + (uint32_t)(16 * (c16 + 1)), r[1]);
                    tmem_wait_ld();
                } else {
#pragma unroll
                    for (int k = 0; k < 16; ++k) r[0][k] = r[1][k] = 0u;
                }
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                    if (u == 1 && !two) break;
#pragma unroll
                    for (int q = 0; q < 4; ++q, ++l) {
                        const uint64_t lo = (uint64_t)r[u][4 * q] + (uint64_t)r[u][4 * q + 1] * 256u;
                        const uint64_t hi = (uint64_t)r[u][4 * q + 2] + (uint64_t)r[u][4 * q + 3] * 256u;
                        const uint64_t t = carry + lo + (hi << 16);
                        if (l < zl) z[l] = (uint32_t)t;
                        carry = t >> 32;
                    }
                }
            }
            if (hf) {
                for (; l < zl; ++l) {
                    z[l] = (uint32_t)carry;
                    carry >>= 32;
                }
            }
            tc_fence_before();
            mbar_arrive(acc_empty + b);  // accumulator b and partial sums b are free again
            if (part.mode != CRT_FULL) {
                // stage the tile's partial rows (zeros for the first block), add this block's
                // integer at limb offset limb0 with one carry chain per coefficient, store back
                uint32_t* zg = part.zp + gpos * zlt;
                for (int w = et; w < TC_M * zlt; w += CRT_EPI_THREADS) {
                    const int mm = w / zlt;
                    zp_s[(size_t)mm * zs + (w - mm * zlt)] =
                        (part.mode == CRT_PARTIAL_FIRST || mm >= cnt) ? 0u : zg[w];
                }
            }
            named_sync(2, CRT_EPI_THREADS);
            if (hf == 0 && valid) {
                for (int k = lh; carry && k < zl; ++k) {  // half 0's carry-out into half 1's limbs
                    const uint64_t t = (uint64_t)z[k] + carry;
                    z[k] = (uint32_t)t;
                    carry = t >> 32;
                }
                if (part.mode == CRT_FULL) {
                    crt_reduce_mod_q(z, zl, P);
                } else {
                    uint32_t* zr = zp_s + (size_t)m * zs;
                    uint64_t c2 = 0;
                    int k = part.limb0;
                    for (int l2 = 0; l2 < zl && k < zlt; ++l2, ++k) {
                        const uint64_t t = (uint64_t)zr[k] + z[l2] + c2;
                        zr[k] = (uint32_t)t;
                        c2 = t >> 32;
                    }
                    for (; c2 && k < zlt; ++k) {
                        const uint64_t t = (uint64_t)zr[k] + c2;
                        zr[k] = (uint32_t)t;
                        c2 = t >> 32;
                    }
                }
            }
            named_sync(2, CRT_EPI_THREADS);
            if (part.mode != CRT_FULL) {
                uint32_t* zg = part.zp + gpos * zlt;
                for (int w = et; w < cnt * zlt; w += CRT_EPI_THREADS) {
                    const int mm = w / zlt;
                    zg[w] = zp_s[(size_t)mm * zs + (w - mm * zlt)];
                }
                continue;
            }
            // coalesced store of the tile's cnt x L limbs (contiguous in the output): thread et takes
            // words et, et + 256, ...; word w is limb col of row mm, tracked incrementally (each sweep
            // advances w by qL rows + rL limbs).  Consecutive threads read consecutive limbs of the
            // odd-stride rows of S.z, so the loads spread over all banks (four consecutive words per
            // thread, for 16-byte stores, put the threads 8 apart on one bank).
            uint32_t* o = out + ((size_t)bt * npos + pos0) * L;
            const int tot = cnt * L;
            const int qL = CRT_EPI_THREADS / L, rL = CRT_EPI_THREADS - qL * L;
            int mm = et / L, col = et - mm * L;
            for (int w = et; w < tot; w += CRT_EPI_THREADS) {
                o[w] = S.z[(size_t)mm * zs + col];
                mm += qL;
                col += rL;
                if (col >= L) {
                    col -= L;
                    ++mm;
                }
            }
        }
    }
    __syncthreads();
    if (threadIdx.x == 0 && *S.abort) {
        flag_error(P.status, DEV_ERR_WAIT);
        // copies and MMAs still in flight must land before this CTA's memory goes away
        if (!b_seen) mbar_wait_bounded(bar_b, 0, P.wait_clocks);
        if (issued) mbar_wait_bounded(mma_done + buf_of(issued - 1), use_of(issued - 1) & 1, P.wait_clocks);
        if (b_pend) mbar_wait_bounded(bar_b, b_par, P.wait_clocks);
    }
    // the last prime block's ab_free arrival (its MMAs are complete: the epilogue waited for them)
    if (threadIdx.x == 0 && ab_commits) mbar_wait_bounded(ab_free, (ab_commits - 1) & 1, P.wait_clocks);
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, nbuf * AS);
}

// ----------------------------------------------------------------------------------------
// CRT with the A operand in tensor memory (points of at most 128 primes and 256 result bytes,
// column chunks of at least 4 columns).  Persistent, warp-specialised, 512 threads.
//   producers (warps 0-7, two threads per position m, one per half of the A columns):
//     * the tile's residues arrive as 16-byte cp.async copies (4 positions of one prime each)
//       into a staging tile [prime][128 positions] in shared memory -- a quarter of the copy
//       instructions of per-residue copies, and decoupled from the MMA: the next tile's copies
//       are issued as soon as this tile's residues have been read out of the staging tile;
//     * each thread reads its position's residues (already y_j, unreduced in [0, 2p)) and writes
//       them straight into one of two A buffers in tensor memory with tcgen05.st: a 32-bit TMEM
//       column of A holds 4 consecutive K bytes, exactly one residue's bytes, so A's column j is
//       y_j and no byte shuffling is needed; sums y_j / p_j in fp32 meanwhile;
//     * v = round(sum) goes into column K (the B image's v column holds the bytes of T_1);
//     * thread 0 issues the MMAs (A from TMEM buffer i & 1, B from shared memory) into the one
//       accumulator once the epilogue has read the previous tile's, and commits to mma_done[i & 1].
//   epilogue (warps 8-15): as in k_crt_tc -- accumulator bytes -> limbs, fold, -q, coalesced
//     stores -- releasing the accumulator (acc_empty) as soon as its TMEM reads are done.
// TMEM: accumulator in columns [0, 256), A buffers at 256 and 384 (ncolA <= 128 columns each).
// smem: [B image][staging KP x 128 words][z 128 x zs][1/p x KP][partial sums 2 x 128]
//       [bars: B, mma_done 2, acc_empty][slot][abort]
// ----------------------------------------------------------------------------------------
namespace {
constexpr uint32_t TM_ACOL = 256;  // first A buffer's TMEM column (the second at +128)

struct CrtTmSmem {
    unsigned char* b;
    uint32_t* stg;
    uint32_t* z;
    float* rcp;
    float* spart;
    uint64_t* bars;
    uint32_t* slot;
    volatile int* abort;
};

__host__ __device__ inline size_t crt_tm_stg_words(const DevPlan& P) { return (size_t)P.KP * TC_M; }

__device__ __forceinline__ CrtTmSmem crt_tm_smem(unsigned char* base, const DevPlan& P) {
    CrtTmSmem m;
    m.b = base;
    m.stg = reinterpret_cast<uint32_t*>(m.b + (size_t)P.crt_nrows * P.crt_kbytes);
    m.z = m.stg + crt_tm_stg_words(P);
    m.rcp = reinterpret_cast<float*>(m.z + (size_t)TC_M * crt_zstride(P.L));
    m.spart = m.rcp + P.KP;
    m.bars = reinterpret_cast<uint64_t*>(m.spart + 2 * TC_M);
    m.slot = reinterpret_cast<uint32_t*>(m.bars + 4);
    m.abort = reinterpret_cast<volatile int*>(m.slot + 1);
    return m;
}
}  // namespace

__global__ void __launch_bounds__(CRT_TC_THREADS, 1) k_crt_tm(DevPlan P, const uint32_t* __restrict__ R, ChunkMap C,
                                                              uint32_t npos, uint32_t nbatch,
                                                              uint32_t* __restrict__ out) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const CrtTmSmem S = crt_tm_smem(smem_raw, P);
    uint64_t *bar_b = S.bars, *mma_done = S.bars + 1, *acc_empty = S.bars + 3;
    const int K = P.K, KP = P.KP, L = P.L, kb = P.crt_kbytes, nrows_b = P.crt_nrows;
    const int ncolA = kb / 4;                 // A columns (multiple of 8, <= 128): primes, v, padding
    const int nblk = ncolA / 8, nb0 = (nblk + 1) / 2;  // 8-column blocks; half 0 owns blocks [0, nb0)
    const int vblk = K / 8;                   // the block holding v's column K
    const int zl = crt_zl(L), zs = crt_zstride(L);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t tiles_per_batch = (npos + TC_M - 1) / TC_M;
    const uint32_t ntiles = tiles_per_batch * nbatch;
    const size_t N = P.N;

    if (threadIdx.x == 0) {
        mbar_init(bar_b, 1);
        mbar_init(mma_done, 1);
        mbar_init(mma_done + 1, 1);
        mbar_init(acc_empty, CRT_EPI_THREADS);
        *S.abort = 0;
        bulk_g2s_all(S.b, P.crt_b, (uint32_t)((size_t)nrows_b * kb), bar_b);
    }
    for (int j = threadIdx.x; j < KP; j += blockDim.x) S.rcp[j] = P.rcp[j];
    if (warp == 0) tmem_alloc(S.slot, 512);
    pdl_wait();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    pdl_trigger();  // after this block's TMEM allocation
    const uint32_t tmem = *S.slot;
    uint32_t issued = 0;   // thread 0: tiles whose MMAs it committed
    bool b_seen = false;   // thread 0: the B image has landed

    // the 16-byte copies of a tile's residues into the staging tile: copy q = (prime j, group c4
    // of 4 positions); groups past the tile's last position re-read the tile's first group
    auto issue_copies = [&](uint32_t tile) {
        const uint32_t bt = tile / tiles_per_batch;
        const uint32_t pos0 = (tile - bt * tiles_per_batch) * TC_M;
        const uint32_t* rb = R + (size_t)bt * P.Kr * N;
        for (int q = threadIdx.x; q < K * (TC_M / 4); q += CRT_PROD_THREADS) {
            const int j = q / (TC_M / 4), c4 = q - j * (TC_M / 4);
            const uint32_t pos = pos0 + 4u * (uint32_t)c4 < npos ? pos0 + 4u * (uint32_t)c4 : pos0;
            cp_async16(S.stg + (size_t)j * TC_M + 4 * c4, rb + (size_t)j * N + chunk_pos_to_n(P, C, pos));
        }
    };

    if (threadIdx.x < CRT_PROD_THREADS) {
        // ---------------- producers ----------------
        const int m = threadIdx.x & (TC_M - 1), h = threadIdx.x >> 7;
        const uint32_t lane_base = (uint32_t)((warp & 3) * 32) << 16;
        const int blk0 = h ? nb0 : 0, blk1 = h ? nblk : nb0;
        uint32_t i = 0;
        if (blockIdx.x < ntiles) issue_copies(blockIdx.x);
        for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++i) {
            if (named_sync_or(1, CRT_PROD_THREADS, *S.abort != 0)) break;
            const int b = (int)(i & 1);
            const uint32_t bt = tile / tiles_per_batch;
            const uint32_t pos0 = (tile - bt * tiles_per_batch) * TC_M;
            cp_async_wait_all();
            named_sync(1, CRT_PROD_THREADS);  // every copy of the tile has landed
            // A buffer b was last read by tile i - 2's MMAs
            if (i >= 2) wait_or_abort(mma_done + b, ((i - 2) >> 1) & 1, S.abort, P.wait_clocks);
            tc_fence_after();
            const uint32_t acol = tmem + lane_base + TM_ACOL + 128u * (uint32_t)b;
            float s = 0.f;
            for (int blk = blk0; blk < blk1; ++blk) {
                if (blk == vblk) continue;  // written with v below
                uint32_t r[8];
#pragma unroll
                for (int c = 0; c < 8; ++c) {
                    const int j = 8 * blk + c;
                    const uint32_t y = j < K ? S.stg[(size_t)j * TC_M + m] : 0u;
                    r[c] = y;
                    s = fmaf((float)y, j < KP ? S.rcp[j] : 0.f, s);
                }
                tmem_st8(acol + 8u * (uint32_t)blk, r);
            }
            // the v block's primes (before column K)
            uint32_t rv[8];
            const bool own_v = vblk >= blk0 && vblk < blk1;
            if (own_v) {
#pragma unroll
                for (int c = 0; c < 8; ++c) {
                    const int j = 8 * vblk + c;
                    const uint32_t y = j < K ? S.stg[(size_t)j * TC_M + m] : 0u;
                    rv[c] = y;
                    s = fmaf((float)y, j < K ? S.rcp[j] : 0.f, s);
                }
            }
            S.spart[h * TC_M + m] = s;
            named_sync(1, CRT_PROD_THREADS);  // staging read out, both halves' sums visible
            const uint32_t nxt = tile + gridDim.x;
            if (nxt < ntiles) issue_copies(nxt);  // overlaps this tile's MMAs and epilogue
            if (own_v) {
                // v = round(sum y'_j / p_j): |x| < M/8 keeps the sum within 1/8 of an integer, further
                // than 1/4 is a failed check; the residues' multiples of p_j make v' <= 2K - 1 < 256
                const float sum = S.spart[m] + S.spart[TC_M + m];
                const float vf = rintf(sum);
                if ((uint32_t)m < npos - pos0 && fabsf(sum - vf) > 0.25f) flag_error(P.status, DEV_ERR_CRT_BOUND);
                rv[K - 8 * vblk] = (uint32_t)min(max((int)vf, 0), 2 * K - 1);
                tmem_st8(acol + 8u * (uint32_t)vblk, rv);
            }
            tmem_wait_st();
            tc_fence_before();
            named_sync(1, CRT_PROD_THREADS);  // A buffer b complete
            if (threadIdx.x == 0) {
                bool ok = *S.abort == 0;
                if (ok && !b_seen) ok = b_seen = wait_or_abort(bar_b, 0, S.abort, P.wait_clocks);
                // the single accumulator: tile i - 1's epilogue must have read it
                if (ok && i > 0) ok = wait_or_abort(acc_empty, (i - 1) & 1, S.abort, P.wait_clocks);
                if (ok) {
                    tc_fence_after();
                    const uint32_t sbo = 8u * (uint32_t)kb;
                    const uint32_t idesc = idesc_u8(nrows_b);
                    const uint32_t a_tm = tmem + TM_ACOL + 128u * (uint32_t)b;
                    for (int kk = 0; kk < kb / 32; ++kk) {
                        const uint64_t bd = sdesc(smem_addr(S.b) + 256u * kk, 128u, sbo);
                        umma_u8_ts(tmem, a_tm + 8u * (uint32_t)kk, bd, idesc, kk > 0 ? 1u : 0u);
                    }
                    umma_commit(mma_done + b);
                    ++issued;
                }
            }
        }
        cp_async_wait_all();  // no copy of this thread may still be in flight at exit
    } else {
        // ---------------- epilogue ----------------
        const int et = threadIdx.x - CRT_PROD_THREADS;
        const int hf = et >> 7, m = (warp & 3) * 32 + lane;
        const int nl = nrows_b / 4;
        const int lh = ((nl + 1) / 2 + 3) / 4 * 4;
        uint32_t* z = S.z + (size_t)m * zs;
        uint32_t i = 0;
        for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++i) {
            if (named_sync_or(2, CRT_EPI_THREADS, *S.abort != 0)) break;
            const uint32_t bt = tile / tiles_per_batch;
            const uint32_t pos0 = (tile - bt * tiles_per_batch) * TC_M;
            const int cnt = (int)min((uint32_t)TC_M, npos - pos0);
            const bool valid = m < cnt;
            const bool got =
                __all_sync(0xffffffffu, wait_or_abort(mma_done + (i & 1), (i >> 1) & 1, S.abort, P.wait_clocks));
            tc_fence_after();
            const uint32_t tacc = tmem + ((uint32_t)((warp & 3) * 32) << 16);
            uint64_t carry = 0;
            const int c0 = hf ? lh / 4 : 0, c1 = hf ? nl / 4 : lh / 4;
            int l = 4 * c0;
            for (int c16 = c0; c16 < c1; c16 += 2) {
                uint32_t r[2][16];
                const bool two = c16 + 1 < c1;
                if (got) {
                    tmem_ld16_async(tacc + (uint32_t)(16 * c16), r[0]);
                    if (two) tmem_ld16_async(tacc + (uint32_t)(16 * (c16 + 1)), r[1]);
                    tmem_wait_ld();
                } else {
#pragma unroll
                    for (int k = 0; k < 16; ++k) r[0][k] = r[1][k] = 0u;
                }
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                    if (u == 1 && !two) break;
#pragma unroll
                    for (int q = 0; q < 4; ++q, ++l) {
                        const uint64_t lo = (uint64_t)r[u][4 * q] + (uint64_t)r[u][4 * q + 1] * 256u;
                        const uint64_t hi = (uint64_t)r[u][4 * q + 2] + (uint64_t)r[u][4 * q + 3] * 256u;
                        const uint64_t t = carry + lo + (hi << 16);
                        if (l < zl) z[l] = (uint32_t)t;
                        carry = t >> 32;
                    }
                }
            }
            if (hf) {
                for (; l < zl; ++l) {
                    z[l] = (uint32_t)carry;
                    carry >>= 32;
                }
            }
            tc_fence_before();
            mbar_arrive(acc_empty);  // the accumulator is free for the next tile's MMAs
            named_sync(2, CRT_EPI_THREADS);
            if (hf == 0 && valid) {
                for (int k = lh; carry && k < zl; ++k) {  // half 0's carry-out into half 1's limbs
                    const uint64_t t = (uint64_t)z[k] + carry;
                    z[k] = (uint32_t)t;
                    carry = t >> 32;
                }
                crt_reduce_mod_q(z, zl, P);
            }
            named_sync(2, CRT_EPI_THREADS);
            uint32_t* o = out + ((size_t)bt * npos + pos0) * L;
            const int tot = cnt * L;
            const int qL = CRT_EPI_THREADS / L, rL = CRT_EPI_THREADS - qL * L;
            int mm = et / L, col = et - mm * L;
            for (int w = et; w < tot; w += CRT_EPI_THREADS) {
                o[w] = S.z[(size_t)mm * zs + col];
                mm += qL;
                col += rL;
                if (col >= L) {
                    col -= L;
                    ++mm;
                }
            }
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (*S.abort) flag_error(P.status, DEV_ERR_WAIT);
        // copies and MMAs still in flight must land before this CTA's memory goes away
        if (!b_seen) mbar_wait_bounded(bar_b, 0, P.wait_clocks);
        if (issued) mbar_wait_bounded(mma_done + ((issued - 1) & 1), ((issued - 1) >> 1) & 1, P.wait_clocks);
    }
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, 512);
}

// Self-test of the bounded waits (pm_selftest_wait): one block waits on an mbarrier that nothing
// arrives on -- thread 0 with mbar_wait_bounded, warp 1 with wait_or_abort, whose first lane to
// time out raises the shared abort flag for the others -- and must give up after `limit` clocks
// with DEV_ERR_WAIT in *status.  Then thread 0 arrives, and every thread's wait on the
// completed phase must succeed (bit 8 of *status if one does not).  No copy or MMA is in flight
// at any point, so giving up leaves nothing behind.
__global__ void __launch_bounds__(64) k_wait_selftest(uint32_t* status, long long limit) {
    __shared__ uint64_t bar;
    __shared__ int abort_f;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        abort_f = 0;
    }
    __syncthreads();
    bool gave_up = false;
    if (threadIdx.x == 0) gave_up = !mbar_wait_bounded(&bar, 0, limit);
    else if (threadIdx.x >= 32) gave_up = !wait_or_abort(&bar, 0, &abort_f, limit);
    if (gave_up) flag_error(status, DEV_ERR_WAIT);
    __syncthreads();
    if (threadIdx.x == 0) mbar_arrive(&bar);
    __syncthreads();
    if (!mbar_wait_bounded(&bar, 0, limit + 1000000ll)) flag_error(status, 1u << 8);
}

size_t rns_tc_smem(const DevPlan& P, int ring) {
    return (size_t)P.dec_nrows * P.dec_kbytes + (size_t)TC_M * P.dec_kbytes + (size_t)ring * TC_M * P.L * 4 +
           (1 + DEC_MAX_RING + 4) * 8 + 8 +
           (size_t)P.KP * 8;
}

size_t crt_tm_smem(const DevPlan& P) {
    return (size_t)P.crt_nrows * P.crt_kbytes + crt_tm_stg_words(P) * 4 + (size_t)TC_M * crt_zstride(P.L) * 4 +
           (size_t)P.KP * 4 + 2 * TC_M * 4 + 4 * 8 + 16;
}

size_t crt_tc_smem(const DevPlan& P, bool partial) {
    return (size_t)P.crt_nrows * P.crt_kbytes + (size_t)TC_M * P.crt_kbytes + crt_z_bytes(P) + (size_t)P.KP * 4 +
           4 * TC_M * 4 + 8 * 8 + 32 + (partial ? crt_z_bytes(P) : 0);
}

// Last step of a CRT computed in blocks: per coefficient, v = round(sum of the blocks'
// partial sums of y_j / p_j) with the |x| < M/8 check, z = partial integer + v T_1, delta fold,
// - q; 128 threads, one coefficient each, rows staged through shared memory so that loads and
// stores are coalesced.
__global__ void __launch_bounds__(TC_M) k_crt_finish(DevPlan P, const uint32_t* __restrict__ zp,
                                                    const float* __restrict__ sp, uint32_t total,
                                                    uint32_t* __restrict__ out) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int L = P.L, zl = crt_zl(L), zs = crt_zstride(L);
    uint32_t* zrow = reinterpret_cast<uint32_t*>(smem_raw);  // [128][zs]
    const size_t c0 = (size_t)blockIdx.x * TC_M;
    const int cnt = (int)min((size_t)TC_M, total - c0);
    pdl_trigger();
    pdl_wait();
    for (int w = threadIdx.x; w < cnt * zl; w += TC_M) {
        const int mm = w / zl;
        zrow[(size_t)mm * zs + (w - mm * zl)] = zp[c0 * zl + w];
    }
    __syncthreads();
    const int m = threadIdx.x;
    if (m < cnt) {
        const float sum = sp[c0 + m];
        const float vf = rintf(sum);
        if (fabsf(sum - vf) > 0.25f) flag_error(P.status, DEV_ERR_CRT_BOUND);
        const uint32_t v = (uint32_t)min(max((int)vf, 0), 2 * P.K);  // residues unreduced: v < 2K
        uint32_t* z = zrow + (size_t)m * zs;
        const uint32_t* T1 = P.t1;
        uint64_t carry = 0;
        for (int l = 0; l < zl; ++l) {
            const uint64_t t = (uint64_t)z[l] + carry + (l < L ? (uint64_t)v * __ldg(T1 + l) : 0ull);
            z[l] = (uint32_t)t;
            carry = t >> 32;
        }
        crt_reduce_mod_q(z, zl, P);
    }
    __syncthreads();
    for (int w = threadIdx.x; w < cnt * L; w += TC_M) {
        const int mm = w / L;
        out[c0 * L + w] = zrow[(size_t)mm * zs + (w - mm * L)];
    }
}

}  // namespace pm
