// pm_kernels.cuh -- declarations of every kernel of the multiply and their launch helpers.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>
#include <cstdint>

#include "pm_device.cuh"

namespace pm {

[[noreturn]] void throw_cuda(cudaError_t e, const char* what);  // throws pm::CudaError

// Launches kernel f.  pdl: with programmatic stream serialization, for a kernel whose previous
// operation in the stream is a kernel: its prologue (up to pdl_wait()) may then run while that
// kernel finishes.  Every kernel of the multiply calls pdl_wait() before it reads data another
// kernel wrote or writes global memory, so the flag changes timing only.
template <class... KArgs, class... Args>
inline cudaError_t launch_kernel(void (*f)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, bool pdl,
                                 Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = pdl ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, f, static_cast<KArgs>(args)...);
}

// ---- NTT (k_ntt.cu).  The kernels are templates, so they are launched only from k_ntt.cu
// (a template kernel launched from another translation unit would bind to a host stub that
// no module registered); these host wrappers are the interface.
void launch_ntt_cols(bool inv, dim3 grid, size_t smem, cudaStream_t s, const DevPlan& P, uint32_t* R, uint32_t col0,
                     int ltc, bool pdl = false);
// mode 0: forward row stages of R; 1 (fused): forward, pointwise product with RA's finished
// transform (batch z of R pairs with transform ra_sel[z] of RA; ra_sel == nullptr: transform z),
// inverse; 2 (both): forward stages of R and of RA (after its column pass) side by side,
// pointwise, inverse stages into R
void launch_ntt_rows(int mode, dim3 grid, cudaStream_t s, const DevPlan& P, uint32_t* R, const uint32_t* RA,
                     const uint32_t* ra_sel = nullptr, bool pdl = false);
// rows of 2^w2 words per row-pass CTA (grid.x = ceil(nrows / this))
int ntt_rows_per_cta(int w2);
// line lengths 2^w1 (columns) and 2^w2 (rows) select the compile-time specialisations
void ntt_set_smem_limit(int bytes, int w1, int w2);  // max dynamic shared memory of their kernels
void ntt_probe_images(int w1, int w2);              // throws CudaError if an image cannot load
size_t ntt_cols_smem(const DevPlan& P, int ltc);

// ---- plain (CUDA-core) RNS decomposition and CRT (k_rns.cu)
// raw input tiles in flight in k_rns_tc at most (a third measured no faster at N=65536, W=1747:
// 12.5-12.9 us per operand either way)
constexpr int DEC_MAX_RING = 2;
constexpr int DEC_TM = 64;   // coefficients per decomposition block (256 threads)
constexpr int CRT_TM = 64;   // coefficients per CRT block (256 threads)
// tab_in_smem: the block stages its constant table (digits x primes) in shared memory
__global__ void k_rns_plain(DevPlan P, const uint32_t* src, ChunkMap C, uint32_t npos, uint32_t* R, int tab_in_smem);
__global__ void k_crt_plain(DevPlan P, const uint32_t* R, ChunkMap C, uint32_t npos, uint32_t* out, int tab_in_smem);
size_t rns_plain_smem(const DevPlan& P, bool tab_in_smem);
size_t crt_plain_smem(const DevPlan& P, bool tab_in_smem);

// ---- tensor-core (tcgen05 kind::i8) RNS decomposition and CRT (k_tc.cu)
constexpr int TC_M = 128;    // coefficients per UMMA tile (TMEM lanes)
// ring: raw input tiles in flight (1 or 2; rns_tc_smem counts them)
__global__ void k_rns_tc(DevPlan P, const uint32_t* src, ChunkMap C, uint32_t npos, uint32_t nbatch, uint32_t* R,
                         int use_bulk, int ring);
// A CRT over more primes than one tile holds runs as a sequence of k_crt_tc launches over
// (prime block, result-byte block) pairs that accumulate exact per-coefficient partial integers
// (zl = L + 3 limbs each) and partial sums of y_j / p_j, then k_crt_finish.
enum : int { CRT_FULL = 0, CRT_PARTIAL_FIRST = 1, CRT_PARTIAL_ADD = 2 };
struct CrtPartial {
    uint32_t* zp;  // [coefficients][L + 3] partial integers (coefficient = batch * npos + position)
    float* sp;     // [coefficients] partial sums of y_j / p_j
    int mode;      // CRT_FULL: the whole CRT, result to `out`
    int limb0;     // the block's first result byte / 4
    int add_s;     // whether this launch adds its sum of y_j / p_j (once per prime block)
};
__global__ void k_crt_tc(DevPlan P, const uint32_t* R, ChunkMap C, uint32_t npos, uint32_t nbatch, uint32_t* out,
                         CrtPartial part, CrtPrimeBlocks pbs);
__global__ void k_crt_finish(DevPlan P, const uint32_t* zp, const float* sp, uint32_t total, uint32_t* out);
// The single-tile CRT with its A operand in tensor memory (k_tc.cu): points with KP <= 128 and
// crt_nrows <= 256, column chunks of at least 4 columns starting on a multiple of 4.
__global__ void k_crt_tm(DevPlan P, const uint32_t* R, ChunkMap C, uint32_t npos, uint32_t nbatch, uint32_t* out);
size_t crt_tm_smem(const DevPlan& P);
// 64-bit digests of `count` arrays of `words` words (k_digest.cu): out_dev[count] (device) is
// cleared and filled on stream s; digest_host computes the same value on the host
void launch_digest(const uint32_t* x, uint64_t words, uint32_t count, uint64_t* out_dev, cudaStream_t s);
uint64_t digest_host(const uint32_t* x, uint64_t words);

// the bounded waits made to run out (pm_selftest_wait): 64 threads, one block
__global__ void k_wait_selftest(uint32_t* status, long long limit);
constexpr long long kWaitClocks = 2000000000ll;  // DevPlan::wait_clocks
constexpr int RNS_TC_THREADS = 640;  // 4 loader warps + 16 epilogue warps (4 lane quarters x 2 prime halves x 2 column sets)
constexpr int CRT_TC_THREADS = 512;  // 256 producers + 256 epilogue threads, two per coefficient each
size_t rns_tc_smem(const DevPlan& P, int ring = 2);
size_t crt_tc_smem(const DevPlan& P, bool partial = false);
// TMEM columns to allocate: a power of two >= max(32, n)
__host__ __device__ inline uint32_t tmem_cols_for(int n) {
    uint32_t c = 32;
    while (c < (uint32_t)n) c <<= 1;
    return c;
}

// Decomposition MMA split: primes [0, KH) -> TMEM columns [0, 4KH), the rest from column
// dec_half1_col; each half is one commit, so the epilogue of half 0 overlaps half 1's MMA.
__host__ __device__ inline int dec_half_primes(int KP) {
    const int h = (KP + 1) / 2;
    return (h + 3) / 4 * 4;
}
__host__ __device__ inline uint32_t dec_half1_col(int n0) { return (uint32_t)((n0 + 31) / 32 * 32); }

// words of one CRT staging row: z needs L + 3 limbs (value < 2^(W + 64)); odd stride
__host__ __device__ inline int crt_zl(int L) { return L + 3; }
__host__ __device__ inline int crt_zstride(int L) { return crt_zl(L) | 1; }


}  // namespace pm
