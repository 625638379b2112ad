// pm_engine.cu -- the multiply's runtime: device tables, scratch, launches, and the host
// pipeline behind the reference-facing call.
//
// Device-resident multiply (run_device), per group of G multiplies sharing one launch each:
//   decompose(a) -> column pass fwd(a) -> row pass fwd(a)
//   decompose(b) -> column pass fwd(b) -> fused row pass (fwd b, * a, inv)
//   column pass inv(b) -> CRT -> c
// Host-operand multiply (run_host), the reference's chunked PCIe pipeline (solve.cu:1022-1243)
// rebuilt around the same kernels: operands go in column chunks (the first NTT pass only
// mixes coefficients within a column), each chunk gathered into pinned memory by the host
// pool while the previous chunk's H2D copy, decomposition and column pass run; a's row pass
// runs while b is still arriving; after b, the fused row pass; then per output column chunk
// the inverse column pass, CRT and a D2H copy, each finished chunk scattered into the
// caller's buffer while the next one is in flight.
#include "pm_engine.h"

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>

#include "pm_kernels.cuh"

// POLYMULT_CRT_TM: the single-tile CRT runs k_crt_tm (A operand in tensor memory) where it applies
#ifndef POLYMULT_CRT_TM
#define POLYMULT_CRT_TM 1
#endif

#if defined(__x86_64__)
#include <immintrin.h>
#endif
#include <sched.h>

namespace pm {

void cuda_check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw_cuda(e, what);
}

void throw_cuda(cudaError_t e, const char* what) { throw CudaError(std::string(what) + ": " + cudaGetErrorString(e)); }

namespace {

int usable_cpus() {
    cpu_set_t set;
    if (sched_getaffinity(0, sizeof(set), &set) == 0) return CPU_COUNT(&set);
    return (int)std::max(1u, std::thread::hardware_concurrency());
}

// pageable <-> pinned copy with non-temporal stores where aligned and `nt` (the destination
// is not read back by this thread, so skipping its read-for-ownership saves host bandwidth);
// with nt = false, ordinary stores leave the staged chunk in the last-level cache, where the
// copy engine's read may find it
#if defined(__x86_64__)
// 32-byte non-temporal stores (AVX2), four loads in flight per iteration
__attribute__((target("avx2"))) void stream_copy_avx2(void* dst, const void* src, size_t bytes) {
    __m256i* d = static_cast<__m256i*>(dst);
    const __m256i* s = static_cast<const __m256i*>(src);
    const size_t n = bytes / 32;
    size_t i = 0;
    for (; i + 4 <= n; i += 4) {
        const __m256i v0 = _mm256_loadu_si256(s + i), v1 = _mm256_loadu_si256(s + i + 1);
        const __m256i v2 = _mm256_loadu_si256(s + i + 2), v3 = _mm256_loadu_si256(s + i + 3);
        _mm256_stream_si256(d + i, v0);
        _mm256_stream_si256(d + i + 1, v1);
        _mm256_stream_si256(d + i + 2, v2);
        _mm256_stream_si256(d + i + 3, v3);
    }
    for (; i < n; ++i) _mm256_stream_si256(d + i, _mm256_loadu_si256(s + i));
    _mm_sfence();
}
const bool g_has_avx2 = __builtin_cpu_supports("avx2");
#endif

void stream_copy(void* dst, const void* src, size_t bytes, bool nt = true) {
#if defined(__x86_64__)
    if (nt && g_has_avx2 && ((uintptr_t)dst & 31) == 0 && (bytes & 31) == 0) {
        stream_copy_avx2(dst, src, bytes);
        return;
    }
    if (nt && ((uintptr_t)dst & 15) == 0 && (bytes & 15) == 0) {
        __m128i* d = static_cast<__m128i*>(dst);
        const __m128i* s = static_cast<const __m128i*>(src);
        const size_t n = bytes / 16;
        for (size_t i = 0; i < n; ++i) _mm_stream_si128(d + i, _mm_loadu_si128(s + i));
        _mm_sfence();
        return;
    }
#endif
    std::memcpy(dst, src, bytes);
}

// `n` column chunks covering [0, ncols): power-of-two widths, narrow ones at the ends named
// by `head` / `tail` (fractions 1/d of ncols) so that the pipeline fills and drains sooner.
std::vector<Chunk> make_chunks(uint32_t ncols, std::initializer_list<uint32_t> head, uint32_t body,
                               std::initializer_list<uint32_t> tail) {
    std::vector<uint32_t> w, t;
    uint32_t rem = ncols;
    for (uint32_t d : head) {
        const uint32_t x = std::min(rem, std::max(1u, ncols / d));
        if (x && rem > x) {
            w.push_back(x);
            rem -= x;
        }
    }
    uint32_t tsum = 0;
    for (uint32_t d : tail) {
        const uint32_t x = std::max(1u, ncols / d);
        if (tsum + x < rem) {
            t.push_back(x);
            tsum += x;
        }
    }
    const uint32_t bw = std::max(1u, ncols / body);
    while (rem > tsum) {
        uint32_t x = std::min(bw, rem - tsum);
        // keep widths powers of two (chunk_pos_to_n divides by cw with a shift)
        while (x & (x - 1)) x &= x - 1;
        w.push_back(x);
        rem -= x;
    }
    w.insert(w.end(), t.begin(), t.end());
    std::vector<Chunk> out;
    uint32_t col = 0;
    for (uint32_t x : w) {
        out.push_back({col, x});
        col += x;
    }
    return out;
}

int ilog2(uint32_t x) {
    int l = 0;
    while ((1u << l) < x) ++l;
    return l;
}

template <class T>
T* dev_alloc(std::vector<void*>& keep, size_t count, size_t* total) {
    T* d = nullptr;
    cuda_check(cudaMalloc(&d, std::max<size_t>(1, count) * sizeof(T)), "cudaMalloc");
    keep.push_back(d);
    if (total) *total += count * sizeof(T);
    return d;
}

template <class T>
T* dev_upload(std::vector<void*>& keep, const std::vector<T>& v, size_t* total) {
    T* d = dev_alloc<T>(keep, v.size(), total);
    if (!v.empty()) cuda_check(cudaMemcpy(d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice), "upload");
    return d;
}

}  // namespace

// ---------------------------------------------------------------------------------------
// construction
// ---------------------------------------------------------------------------------------
Engine::Engine(uint32_t N, uint32_t W, uint32_t L, const uint32_t* q, int gemm_request, int device,
               const EngineOptions& opt)
    : plan_(make_plan(N, W, L, q)), device_(device) {
    if (opt.w1 >= 0) set_split(plan_, opt.w1);
    int ndev = 0;
    cuda_check(cudaGetDeviceCount(&ndev), "no CUDA device");
    if (device < 0 || device >= ndev) throw CudaError("device index out of range");
    cuda_check(cudaSetDevice(device), "cudaSetDevice");
    cudaDeviceProp prop{};
    cuda_check(cudaGetDeviceProperties(&prop, device), "cudaGetDeviceProperties");
    if (prop.major != 10) throw Unsupported("this library is built for sm_100a (B200); device is sm_" +
                                            std::to_string(prop.major * 10 + prop.minor));
    num_sms_ = prop.multiProcessorCount;
    smem_optin_ = prop.sharedMemPerBlockOptin;
    try {
        upload_tables();
        setup_launch_shapes();
        // The tensor-core decomposition runs in prime blocks of at most 128 primes (TMEM holds
        // 4 byte columns per prime) whose B image fits shared memory; the tensor-core CRT needs
        // every prime in one tile (K <= 128) and a result of at most 256 bytes.  Points beyond
        // the CRT's reach (K > 128: W above about 1900 bits) take the mixed form: tensor-core
        // decomposition, CUDA-core CRT.
        const bool dec_fits = make_dec_blocks();
        const bool crt_fits = crt_tc_smem(dp_) <= smem_optin_ && plan_.KP <= 128 && dp_.crt_nrows <= 256;
        const bool crt_blocks = !crt_fits && dec_fits && make_crt_blocks();
        if (crt_blocks) make_crt_wide();
        if (gemm_request == GEMM_TENSOR && !(dec_fits && (crt_fits || crt_blocks)))
            throw Unsupported("tensor-core GEMM form does not cover this point (shared memory / TMEM)");
        if (gemm_request == GEMM_MIXED && !dec_fits)
            throw Unsupported("tensor-core decomposition does not cover this point (shared memory)");
        dec_tc_ = gemm_request != GEMM_PLAIN && dec_fits;
        crt_tc_ = dec_tc_ && crt_fits && gemm_request != GEMM_MIXED;
        crt_blocked_ = dec_tc_ && !crt_fits && crt_blocks && gemm_request != GEMM_MIXED;
        form_ = (crt_tc_ || crt_blocked_) ? GEMM_TENSOR : dec_tc_ ? GEMM_MIXED : GEMM_PLAIN;
        if (dec_tc_) {
            smem_dec_ = 0;
            for (const DecBlock& b : dec_blocks_) smem_dec_ = std::max(smem_dec_, b.smem);
        }
        if (crt_tc_) smem_crt_ = crt_tc_smem(dp_);
        // the single-tile CRT with its A operand in tensor memory where it applies (POLYMULT_CRT_TM)
        crt_tm_ok_ = crt_tc_ && plan_.KP <= 128 && dp_.crt_nrows <= 256 && dp_.crt_kbytes <= 512 &&
                     crt_tm_smem(dp_) <= smem_optin_;
        crt_tm_ = POLYMULT_CRT_TM && crt_tm_ok_;
        // multiplies per launch group of run_device: up to POLYMULT_GROUP_WORDS residue words
        // per operand (default 256 Mi: 32 multiplies at N = 65536, W = 1747, 2 GB of residue
        // scratch), at most 256.  Measured there: 8 per group 9081 mults/s, 16 9435, 32 9646 --
        // every kernel's fixed costs (B images, twiddle reads, ramp, last partial wave)
        // amortise over the group.
        size_t group_words = size_t(256) << 20;
        if (const char* e = std::getenv("POLYMULT_GROUP_WORDS")) group_words = std::max<size_t>(1, std::strtoull(e, nullptr, 10));
        const size_t per_mult = (size_t)plan_.K * plan_.N;
        group_cap_ = (uint32_t)std::max<size_t>(1, std::min<size_t>(256, group_words / std::max<size_t>(1, per_mult)));
        if (crt_blocked_) reserve_crt_partials((size_t)group_cap_ * plan_.N);
        if (opt.host_pipeline) {
            ensure_scratch(1);
            setup_host_pipeline();
        }
    } catch (...) {
        for (void* d : dev_allocs_) cudaFree(d);
        dev_allocs_.clear();
        throw;
    }
}

Engine::~Engine() {
    cudaSetDevice(device_);
    cudaDeviceSynchronize();
    pool_.reset();
    for (auto e : ev_in_) cudaEventDestroy(e);
    for (auto e : ev_done_in_) cudaEventDestroy(e);
    for (auto e : ev_crt_) cudaEventDestroy(e);
    for (auto e : ev_out_) cudaEventDestroy(e);
    for (auto e : trace_ev_) cudaEventDestroy(e);
    if (ev_fused_) cudaEventDestroy(ev_fused_);
    for (auto s : s_comp_)
        if (s) cudaStreamDestroy(s);
    if (s_h2d_) cudaStreamDestroy(s_h2d_);
    if (s_d2h_) cudaStreamDestroy(s_d2h_);
    for (void* d : dev_allocs_) cudaFree(d);
    if (d_ra_) cudaFree(d_ra_);
    if (d_rb_) cudaFree(d_rb_);
    if (d_zp_) cudaFree(d_zp_);
    if (d_sp_) cudaFree(d_sp_);
    for (auto h : h_in_)
        if (h) cudaFreeHost(h);
    if (h_out_) cudaFreeHost(h_out_);
    if (h_status_) cudaFreeHost(h_status_);
}

void Engine::upload_tables() {
    const Plan& P = plan_;
    DevPlan& d = dp_;
    d.N = P.N;
    d.nrows = P.nrows;
    d.ncols = P.ncols;
    d.logN = P.logN;
    d.w1 = P.w1;
    d.w2 = P.w2;
    d.K = P.K;
    d.Kr = P.K;
    d.KP = P.KP;
    d.L = (int)P.L;
    d.W = (int)P.W;
    d.D = P.D;
    d.DP = P.DP;
    d.fold_count = P.fold_count;
    d.delta = P.delta;
    size_t* tb = &table_bytes_;
    d.p = dev_upload(dev_allocs_, P.p, tb);
    d.pinv = dev_upload(dev_allocs_, P.pinv, tb);
    d.crt_c = dev_upload(dev_allocs_, P.crt_c, tb);
    d.crt_cc = dev_upload(dev_allocs_, P.crt_cc, tb);
    d.rcp = dev_upload(dev_allocs_, P.rcp, tb);
    d.tw = reinterpret_cast<const uint2*>(dev_upload(dev_allocs_, P.tw, tb));
    d.dec24 = dev_upload(dev_allocs_, P.dec24, tb);
    d.crt24 = dev_upload(dev_allocs_, P.crt24, tb);
    d.t1 = dev_upload(dev_allocs_, P.t1, tb);
    d.q = dev_upload(dev_allocs_, P.q, tb);
    d.dec_b = dev_upload(dev_allocs_, P.dec_b, tb);
    d.dec_b_ra = dev_upload(dev_allocs_, P.dec_b_ra, tb);
    d.crt_b = dev_upload(dev_allocs_, P.crt_b, tb);
    d.crt_kv = P.crt_kv;
    d.dec_nrows = P.dec_gemm.n_rows;
    d.dec_kbytes = P.dec_gemm.k_bytes;
    d.crt_nrows = P.crt_gemm.n_rows;
    d.crt_kbytes = P.crt_gemm.k_bytes;
    uint32_t* st = dev_alloc<uint32_t>(dev_allocs_, 1, nullptr);
    cuda_check(cudaMemset(st, 0, 4), "memset status");
    d.status = st;
    d.wait_clocks = kWaitClocks;
    // POLYMULT_COL_TMA=0: the column passes keep the one-tile-per-CTA kernels
    d.col_tma = !(std::getenv("POLYMULT_COL_TMA") && std::getenv("POLYMULT_COL_TMA")[0] == '0');
}

void Engine::set_status_for_test(uint32_t bits) {
    cuda_check(cudaSetDevice(device_), "cudaSetDevice");
    cuda_check(cudaDeviceSynchronize(), "device synchronize");
    cuda_check(cudaMemcpy(dp_.status, &bits, 4, cudaMemcpyHostToDevice), "status write");
}

uint32_t wait_selftest(int device, long long limit) {
    cuda_check(cudaSetDevice(device), "cudaSetDevice");
    uint32_t* st = nullptr;
    cuda_check(cudaMalloc(&st, 4), "cudaMalloc");
    uint32_t out = 0;
    cudaError_t e = cudaMemset(st, 0, 4);
    if (e == cudaSuccess) e = launch_kernel(k_wait_selftest, dim3(1), dim3(64), 0, nullptr, false, st, limit);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(&out, st, 4, cudaMemcpyDeviceToHost);
    cudaFree(st);
    if (e != cudaSuccess) throw_cuda(e, "wait self-test");
    return out;
}

void Engine::setup_launch_shapes() {
    rpb_ = ntt_rows_per_cta(plan_.w2);
    // the widest tile launch_cols uses: 64 columns for lines of 128 or 256 rows, else 32
    const uint32_t widest = plan_.w1 >= 7 && plan_.w1 <= 8 ? 64 : 32;
    smem_cols_ = std::max(ntt_cols_smem(dp_, ilog2(std::min<uint32_t>(32, plan_.ncols))),
                          ntt_cols_smem(dp_, ilog2(std::min<uint32_t>(widest, plan_.ncols))));
    if (smem_cols_ > smem_optin_) throw Unsupported("NTT tile exceeds shared memory");
    // the plain kernels stage their constant tables in shared memory while two blocks still fit
    // an SM (up to W = 1747 or so); beyond that they read them through L1
    dec_tab_smem_ = rns_plain_smem(dp_, true) <= 110 * 1024;
    smem_dec_ = rns_plain_smem(dp_, dec_tab_smem_);
    crt_tab_smem_ = crt_plain_smem(dp_, true) <= 110 * 1024;
    smem_crt_ = crt_plain_smem(dp_, crt_tab_smem_);
    if (smem_dec_ > smem_optin_ || smem_crt_ > smem_optin_) throw Unsupported("plain GEMM tile exceeds shared memory");
    // Every kernel may use up to the device's opt-in maximum: contexts for different points
    // share these kernels, so a per-point limit set by one context could fail another's launch.
    const int mx = (int)smem_optin_;
    ntt_probe_images(plan_.w1, plan_.w2);
    struct Probe {
        const void* fn;
        const char* name;
    };
    const Probe probes[] = {{(const void*)k_rns_plain, "k_rns_plain"},
                            {(const void*)k_crt_plain, "k_crt_plain"},
                            {(const void*)k_rns_tc, "k_rns_tc"},
                            {(const void*)k_crt_tc, "k_crt_tc"},
                            {(const void*)k_crt_tm, "k_crt_tm"}};
    for (const Probe& pr : probes) {
        cudaFuncAttributes fa{};
        cuda_check(cudaFuncGetAttributes(&fa, pr.fn), (std::string("kernel image ") + pr.name).c_str());
    }
    ntt_set_smem_limit(mx, plan_.w1, plan_.w2);
    cuda_check(cudaFuncSetAttribute(k_rns_plain, cudaFuncAttributeMaxDynamicSharedMemorySize, mx), "smem attr");
    cuda_check(cudaFuncSetAttribute(k_crt_plain, cudaFuncAttributeMaxDynamicSharedMemorySize, mx), "smem attr");
    cuda_check(cudaFuncSetAttribute(k_rns_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, mx), "smem attr");
    cuda_check(cudaFuncSetAttribute(k_crt_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, mx), "smem attr");
    cuda_check(cudaFuncSetAttribute(k_crt_tm, cudaFuncAttributeMaxDynamicSharedMemorySize, mx), "smem attr");
    cuda_check(cudaFuncSetAttribute(k_crt_finish, cudaFuncAttributeMaxDynamicSharedMemorySize, mx), "smem attr");
}

// Test hook (pm_test_fail_scratch_allocs): after `skip` more residue-scratch allocations, the
// next `n` fail on the host as if cudaMalloc had run out of memory.
static std::mutex g_inject_mutex;
static int g_inject_skip = 0, g_inject_fail = 0;
void inject_scratch_alloc_failures(int skip, int n) {
    std::lock_guard<std::mutex> lk(g_inject_mutex);
    g_inject_skip = std::max(0, skip);
    g_inject_fail = std::max(0, n);
}

static cudaError_t scratch_malloc(void** p, size_t bytes) {
    {
        std::lock_guard<std::mutex> lk(g_inject_mutex);
        if (g_inject_skip > 0) --g_inject_skip;
        else if (g_inject_fail > 0) {
            --g_inject_fail;
            *p = nullptr;
            return cudaErrorMemoryAllocation;
        }
    }
    return cudaMalloc(p, bytes);
}

void Engine::ensure_scratch(uint32_t group) {
    if (group <= group_) return;
    // the engine holds no scratch from here until both arrays exist: a failed allocation leaves
    // group_ = 0, so the next call allocates again instead of launching on missing arrays
    if (d_ra_) cudaFree(d_ra_);
    if (d_rb_) cudaFree(d_rb_);
    d_ra_ = d_rb_ = nullptr;
    group_ = 0;
    scratch_words_ = 0;
    const size_t words = (size_t)group * plan_.K * plan_.N;
    cuda_check(scratch_malloc(reinterpret_cast<void**>(&d_ra_), words * 4), "cudaMalloc residues");
    const cudaError_t e = scratch_malloc(reinterpret_cast<void**>(&d_rb_), words * 4);
    if (e != cudaSuccess) {
        cudaFree(d_ra_);
        d_ra_ = nullptr;
        throw_cuda(e, "cudaMalloc residues");
    }
    scratch_words_ = 2 * words;
    group_ = group;
}

// Column-chunk schedule of the host pipeline.  Staged calls (kind 0): input chunks of
// ncols / in_body columns after narrow head chunks (1/32, 1/32, 1/16), output chunks of
// ncols / out_body columns between narrow head and tail chunks (1/64, 1/32 ... 1/32, 1/64),
// so that the host staging starts and the host scatter ends sooner.  Direct-copy calls
// (kind 1): b in chunks of ncols / in_body (a moves whole), output in chunks of
// ncols / out_body, no narrow heads or tails: nothing on the host precedes an H2D or follows
// a D2H, the first output chunk's latency (inverse column pass + CRT, ~30 us at N = 65536)
// hardly depends on its width, and each copy costs a few microseconds of DMA set-up.  Events
// sized for the longer schedule.
// Direct-copy calls also take divisor 3 for either side: b in [1/2, 1/4, 1/4] (the last chunk,
// whose compute is exposed, a quarter) and the output in [1/4, 1/4, 1/2] (the first, which gates
// the first D2H, a quarter) -- three copies each; and divisor 5, geometric: b in
// [1/2, 1/4, 1/8, 1/8] and the output in [1/8, 1/8, 1/4, 1/2] -- four copies each, an eighth of
// the transform exposed at either end of the device tail.
void Engine::set_chunk_schedule(uint32_t in_body, uint32_t out_body, int kind) {
    if (kind != 0 && kind != 1) throw InvalidPoint("pipeline kind must be 0 (staged) or 1 (direct)");
    auto ok = [&](uint32_t d) { return d != 0 && ((d & (d - 1)) == 0 || (kind == 1 && (d == 3 || d == 5))); };
    if (!ok(in_body) || !ok(out_body))
        throw InvalidPoint("chunk divisors must be powers of two (or 3 or 5 for direct-copy calls)");
    const uint32_t nc = plan_.ncols;
    if (kind == 0) {
        // narrow head (and output tail) chunks only under a fine body: they start the staging
        // sooner, but each chunk costs its own copy set-up and launches
        cin_[kind] = in_body >= 8 ? make_chunks(nc, {32, 32, 16}, in_body, {}) : make_chunks(nc, {}, in_body, {});
        cout_[kind] = out_body >= 8 ? make_chunks(nc, {64, 32}, out_body, {32, 64}) : make_chunks(nc, {}, out_body, {});
    } else {
        cin_[kind] = in_body == 3   ? make_chunks(nc, {2}, 4, {})
                     : in_body == 5 ? make_chunks(nc, {2, 4, 8}, 8, {})
                                    : make_chunks(nc, {}, in_body, {});
        cout_[kind] = out_body == 3   ? make_chunks(nc, {}, 4, {2})
                      : out_body == 5 ? make_chunks(nc, {8}, 8, {4, 2})
                                      : make_chunks(nc, {}, out_body, {});
    }
    in_body_[kind] = in_body;
    out_body_[kind] = out_body;
    // input items: both operands' chunks (kind 0), or a whole plus b's chunks (kind 1)
    const size_t nin = std::max(2 * cin_[0].size(), 1 + cin_[1].size());
    const size_t nco = std::max(cout_[0].size(), cout_[1].size());
    auto mk = [](std::vector<cudaEvent_t>& v, size_t n, unsigned flags) {
        if (v.size() == n) return;
        for (auto e : v) cudaEventDestroy(e);
        v.assign(n, nullptr);
        for (auto& e : v) cuda_check(cudaEventCreateWithFlags(&e, flags), "event");
    };
    mk(ev_in_, nin, cudaEventDisableTiming);
    mk(ev_done_in_, nin, cudaEventDisableTiming);
    mk(ev_crt_, nco, cudaEventDisableTiming);
    mk(ev_out_, nco, cudaEventDisableTiming);
    if (profile_) mk(trace_ev_, 8 + 2 * nin + 2 * nco, cudaEventDefault);
}

double Engine::tune_host_pipeline(int reps, int kind) {
    if (!pool_) throw Unsupported("this context has no host pipeline");
    if (kind != 0 && kind != 1) throw InvalidPoint("pipeline kind must be 0 (staged) or 1 (direct)");
    reps = std::max(1, reps);
    // timing operand: pseudo-random limbs with the top limb of every coefficient zero, so that
    // each coefficient is below 2^(32(L-1)) < q (the kernels' bounds assume inputs below q);
    // kind 1 times page-locked buffers (the direct-copy path)
    const size_t words = plan_.coeff_words();
    std::vector<uint32_t> va, vc;
    uint32_t *a = nullptr, *c = nullptr;
    if (kind == 1) {
        cuda_check(cudaHostAlloc(&a, words * 4, cudaHostAllocDefault), "cudaHostAlloc");
        if (cudaHostAlloc(&c, words * 4, cudaHostAllocDefault) != cudaSuccess) {
            cudaFreeHost(a);
            throw CudaError("cudaHostAlloc failed");
        }
    } else {
        va.resize(words);
        vc.resize(words);
        a = va.data();
        c = vc.data();
    }
    for (size_t i = 0; i < words; ++i) a[i] = (i % plan_.L == plan_.L - 1) ? 0u : (uint32_t)(i * 2654435761u);
    double best = 1e30;
    uint32_t bi = in_body_[kind], bo = out_body_[kind];
    // body divisors 1, 2, 4, 8, 16; direct-copy calls also 3 and 5 (the uneven three- and
    // four-chunk shapes of set_chunk_schedule): fewer copies, each ~4 us of DMA set-up, against
    // more compute exposed after the last input chunk and before the first output one
    const uint32_t cand[7] = {1, 2, 3, 4, 5, 8, 16};
    try {
        for (uint32_t ib : cand)
            for (uint32_t ob : cand) {
                if ((ib == 5 ? 8 : ib) > plan_.ncols || (ob == 5 ? 8 : ob) > plan_.ncols) continue;
                if (kind == 0 && (ib == 3 || ob == 3 || ib == 5 || ob == 5)) continue;
                set_chunk_schedule(ib, ob, kind);
                run_host(a, a, c);
                std::vector<double> t;
                for (int r = 0; r < reps; ++r) {
                    const auto t0 = std::chrono::steady_clock::now();
                    run_host(a, a, c);
                    t.push_back(
                        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count());
                }
                std::sort(t.begin(), t.end());
                const double med = t[t.size() / 2];
                if (med < best) {
                    best = med;
                    bi = ib;
                    bo = ob;
                }
            }
    } catch (...) {
        if (kind == 1) {
            cudaFreeHost(a);
            cudaFreeHost(c);
        }
        throw;
    }
    if (kind == 1) {
        cudaFreeHost(a);
        cudaFreeHost(c);
    }
    set_chunk_schedule(bi, bo, kind);
    return best;
}

void Engine::setup_host_pipeline() {
    const size_t bytes = plan_.coeff_words() * 4;
    for (int i = 0; i < 2; ++i) {
        d_in_[i] = dev_alloc<uint32_t>(dev_allocs_, plan_.coeff_words(), nullptr);
        cuda_check(cudaHostAlloc(&h_in_[i], bytes, cudaHostAllocDefault), "cudaHostAlloc");
    }
    d_out_ = dev_alloc<uint32_t>(dev_allocs_, plan_.coeff_words(), nullptr);
    cuda_check(cudaHostAlloc(&h_out_, bytes, cudaHostAllocDefault), "cudaHostAlloc");
    cuda_check(cudaHostAlloc(&h_status_, 16, cudaHostAllocDefault), "cudaHostAlloc");
    *h_status_ = 0;
    profile_ = std::getenv("POLYMULT_PROFILE") != nullptr;
    if (const char* e = std::getenv("POLYMULT_GATHER_STORES")) nt_gather_ = std::strcmp(e, "cached") != 0;
    if (const char* e = std::getenv("POLYMULT_MERGE_COPIES")) merge_copies_ = std::strcmp(e, "0") != 0;
    for (auto& s : s_comp_) cuda_check(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "stream");
    cuda_check(cudaStreamCreateWithFlags(&s_h2d_, cudaStreamNonBlocking), "stream");
    cuda_check(cudaStreamCreateWithFlags(&s_d2h_, cudaStreamNonBlocking), "stream");
    // default schedules by operand size (the tuner refines them): a point of a few hundred KB
    // moves in one chunk each way (its copies take microseconds, each chunk costs a few of set-up
    // and four launches), a few MB in quarters, larger points in eighths with narrow heads
    const size_t opb = plan_.coeff_words() * 4;
    const uint32_t body = opb < (1u << 20) ? 1 : opb < (8u << 20) ? 4 : 8;
    set_chunk_schedule(std::min<uint32_t>(body, plan_.ncols), std::min<uint32_t>(body, plan_.ncols), 0);
    set_chunk_schedule(std::min<uint32_t>(body, plan_.ncols), std::min<uint32_t>(body, plan_.ncols), 1);
    cuda_check(cudaEventCreateWithFlags(&ev_fused_, cudaEventDisableTiming), "event");
    // 7 workers by default: they copy while the caller issues a chunk's CUDA calls, and the caller
    // joins them once it is done (8 copying threads at most).  On the 16-CPU B200 hosts measured,
    // 12 threads stage an operand pair faster in isolation (0.63 ms against 1.0 ms) but made the
    // end-to-end call slower and far more variable inside a full process (p50 1.51 ms, p99 5.6 ms
    // against 1.13 / 1.2 ms): spinning workers then compete with the process's other threads.
    // POLYMULT_HOST_THREADS overrides.
    int workers = std::max(0, std::min(7, usable_cpus() - 2));
    if (const char* e = std::getenv("POLYMULT_HOST_THREADS")) workers = std::max(0, std::min(63, std::atoi(e) - 1));
    pool_.reset(new HostPool(workers));
}

// Prime blocks of the tensor-core decomposition: the largest block (a multiple of 4 primes,
// at most 128) whose B image slice fits shared memory next to the A tile and the raw ring.
// A block's B operand is a contiguous slice of the full image (rows 4j + t, 4 j0 a multiple
// of 8); its kernel sees K = the block's primes, p / pinv from j0, and writes residue rows
// j0.. of the full arrays.  False if no block fits.
//
// A point that needs several blocks takes a one-tile raw ring where that makes the blocks wider
// (fewer blocks: each re-reads the operand), e.g. 84 instead of 52 primes at W = 3000.
bool Engine::make_dec_blocks() {
    dec_blocks_.clear();
    auto block_primes = [&](int ring) {
        int k = std::min(plan_.KP, 128) & ~3;
        for (; k >= 4; k -= 4) {
            DevPlan t = dp_;
            t.KP = k;
            t.dec_nrows = 4 * k;
            if (rns_tc_smem(t, ring) <= smem_optin_) break;
        }
        return k;
    };
    int kpb = block_primes(2), ring = 2;
    if (kpb < 4) return false;
    if (kpb < plan_.K) {
        const int kpb1 = block_primes(1);
        if ((plan_.K + kpb1 - 1) / kpb1 < (plan_.K + kpb - 1) / kpb) {
            kpb = kpb1;
            ring = 1;
        }
    }
    for (int j0 = 0; j0 < plan_.K; j0 += kpb) {
        DecBlock b;
        b.j0 = (uint32_t)j0;
        b.dp = dp_;
        b.dp.K = std::min(kpb, plan_.K - j0);
        b.dp.KP = (b.dp.K + 3) & ~3;
        b.dp.p += j0;
        b.dp.pinv += j0;
        b.dp.dec_b += (size_t)4 * j0 * dp_.dec_kbytes;
        b.dp.dec_b_ra += (size_t)4 * j0 * dp_.dec_kbytes;
        b.dp.dec_nrows = 4 * b.dp.KP;
        b.ring = ring;
        b.smem = rns_tc_smem(b.dp, ring);
        dec_blocks_.push_back(b);
    }
    return true;
}

// Blocks of a CRT whose primes do not fit one tile: prime blocks of the largest multiple of 4
// (at most 128) and result-byte blocks of at most 256 bytes (TMEM columns) such that the
// partial-mode kernel fits shared memory.  Each block gets its own B image -- rows v0.. of the
// full image, K columns 4 j0.. -- re-packed into the canonical layout with the block's K width.
bool Engine::make_crt_blocks() {
    crt_blocks_.clear();
    const int nrows_full = plan_.crt_gemm.n_rows, kb_full = plan_.crt_gemm.k_bytes;
    auto round_up = [](int x, int m) { return (x + m - 1) / m * m; };
    int kpb = std::min(plan_.KP, 128) & ~3;
    for (; kpb >= 4; kpb -= 4) {
        DevPlan t = dp_;  // KP: the whole plan's 1/p table, which a byte-block launch stages
        t.crt_kbytes = round_up(4 * kpb, 32);
        t.crt_nrows = std::min(256, nrows_full);
        if (crt_tc_smem(t, true) <= smem_optin_) break;
    }
    if (kpb < 4) return false;
    for (int j0 = 0; j0 < plan_.K; j0 += kpb) {
        const int cnt = std::min(kpb, plan_.K - j0), kp = (cnt + 3) & ~3, kb = round_up(4 * kp, 32);
        for (int v0 = 0; v0 < nrows_full; v0 += 256) {
            const int nr = std::min(256, nrows_full - v0);
            std::vector<uint8_t> img((size_t)nr * kb, 0);
            for (int v = 0; v < nr; ++v)
                for (int kbyte = 0; kbyte < 4 * kp; ++kbyte) {
                    const int fk = 4 * j0 + kbyte;
                    // (not the v column: the blocks' partial integers leave v T_1 to k_crt_finish)
                    if (fk < kb_full && fk != plan_.crt_kv)
                        img[umma_kmajor_offset(v, kbyte, kb)] = plan_.crt_b[umma_kmajor_offset(v0 + v, fk, kb_full)];
                }
            CrtBlock b;
            b.j0 = (uint32_t)j0;
            b.dp = dp_;
            b.dp.K = cnt;
            b.dp.KP = kp;
            b.dp.p += j0;
            b.dp.pinv += j0;
            b.dp.crt_c += j0;
            b.dp.crt_cc += j0;
            b.dp.rcp += j0;
            b.dp.crt_b = dev_upload(dev_allocs_, img, &table_bytes_);
            b.dp.crt_nrows = nr;
            b.dp.crt_kbytes = kb;
            b.mode = (j0 == 0 && v0 == 0) ? CRT_PARTIAL_FIRST : CRT_PARTIAL_ADD;
            b.limb0 = v0 / 4;
            b.add_s = v0 == 0;
            b.smem = crt_tc_smem(b.dp, true);
            crt_blocks_.push_back(b);
        }
    }
    // group the blocks by result-byte block: one launch each, its prime blocks in TMEM
    crt_byte_launches_.clear();
    for (int v0 = 0; v0 < nrows_full; v0 += 256) {
        CrtByteLaunch bl;
        bl.dp = dp_;
        bl.dp.crt_nrows = std::min(256, nrows_full - v0);
        bl.dp.crt_kbytes = 0;
        for (const CrtBlock& b : crt_blocks_) {
            if (b.limb0 != v0 / 4) continue;
            if (bl.pbs.n == CrtPrimeBlocks::MAX) {
                crt_byte_launches_.clear();
                return true;
            }
            const int q = bl.pbs.n++;
            bl.pbs.j0[q] = (int)b.j0;
            bl.pbs.k[q] = b.dp.K;
            bl.pbs.kp[q] = b.dp.KP;
            bl.pbs.kb[q] = b.dp.crt_kbytes;
            bl.pbs.b[q] = b.dp.crt_b;
            bl.dp.crt_kbytes = std::max(bl.dp.crt_kbytes, b.dp.crt_kbytes);
        }
        bl.mode = v0 == 0 ? CRT_PARTIAL_FIRST : CRT_PARTIAL_ADD;
        bl.limb0 = v0 / 4;
        bl.add_s = v0 == 0;
        bl.smem = crt_tc_smem(bl.dp, true);  // the whole plan's 1/p table
        if (bl.pbs.n == 0 || bl.smem > smem_optin_) {
            crt_byte_launches_.clear();
            return true;
        }
        crt_byte_launches_.push_back(bl);
    }
    return true;
}

// The CRT of a point with more than 128 primes and at most 512 result bytes in one launch: one
// TMEM accumulator holds every result byte of a tile (its epilogue no longer overlaps the next
// tile's MMAs), the tile's prime blocks accumulate into it in turn, and the epilogue is the
// single-block one (v column, fold, -q) -- no partial integers, no k_crt_finish.  Each prime
// block's B image covers all result rows and the block's own K bytes; the last block's also
// the v column (its K bytes extended to reach it).  False where the blocks or shared memory do
// not allow it.
bool Engine::make_crt_wide() {
    crt_wide_ok_ = false;
    const int nrows_full = plan_.crt_gemm.n_rows, kb_full = plan_.crt_gemm.k_bytes;
    if (nrows_full > 512 || tmem_cols_for(nrows_full) > 512) return false;
    auto round_up = [](int x, int m) { return (x + m - 1) / m * m; };
    int kpb = std::min(plan_.KP, 128) & ~3;
    for (; kpb >= 4; kpb -= 4) {
        DevPlan t = dp_;
        t.crt_kbytes = round_up(4 * kpb + 32, 32);  // room for the last block's v column
        t.crt_nrows = nrows_full;
        if (crt_tc_smem(t, false) <= smem_optin_) break;
    }
    if (kpb < 4) return false;
    CrtByteLaunch w;
    w.dp = dp_;
    w.dp.crt_nrows = nrows_full;
    w.dp.crt_kbytes = 0;
    std::vector<std::pair<int, int>> blocks;  // (j0, count)
    for (int j0 = 0; j0 < plan_.K; j0 += kpb) blocks.push_back({j0, std::min(kpb, plan_.K - j0)});
    if ((int)blocks.size() > CrtPrimeBlocks::MAX) return false;
    for (size_t q = 0; q < blocks.size(); ++q) {
        const int j0 = blocks[q].first, cnt = blocks[q].second, kp = (cnt + 3) & ~3;
        const bool last = q + 1 == blocks.size();
        // v = round(sum y'_j / p_j) <= 2K - 1 needs two bytes once K > 128: A's v column kvl
        // takes v mod 256 against T_1's bytes, column kvl + 1 takes v / 256 against T_1's bytes
        // one result byte up (256 T_1), so that the MMA adds v T_1
        const int kvl = plan_.crt_kv - 4 * j0;  // the v column in this block's K bytes (last block)
        const int kb = round_up(last ? std::max(4 * kp, kvl + 2) : 4 * kp, 32);
        std::vector<uint8_t> img((size_t)nrows_full * kb, 0);
        for (int v = 0; v < nrows_full; ++v)
            for (int kbyte = 0; kbyte < kb; ++kbyte) {
                const int fk = 4 * j0 + kbyte;
                if (last && kbyte == kvl + 1) {
                    if (v > 0) img[umma_kmajor_offset(v, kbyte, kb)] =
                                   plan_.crt_b[umma_kmajor_offset(v - 1, plan_.crt_kv, kb_full)];
                } else if (fk < kb_full && (kbyte < 4 * kp || (last && kbyte == kvl))) {
                    // the block's own primes, and the v column in the last block
                    img[umma_kmajor_offset(v, kbyte, kb)] = plan_.crt_b[umma_kmajor_offset(v, fk, kb_full)];
                }
            }
        const int n = w.pbs.n++;
        w.pbs.j0[n] = j0;
        w.pbs.k[n] = cnt;
        w.pbs.kp[n] = kp;
        w.pbs.kb[n] = kb;
        w.pbs.b[n] = dev_upload(dev_allocs_, img, &table_bytes_);
        w.dp.crt_kbytes = std::max(w.dp.crt_kbytes, kb);
    }
    w.mode = CRT_FULL;
    w.smem = crt_tc_smem(w.dp, false);
    if (w.smem > smem_optin_) return false;
    crt_wide_ = w;
    crt_wide_ok_ = true;
    return true;
}

void Engine::reserve_crt_partials(size_t coeffs) {
    if (!crt_blocked_ || coeffs <= partial_coeffs_) return;
    if (d_zp_) cudaFree(d_zp_);
    if (d_sp_) cudaFree(d_sp_);
    d_zp_ = nullptr;
    d_sp_ = nullptr;
    partial_coeffs_ = 0;
    cuda_check(cudaMalloc(&d_zp_, coeffs * crt_zl(plan_.L) * 4), "cudaMalloc CRT partials");
    cuda_check(cudaMalloc(&d_sp_, coeffs * 4), "cudaMalloc CRT partials");
    partial_coeffs_ = coeffs;
}

void Engine::set_variant(bool col_tma, bool crt_tm) {
    dp_.col_tma = col_tma ? 1 : 0;
    crt_tm_ = crt_tm && crt_tm_ok_;
}

bool Engine::col_tma_applies() const {
    // the TMA column pass: lines of 256 rows, tiles of 64 columns (launch_cols_tma)
    return plan_.w1 == 8 && plan_.ncols >= 64;
}

int Engine::kernel_launches_per_group() const {
    const int dec = dec_tc_ ? (int)dec_blocks_.size() : 1;
    const int crt = !crt_blocked_ || crt_wide_ok_
                        ? 1
                        : (int)(crt_byte_launches_.empty() ? crt_blocks_.size() : crt_byte_launches_.size()) + 1;
    // column passes of a, b and the inverse, and one row pass for both operands
    return 2 * dec + crt + (plan_.w1 > 0 ? 4 : 1);
}

ChunkMap Engine::chunk_map(Chunk ch) const {
    ChunkMap m;
    m.col0 = ch.col0;
    m.cw = ch.cw;
    m.lcw = ilog2(ch.cw);
    return m;
}

// ---------------------------------------------------------------------------------------
// launches
// ---------------------------------------------------------------------------------------
// ra: src is the operand whose transform the fused row pass reads (RA).  In the tensor form its
// residues are decomposed times gamma_j, the tcgen05 CRT's per-prime factor (dec_b_ra), so that
// the inverse transform delivers the CRT's y_j directly.
void Engine::launch_dec(const uint32_t* src, Chunk ch, uint32_t nb, uint32_t* R, cudaStream_t s, bool ra,
                        bool pdl) const {
    const uint32_t npos = plan_.nrows * ch.cw;
    if (dec_tc_) {
        const uint32_t tiles = (npos + TC_M - 1) / TC_M * nb;
        const uint32_t grid = std::min<uint32_t>(tiles, (uint32_t)num_sms_);
        const int bulk = ((uintptr_t)src % 16 == 0) && ((size_t)npos * plan_.L * 4) % 16 == 0;
        const bool scaled = ra && (crt_tc_ || crt_blocked_);
        for (const DecBlock& b : dec_blocks_) {
            DevPlan d = b.dp;
            if (scaled) d.dec_b = d.dec_b_ra;
            cuda_check(launch_kernel(k_rns_tc, dim3(grid), dim3(RNS_TC_THREADS), b.smem, s, pdl, d, src,
                                     chunk_map(ch), npos, nb, R + (size_t)b.j0 * plan_.N, bulk, b.ring),
                       "launch k_rns_tc");
            pdl = true;  // the next prime block follows this launch
        }
    } else {
        dim3 grid((npos + DEC_TM - 1) / DEC_TM, 1, nb);
        cuda_check(launch_kernel(k_rns_plain, grid, dim3(256), smem_dec_, s, pdl, dp_, src, chunk_map(ch), npos, R,
                                 dec_tab_smem_ ? 1 : 0),
                   "launch k_rns_plain");
    }
}

void Engine::launch_cols(bool inv, uint32_t* R, Chunk ch, uint32_t nb, cudaStream_t s, bool pdl) const {
    if (plan_.w1 == 0) return;
    // tiles of 32 columns (64 for the two-column kernel of lines of >= 128 rows, where the chunk
    // is at least that wide)
    const int ltc = ilog2(std::min<uint32_t>(plan_.w1 >= 7 && plan_.w1 <= 8 && ch.cw >= 64 ? 64 : 32, ch.cw));
    dim3 grid(ch.cw >> ltc, plan_.K, nb);
    const size_t smem = ntt_cols_smem(dp_, ltc);
    launch_ntt_cols(inv, grid, smem, s, dp_, R, ch.col0, ltc, pdl);
}

void Engine::launch_rows(bool fused, uint32_t* R, const uint32_t* RA, uint32_t nb, cudaStream_t s,
                         const uint32_t* ra_sel, bool pdl) const {
    dim3 grid((plan_.nrows + rpb_ - 1) / rpb_, plan_.K, nb);
    launch_ntt_rows(fused, grid, s, dp_, R, RA, ra_sel, pdl);
}

void Engine::launch_rows_both(uint32_t* R, const uint32_t* RA, uint32_t nb, cudaStream_t s, bool pdl) const {
    dim3 grid((plan_.nrows + rpb_ - 1) / rpb_, plan_.K, nb);
    launch_ntt_rows(2, grid, s, dp_, R, RA, nullptr, pdl);
}

void Engine::launch_crt(const uint32_t* R, Chunk ch, uint32_t nb, uint32_t* out, cudaStream_t s, size_t poff,
                        bool pdl) const {
    const uint32_t npos = plan_.nrows * ch.cw;
    if (crt_tm_ && ch.cw >= 4 && ch.col0 % 4 == 0) {
        const uint32_t tiles = (npos + TC_M - 1) / TC_M * nb;
        const uint32_t grid = std::min<uint32_t>(tiles, (uint32_t)num_sms_);
        cuda_check(launch_kernel(k_crt_tm, dim3(grid), dim3(CRT_TC_THREADS), crt_tm_smem(dp_), s, pdl, dp_, R,
                                 chunk_map(ch), npos, nb, out),
                   "launch k_crt_tm");
    } else if (crt_tc_) {
        const uint32_t tiles = (npos + TC_M - 1) / TC_M * nb;
        const uint32_t grid = std::min<uint32_t>(tiles, (uint32_t)num_sms_);
        const CrtPartial full{nullptr, nullptr, CRT_FULL, 0, 0};
        cuda_check(launch_kernel(k_crt_tc, dim3(grid), dim3(CRT_TC_THREADS), smem_crt_, s, pdl, dp_, R, chunk_map(ch),
                                 npos, nb, out, full, CrtPrimeBlocks{}),
                   "launch k_crt_tc");
    } else if (crt_blocked_ && crt_wide_ok_) {
        const uint32_t tiles = (npos + TC_M - 1) / TC_M * nb;
        const uint32_t grid = std::min<uint32_t>(tiles, (uint32_t)num_sms_);
        const CrtPartial full{nullptr, nullptr, CRT_FULL, 0, 0};
        cuda_check(launch_kernel(k_crt_tc, dim3(grid), dim3(CRT_TC_THREADS), crt_wide_.smem, s, pdl, crt_wide_.dp, R,
                                 chunk_map(ch), npos, nb, out, full, crt_wide_.pbs),
                   "launch k_crt_tc (wide)");
    } else if (crt_blocked_) {
        const size_t coeffs = (size_t)npos * nb;
        if (poff + coeffs > partial_coeffs_) throw Unsupported("blocked CRT: partial buffers reserved for fewer coefficients");
        uint32_t* zp = d_zp_ + poff * crt_zl(plan_.L);
        float* sp = d_sp_ + poff;
        const uint32_t tiles = (npos + TC_M - 1) / TC_M * nb;
        const uint32_t grid = std::min<uint32_t>(tiles, (uint32_t)num_sms_);
        if (!crt_byte_launches_.empty()) {
            for (const CrtByteLaunch& bl : crt_byte_launches_) {
                const CrtPartial part{zp, sp, bl.mode, bl.limb0, bl.add_s};
                cuda_check(launch_kernel(k_crt_tc, dim3(grid), dim3(CRT_TC_THREADS), bl.smem, s, pdl, bl.dp, R,
                                         chunk_map(ch), npos, nb, out, part, bl.pbs),
                           "launch k_crt_tc (byte block)");
                pdl = true;  // each later launch follows the previous one
            }
        } else {
            for (const CrtBlock& b : crt_blocks_) {
                const CrtPartial part{zp, sp, b.mode, b.limb0, b.add_s};
                cuda_check(launch_kernel(k_crt_tc, dim3(grid), dim3(CRT_TC_THREADS), b.smem, s, pdl, b.dp,
                                         R + (size_t)b.j0 * plan_.N, chunk_map(ch), npos, nb, out, part,
                                         CrtPrimeBlocks{}),
                           "launch k_crt_tc (block)");
                pdl = true;  // each later launch follows the previous block's
            }
        }
        const size_t fsmem = (size_t)TC_M * crt_zstride(plan_.L) * 4;
        cuda_check(launch_kernel(k_crt_finish, dim3((unsigned)((coeffs + TC_M - 1) / TC_M)), dim3(TC_M), fsmem, s,
                                 true, dp_, zp, sp, (uint32_t)coeffs, out),
                   "launch k_crt_finish");
    } else {
        dim3 grid((npos + CRT_TM - 1) / CRT_TM, 1, nb);
        cuda_check(launch_kernel(k_crt_plain, grid, dim3(256), smem_crt_, s, pdl, dp_, R, chunk_map(ch), npos, out,
                                 crt_tab_smem_ ? 1 : 0),
                   "launch k_crt_plain");
    }
}

// ---------------------------------------------------------------------------------------
// device-resident multiply
// ---------------------------------------------------------------------------------------
void Engine::run_device(const uint32_t* a, const uint32_t* b, uint32_t* c, uint32_t count, cudaStream_t s) {
    cuda_check(cudaSetDevice(device_), "cudaSetDevice");
    if (count == 0) return;
    const uint32_t g = std::min(count, group_cap_);
    ensure_scratch(g);
    const Chunk all{0, plan_.ncols};
    const size_t cw = plan_.coeff_words();
    for (uint32_t i = 0; i < count; i += g) {
        const uint32_t nb = std::min(g, count - i);
        const uint32_t* ai = a + (size_t)i * cw;
        const uint32_t* bi = b + (size_t)i * cw;
        // every launch but the call's first follows a kernel of this sequence
        launch_dec(ai, all, nb, d_ra_, s, true, i > 0);
        launch_cols(false, d_ra_, all, nb, s, true);
        launch_dec(bi, all, nb, d_rb_, s, false, true);
        launch_cols(false, d_rb_, all, nb, s, true);
        launch_rows_both(d_rb_, d_ra_, nb, s, true);
        launch_cols(true, d_rb_, all, nb, s, true);
        launch_crt(d_rb_, all, nb, c + (size_t)i * cw, s, 0, true);
    }
    cuda_check(cudaGetLastError(), "kernel launch");
}

void Engine::time_stages(const uint32_t* a, const uint32_t* b, uint32_t* c, uint32_t count, int reps,
                         cudaStream_t s, float* ms_out) {
    cuda_check(cudaSetDevice(device_), "cudaSetDevice");
    if (count == 0 || count > group_cap_) throw InvalidPoint("count must be in [1, group]");
    if (reps < 1) throw InvalidPoint("reps must be >= 1");
    ensure_scratch(count);
    const Chunk all{0, plan_.ncols};
    constexpr int S = 8;
    cudaEvent_t ev[S + 1];
    for (auto& e : ev) cuda_check(cudaEventCreate(&e), "event");
    double acc[S] = {0};
    try {
        for (int r = 0; r < reps; ++r) {
            // the sequence of run_device; stage 2 (a's own row pass) is empty, as the row pass
            // of stage 5 transforms both operands' rows
            cuda_check(cudaEventRecord(ev[0], s), "record");
            launch_dec(a, all, count, d_ra_, s, true);
            cuda_check(cudaEventRecord(ev[1], s), "record");
            launch_cols(false, d_ra_, all, count, s);
            cuda_check(cudaEventRecord(ev[2], s), "record");
            cuda_check(cudaEventRecord(ev[3], s), "record");
            launch_dec(b, all, count, d_rb_, s);
            cuda_check(cudaEventRecord(ev[4], s), "record");
            launch_cols(false, d_rb_, all, count, s);
            cuda_check(cudaEventRecord(ev[5], s), "record");
            launch_rows_both(d_rb_, d_ra_, count, s);
            cuda_check(cudaEventRecord(ev[6], s), "record");
            launch_cols(true, d_rb_, all, count, s);
            cuda_check(cudaEventRecord(ev[7], s), "record");
            launch_crt(d_rb_, all, count, c, s);
            cuda_check(cudaEventRecord(ev[8], s), "record");
            cuda_check(cudaGetLastError(), "kernel launch");
            cuda_check(cudaEventSynchronize(ev[S]), "sync");
            for (int k = 0; k < S; ++k) {
                if (k == 2) continue;  // no kernel between ev[2] and ev[3]
                float ms = 0;
                cuda_check(cudaEventElapsedTime(&ms, ev[k], ev[k + 1]), "elapsed");
                acc[k] += ms;
            }
        }
    } catch (...) {
        for (auto e : ev) cudaEventDestroy(e);
        throw;
    }
    for (auto e : ev) cudaEventDestroy(e);
    for (int k = 0; k < S; ++k) ms_out[k] = (float)(acc[k] / reps);
    throw_if_status();
}

void Engine::run_device_with_scratch(const uint32_t* a, const uint32_t* b, uint32_t* c, uint32_t* ra, uint32_t* rb,
                                     cudaStream_t s) {
    cuda_check(cudaSetDevice(device_), "cudaSetDevice");
    run_group(a, b, c, 1, ra, rb, s);
}

void Engine::run_group(const uint32_t* a, const uint32_t* b, uint32_t* c, uint32_t nb, uint32_t* ra, uint32_t* rb,
                       cudaStream_t s) const {
    if (nb == 0) return;
    const Chunk all{0, plan_.ncols};
    launch_dec(a, all, nb, ra, s, true);
    launch_cols(false, ra, all, nb, s, true);
    launch_dec(b, all, nb, rb, s, false, true);
    launch_cols(false, rb, all, nb, s, true);
    launch_rows_both(rb, ra, nb, s, true);
    launch_cols(true, rb, all, nb, s, true);
    launch_crt(rb, all, nb, c, s, 0, true);
    cuda_check(cudaGetLastError(), "kernel launch");
}

uint32_t Engine::take_status() {
    cuda_check(cudaSetDevice(device_), "cudaSetDevice");
    uint32_t st = 0;
    cuda_check(cudaDeviceSynchronize(), "device synchronize");
    cuda_check(cudaMemcpy(&st, dp_.status, 4, cudaMemcpyDeviceToHost), "status read");
    if (st) cuda_check(cudaMemset(dp_.status, 0, 4), "status clear");
    return st;
}

void Engine::throw_if_status() {
    const uint32_t st = take_status();
    if (st) {
        std::string what = "device-side check failed:";
        if (st & DEV_ERR_CRT_BOUND) what += " CRT estimate outside its exactness bound;";
        if (st & DEV_ERR_FOLD) what += " CRT value outside its bound after folding;";
        if (st & DEV_ERR_WAIT) what += " tensor-core wait timed out;";
        throw DeviceCheckError(what);
    }
}

// ---------------------------------------------------------------------------------------
// host-operand multiply: the chunked pipeline
// ---------------------------------------------------------------------------------------
// True if [p, p + bytes) is page-locked host memory this device can copy from / to directly.
static bool host_range_pinned(const void* p, size_t bytes) {
    auto pinned = [](const void* q) {
        cudaPointerAttributes at;
        if (cudaPointerGetAttributes(&at, q) != cudaSuccess) {
            cudaGetLastError();  // an unknown pointer is not an error here
            return false;
        }
        return at.type == cudaMemoryTypeHost;
    };
    return bytes > 0 && pinned(p) && pinned(static_cast<const char*>(p) + bytes - 1);
}

void Engine::run_host(const uint32_t* a, const uint32_t* b, uint32_t* c) {
    if (!pool_) throw Unsupported("this context has no host pipeline");
    cuda_check(cudaSetDevice(device_), "cudaSetDevice");
    ensure_scratch(1);
    const uint32_t nrows = plan_.nrows, ncols = plan_.ncols, L = plan_.L;
    const uint32_t* src[2] = {a, b};
    // copy jobs of one column chunk: tasks of at least 64 KB of the chunk each (up to 64, one
    // row at most), taken from the pool's word by whichever thread is free
    auto tasks_for = [&](uint32_t cw) {
        const size_t bytes = (size_t)nrows * cw * L * 4;
        return (uint32_t)std::max<size_t>(1, std::min<size_t>({(size_t)nrows, 64, bytes >> 16}));
    };
    // operands already in page-locked memory skip the host staging: each column chunk moves
    // with one strided DMA copy (rows of cw * L words at a pitch of ncols * L words); with all
    // three page-locked the call runs the direct-copy schedule
    const size_t opbytes = plan_.coeff_words() * 4, pitch = (size_t)ncols * L * 4;
    const bool direct_in[2] = {host_range_pinned(a, opbytes), host_range_pinned(b, opbytes)};
    const bool direct_out = host_range_pinned(c, opbytes);
    const int kind = direct_in[0] && direct_in[1] && direct_out ? 1 : 0;
    const std::vector<Chunk>& cout = cout_[kind];
    const size_t nout = cout.size();
    // input items (operand, column chunk): both operands in the schedule's input chunks; with
    // direct copies a moves in one piece (each copy costs a few microseconds of DMA set-up, and
    // a's transform is hidden under b's transfer anyway) and only b is chunked
    std::vector<std::pair<int, Chunk>> items;
    if (kind == 1) items.push_back({0, Chunk{0, ncols}});
    else
        for (const Chunk& ch : cin_[kind]) items.push_back({0, ch});
    const int na = (int)items.size();
    for (const Chunk& ch : cin_[kind]) items.push_back({1, ch});
    const int nin = (int)items.size();

    // The pool's open copy job.  The workers copy chunk i + 1 (or scatter output chunk oc)
    // while this thread issues chunk i's copies and kernels (12-20 us of API calls per chunk),
    // then joins in with wait(); the guard, declared after the job, waits for it before the
    // job goes out of scope if anything below throws.
    std::function<void(int)> job;
    struct JoinPool {
        HostPool* p;
        ~JoinPool() { p->wait(); }
    } join_pool{pool_.get()};
    const bool ntg = nt_gather_;
    // opens the staging job of input item i: layout [row][col-in-chunk][limb] in pinned memory
    // (nothing to do for an operand already page-locked)
    auto stage_start = [&](int i) {
        const int P = items[i].first;
        if (direct_in[P]) return false;
        const Chunk ch = items[i].second;
        uint32_t* dst = h_in_[P] + (size_t)ch.col0 * nrows * L;
        const uint32_t* s = src[P];
        const size_t seg = (size_t)ch.cw * L;
        const uint32_t nt = tasks_for(ch.cw), rpt = (nrows + nt - 1) / nt;
        job = [=](int t) {
            const uint32_t r1 = std::min<uint32_t>(nrows, (uint32_t)(t + 1) * rpt);
            for (uint32_t r = (uint32_t)t * rpt; r < r1; ++r)
                stream_copy(dst + r * seg, s + ((size_t)r * ncols + ch.col0) * L, seg * 4, ntg);
        };
        pool_->start((int)nt, job);
        return true;
    };
    // opens the job that scatters output chunk oc from pinned memory into c
    auto scatter_start = [&](size_t oc) {
        const Chunk ch = cout[oc];
        const uint32_t* srcc = h_out_ + (size_t)ch.col0 * nrows * L;
        const size_t seg = (size_t)ch.cw * L;
        const uint32_t nt = tasks_for(ch.cw), rpt = (nrows + nt - 1) / nt;
        job = [=](int t) {
            const uint32_t r1 = std::min<uint32_t>(nrows, (uint32_t)(t + 1) * rpt);
            for (uint32_t r = (uint32_t)t * rpt; r < r1; ++r)
                stream_copy(c + ((size_t)r * ncols + ch.col0) * L, srcc + r * seg, seg * 4);
        };
        pool_->start((int)nt, job);
    };
    uint32_t* dR[2] = {d_ra_, d_rb_};
    using clk = std::chrono::steady_clock;
    const auto t0 = clk::now();
    auto us = [&](clk::time_point t) { return std::chrono::duration<double, std::micro>(t - t0).count(); };
    clk::time_point t_stage0, t_inputs, t_first_out, t_last_out;
    // POLYMULT_PROFILE: device timeline from timing events on the pipeline's streams
    std::vector<std::pair<std::string, cudaEvent_t>> marks;
    std::vector<double> staged_us;  // host time each input chunk finished staging
    std::vector<double> issued_us;  // host time each input chunk's copies and kernels were issued
    auto mark = [&](const std::string& name, cudaStream_t st) {
        if (!profile_ || marks.size() >= trace_ev_.size()) return;
        cuda_check(cudaEventRecord(trace_ev_[marks.size()], st), "record");
        marks.emplace_back(name, trace_ev_[marks.size()]);
    };
    mark("start", s_h2d_);
    if (stage_start(0)) pool_->wait();
    t_stage0 = clk::now();
    // the kernels of input item k, once its copy is issued (the copy's event: ev_in_[hi])
    auto issue_compute = [&](int k, int hi) {
        const int P = items[k].first;
        const Chunk ch = items[k].second;
        const size_t off = (size_t)ch.col0 * nrows * L;
        // the last input chunk runs on stream 0, after a's row pass and b's other chunks, so
        // that its kernels, the fused row pass and the first output chunk's follow each other
        // in one stream (each launch overlapping the previous kernel's tail)
        const bool last = k + 1 == nin;
        cudaStream_t sc = last ? s_comp_[0] : s_comp_[k % 3];
        if (last)
            for (int q = na; q < k; ++q) cuda_check(cudaStreamWaitEvent(sc, ev_done_in_[q], 0), "wait");
        cuda_check(cudaStreamWaitEvent(sc, ev_in_[hi], 0), "wait");
        launch_dec(d_in_[P] + off, ch, 1, dR[P], sc, P == 0);
        launch_cols(false, dR[P], ch, 1, sc, true);
        if (!last) {
            cuda_check(cudaEventRecord(ev_done_in_[k], sc), "record");
            mark("in" + std::to_string(k), sc);
        }
        if (k == na - 1) {  // a complete: its row pass overlaps b's transfer
            for (int q = 0; q < na; ++q) cuda_check(cudaStreamWaitEvent(s_comp_[0], ev_done_in_[q], 0), "wait");
            launch_rows(false, d_ra_, nullptr, 1, s_comp_[0]);
            mark("rowA", s_comp_[0]);
        }
    };
    // Staged items of one operand lie side by side in pinned and in device memory, so the items
    // staged since the last copy go as one copy: a copy is issued when at most one is still in
    // flight (so the DMA engine always has the next one queued), and at the end of each operand.
    // Fewer, larger copies pay the per-copy set-up less often; items whose operand is page-locked
    // go one strided copy each.
    int pend = 0;                 // first item staged but not yet copied
    int fl_prev = -1, fl_last = -1;  // last items of the two latest copies (their ev_in_ mark completion)
    auto in_flight = [&](int hi) {
        if (hi < 0) return false;
        const cudaError_t q = cudaEventQuery(ev_in_[hi]);
        if (q == cudaErrorNotReady) {
            if (cudaPeekAtLastError() == cudaErrorNotReady) cudaGetLastError();  // the query's answer
            return true;
        }
        return false;
    };
    for (int i = 0; i < nin; ++i) {
        const int P = items[i].first;
        // the next chunk is copied by the workers while this thread issues this one
        const bool staging = i + 1 < nin && stage_start(i + 1);
        const bool op_end = i + 1 == nin || items[i + 1].first != P;
        const bool flush = op_end || direct_in[P] || !merge_copies_ || !(in_flight(fl_prev) && in_flight(fl_last));
        if (flush) {
            const Chunk c0 = items[pend].second;
            const size_t off = (size_t)c0.col0 * nrows * L;
            size_t words = 0;
            for (int k = pend; k <= i; ++k) words += (size_t)items[k].second.cw * nrows * L;
            if (direct_in[P])
                cuda_check(cudaMemcpy2DAsync(d_in_[P] + off, (size_t)c0.cw * L * 4, src[P] + (size_t)c0.col0 * L, pitch,
                                             (size_t)c0.cw * L * 4, nrows, cudaMemcpyHostToDevice, s_h2d_),
                           "H2D");
            else
                cuda_check(cudaMemcpyAsync(d_in_[P] + off, h_in_[P] + off, words * 4, cudaMemcpyHostToDevice, s_h2d_),
                           "H2D");
            cuda_check(cudaEventRecord(ev_in_[i], s_h2d_), "record");
            mark("h2d" + std::to_string(i), s_h2d_);
            for (int k = pend; k <= i; ++k) issue_compute(k, i);
            fl_prev = fl_last;
            fl_last = i;
            pend = i + 1;
        }
        if (profile_ && i + 1 < nin) issued_us.push_back(us(clk::now()));
        if (staging) pool_->wait();
        if (profile_ && i + 1 < nin) staged_us.push_back(us(clk::now()));
    }
    // stream 0 has run a's row pass and b's last chunk after the others
    cudaStream_t s0 = s_comp_[0];
    launch_rows(true, d_rb_, d_ra_, 1, s0, nullptr, true);
    if (kind == 0) cuda_check(cudaEventRecord(ev_fused_, s0), "record");
    mark("fused", s0);
    auto issue_out = [&](size_t oc) {
        const Chunk ch = cout[oc];
        const size_t off = (size_t)ch.col0 * nrows * L, words = (size_t)ch.cw * nrows * L;
        // staged calls spread the output chunks over three streams; direct-copy calls run them
        // in order on one stream: each chunk's compute is shorter than its D2H, and the first
        // chunk, which gates the first D2H, then has the GPU to itself
        const int si = kind == 1 ? 0 : (int)(oc % 3);
        cudaStream_t sc = s_comp_[si];
        if (si != 0) cuda_check(cudaStreamWaitEvent(sc, ev_fused_, 0), "wait");
        launch_cols(true, d_rb_, ch, 1, sc, si == 0);
        // output chunks run on three streams: each gets its own region of the partial buffers
        launch_crt(d_rb_, ch, 1, d_out_ + off, sc, (size_t)ch.col0 * nrows, true);
        cuda_check(cudaEventRecord(ev_crt_[oc], sc), "record");
        mark("crt" + std::to_string(oc), sc);
        cuda_check(cudaStreamWaitEvent(s_d2h_, ev_crt_[oc], 0), "wait");
        if (direct_out)
            cuda_check(cudaMemcpy2DAsync(c + (size_t)ch.col0 * L, pitch, d_out_ + off, (size_t)ch.cw * L * 4,
                                         (size_t)ch.cw * L * 4, nrows, cudaMemcpyDeviceToHost, s_d2h_),
                       "D2H");
        else
            cuda_check(cudaMemcpyAsync(h_out_ + off, d_out_ + off, words * 4, cudaMemcpyDeviceToHost, s_d2h_),
                       "D2H");
        cuda_check(cudaEventRecord(ev_out_[oc], s_d2h_), "record");
        mark("d2h" + std::to_string(oc), s_d2h_);
        if (oc + 1 == nout) {
            // device status word -> pinned memory behind the last D2H (s_d2h has waited on every CRT)
            cuda_check(cudaMemcpyAsync(h_status_, dp_.status, 4, cudaMemcpyDeviceToHost, s_d2h_), "status D2H");
            cuda_check(cudaMemsetAsync(dp_.status, 0, 4, s_d2h_), "status clear");
            cuda_check(cudaEventRecord(ev_out_[oc], s_d2h_), "record");  // re-recorded: the host waits on it
        }
    };
    // Output chunks issued before the host waits on the first: all of them when nothing is
    // scattered on the host; else the first three (one per compute stream), then more for as
    // long as the first D2H has not finished (the host usually waits here for the device's
    // last input chunk), and the rest two at a time while the workers scatter earlier ones.
    // The first scatter is then not held up behind the API calls of every output chunk, and
    // the device stays ahead of the scatter.
    size_t issued = direct_out ? nout : std::min<size_t>(3, nout);
    for (size_t oc = 0; oc < issued; ++oc) issue_out(oc);
    while (issued < nout && cudaEventQuery(ev_out_[0]) == cudaErrorNotReady) issue_out(issued++);
    if (cudaPeekAtLastError() == cudaErrorNotReady) cudaGetLastError();  // the query's answer, not a failure
    cuda_check(cudaGetLastError(), "kernel launch");
    t_inputs = clk::now();
    for (size_t oc = 0; oc < nout; ++oc) {
        cuda_check(cudaEventSynchronize(ev_out_[oc]), "D2H chunk");
        if (oc == 0) t_first_out = clk::now();
        if (oc + 1 == nout) t_last_out = clk::now();
        if (!direct_out) scatter_start(oc);
        for (int k = 0; k < 2 && issued < nout; ++k) issue_out(issued++);
        pool_->wait();
    }
    cuda_check(cudaGetLastError(), "kernel launch");
    if (profile_) {
        std::fprintf(stderr,
                     "polymult: host: stage0 %.1f us | inputs issued %.1f | first out %.1f | last out %.1f | done %.1f"
                     " | direct copies a %d b %d c %d\n",
                     us(t_stage0), us(t_inputs), us(t_first_out), us(t_last_out), us(clk::now()), (int)direct_in[0],
                     (int)direct_in[1], (int)direct_out);
        std::string line = "polymult: device (us after start):";
        for (size_t k = 1; k < marks.size(); ++k) {
            float ms = 0;
            if (cudaEventElapsedTime(&ms, marks[0].second, marks[k].second) == cudaSuccess) {
                char buf[64];
                std::snprintf(buf, sizeof buf, " %s %.1f", marks[k].first.c_str(), 1000.0 * ms);
                line += buf;
            }
        }
        std::fprintf(stderr, "%s\n", line.c_str());
        std::string st = "polymult: host chunk issued / next chunk staged (us):";
        for (size_t k = 0; k < staged_us.size(); ++k) {
            char buf[48];
            std::snprintf(buf, sizeof buf, " %.1f/%.1f", issued_us[k], staged_us[k]);
            st += buf;
        }
        std::fprintf(stderr, "%s\n", st.c_str());
    }
    const uint32_t st = *h_status_;
    if (st) {
        *h_status_ = 0;
        std::string what = "device-side check failed:";
        if (st & DEV_ERR_CRT_BOUND) what += " CRT estimate outside its exactness bound;";
        if (st & DEV_ERR_FOLD) what += " CRT value outside its bound after folding;";
        if (st & DEV_ERR_WAIT) what += " tensor-core wait timed out;";
        throw DeviceCheckError(what);
    }
}

}  // namespace pm
