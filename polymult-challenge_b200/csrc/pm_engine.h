// pm_engine.h -- one multiplication context: the plan's tables on the device, scratch
// residue arrays, streams, pinned staging, and the two ways of running the multiply
// (device-resident operands, or host operands through the chunked PCIe pipeline).
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <functional>
#include <memory>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "pm_device.cuh"
#include "pm_hostpool.h"
#include "pm_plan.h"

namespace pm {

struct CudaError : std::runtime_error {
    explicit CudaError(const std::string& s) : std::runtime_error(s) {}
};
struct DeviceCheckError : std::runtime_error {
    explicit DeviceCheckError(const std::string& s) : std::runtime_error(s) {}
};
struct Unsupported : std::runtime_error {
    explicit Unsupported(const std::string& s) : std::runtime_error(s) {}
};

void cuda_check(cudaError_t e, const char* what);
// Test hook: after `skip` more residue-scratch allocations of any engine, the next `n` fail
// (host-side injection).
void inject_scratch_alloc_failures(int skip, int n);

class Engine;
// pm_run_device_static's body (pm_static_scratch.cu): one multiply with the library's static
// residue scratch; throws InvalidPoint for a point beyond it.
void run_device_static(Engine& e, const uint32_t* d_a, const uint32_t* d_b, uint32_t* d_c, cudaStream_t stream);
// drops the cached device address of the static scratch on `device` (pm_free)
void forget_static_scratch_address(int device);
// runs k_wait_selftest on `device` with a wait limit of `limit` clocks; returns its status word
uint32_t wait_selftest(int device, long long limit);
// Harvey-Shoup butterflies per second on `device` with operands in registers (k_peak.cu), per
// clock per SM, and whether the kernel's checksum matched the host's
void butterfly_peak(int device, double* per_s, double* per_clk_sm, bool* checked);

enum GemmForm : int { GEMM_AUTO = 0, GEMM_PLAIN = 1, GEMM_TENSOR = 2, GEMM_MIXED = 3 };

struct Chunk {
    uint32_t col0, cw;
};

// Construction options beyond the point itself.
struct EngineOptions {
    bool host_pipeline = true;  // pinned staging + streams for run_host (not needed by batches)
    int w1 = -1;                // 4-step split nrows = 2^w1 (-1: logN / 2)
};

class Engine {
  public:
    Engine(uint32_t N, uint32_t W, uint32_t L, const uint32_t* q, int gemm_request, int device,
           const EngineOptions& opt = EngineOptions());
    ~Engine();
    Engine(const Engine&) = delete;
    Engine& operator=(const Engine&) = delete;

    // c[i] = a[i] * b[i] for i < count; operands contiguous [count][N][L] in device memory.
    // Asynchronous on `stream`; check_status() reports device-side check failures.
    void run_device(const uint32_t* a, const uint32_t* b, uint32_t* c, uint32_t count, cudaStream_t stream);
    // One multiply with residue scratch supplied by the caller (two arrays of K*N words);
    // allocates nothing.  Asynchronous on `stream`.
    void run_device_with_scratch(const uint32_t* a, const uint32_t* b, uint32_t* c, uint32_t* ra, uint32_t* rb,
                                 cudaStream_t stream);
    // nb multiplies in one launch per kernel, residue scratch supplied by the caller (two
    // arrays of nb*K*N words); allocates nothing and may be captured in a CUDA graph.
    void run_group(const uint32_t* a, const uint32_t* b, uint32_t* c, uint32_t nb, uint32_t* ra, uint32_t* rb,
                   cudaStream_t stream) const;
    // Per-kernel mean durations (ms) of `reps` groups of `count` multiplies (CUDA events).
    void time_stages(const uint32_t* a, const uint32_t* b, uint32_t* c, uint32_t count, int reps, cudaStream_t s,
                     float* ms_out);
    // One multiply from host (pageable) operands to a host result; synchronous.
    void run_host(const uint32_t* a, const uint32_t* b, uint32_t* c);
    // Device memory for `coeffs` coefficients of a blocked CRT per launch (no-op otherwise);
    // called before a CUDA-graph capture so that no allocation happens inside it.
    void reserve(size_t coeffs) { reserve_crt_partials(coeffs); }
    // Host pipeline column-chunk schedule (powers of two: body chunks of ncols / divisor).
    // Host-pipeline schedules per kind of call: kind 0 = operands staged through the host pool
    // (pageable buffers), kind 1 = operands and result page-locked, moved by direct copies.
    void set_chunk_schedule(uint32_t in_body, uint32_t out_body, int kind = 0);
    // Measures the candidate schedules on run_host and keeps the fastest; median ms.
    double tune_host_pipeline(int reps, int kind = 0);
    uint32_t in_body(int kind = 0) const { return in_body_[kind]; }
    uint32_t out_body(int kind = 0) const { return out_body_[kind]; }
    // Reads (and clears) the device status word; synchronises with the device.
    uint32_t take_status();
    void throw_if_status();
    // Test hook: writes `bits` into the device status word (after the device is idle), as a
    // failed device-side check would.
    void set_status_for_test(uint32_t bits);

    // Kernel variants the batch autotuner chooses between: the column passes of 256-row lines by
    // the TMA-pipelined kernel or one tile per CTA; the single-tile CRT GEMM with its A operand
    // in tensor memory (k_crt_tm) or in shared memory (k_crt_tc).  A variant that does not
    // apply to the point is ignored.
    void set_variant(bool col_tma, bool crt_tm);
    bool col_tma() const { return dp_.col_tma != 0; }
    bool crt_tm() const { return crt_tm_; }
    bool col_tma_applies() const;
    bool crt_tm_applies() const { return crt_tm_ok_; }

    const Plan& plan() const { return plan_; }
    const DevPlan& dev() const { return dp_; }
    int gemm_form() const { return form_; }
    int device() const { return device_; }
    size_t scratch_bytes() const { return scratch_words_ * 4; }
    size_t table_bytes() const { return table_bytes_; }
    uint32_t group() const { return group_cap_; }  // multiplies per launch group of run_device
    int kernel_launches_per_group() const;
    const std::vector<Chunk>& in_chunks(int kind = 0) const { return cin_[kind]; }
    const std::vector<Chunk>& out_chunks(int kind = 0) const { return cout_[kind]; }

    // launch helpers (also used by the tests' stage-by-stage checks)
    // ra: src is the operand whose transform the fused row pass reads (RA); see pm_engine.cu
    // pdl: the previous operation in stream s is a kernel; the launch may overlap its tail
    // (programmatic dependent launch, see launch_kernel)
    void launch_dec(const uint32_t* src, Chunk ch, uint32_t nb, uint32_t* R, cudaStream_t s, bool ra = false,
                    bool pdl = false) const;
    void launch_cols(bool inv, uint32_t* R, Chunk ch, uint32_t nb, cudaStream_t s, bool pdl = false) const;
    void launch_rows(bool fused, uint32_t* R, const uint32_t* RA, uint32_t nb, cudaStream_t s,
                     const uint32_t* ra_sel = nullptr, bool pdl = false) const;
    // both operands' row passes in one kernel: forward rows of R (b) and RA (a, after its column
    // pass, read only), pointwise product, inverse rows into R
    void launch_rows_both(uint32_t* R, const uint32_t* RA, uint32_t nb, cudaStream_t s, bool pdl = false) const;
    // `poff`: first coefficient of this launch's region of the blocked CRT's partial buffers --
    // launches that may run concurrently (other streams) must use disjoint regions
    void launch_crt(const uint32_t* R, Chunk ch, uint32_t nb, uint32_t* out, cudaStream_t s, size_t poff = 0,
                    bool pdl = false) const;

  private:
    struct DecBlock {
        DevPlan dp;        // the block's view of the plan (primes j0 .. j0 + dp.K)
        uint32_t j0 = 0;
        size_t smem = 0;
        int ring = 2;      // raw input tiles in flight
    };
    bool make_dec_blocks();
    // (prime block, result-byte block) launches of a CRT too large for one tile
    struct CrtBlock {
        DevPlan dp;
        uint32_t j0 = 0;
        int mode = 0, limb0 = 0, add_s = 0;
        size_t smem = 0;
    };
    // one launch per result-byte block with every prime block accumulated in TMEM (empty: one
    // launch per (prime block, byte block), where a byte block would need more than
    // CrtPrimeBlocks::MAX)
    struct CrtByteLaunch {
        DevPlan dp;
        CrtPrimeBlocks pbs{};
        int mode = 0, limb0 = 0, add_s = 0;
        size_t smem = 0;
    };
    std::vector<CrtByteLaunch> crt_byte_launches_;
    // all result bytes of a wide point in one accumulator of up to 512 TMEM columns (no double
    // buffering), every prime block accumulated, the full CRT in one launch: no partial integers
    CrtByteLaunch crt_wide_;
    bool crt_wide_ok_ = false;
    bool make_crt_wide();
    bool make_crt_blocks();
    void reserve_crt_partials(size_t coeffs);
    void upload_tables();
    void setup_launch_shapes();
    void ensure_scratch(uint32_t group);
    void setup_host_pipeline();
    ChunkMap chunk_map(Chunk ch) const;

    Plan plan_;
    DevPlan dp_{};
    int device_ = 0;
    int form_ = GEMM_PLAIN;
    bool dec_tc_ = false, crt_tc_ = false;  // which contractions run on the tensor cores
    bool crt_tm_ = false;                   // the single-tile CRT takes k_crt_tm (A in tensor memory)
    bool crt_tm_ok_ = false;                // k_crt_tm applies to this point
    bool crt_blocked_ = false;              // the tensor-core CRT runs in blocks (K > one tile)
    std::vector<DecBlock> dec_blocks_;
    std::vector<CrtBlock> crt_blocks_;
    uint32_t* d_zp_ = nullptr;              // blocked CRT: partial integers [coefficients][L + 3]
    float* d_sp_ = nullptr;                 // blocked CRT: partial sums [coefficients]
    size_t partial_coeffs_ = 0;
    int num_sms_ = 148;
    size_t smem_optin_ = 227 * 1024;
    std::vector<void*> dev_allocs_;
    size_t table_bytes_ = 0;

    // scratch residues for `group_` multiplies: R_a, R_b [group][K][N]
    uint32_t* d_ra_ = nullptr;
    uint32_t* d_rb_ = nullptr;
    size_t scratch_words_ = 0;
    uint32_t group_ = 0;
    uint32_t group_cap_ = 1;

    // launch shapes
    int rpb_ = 1;
    size_t smem_cols_ = 0;
    size_t smem_dec_ = 0, smem_crt_ = 0;
    bool dec_tab_smem_ = false, crt_tab_smem_ = false;

    // host pipeline
    std::vector<Chunk> cin_[2], cout_[2];
    uint32_t in_body_[2] = {8, 8}, out_body_[2] = {8, 8};
    uint32_t* d_in_[2] = {nullptr, nullptr};
    uint32_t* d_out_ = nullptr;
    uint32_t* h_in_[2] = {nullptr, nullptr};
    uint32_t* h_out_ = nullptr;
    cudaStream_t s_comp_[3] = {nullptr, nullptr, nullptr};
    cudaStream_t s_h2d_ = nullptr, s_d2h_ = nullptr;
    std::vector<cudaEvent_t> ev_in_, ev_done_in_, ev_crt_, ev_out_;
    uint32_t* h_status_ = nullptr;  // pinned copy of the device status word, written after each run_host
    bool profile_ = false;          // POLYMULT_PROFILE: per-call host and device timeline on stderr
    bool nt_gather_ = true;         // POLYMULT_GATHER_STORES=cached: ordinary stores when staging inputs
    bool merge_copies_ = true;      // POLYMULT_MERGE_COPIES=0: one H2D copy per staged input chunk
    std::vector<cudaEvent_t> trace_ev_;  // timing events of that timeline
    cudaEvent_t ev_fused_ = nullptr;
    std::unique_ptr<HostPool> pool_;
};

}  // namespace pm
