// pm_capi.cpp -- the extern "C" boundary (include/polymult_b200.h).  Exceptions never cross
// it: each entry point maps them to a status code and keeps the message per thread.
#include <cuda_runtime.h>

#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/polymult_b200.h"
#include "pm_context.h"
#include "pm_kernels.cuh"

namespace pm {

thread_local std::string g_last_error;

int fail(int code, const char* what) {
    g_last_error = what ? what : "";
    return code;
}

}  // namespace pm

using pm::fail;
using pm::g_last_error;

namespace {

// Restores the caller's current device on scope exit: the entry points that run an engine
// switch to the engine's device, which a framework calling them does not expect to change.
struct DeviceScope {
    int saved = -1;
    DeviceScope() {
        if (cudaGetDevice(&saved) != cudaSuccess) {
            saved = -1;
            cudaGetLastError();
        }
    }
    ~DeviceScope() {
        if (saved >= 0) cudaSetDevice(saved);
    }
};

template <class F>
int guarded(F&& f) {
    try {
        f();
        g_last_error.clear();
        return PM_OK;
    } catch (const pm::InvalidPoint& e) {
        return fail(PM_ERR_INVALID, e.what());
    } catch (const pm::Unsupported& e) {
        return fail(PM_ERR_UNSUPPORTED, e.what());
    } catch (const pm::DeviceCheckError& e) {
        return fail(PM_ERR_DEVICE, e.what());
    } catch (const pm::CudaError& e) {
        return fail(PM_ERR_CUDA, e.what());
    } catch (const std::bad_alloc&) {
        return fail(PM_ERR_INTERNAL, "host allocation failed");
    } catch (const std::exception& e) {
        return fail(PM_ERR_INTERNAL, e.what());
    } catch (...) {
        return fail(PM_ERR_INTERNAL, "unknown exception");
    }
}

}  // namespace

extern "C" {

int pm_init(uint32_t N, uint32_t W, uint32_t L, const uint32_t* q, int gemm_form, int device, pm_context** out) {
    if (!out) return fail(PM_ERR_INVALID, "out is null");
    *out = nullptr;
    if (gemm_form < PM_GEMM_AUTO || gemm_form > PM_GEMM_MIXED) return fail(PM_ERR_INVALID, "bad gemm_form");
    return guarded([&] {
        pm::Engine* e = new pm::Engine(N, W, L, q, gemm_form, device);
        try {
            // warm-up on zero operands: loads the module, touches every buffer
            std::vector<uint32_t> zeros((size_t)N * L, 0), sink((size_t)N * L);
            e->run_host(zeros.data(), zeros.data(), sink.data());
        } catch (...) {
            delete e;
            throw;
        }
        *out = new pm_context{e};
    });
}

int pm_run(pm_context* ctx, const uint32_t* a, const uint32_t* b, uint32_t* c) {
    if (!ctx || !ctx->engine) return fail(PM_ERR_INVALID, "null context");
    if (!a || !b || !c) return fail(PM_ERR_INVALID, "null operand");
    DeviceScope keep;
    return guarded([&] { ctx->engine->run_host(a, b, c); });
}

int pm_run_device(pm_context* ctx, const uint32_t* d_a, const uint32_t* d_b, uint32_t* d_c, uint32_t count,
                  void* stream) {
    if (!ctx || !ctx->engine) return fail(PM_ERR_INVALID, "null context");
    if (count && (!d_a || !d_b || !d_c)) return fail(PM_ERR_INVALID, "null operand");
    DeviceScope keep;
    return guarded([&] { ctx->engine->run_device(d_a, d_b, d_c, count, static_cast<cudaStream_t>(stream)); });
}

int pm_run_device_static(pm_context* ctx, const uint32_t* d_a, const uint32_t* d_b, uint32_t* d_c, void* stream) {
    if (!ctx || !ctx->engine) return fail(PM_ERR_INVALID, "null context");
    if (!d_a || !d_b || !d_c) return fail(PM_ERR_INVALID, "null operand");
    DeviceScope keep;
    return guarded([&] { pm::run_device_static(*ctx->engine, d_a, d_b, d_c, static_cast<cudaStream_t>(stream)); });
}

int pm_time_stages(pm_context* ctx, const uint32_t* d_a, const uint32_t* d_b, uint32_t* d_c, uint32_t count,
                   int reps, void* stream, float* ms_out) {
    if (!ctx || !ctx->engine || !ms_out) return fail(PM_ERR_INVALID, "null argument");
    if (!d_a || !d_b || !d_c) return fail(PM_ERR_INVALID, "null operand");
    DeviceScope keep;
    return guarded(
        [&] { ctx->engine->time_stages(d_a, d_b, d_c, count, reps, static_cast<cudaStream_t>(stream), ms_out); });
}

int pm_sync(pm_context* ctx) {
    if (!ctx || !ctx->engine) return fail(PM_ERR_INVALID, "null context");
    DeviceScope keep;
    return guarded([&] { ctx->engine->throw_if_status(); });
}

void pm_free(pm_context* ctx) {
    if (!ctx) return;
    DeviceScope keep;
    if (ctx->engine) pm::forget_static_scratch_address(ctx->engine->device());
    delete ctx->engine;
    delete ctx;
}

void pm_test_fail_scratch_allocs(int skip, int n) { pm::inject_scratch_alloc_failures(skip, n); }

int pm_test_set_status(pm_context* ctx, uint32_t bits) {
    if (!ctx || !ctx->engine) return fail(PM_ERR_INVALID, "null context");
    DeviceScope keep;
    return guarded([&] { ctx->engine->set_status_for_test(bits); });
}

int pm_selftest_wait(int device, uint64_t limit_clocks, uint32_t* status_out) {
    if (!status_out || limit_clocks == 0 || limit_clocks > (uint64_t)pm::kWaitClocks)
        return fail(PM_ERR_INVALID, "bad self-test arguments");
    DeviceScope keep;
    return guarded([&] { *status_out = pm::wait_selftest(device, (long long)limit_clocks); });
}

int pm_butterfly_peak(int device, double* bfly_per_s, double* bfly_per_clk_sm) {
    if (!bfly_per_s || !bfly_per_clk_sm) return fail(PM_ERR_INVALID, "null argument");
    DeviceScope keep;
    return guarded([&] {
        bool ok = false;
        pm::butterfly_peak(device, bfly_per_s, bfly_per_clk_sm, &ok);
        if (!ok) throw pm::DeviceCheckError("butterfly peak: the kernel's checksum differs from the host's");
    });
}

int pm_get_info(const pm_context* ctx, pm_info* out) {
    if (!ctx || !ctx->engine || !out) return fail(PM_ERR_INVALID, "null argument");
    const pm::Engine& e = *ctx->engine;
    const pm::Plan& P = e.plan();
    std::memset(out, 0, sizeof *out);
    out->N = P.N;
    out->W = P.W;
    out->L = P.L;
    out->K = P.K;
    out->logN = P.logN;
    out->w1 = P.w1;
    out->w2 = P.w2;
    out->gemm_form = e.gemm_form();
    out->device = e.device();
    out->delta = P.delta;
    out->table_bytes = e.table_bytes();
    out->scratch_bytes = e.scratch_bytes();
    out->launches_per_multiply = e.kernel_launches_per_group();
    out->group = (int32_t)e.group();
    return PM_OK;
}

static void fill_pipeline(const pm::Engine& e, int kind, double ms, pm_pipeline_info* out) {
    std::memset(out, 0, sizeof *out);
    out->in_chunks = (int32_t)e.in_chunks(kind).size();
    out->out_chunks = (int32_t)e.out_chunks(kind).size();
    out->in_body = (int32_t)e.in_body(kind);
    out->out_body = (int32_t)e.out_body(kind);
    out->tuned_ms = ms;
}

int pm_tune_pipeline(pm_context* ctx, int reps, int flags, pm_pipeline_info* out) {
    if (!ctx || !ctx->engine) return fail(PM_ERR_INVALID, "null context");
    if (flags & ~PM_PIPELINE_PINNED) return fail(PM_ERR_INVALID, "unknown pipeline flags");
    const int kind = (flags & PM_PIPELINE_PINNED) ? 1 : 0;
    return guarded([&] {
        const double ms = ctx->engine->tune_host_pipeline(reps, kind);
        ctx->tuned_ms[kind] = ms;
        if (out) fill_pipeline(*ctx->engine, kind, ms, out);
    });
}

int pm_set_pipeline(pm_context* ctx, int flags, int32_t in_body, int32_t out_body) {
    if (!ctx || !ctx->engine) return fail(PM_ERR_INVALID, "null context");
    if (flags & ~PM_PIPELINE_PINNED) return fail(PM_ERR_INVALID, "unknown pipeline flags");
    if (in_body <= 0 || out_body <= 0) return fail(PM_ERR_INVALID, "chunk divisors must be positive");
    const int kind = (flags & PM_PIPELINE_PINNED) ? 1 : 0;
    const uint32_t nc = ctx->engine->plan().ncols;
    if ((uint32_t)in_body > nc || (uint32_t)out_body > nc) return fail(PM_ERR_INVALID, "chunk divisor above ncols");
    return guarded([&] {
        ctx->engine->set_chunk_schedule((uint32_t)in_body, (uint32_t)out_body, kind);
        ctx->tuned_ms[kind] = 0.0;
    });
}

int pm_get_pipeline(const pm_context* ctx, int flags, pm_pipeline_info* out) {
    if (!ctx || !ctx->engine || !out) return fail(PM_ERR_INVALID, "null argument");
    if (flags & ~PM_PIPELINE_PINNED) return fail(PM_ERR_INVALID, "unknown pipeline flags");
    const int kind = (flags & PM_PIPELINE_PINNED) ? 1 : 0;
    fill_pipeline(*ctx->engine, kind, ctx->tuned_ms[kind], out);
    return PM_OK;
}

int pm_batch_init(const pm_batch_class* classes, uint32_t nclasses, int gemm_form, int flags, int device,
                  pm_batch** out) {
    if (!out) return fail(PM_ERR_INVALID, "out is null");
    *out = nullptr;
    if (!classes || nclasses == 0) return fail(PM_ERR_INVALID, "no classes");
    if (gemm_form < PM_GEMM_AUTO || gemm_form > PM_GEMM_MIXED) return fail(PM_ERR_INVALID, "bad gemm_form");
    if (flags & ~(PM_BATCH_TUNE | PM_BATCH_NO_GRAPH)) return fail(PM_ERR_INVALID, "unknown flags");
    return guarded([&] { *out = new pm_batch{new pm::Batch(classes, nclasses, gemm_form, flags, device)}; });
}

int pm_batch_run(pm_batch* batch, void* stream) {
    if (!batch || !batch->batch) return fail(PM_ERR_INVALID, "null batch");
    return guarded([&] { batch->batch->run(static_cast<cudaStream_t>(stream)); });
}

int pm_batch_sync(pm_batch* batch) {
    if (!batch || !batch->batch) return fail(PM_ERR_INVALID, "null batch");
    return guarded([&] { batch->batch->sync(); });
}

int pm_batch_get_info(const pm_batch* batch, pm_batch_info* out) {
    if (!batch || !batch->batch || !out) return fail(PM_ERR_INVALID, "null argument");
    const pm::Batch& b = *batch->batch;
    std::memset(out, 0, sizeof *out);
    out->classes = (uint32_t)b.classes();
    out->streams = (uint32_t)b.streams();
    out->kernel_launches = b.kernel_launches();
    out->graph_nodes = b.graph_nodes();
    out->scratch_bytes = b.scratch_bytes();
    return PM_OK;
}

int pm_batch_get_class(const pm_batch* batch, uint32_t index, pm_batch_class_info* out) {
    if (!batch || !batch->batch || !out) return fail(PM_ERR_INVALID, "null argument");
    const pm::Batch& b = *batch->batch;
    if (index >= b.classes()) return fail(PM_ERR_INVALID, "class index out of range");
    const pm::Engine& e = b.engine(index);
    std::memset(out, 0, sizeof *out);
    out->K = e.plan().K;
    out->w1 = e.plan().w1;
    out->w2 = e.plan().w2;
    out->gemm_form = e.gemm_form();
    out->tuned_ms = b.tuned_ms(index);
    out->col_tma = e.col_tma() && e.col_tma_applies() ? 1 : 0;
    out->crt_tm = e.crt_tm() ? 1 : 0;
    out->launch_groups = b.launch_groups(index);
    return PM_OK;
}

void pm_batch_free(pm_batch* batch) {
    if (!batch) return;
    delete batch->batch;
    delete batch;
}

int pm_server_init(uint32_t N, uint32_t W, uint32_t L, const uint32_t* q, const uint32_t* resident, uint32_t nresident,
                   uint64_t hbm_budget, uint32_t max_batch, uint32_t streams, int gemm_form, int device,
                   pm_server** out) {
    if (!out) return fail(PM_ERR_INVALID, "out is null");
    *out = nullptr;
    if (!resident || nresident == 0) return fail(PM_ERR_INVALID, "no resident operands");
    if (gemm_form < PM_GEMM_AUTO || gemm_form > PM_GEMM_MIXED) return fail(PM_ERR_INVALID, "bad gemm_form");
    return guarded([&] {
        *out = new pm_server{
            new pm::Server(N, W, L, q, resident, nresident, hbm_budget, max_batch, streams, gemm_form, device)};
    });
}

int pm_server_run(pm_server* server, uint32_t n, const double* t_arrive, const uint32_t* sel,
                  const uint32_t* const* a, uint32_t* const* c, double* latency, pm_serve_stats* stats,
                  uint64_t* digest) {
    if (!server || !server->server) return fail(PM_ERR_INVALID, "null server");
    if (n && (!t_arrive || !sel || !a || !c || !latency)) return fail(PM_ERR_INVALID, "null argument");
    DeviceScope keep;
    return guarded([&] { server->server->run(n, t_arrive, sel, a, c, latency, stats, digest); });
}

int pm_digest(const uint32_t* d_words, uint64_t words, uint32_t count, void* stream, uint64_t* out) {
    if ((count && !d_words) || (count && !out)) return fail(PM_ERR_INVALID, "null argument");
    return guarded([&] {
        if (count == 0) return;
        const cudaStream_t s = static_cast<cudaStream_t>(stream);
        uint64_t* d = nullptr;
        pm::cuda_check(cudaMallocAsync(reinterpret_cast<void**>(&d), (size_t)count * 8, s), "cudaMallocAsync");
        try {
            pm::launch_digest(d_words, words, count, d, s);
            pm::cuda_check(cudaMemcpyAsync(out, d, (size_t)count * 8, cudaMemcpyDeviceToHost, s), "digest D2H");
            pm::cuda_check(cudaStreamSynchronize(s), "digest");
        } catch (...) {
            cudaFreeAsync(d, s);
            throw;
        }
        pm::cuda_check(cudaFreeAsync(d, s), "cudaFreeAsync");
    });
}

uint64_t pm_digest_host(const uint32_t* words, uint64_t n) { return words ? pm::digest_host(words, n) : 0; }

int pm_server_host_alloc(pm_server* server, size_t bytes, void** out) {
    if (!server || !server->server || !out) return fail(PM_ERR_INVALID, "null argument");
    return guarded([&] { *out = server->server->host_alloc(bytes); });
}

int pm_server_host_free(pm_server* server, void* p) {
    if (!server || !server->server) return fail(PM_ERR_INVALID, "null server");
    return guarded([&] { server->server->host_free(p); });
}

void pm_server_free(pm_server* server) {
    if (!server) return;
    delete server->server;
    delete server;
}

const char* pm_last_error(void) { return g_last_error.c_str(); }

int pm_selftest_host_pool(uint32_t pools, uint32_t runs, uint32_t workers, int vary, uint64_t* failures) {
    if (!failures || workers > 63) return fail(PM_ERR_INVALID, "bad self-test arguments");
    return guarded(
        [&] { *failures = pm::host_pool_selftest(pools, runs, (int)workers, (vary & 1) != 0, (vary & 2) != 0,
                                                     (vary & 4) != 0); });
}

int pm_plan_selfcheck(uint32_t N, uint32_t W, uint32_t L, const uint32_t* q, int32_t* K_out) {
    return guarded([&] {
        pm::Plan P = pm::make_plan(N, W, L, q);
        if (K_out) *K_out = P.K;
        const std::string why = pm::check_plan(P);
        if (!why.empty()) throw std::runtime_error("plan self-check failed: " + why);
    });
}

}  // extern "C"
