// pm_server.cpp -- serving: a request loop with continuous batching, admission by an HBM
// budget, and operands kept resident on the device in NTT form.
//
// No reference counterpart: the reference serves one fherma_run call at a time
// (main.cpp:181-186 times each call alone).  Here a server holds one point and R fixed
// operands b_0 .. b_{R-1}, each already through decomposition, column pass and row pass (the
// forward transform a multiply otherwise recomputes per call: k_row_fwd's output,
// solve.cu:341-355).  A request multiplies a fresh operand a by one of them, so it costs one
// decomposition, one forward column pass, the fused row pass (forward a, pointwise with the
// resident b_k, inverse), the inverse column pass and the CRT -- five kernels instead of
// eight -- plus its own H2D and D2H copy.
//
// Admission: every in-flight request holds its input, residue and output buffers
// (8NL + 4KN bytes); the budget minus the resident transforms and the tables bounds the
// requests in flight (max_inflight).  Device memory is carved at start-up into `streams`
// slots of cap = min(max_batch, max_inflight / streams) requests each.
//
// Continuous batching: the caller's thread runs the loop.  Requests join a FIFO queue at
// their arrival time; whenever a slot is free and the in-flight count allows, the slot takes
// every queued request up to its capacity -- whatever their resident operand (the fused row
// kernel reads resident transform sel[z] for batch entry z) -- and launches the batch on its
// own stream: H2D copies, the five kernels, D2H copies, an event.  Batches of different slots
// overlap on the device and on the copy engines; a slot's requests complete when its event
// has fired, and the slot takes the next batch at once.  Latency = completion seen by the
// loop - arrival time.
#include "pm_server.h"

#include "pm_kernels.cuh"

#include <algorithm>
#include <chrono>
#include <deque>
#include <thread>

namespace pm {

Server::Server(uint32_t N, uint32_t W, uint32_t L, const uint32_t* q, const uint32_t* resident, uint32_t nresident,
               uint64_t hbm_budget, uint32_t max_batch, uint32_t streams, int gemm_request, int device)
    : device_(device), nres_(nresident), max_batch_(std::max(1u, max_batch)) {
    if (!resident || nresident == 0) throw InvalidPoint("a server needs at least one resident operand");
    if (streams == 0) throw InvalidPoint("streams must be >= 1");
    EngineOptions opt;
    opt.host_pipeline = false;
    eng_.reset(new Engine(N, W, L, q, gemm_request, device, opt));
    try {
        const Plan& P = eng_->plan();
        const size_t cw = P.coeff_words(), rw = P.residue_words();
        const uint64_t fixed = (uint64_t)nres_ * rw * 4 + eng_->table_bytes();
        const uint64_t per_req = (uint64_t)(2 * cw + rw) * 4;
        if (hbm_budget <= fixed + per_req)
            throw InvalidPoint("HBM budget too small: resident operands and tables need " + std::to_string(fixed) +
                               " bytes and one request " + std::to_string(per_req));
        max_inflight_ = (uint32_t)std::min<uint64_t>((hbm_budget - fixed) / per_req, 1u << 30);
        const uint32_t ns = std::min(streams, max_inflight_);
        cap_ = std::max(1u, std::min(max_batch_, max_inflight_ / ns));
        auto dalloc = [&](size_t words) {
            void* p = nullptr;
            cuda_check(cudaMalloc(&p, std::max<size_t>(words, 1) * 4), "cudaMalloc server");
            dev_.push_back(p);
            return static_cast<uint32_t*>(p);
        };
        resident_ = dalloc((size_t)nres_ * rw);
        eng_->reserve((size_t)ns * cap_ * P.N);  // a blocked CRT's partials: one region per slot
        slots_.resize(ns);
        for (Slot& s : slots_) {
            cuda_check(cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking), "stream");
            cuda_check(cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming), "event");
            s.in = dalloc((size_t)cap_ * cw);
            s.res = dalloc((size_t)cap_ * rw);
            s.out = dalloc((size_t)cap_ * cw);
            s.sel_d = dalloc(cap_);
            s.dig_d = reinterpret_cast<uint64_t*>(dalloc(2 * (size_t)cap_));
            cuda_check(cudaHostAlloc(&s.sel_h, cap_ * 4, cudaHostAllocDefault), "cudaHostAlloc");
            cuda_check(cudaHostAlloc(&s.dig_h, cap_ * 8, cudaHostAllocDefault), "cudaHostAlloc");
        }
        // resident operands -> forward transforms, through slot 0's input buffer
        const Chunk all{0, P.ncols};
        Slot& s0 = slots_[0];
        for (uint32_t k = 0; k < nres_; ++k) {
            cuda_check(cudaMemcpyAsync(s0.in, resident + (size_t)k * cw, cw * 4, cudaMemcpyHostToDevice, s0.stream),
                       "resident upload");
            uint32_t* rk = resident_ + (size_t)k * rw;
            eng_->launch_dec(s0.in, all, 1, rk, s0.stream, /*ra=*/true);  // the fused pass's RA operand
            eng_->launch_cols(false, rk, all, 1, s0.stream);
            eng_->launch_rows(false, rk, nullptr, 1, s0.stream);
            cuda_check(cudaStreamSynchronize(s0.stream), "resident transform");
        }
        eng_->throw_if_status();
    } catch (...) {
        release();
        throw;
    }
}

Server::~Server() { release(); }

void Server::release() {
    cudaSetDevice(device_);
    cudaDeviceSynchronize();
    for (Slot& s : slots_) {
        if (s.stream) cudaStreamDestroy(s.stream);
        if (s.done) cudaEventDestroy(s.done);
        if (s.sel_h) cudaFreeHost(s.sel_h);
        if (s.dig_h) cudaFreeHost(s.dig_h);
    }
    slots_.clear();
    for (void* p : dev_) cudaFree(p);
    dev_.clear();
    for (void* p : host_) cudaFreeHost(p);
    host_.clear();
    eng_.reset();
}

void* Server::host_alloc(size_t bytes) {
    void* p = nullptr;
    cuda_check(cudaSetDevice(device_), "cudaSetDevice");
    cuda_check(cudaHostAlloc(&p, std::max<size_t>(bytes, 1), cudaHostAllocPortable), "cudaHostAlloc");
    host_.push_back(p);
    return p;
}

void Server::host_free(void* p) {
    auto it = std::find(host_.begin(), host_.end(), p);
    if (it == host_.end()) throw InvalidPoint("pointer was not allocated by this server");
    cudaFreeHost(p);
    host_.erase(it);
}

void Server::launch(Slot& s, const uint32_t* sel, const uint32_t* const* a, uint32_t* const* c, bool digest) {
    const Plan& P = eng_->plan();
    const size_t cw = P.coeff_words();
    const uint32_t nb = (uint32_t)s.reqs.size();
    for (uint32_t i = 0; i < nb; ++i) {
        const uint32_t r = s.reqs[i];
        if (sel[r] >= nres_) throw InvalidPoint("request " + std::to_string(r) + ": resident index out of range");
        s.sel_h[i] = sel[r];
        cuda_check(cudaMemcpyAsync(s.in + i * cw, a[r], cw * 4, cudaMemcpyHostToDevice, s.stream), "request H2D");
    }
    cuda_check(cudaMemcpyAsync(s.sel_d, s.sel_h, nb * 4, cudaMemcpyHostToDevice, s.stream), "selector H2D");
    const Chunk all{0, P.ncols};
    // after the copies the launches follow one another (each may overlap the previous one's tail)
    eng_->launch_dec(s.in, all, nb, s.res, s.stream);
    eng_->launch_cols(false, s.res, all, nb, s.stream, true);
    eng_->launch_rows(true, s.res, resident_, nb, s.stream, s.sel_d, true);
    eng_->launch_cols(true, s.res, all, nb, s.stream, true);
    eng_->launch_crt(s.res, all, nb, s.out, s.stream, (size_t)(&s - slots_.data()) * cap_ * P.N, true);
    if (digest) {
        launch_digest(s.out, cw, nb, s.dig_d, s.stream);
        cuda_check(cudaMemcpyAsync(s.dig_h, s.dig_d, nb * 8, cudaMemcpyDeviceToHost, s.stream), "digest D2H");
    }
    for (uint32_t i = 0; i < nb; ++i)
        cuda_check(cudaMemcpyAsync(c[s.reqs[i]], s.out + i * cw, cw * 4, cudaMemcpyDeviceToHost, s.stream),
                   "result D2H");
    cuda_check(cudaEventRecord(s.done, s.stream), "record");
    s.busy = true;
}

void Server::run(uint32_t n, const double* t_arrive, const uint32_t* sel, const uint32_t* const* a,
                 uint32_t* const* c, double* latency, pm_serve_stats* stats, uint64_t* digest) {
    cuda_check(cudaSetDevice(device_), "cudaSetDevice");
    for (uint32_t i = 0; i < n; ++i) {
        if (!a[i] || !c[i]) throw InvalidPoint("request " + std::to_string(i) + ": null operand");
        if (i && t_arrive[i] < t_arrive[i - 1]) throw InvalidPoint("arrival times must not decrease");
    }
    using clk = std::chrono::steady_clock;
    const auto t0 = clk::now();
    auto now = [&] { return std::chrono::duration<double>(clk::now() - t0).count(); };
    std::deque<uint32_t> queue;
    uint32_t next = 0, done = 0, inflight = 0, peak = 0;
    uint64_t batches = 0, batched = 0;
    double t_last = 0.0;
    try {
        while (done < n) {
            bool progressed = false;
            const double t = now();
            while (next < n && t_arrive[next] <= t) queue.push_back(next++);
            for (Slot& s : slots_) {
                if (!s.busy) continue;
                const cudaError_t q = cudaEventQuery(s.done);
                if (q == cudaErrorNotReady) continue;
                cuda_check(q, "batch");
                const double tc = now();
                for (uint32_t r : s.reqs) latency[r] = tc - t_arrive[r];
                if (digest)
                    for (size_t i = 0; i < s.reqs.size(); ++i) digest[s.reqs[i]] = s.dig_h[i];
                done += (uint32_t)s.reqs.size();
                inflight -= (uint32_t)s.reqs.size();
                t_last = tc;
                s.reqs.clear();
                s.busy = false;
                progressed = true;
            }
            for (Slot& s : slots_) {
                if (s.busy || queue.empty() || inflight >= max_inflight_) continue;
                const uint32_t nb = std::min<uint32_t>({cap_, (uint32_t)queue.size(), max_inflight_ - inflight});
                for (uint32_t i = 0; i < nb; ++i) {
                    s.reqs.push_back(queue.front());
                    queue.pop_front();
                }
                launch(s, sel, a, c, digest != nullptr);
                inflight += nb;
                peak = std::max(peak, inflight);
                ++batches;
                batched += nb;
                progressed = true;
            }
            if (!progressed) {
                // nothing to do before the next arrival or completion: yield briefly
                if (next < n && queue.empty() && inflight == 0 && t_arrive[next] - now() > 200e-6)
                    std::this_thread::sleep_for(std::chrono::microseconds(50));
#if defined(__x86_64__)
                else
                    __builtin_ia32_pause();
#endif
            }
        }
    } catch (...) {
        cudaDeviceSynchronize();
        for (Slot& s : slots_) {
            s.reqs.clear();
            s.busy = false;
        }
        throw;
    }
    eng_->throw_if_status();
    if (stats) {
        stats->requests = n;
        stats->batches = batches;
        stats->mean_batch = batches ? (double)batched / batches : 0.0;
        stats->peak_inflight = peak;
        stats->max_inflight = max_inflight_;
        stats->seconds = n ? t_last - t_arrive[0] : 0.0;
    }
}

}  // namespace pm
