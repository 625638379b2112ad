// pm_server.h -- the serving loop behind pm_server_* (see pm_server.cpp).
#pragma once

#include <memory>
#include <vector>

#include "../../include/polymult_b200.h"
#include "pm_engine.h"

namespace pm {

class Server {
  public:
    Server(uint32_t N, uint32_t W, uint32_t L, const uint32_t* q, const uint32_t* resident, uint32_t nresident,
           uint64_t hbm_budget, uint32_t max_batch, uint32_t streams, int gemm_request, int device);
    ~Server();
    Server(const Server&) = delete;
    Server& operator=(const Server&) = delete;

    // digest: optional; digest[i] receives the device digest (launch_digest) of c[i]
    void run(uint32_t n, const double* t_arrive, const uint32_t* sel, const uint32_t* const* a, uint32_t* const* c,
             double* latency, pm_serve_stats* stats, uint64_t* digest = nullptr);
    void* host_alloc(size_t bytes);
    void host_free(void* p);

    const Engine& engine() const { return *eng_; }
    uint32_t max_inflight() const { return max_inflight_; }
    uint32_t slots() const { return (uint32_t)slots_.size(); }
    uint32_t slot_capacity() const { return cap_; }

  private:
    struct Slot {
        cudaStream_t stream = nullptr;
        cudaEvent_t done = nullptr;
        uint32_t* in = nullptr;    // [cap][N][L]
        uint32_t* res = nullptr;   // [cap][K][N]
        uint32_t* out = nullptr;   // [cap][N][L]
        uint32_t* sel_d = nullptr; // [cap] resident index per batch entry
        uint32_t* sel_h = nullptr; // pinned staging of sel_d
        uint64_t* dig_d = nullptr; // [cap] digests of the batch's results
        uint64_t* dig_h = nullptr; // pinned copy of dig_d
        std::vector<uint32_t> reqs;
        bool busy = false;
    };
    void launch(Slot& s, const uint32_t* sel, const uint32_t* const* a, uint32_t* const* c, bool digest);
    void release();

    std::unique_ptr<Engine> eng_;
    int device_ = 0;
    uint32_t nres_ = 0;
    uint32_t* resident_ = nullptr;  // [nres][K][N] forward transforms (row-pass output)
    uint32_t max_batch_ = 1, max_inflight_ = 1, cap_ = 1;
    std::vector<Slot> slots_;
    std::vector<void*> dev_, host_;
};

}  // namespace pm
