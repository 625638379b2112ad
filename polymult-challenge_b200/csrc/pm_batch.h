// pm_batch.h -- a batch of multiplications of uneven points behind pm_batch_* (see
// pm_batch.cpp for the schedule, the CUDA graph and the autotuner).
#pragma once

#include <memory>
#include <string>
#include <vector>

#include "../../include/polymult_b200.h"
#include "pm_engine.h"

namespace pm {

class Batch {
  public:
    Batch(const pm_batch_class* classes, uint32_t n, int gemm_request, int flags, int device);
    ~Batch();
    Batch(const Batch&) = delete;
    Batch& operator=(const Batch&) = delete;

    // Every class's multiplications; one graph launch on `s` (or the launches themselves
    // with PM_BATCH_NO_GRAPH).  Asynchronous.
    void run(cudaStream_t s);
    // Waits and reports device-side check failures of any class.
    void sync();

    size_t classes() const { return cls_.size(); }
    const Engine& engine(size_t i) const { return *cls_[i].eng; }
    double tuned_ms(size_t i) const { return cls_[i].tuned_ms; }
    uint32_t launch_groups(size_t i) const { return cls_[i].groups; }
    int kernel_launches() const;
    size_t graph_nodes() const { return graph_nodes_; }
    size_t streams() const { return streams_.size(); }
    size_t scratch_bytes() const {
        size_t b = 0;
        for (size_t w : scratch_words_) b += 2 * w * 4;
        return b;
    }

    static constexpr size_t kMaxStreams = 8;

  private:
    struct Cls {
        pm_batch_class src{};
        std::vector<uint32_t> q;
        std::unique_ptr<Engine> eng;
        double tuned_ms = 0.0;  // measured time of the chosen configuration (0: not tuned, -1: cached)
        uint32_t groups = 1;    // launch groups the class's multiplications run in
    };
    void choose_configs(int gemm_request);
    static void run_class(const Engine& e, const pm_batch_class& s, uint32_t groups, uint32_t* ra, uint32_t* rb,
                          cudaStream_t st);
    static double time_class(const Engine& e, const pm_batch_class& s, uint32_t* ra, uint32_t* rb, uint32_t groups = 1);
    void alloc_scratch();
    void enqueue(cudaStream_t origin);
    void capture();
    void release();

    int device_ = 0;
    int flags_ = 0;
    std::vector<Cls> cls_;
    std::vector<std::vector<size_t>> sched_;  // classes per stream, in launch order
    std::vector<cudaStream_t> streams_;
    std::vector<uint32_t*> scratch_;
    std::vector<size_t> scratch_words_;
    cudaStream_t capture_ = nullptr;
    cudaEvent_t fork_ = nullptr;
    std::vector<cudaEvent_t> joins_;
    cudaGraph_t graph_ = nullptr;
    cudaGraphExec_t exec_ = nullptr;
    size_t graph_nodes_ = 0;
};

}  // namespace pm
