// pm_hostpool.h -- the host threads that stage pm_run's pageable operands and results.
//
// HostPool::run(n, fn) runs fn(0) .. fn(n - 1) on the pool's workers and the calling thread
// and returns once every call has returned.  start(n, fn) opens the same job on the workers
// alone and returns at once, so that the caller can do other work (issue the CUDA calls of
// the previous chunk) while the workers copy; wait() then joins in on the tickets left and
// returns once every call has returned.  One job is open at a time, and fn must outlive it.
// The pipeline issues a job every few tens of microseconds (one per column chunk), so idle
// workers spin between jobs and only park (on a futex) after `idle_us` without work.
//
// One 64-bit word describes the open job: (job id << 48) | (task count << 32) | next ticket.
// A worker that sees next < count takes a ticket with fetch_add; the word it gets back names
// the job and its count, so a ticket at or past the count is simply dropped, and a ticket
// below it is a task of exactly that job.  The job's function pointer is written before the
// word that opens the job (release) and is replaced only after every task of the job has
// finished, so a worker holding a live ticket always reads its own job's function.  There is
// no compare-and-swap loop and no per-job handshake with workers that were preempted: a late
// worker's fetch_add on a finished job's word only moves its ticket further past the count.
#pragma once

#include <atomic>
#include <cstdint>
#include <functional>
#include <thread>
#include <vector>

namespace pm {

class HostPool {
  public:
    explicit HostPool(int workers, int idle_us = 200000);
    ~HostPool();
    HostPool(const HostPool&) = delete;
    HostPool& operator=(const HostPool&) = delete;
    // at most 65535 tasks per job
    void run(int n, const std::function<void(int)>& fn);
    void start(int n, const std::function<void(int)>& fn);
    void wait();  // returns at once if no job is open
    bool open() const { return open_; }
    int size() const { return (int)threads_.size() + 1; }

  private:
    void worker();
    // takes and runs one ticket of the open job; false if the job has no ticket left
    bool take_one();

    std::vector<std::thread> threads_;
    alignas(64) std::atomic<uint64_t> word_{0};   // job << 48 | count << 32 | next ticket
    alignas(64) std::atomic<uint32_t> finished_{0};
    alignas(64) std::atomic<uint32_t> wake_seq_{0};  // futex word: bumped by every published job
    std::atomic<int> parked_{0};
    std::atomic<bool> stop_{false};
    const std::function<void(int)>* fn_ = nullptr;  // the open job's function
    uint64_t job_ = 0;
    bool open_ = false;  // a job was started and not yet waited for
    uint32_t open_n_ = 0;
    int idle_us_;
};

// Stress test of HostPool (pm_selftest_host_pool): task sets whose tasks did not each run
// exactly once, or were still running when run() / wait() returned.  vary: task counts 1..64
// instead of 64; park: workers park between task sets and are woken by the next one; split:
// every other set is opened with start() and joined with wait() after some work of the caller.
uint64_t host_pool_selftest(uint32_t pools, uint32_t runs, int workers, bool vary, bool park, bool split = false);

}  // namespace pm
