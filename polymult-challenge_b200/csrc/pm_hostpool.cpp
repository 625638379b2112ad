// pm_hostpool.cpp -- HostPool (see pm_hostpool.h).
#include "pm_hostpool.h"

#include <linux/futex.h>
#include <sys/syscall.h>
#include <unistd.h>

#include <chrono>
#include <climits>
#include <stdexcept>

namespace pm {
namespace {

constexpr uint64_t kTicketMask = 0xFFFFFFFFull;

inline uint32_t ticket_of(uint64_t w) { return (uint32_t)(w & kTicketMask); }
inline uint32_t count_of(uint64_t w) { return (uint32_t)((w >> 32) & 0xFFFFu); }

inline void relax() {
#if defined(__x86_64__)
    __builtin_ia32_pause();
#endif
}

void futex_wait(std::atomic<uint32_t>* addr, uint32_t expected, long timeout_ns) {
    timespec ts{timeout_ns / 1000000000L, timeout_ns % 1000000000L};
    syscall(SYS_futex, reinterpret_cast<uint32_t*>(addr), FUTEX_WAIT_PRIVATE, expected, &ts, nullptr, 0);
}

void futex_wake_all(std::atomic<uint32_t>* addr) {
    syscall(SYS_futex, reinterpret_cast<uint32_t*>(addr), FUTEX_WAKE_PRIVATE, INT_MAX, nullptr, nullptr, 0);
}

}  // namespace

HostPool::HostPool(int workers, int idle_us) : idle_us_(idle_us) {
    threads_.reserve((size_t)workers);
    for (int i = 0; i < workers; ++i) threads_.emplace_back([this] { worker(); });
}

HostPool::~HostPool() {
    stop_.store(true);
    wake_seq_.fetch_add(1);
    futex_wake_all(&wake_seq_);
    for (auto& t : threads_) t.join();
}

bool HostPool::take_one() {
    const uint64_t seen = word_.load(std::memory_order_acquire);
    if (ticket_of(seen) >= count_of(seen)) return false;
    const uint64_t got = word_.fetch_add(1, std::memory_order_acq_rel);
    const uint32_t t = ticket_of(got);
    if (t >= count_of(got)) return false;
    (*fn_)((int)t);  // fn_ is this ticket's job's: it changes only after the job finished
    finished_.fetch_add(1, std::memory_order_acq_rel);
    return true;
}

void HostPool::run(int n, const std::function<void(int)>& fn) {
    start(n, fn);
    wait();
}

void HostPool::start(int n, const std::function<void(int)>& fn) {
    if (open_) throw std::logic_error("HostPool: a job is already open");
    if (n <= 0) return;
    if (n > 0xFFFF) throw std::length_error("HostPool: more than 65535 tasks in one job");
    // The previous job is finished (its run() returned), so no live ticket reads fn_ now; late
    // fetch_adds on its word only move the ticket further past its count.
    fn_ = &fn;
    finished_.store(0, std::memory_order_relaxed);
    job_ = (job_ + 1) & 0xFFFFu;
    // publishes fn_ too; sequentially consistent against a parking worker's parked_ / word_ pair
    word_.store((job_ << 48) | ((uint64_t)n << 32), std::memory_order_seq_cst);
    if (parked_.load(std::memory_order_seq_cst) > 0) {
        wake_seq_.fetch_add(1, std::memory_order_seq_cst);
        futex_wake_all(&wake_seq_);
    }
    open_ = true;
    open_n_ = (uint32_t)n;
}

void HostPool::wait() {
    if (!open_) return;
    while (take_one()) {
    }
    while (finished_.load(std::memory_order_acquire) < open_n_) relax();
    open_ = false;
}

void HostPool::worker() {
    using clock = std::chrono::steady_clock;
    auto last_work = clock::now();
    uint32_t spins = 0;
    while (!stop_.load(std::memory_order_relaxed)) {
        if (take_one()) {
            last_work = clock::now();
            continue;
        }
        relax();
        if ((++spins & 2047u) != 0) continue;
        if (clock::now() - last_work < std::chrono::microseconds(idle_us_)) continue;
        // park: announce first, then re-check for work, then sleep while no job was published
        const uint32_t seq = wake_seq_.load(std::memory_order_seq_cst);
        parked_.fetch_add(1, std::memory_order_seq_cst);
        const uint64_t w = word_.load(std::memory_order_seq_cst);
        if (ticket_of(w) >= count_of(w) && !stop_.load()) futex_wait(&wake_seq_, seq, 100000000L);
        parked_.fetch_sub(1, std::memory_order_seq_cst);
        last_work = clock::now();
    }
}

uint64_t host_pool_selftest(uint32_t pools, uint32_t runs, int workers, bool vary, bool park, bool split) {
    uint64_t bad = 0;
    std::vector<std::atomic<int>> hits(64);
    for (uint32_t pi = 0; pi < pools; ++pi) {
        // park: workers give up spinning after 20 us, and every third task set comes after a
        // pause long enough for them to be asleep, so that run() has to wake them
        HostPool pool(workers, park ? 20 : 200000);
        for (uint32_t it = 0; it < runs; ++it) {
            if (park && it % 3 == 0) std::this_thread::sleep_for(std::chrono::microseconds(300));
            const int n = vary ? 1 + (int)((it * 37u + pi) % 64u) : 64;
            for (auto& h : hits) h.store(0, std::memory_order_relaxed);
            std::atomic<int> inflight{0};
            const std::function<void(int)> fn = [&](int t) {
                inflight.fetch_add(1);
                if (t >= 0 && t < 64) hits[t].fetch_add(1);
                inflight.fetch_sub(1);
            };
            if (split && it % 2 == 1) {
                pool.start(n, fn);
                // the caller's own work between start() and wait()
                volatile uint64_t x = it;
                for (int k = 0; k < 2000; ++k) x = x * 6364136223846793005ull + 1442695040888963407ull;
                pool.wait();
            } else {
                pool.run(n, fn);
            }
            bool ok = inflight.load() == 0 && !pool.open();
            for (int t = 0; t < 64 && ok; ++t) ok = hits[t].load() == (t < n ? 1 : 0);
            if (!ok) ++bad;
        }
    }
    return bad;
}

}  // namespace pm
