// pm_batch.cpp -- many multiplications of uneven points (N, W, q) in one CUDA-graph launch,
// with a measured choice of the 4-step split, the GEMM form, the kernel variants and the launch
// groups per point (the autotuner).
//
// The reference has no batch path (it multiplies one pair per fherma_run call,
// solve.cu:1480-1498, with fixed heuristics for the split and the chunking,
// solve.cu:85-87, 917-918, 1403-1419).  Here a batch is a list of CLASSES -- one point and
// `count` multiplications of it whose operands lie contiguously in device memory -- and:
//   * every class runs as one launch per kernel covering all of its multiplications
//     (grid.z / the persistent tile range spans the class's batch), so the 8 kernels of a
//     class see count x the work of one multiply -- or as 2 or 4 such launch groups in a row
//     where the tuner measured that faster;
//   * classes are spread over a few streams (largest work first, each class to the stream
//     with the least work so far) so that small classes overlap one another on the GPU;
//   * the whole schedule -- every class's launches, the fork and join between streams -- is
//     captured once into a CUDA graph and replayed by pm_batch_run with one launch call;
//   * residue scratch is allocated once at init: per stream, the largest class on it (the
//     classes of one stream run one after the other and reuse it).
// The autotuner (PM_BATCH_TUNE) times, per class, every split w1 in logN/2 - 1 .. logN/2 + 1
// that the kernels support and both GEMM forms (where the tensor-core form fits) on the
// class's own operands, CUDA events around 3 repetitions after a warm-up, and keeps the
// fastest; then, on that engine, the column-pass kernel (TMA pipeline / one tile per CTA), the
// CRT GEMM's A placement (tensor / shared memory) and 1, 2 or 4 launch groups per class.
// Results are cached per (N, W, count, device) in a text file ($POLYMULT_TUNE_CACHE, default
// ~/.cache/polymult_b200/tune.txt).
#include "pm_batch.h"

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <map>
#include <sstream>
#include <sys/stat.h>

namespace pm {

namespace {

struct TuneKey {
    uint32_t N, W, count;
    std::string dev;
    std::string str() const {
        std::ostringstream o;
        o << N << ' ' << W << ' ' << count << ' ' << dev;
        return o.str();
    }
};

std::string cache_path() {
    if (const char* p = std::getenv("POLYMULT_TUNE_CACHE")) return p;
    const char* home = std::getenv("HOME");
    return std::string(home ? home : "/tmp") + "/.cache/polymult_b200/tune.txt";
}

// The tuner's choice for one class.  col_tma / crt_tm: -1 = the engine's default.
struct Choice {
    int gemm = 0, w1 = 0;
    int col_tma = -1, crt_tm = -1;
    uint32_t groups = 1;
};

// "N W count device-name-with-underscores gemm w1 ms [col_tma crt_tm groups]" per line (lines
// written before the variant fields existed keep the engine's defaults and one launch group)
std::map<std::string, Choice> read_cache() {
    std::map<std::string, Choice> m;
    std::ifstream f(cache_path());
    std::string line;
    while (std::getline(f, line)) {
        std::istringstream in(line);
        TuneKey k;
        Choice c;
        double ms = 0;
        if (!(in >> k.N >> k.W >> k.count >> k.dev >> c.gemm >> c.w1 >> ms)) continue;
        int ct = -1, cm = -1;
        uint32_t g = 1;
        if (in >> ct >> cm >> g) {
            c.col_tma = ct;
            c.crt_tm = cm;
            c.groups = std::max<uint32_t>(1, g);
        }
        m[k.str()] = c;
    }
    return m;
}

void append_cache(const TuneKey& k, const Choice& c, double ms) {
    const std::string p = cache_path();
    for (size_t i = 1; i < p.size(); ++i)
        if (p[i] == '/') mkdir(p.substr(0, i).c_str(), 0755);
    std::ofstream f(p, std::ios::app);
    if (f)
        f << k.str() << ' ' << c.gemm << ' ' << c.w1 << ' ' << ms << ' ' << c.col_tma << ' ' << c.crt_tm << ' '
          << c.groups << '\n';
}

// multiplies per launch group when `count` runs in `groups` launch groups
uint32_t per_group(uint32_t count, uint32_t groups) { return (count + groups - 1) / std::max<uint32_t>(1, groups); }

std::string device_tag(int device) {
    cudaDeviceProp prop{};
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return "unknown";
    std::string s = prop.name;
    for (char& ch : s)
        if (ch == ' ') ch = '_';
    return s;
}

}  // namespace

Batch::Batch(const pm_batch_class* classes, uint32_t n, int gemm_request, int flags, int device)
    : device_(device), flags_(flags) {
    if (n == 0 || !classes) throw InvalidPoint("a batch needs at least one class");
    cuda_check(cudaSetDevice(device), "cudaSetDevice");
    try {
        for (uint32_t i = 0; i < n; ++i) {
            const pm_batch_class& c = classes[i];
            if (!c.q) throw InvalidPoint("class " + std::to_string(i) + ": q is null");
            if (c.count && (!c.d_a || !c.d_b || !c.d_c))
                throw InvalidPoint("class " + std::to_string(i) + ": null operand");
            Cls k;
            k.src = c;
            k.q.assign(c.q, c.q + c.L);
            k.src.q = k.q.data();
            cls_.push_back(std::move(k));
        }
        choose_configs(gemm_request);
        alloc_scratch();
        cuda_check(cudaStreamCreateWithFlags(&capture_, cudaStreamNonBlocking), "stream");
        for (auto& s : streams_) cuda_check(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "stream");
        cuda_check(cudaEventCreateWithFlags(&fork_, cudaEventDisableTiming), "event");
        joins_.resize(streams_.size());
        for (auto& e : joins_) cuda_check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
        if (!(flags_ & PM_BATCH_NO_GRAPH)) capture();
    } catch (...) {
        release();
        throw;
    }
}

Batch::~Batch() { release(); }

void Batch::release() {
    cudaSetDevice(device_);
    cudaDeviceSynchronize();
    if (exec_) cudaGraphExecDestroy(exec_);
    if (graph_) cudaGraphDestroy(graph_);
    exec_ = nullptr;
    graph_ = nullptr;
    for (auto e : joins_) cudaEventDestroy(e);
    joins_.clear();
    if (fork_) cudaEventDestroy(fork_);
    fork_ = nullptr;
    for (auto s : streams_)
        if (s) cudaStreamDestroy(s);
    streams_.clear();
    if (capture_) cudaStreamDestroy(capture_);
    capture_ = nullptr;
    for (auto p : scratch_) cudaFree(p);
    scratch_.clear();
    for (auto& c : cls_) c.eng.reset();
}

// Picks per class -- from the tuning cache, by measurement, or the defaults -- the gemm form
// and split (first stage: one engine per candidate), then the kernel variants and the number
// of launch groups (second stage: switched on the chosen engine), and builds the class's
// engine with them.
void Batch::choose_configs(int gemm_request) {
    const std::string dev = device_tag(device_);
    std::map<std::string, Choice> cache;
    if (flags_ & PM_BATCH_TUNE) cache = read_cache();
    // one probe scratch, sized for the largest class, while tuning
    uint32_t* probe = nullptr;
    try {
        for (auto& c : cls_) {
            const pm_batch_class& s = c.src;
            EngineOptions opt;
            opt.host_pipeline = false;
            opt.w1 = s.w1 < 0 ? -1 : s.w1;
            if (!(flags_ & PM_BATCH_TUNE) || s.count == 0 || s.w1 >= 0) {  // explicit split: not tuned
                c.eng.reset(new Engine(s.N, s.W, s.L, s.q, gemm_request, device_, opt));
                continue;
            }
            const TuneKey key{s.N, s.W, s.count, dev};
            auto hit = cache.find(key.str());
            if (hit != cache.end()) {
                const Choice& ch = hit->second;
                opt.w1 = ch.w1;
                c.eng.reset(new Engine(s.N, s.W, s.L, s.q, ch.gemm, device_, opt));
                c.eng->set_variant(ch.col_tma < 0 ? c.eng->col_tma() : ch.col_tma != 0,
                                   ch.crt_tm < 0 ? c.eng->crt_tm() : ch.crt_tm != 0);
                c.groups = std::min<uint32_t>(std::max<uint32_t>(1, ch.groups), s.count);
                c.tuned_ms = -1.0;
                continue;
            }
            // candidates: splits around logN/2, both forms (tensor only where it fits)
            int logN = 0;
            while ((1u << logN) < s.N) ++logN;
            std::vector<std::pair<int, int>> cand;
            // AUTO resolves to the tensor-core form, or the mixed one where the CRT does not fit
            const int forms[2] = {GEMM_AUTO, GEMM_PLAIN};
            for (int f : forms) {
                if (gemm_request != GEMM_AUTO && f != gemm_request) continue;
                for (int w1 = logN / 2 - 1; w1 <= logN / 2 + 1; ++w1)
                    if (w1 >= 0 && w1 <= 10 && logN - w1 >= (logN > 0 ? 1 : 0) && logN - w1 <= 10)
                        cand.push_back({f, w1});
            }
            double best = 1e30;
            std::unique_ptr<Engine> best_eng;
            int best_form = 0, best_w1 = 0;
            for (auto [f, w1] : cand) {
                std::unique_ptr<Engine> e;
                try {
                    EngineOptions o = opt;
                    o.w1 = w1;
                    e.reset(new Engine(s.N, s.W, s.L, s.q, f, device_, o));
                } catch (const Unsupported&) {
                    continue;  // this form / split does not fit the point
                } catch (const InvalidPoint&) {
                    continue;
                }
                e->reserve((size_t)s.count * e->plan().N);
                const size_t words = (size_t)s.count * e->plan().K * e->plan().N;
                if (probe) cudaFree(probe);
                probe = nullptr;
                cuda_check(cudaMalloc(&probe, 2 * words * 4), "cudaMalloc tuning scratch");
                const double ms = time_class(*e, s, probe, probe + words);
                if (ms < best) {
                    best = ms;
                    best_eng = std::move(e);
                    best_form = f;
                    best_w1 = w1;
                }
            }
            if (!best_eng) throw Unsupported("no kernel configuration fits this point");
            // second stage on the chosen engine: column-pass kernel (TMA pipeline or one tile per
            // CTA), CRT GEMM operand placement (A in tensor or shared memory), and the class in
            // 1, 2 or 4 launch groups (less scratch, the groups' residues closer to L2 size,
            // against each kernel's fixed costs spread over fewer multiplies)
            Engine& e = *best_eng;
            Choice ch;
            ch.gemm = best_form;
            ch.w1 = best_w1;
            ch.col_tma = e.col_tma() ? 1 : 0;
            ch.crt_tm = e.crt_tm() ? 1 : 0;
            std::vector<int> cols{ch.col_tma}, crts{ch.crt_tm};
            if (e.col_tma_applies()) cols.push_back(1 - ch.col_tma);
            if (e.crt_tm_applies()) crts.push_back(1 - ch.crt_tm);
            const size_t words = (size_t)s.count * e.plan().K * e.plan().N;
            for (uint32_t g : {1u, 2u, 4u}) {
                if (g > s.count) break;
                e.reserve((size_t)per_group(s.count, g) * e.plan().N);
                for (int ct : cols)
                    for (int cm : crts) {
                        if (g == 1 && ct == ch.col_tma && cm == ch.crt_tm) continue;  // timed above
                        e.set_variant(ct != 0, cm != 0);
                        const double ms = time_class(e, s, probe, probe + words, g);
                        if (ms < best) {
                            best = ms;
                            ch.col_tma = ct;
                            ch.crt_tm = cm;
                            ch.groups = g;
                        }
                    }
            }
            e.set_variant(ch.col_tma != 0, ch.crt_tm != 0);
            c.groups = ch.groups;
            c.eng = std::move(best_eng);
            c.tuned_ms = best;
            append_cache(key, ch, best);
        }
    } catch (...) {
        if (probe) cudaFree(probe);
        throw;
    }
    if (probe) cudaFree(probe);
    cuda_check(cudaDeviceSynchronize(), "tuning");
    for (auto& c : cls_) c.eng->throw_if_status();
}

// The class's multiplications as `groups` launch groups, one after another on `st`, each
// reusing the same residue scratch (sized for one group).
void Batch::run_class(const Engine& e, const pm_batch_class& s, uint32_t groups, uint32_t* ra, uint32_t* rb,
                      cudaStream_t st) {
    const uint32_t per = per_group(s.count, groups);
    const size_t words = (size_t)e.plan().N * e.plan().L;
    for (uint32_t i0 = 0; i0 < s.count; i0 += per) {
        const uint32_t n = std::min(per, s.count - i0);
        e.run_group(s.d_a + i0 * words, s.d_b + i0 * words, s.d_c + i0 * words, n, ra, rb, st);
    }
}

// Mean time (ms) of the class's multiplications in `groups` launch groups on a scratch
// stream: 1 warm-up, 3 timed.
double Batch::time_class(const Engine& e, const pm_batch_class& s, uint32_t* ra, uint32_t* rb, uint32_t groups) {
    cudaStream_t st = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cuda_check(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "stream");
    float ms = 0;
    try {
        cuda_check(cudaEventCreate(&e0), "event");
        cuda_check(cudaEventCreate(&e1), "event");
        run_class(e, s, groups, ra, rb, st);
        cuda_check(cudaEventRecord(e0, st), "record");
        for (int r = 0; r < 3; ++r) run_class(e, s, groups, ra, rb, st);
        cuda_check(cudaEventRecord(e1, st), "record");
        cuda_check(cudaEventSynchronize(e1), "sync");
        cuda_check(cudaEventElapsedTime(&ms, e0, e1), "elapsed");
    } catch (...) {
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        cudaStreamDestroy(st);
        throw;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaStreamDestroy(st);
    return ms / 3.0;
}

// Streams and scratch: classes by decreasing work, each to the least-loaded stream; a
// stream's scratch is the largest residue footprint among its classes.
void Batch::alloc_scratch() {
    std::vector<size_t> order(cls_.size());
    for (size_t i = 0; i < order.size(); ++i) order[i] = i;
    auto work = [&](size_t i) {
        const Plan& P = cls_[i].eng->plan();
        return (double)cls_[i].src.count * P.K * P.N;
    };
    std::stable_sort(order.begin(), order.end(), [&](size_t x, size_t y) { return work(x) > work(y); });
    const size_t ns = std::max<size_t>(1, std::min<size_t>(kMaxStreams, cls_.size()));
    for (auto& c : cls_) c.eng->reserve((size_t)per_group(c.src.count, c.groups) * c.eng->plan().N);
    std::vector<double> load(ns, 0.0);
    std::vector<size_t> need(ns, 0);
    sched_.assign(ns, {});
    for (size_t i : order) {
        if (cls_[i].src.count == 0) continue;
        const size_t s = (size_t)(std::min_element(load.begin(), load.end()) - load.begin());
        load[s] += work(i);
        sched_[s].push_back(i);
        const Plan& P = cls_[i].eng->plan();
        need[s] = std::max(need[s], (size_t)per_group(cls_[i].src.count, cls_[i].groups) * P.K * P.N);
    }
    streams_.assign(ns, nullptr);
    scratch_.assign(ns, nullptr);
    scratch_words_.assign(ns, 0);
    for (size_t s = 0; s < ns; ++s) {
        if (!need[s]) continue;
        cuda_check(cudaMalloc(&scratch_[s], 2 * need[s] * 4), "cudaMalloc batch scratch");
        scratch_words_[s] = need[s];
    }
}

// The whole schedule on the streams: fork from `origin`, every class's group, join.
void Batch::enqueue(cudaStream_t origin) {
    cuda_check(cudaEventRecord(fork_, origin), "record");
    for (size_t s = 0; s < streams_.size(); ++s) {
        cuda_check(cudaStreamWaitEvent(streams_[s], fork_, 0), "wait");
        for (size_t i : sched_[s]) {
            const Cls& c = cls_[i];
            run_class(*c.eng, c.src, c.groups, scratch_[s], scratch_[s] + scratch_words_[s], streams_[s]);
        }
        cuda_check(cudaEventRecord(joins_[s], streams_[s]), "record");
        cuda_check(cudaStreamWaitEvent(origin, joins_[s], 0), "wait");
    }
}

void Batch::capture() {
    cuda_check(cudaStreamBeginCapture(capture_, cudaStreamCaptureModeThreadLocal), "begin capture");
    try {
        enqueue(capture_);
    } catch (...) {
        cudaGraph_t g = nullptr;
        cudaStreamEndCapture(capture_, &g);
        if (g) cudaGraphDestroy(g);
        throw;
    }
    cuda_check(cudaStreamEndCapture(capture_, &graph_), "end capture");
    cuda_check(cudaGraphInstantiate(&exec_, graph_, 0), "graph instantiate");
    size_t nodes = 0;
    cuda_check(cudaGraphGetNodes(graph_, nullptr, &nodes), "graph nodes");
    graph_nodes_ = nodes;
}

void Batch::run(cudaStream_t s) {
    cuda_check(cudaSetDevice(device_), "cudaSetDevice");
    if (exec_) cuda_check(cudaGraphLaunch(exec_, s), "graph launch");
    else enqueue(s);
}

void Batch::sync() {
    cuda_check(cudaSetDevice(device_), "cudaSetDevice");
    cuda_check(cudaDeviceSynchronize(), "device synchronize");
    for (auto& c : cls_) c.eng->throw_if_status();
}

int Batch::kernel_launches() const {
    int n = 0;
    for (const auto& c : cls_)
        if (c.src.count) n += (int)c.groups * c.eng->kernel_launches_per_group();
    return n;
}

}  // namespace pm
