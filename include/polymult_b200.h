/*
 * polymult_b200.h -- C ABI of the B200 negacyclic multiplier c = a*b mod (X^N + 1, q).
 *
 * Coefficients are W-bit integers in [0, q) stored as L = ceil(W/32) little-endian u32
 * limbs; a polynomial is N x L words, row-major [N][L] (the reference's Tensor<u32> of
 * shape {N, L}, fherma.h:31-40).  q must lie just below 2^W: delta = 2^W - q < 2^63 (the
 * spec-derived prime: the largest prime below 2^W with q == 1 mod 2N).
 *
 * The reference binds three C++ symbols, fherma_init / fherma_run / fherma_free
 * (fherma.h:45-48, fherma.toml:7-10).  This header is the plain-C boundary underneath
 * them: pointers and sizes only, status codes instead of exceptions.  The C++ symbols
 * themselves are declared in fherma_abi.h and implemented on top of these functions.
 *
 * Every call returns PM_OK (0) or a positive error code; pm_last_error() gives the
 * message of the last failure on the calling thread.
 */
#ifndef POLYMULT_B200_H
#define POLYMULT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct pm_context pm_context;

enum pm_status {
    PM_OK = 0,
    PM_ERR_INVALID = 1,     /* invalid point or argument (reference: runtime_error from precompute,
                               solve.cu:873-913, or the size check of fherma_run, solve.cu:1482-1483) */
    PM_ERR_CUDA = 2,        /* CUDA runtime failure (reference: check(), solve.cu:814-816) */
    PM_ERR_DEVICE = 3,      /* a device-side check failed: CRT estimate bound, fold bound, wait timeout */
    PM_ERR_UNSUPPORTED = 4, /* e.g. the tensor-core form requested for a point it does not cover */
    PM_ERR_INTERNAL = 5
};

/* GEMM form of the RNS decomposition and the CRT. */
enum pm_gemm_form {
    PM_GEMM_AUTO = 0,   /* tensor cores where the point fits, else CUDA cores */
    PM_GEMM_PLAIN = 1,  /* int32 CUDA-core kernels */
    PM_GEMM_TENSOR = 2, /* tcgen05 kind::i8 byte-sliced GEMMs (error if the point does not fit) */
    PM_GEMM_MIXED = 3   /* tensor-core decomposition (in prime blocks where K > 128), CUDA-core
                           CRT; also what PM_GEMM_AUTO resolves to where only the decomposition
                           fits the tensor-core kernels */
};

typedef struct pm_info {
    uint32_t N, W, L;
    int32_t K;             /* RNS primes */
    int32_t logN, w1, w2;  /* 4-step split: nrows = 2^w1, ncols = 2^w2 */
    int32_t gemm_form;     /* resolved form: PM_GEMM_PLAIN, PM_GEMM_TENSOR or PM_GEMM_MIXED */
    int32_t device;
    uint64_t delta;        /* 2^W - q */
    uint64_t table_bytes;  /* device memory of the per-point tables */
    uint64_t scratch_bytes;/* device memory of the residue scratch */
    int32_t launches_per_multiply; /* kernels launched per device-resident multiply group */
    int32_t group;         /* multiplies per launch group of pm_run_device (its scratch grows to this on use) */
} pm_info;

/* Replaces fherma_init (solve.cu:1392-1478): validates the point, builds every table,
 * uploads them, allocates scratch and pinned staging, and runs one warm-up multiply. */
int pm_init(uint32_t N, uint32_t W, uint32_t L, const uint32_t* q, int gemm_form, int device, pm_context** out);

/* Replaces fherma_run (solve.cu:1480-1498): c = a*b for host operands through the chunked
 * PCIe pipeline.  a, b, c: N*L words of host memory (pageable is fine).  Synchronous. */
int pm_run(pm_context* ctx, const uint32_t* a, const uint32_t* b, uint32_t* c);

/* No reference counterpart (the reference only takes host operands): c[i] = a[i]*b[i] for
 * i < count, operands already in device memory as [count][N][L].  Asynchronous on
 * `stream` (a cudaStream_t; NULL = legacy default stream); pm_sync() waits and reports
 * device-side check failures. */
int pm_run_device(pm_context* ctx, const uint32_t* d_a, const uint32_t* d_b, uint32_t* d_c, uint32_t count,
                  void* stream);

/* Kernels of one device-resident multiply group, in launch order (pm_time_stages). */
#define PM_STAGE_COUNT 8
enum pm_stage {
    PM_STAGE_DEC_A = 0,    /* RNS decomposition of a */
    PM_STAGE_COLS_A = 1,   /* forward column pass of a */
    PM_STAGE_ROWS_A = 2,   /* forward row pass of a: 0 in device-resident groups, whose row pass
                              (PM_STAGE_FUSED) transforms both operands' rows */
    PM_STAGE_DEC_B = 3,    /* RNS decomposition of b */
    PM_STAGE_COLS_B = 4,   /* forward column pass of b */
    PM_STAGE_FUSED = 5,    /* fused row pass: forward rows of b and a, pointwise, inverse */
    PM_STAGE_COLS_INV = 6, /* inverse column pass */
    PM_STAGE_CRT = 7       /* CRT straight to mod q */
};

/* No reference counterpart (the reference's PM_PROFILE timer is host-side, solve.cu:1238-1242):
 * runs `reps` device-resident multiply groups of `count` (<= pm_info.group) multiplies on
 * `stream` and writes each kernel's mean duration in milliseconds, measured with CUDA events
 * on that stream, to ms_out[PM_STAGE_COUNT].  Synchronous. */
int pm_time_stages(pm_context* ctx, const uint32_t* d_a, const uint32_t* d_b, uint32_t* d_c, uint32_t count,
                   int reps, void* stream, float* ms_out);

/* No counterpart in the reference.  One device-resident multiply, c = a*b with d_a, d_b, d_c
 * of N*L words in device memory, that allocates nothing: its residue scratch is a fixed 64 MiB
 * device array inside this library (held on every GPU that loads the library until exit), so
 * it serves callers that cannot call cudaMalloc while computing -- e.g. a host framework whose
 * caching allocator owns the device memory, or a latency-critical path that cannot take
 * cudaMalloc's implicit synchronisation (pm_run_device may allocate to grow its scratch).
 * Limit: K*N <= 8,388,608 residue words per operand (N = 65536 up to W = 1747); larger points
 * return PM_ERR_INVALID.  Asynchronous on `stream`; pm_sync() reports device-side checks.
 * All calls share the scratch array: calls that overlap on the GPU race, so serialise them.
 * The first call on a device looks up the array's device address; make it before any stream
 * capture.  pm_free forgets that address (free every context of a device before a
 * cudaDeviceReset, after which it would be stale).  The context must come from an earlier
 * pm_init (which does allocate).  Like the other entry points that run a context, it leaves the
 * caller's current device as it found it; errors map as pm_run_device's do. */
int pm_run_device_static(pm_context* ctx, const uint32_t* d_a, const uint32_t* d_b, uint32_t* d_c, void* stream);

/* ---- Batches of multiplications of uneven points.  No reference counterpart: the reference
 * multiplies one pair per fherma_run call (solve.cu:1480-1498) with fixed split and chunking
 * heuristics (solve.cu:85-87, 917-918, 1403-1419).
 *
 * A batch is a list of classes, each one point (N, W, q) and `count` multiplications of it
 * whose operands lie contiguously in device memory.  pm_batch_init builds every class's
 * tables, allocates the residue scratch once, and captures the whole schedule -- one launch
 * per kernel per class, classes spread over up to 8 streams -- into a CUDA graph;
 * pm_batch_run replays it with one graph launch.  The operand pointers are captured: write
 * new inputs into the same buffers between runs.  With PM_BATCH_TUNE each class's
 * configuration is chosen by timing the candidates on the class's operands: first the 4-step
 * split and the GEMM form, then the column-pass kernel (TMA pipeline or one tile per CTA), the
 * CRT GEMM's A-operand placement (tensor or shared memory) and the number of launch groups the
 * class runs in (1, 2 or 4; fewer multiplies per group need less scratch).  Results are cached
 * in $POLYMULT_TUNE_CACHE (default ~/.cache/polymult_b200/tune.txt); the tuning runs write the
 * outputs.  Results are bit-identical whatever the choice. */
typedef struct pm_batch pm_batch;

typedef struct pm_batch_class {
    uint32_t N, W, L;
    const uint32_t* q;   /* host memory, L limbs (copied by pm_batch_init) */
    uint32_t count;      /* multiplications of this point (0 allowed) */
    const uint32_t* d_a; /* device memory, [count][N][L] */
    const uint32_t* d_b; /* device memory, [count][N][L] */
    uint32_t* d_c;       /* device memory, [count][N][L] */
    int32_t w1;          /* 4-step split nrows = 2^w1 (both line lengths <= 2^10); -1: default or tuned */
} pm_batch_class;

enum pm_batch_flags {
    PM_BATCH_TUNE = 1,     /* measure and choose split, GEMM form, kernel variants and launch groups per class */
    PM_BATCH_NO_GRAPH = 2  /* launch the schedule directly on every run instead of a graph */
};

typedef struct pm_batch_info {
    uint32_t classes;
    uint32_t streams;        /* streams the classes are spread over */
    int32_t kernel_launches; /* kernels per run */
    uint64_t graph_nodes;    /* nodes of the captured graph (0 with PM_BATCH_NO_GRAPH) */
    uint64_t scratch_bytes;  /* device residue scratch of the batch */
} pm_batch_info;

typedef struct pm_batch_class_info {
    int32_t K, w1, w2;
    int32_t gemm_form;  /* PM_GEMM_PLAIN or PM_GEMM_TENSOR */
    double tuned_ms;    /* measured ms of the chosen configuration; 0 untuned, -1 from the cache */
    int32_t col_tma;    /* 1: column passes by the TMA-pipelined kernel (256-row lines), 0: one tile per CTA */
    int32_t crt_tm;     /* 1: CRT GEMM with its A operand in tensor memory, 0: in shared memory (or plain) */
    uint32_t launch_groups; /* the class's multiplications run as this many launch groups */
} pm_batch_class_info;

int pm_batch_init(const pm_batch_class* classes, uint32_t nclasses, int gemm_form, int flags, int device,
                  pm_batch** out);
/* Asynchronous on `stream` (NULL = legacy default stream); pm_batch_sync waits. */
int pm_batch_run(pm_batch* batch, void* stream);
/* Waits for the batch's device work; PM_ERR_DEVICE if a device-side check failed. */
int pm_batch_sync(pm_batch* batch);
int pm_batch_get_info(const pm_batch* batch, pm_batch_info* out);
int pm_batch_get_class(const pm_batch* batch, uint32_t index, pm_batch_class_info* out);
void pm_batch_free(pm_batch* batch);

/* ---- Serving.  No reference counterpart (the reference serves one fherma_run call at a time,
 * main.cpp:181-186).  A server holds one point and `nresident` fixed operands, uploaded once and
 * kept on the device in NTT form (decomposed and forward-transformed).  pm_server_run plays a
 * stream of requests: request i arrives t_arrive[i] seconds after the call starts and asks for
 * c[i] = a[i] * resident[sel[i]] (a[i], c[i]: host buffers of N*L words; pinned ones from
 * pm_server_host_alloc let the copies run asynchronously).  Continuous batching: whenever one of
 * the server's `streams` slots is free, it takes every queued request up to its capacity,
 * whatever their resident operand, and runs them as one batch while other slots' batches are on
 * the GPU.  Admission: each request in flight holds 8NL + 4KN bytes of device memory; with the
 * resident transforms and tables, the total stays within hbm_budget bytes.  Each result is
 * bit-identical to the same multiplication run alone.  Synchronous; fills latency[i] (seconds,
 * completion - arrival) and *stats. */
typedef struct pm_server pm_server;

typedef struct pm_serve_stats {
    uint64_t requests;
    uint64_t batches;
    double mean_batch;       /* requests per launched batch */
    uint32_t peak_inflight;  /* most requests in flight at once */
    uint32_t max_inflight;   /* the admission limit the budget gives */
    double seconds;          /* first arrival to last completion */
} pm_serve_stats;

int pm_server_init(uint32_t N, uint32_t W, uint32_t L, const uint32_t* q, const uint32_t* resident, uint32_t nresident,
                   uint64_t hbm_budget, uint32_t max_batch, uint32_t streams, int gemm_form, int device,
                   pm_server** out);
/* digest: NULL, or n entries; digest[i] receives pm_digest of request i's result, computed on the
 * device from the result itself before its copy to c[i] (so a long stream can reuse its host
 * result buffers and still have every result checked). */
int pm_server_run(pm_server* server, uint32_t n, const double* t_arrive, const uint32_t* sel,
                  const uint32_t* const* a, uint32_t* const* c, double* latency, pm_serve_stats* stats,
                  uint64_t* digest);
/* Pinned host memory owned by the server (freed by pm_server_free if not before). */
int pm_server_host_alloc(pm_server* server, size_t bytes, void** out);
int pm_server_host_free(pm_server* server, void* p);
void pm_server_free(pm_server* server);

/* The host pipeline's column-chunk schedule.  The reference fixes it (make_chunks,
 * solve.cu:1085-1108, with the divisors of solve.cu:1403-1405). */
typedef struct pm_pipeline_info {
    int32_t in_chunks, out_chunks;  /* column chunks per input operand / of the output */
    int32_t in_body, out_body;      /* body chunk = ncols / divisor */
    double tuned_ms;                /* median pm_run time of the chosen schedule (0: not tuned) */
} pm_pipeline_info;

/* pm_run keeps two schedules: one for calls whose buffers it stages through its host threads
 * (pageable memory; the reference's case) and one for calls whose a, b and c are all
 * page-locked (cudaHostAlloc / cudaHostRegister), which it copies chunk by chunk with strided
 * DMA copies and no host staging.  `flags` selects the second with PM_PIPELINE_PINNED. */
#define PM_PIPELINE_PINNED 1

/* No reference counterpart: the autotuner of the host pipeline.  Runs `reps` pm_run calls (plus
 * a warm-up) for every schedule with body divisors in {1, 2, 4, 8, 16} x {1, 2, 4, 8, 16} on
 * pageable timing buffers (narrow head chunks only with a body of 8 or more; with
 * PM_PIPELINE_PINNED: {1, 2, 3, 4, 5, 8, 16} squared on page-locked ones, 3 standing for the
 * chunks 1/2, 1/4, 1/4 of b and 1/4, 1/4, 1/2 of c, and 5 for 1/2, 1/4, 1/8, 1/8 of b and
 * 1/8, 1/8, 1/4, 1/2 of c), keeps the one with the lowest median wall time for that kind of
 * call, and describes it in *out.  Before any tuning the schedules follow the operand size (one
 * chunk below 1 MB, quarters below 8 MB, eighths above).  Synchronous; up to 25
 * (PM_PIPELINE_PINNED: 49) x (reps + 1) calls. */
int pm_tune_pipeline(pm_context* ctx, int reps, int flags, pm_pipeline_info* out);
int pm_get_pipeline(const pm_context* ctx, int flags, pm_pipeline_info* out);
/* No reference counterpart: sets the schedule of one kind of call (flags as above) to body
 * divisors `in_body` / `out_body` -- powers of two up to ncols, or for PM_PIPELINE_PINNED also
 * 3 and 5 (the uneven shapes of pm_tune_pipeline) -- without measuring, e.g. to reuse a
 * schedule tuned earlier.  PM_ERR_INVALID for another divisor. */
int pm_set_pipeline(pm_context* ctx, int flags, int32_t in_body, int32_t out_body);

/* Waits for the context's device work and returns PM_ERR_DEVICE if a device-side check
 * failed since the last call. */
int pm_sync(pm_context* ctx);

/* Replaces fherma_free (solve.cu:1530-1534). NULL is accepted. */
void pm_free(pm_context* ctx);

int pm_get_info(const pm_context* ctx, pm_info* out);

/* Message of the last failure on this thread ("" if none). */
const char* pm_last_error(void);

/* Host-only: builds the plan of a point without touching a GPU and runs its self-checks
 * (primes, roots of unity, CRT reconstruction of random values through the tables).
 * Fills *K_out with the prime count.  Usable on a machine without a GPU. */
int pm_plan_selfcheck(uint32_t N, uint32_t W, uint32_t L, const uint32_t* q, int32_t* K_out);

/* Host-only: stress test of the thread pool that stages pm_run's pageable operands.  Creates
 * `pools` pools of `workers` threads and runs `runs` task sets on each, counting task sets where
 * a task ran other than once or was still running when the set returned.  *failures gets that
 * count (0 expected).  `vary` bit 0: task counts 1..64 instead of 64 every time; bit 1: workers
 * park between task sets (20 us idle limit, a 300 us pause before every third set) so that each
 * set has to wake them; bit 2: every other set is opened without the caller (the pipeline's
 * asynchronous staging) and joined after some work of the caller.  No GPU needed. */
int pm_selftest_host_pool(uint32_t pools, uint32_t runs, uint32_t workers, int vary, uint64_t* failures);

/* Test hook, host-only: after `skip` more residue-scratch allocations of any context (each
 * context's scratch is two arrays), the next `n` fail as if cudaMalloc had run out of device
 * memory; the calls that needed them return PM_ERR_CUDA and the context holds no scratch until
 * a later call allocates it again.  Lets tests drive the allocation-failure path without
 * exhausting a shared GPU.  (0, 0) switches the injection off. */
void pm_test_fail_scratch_allocs(int skip, int n);

/* No reference counterpart: 64-bit digests of `count` arrays of `words` u32 words each, lying
 * contiguously in device memory (results of pm_run_device, for instance), into out[count] (host
 * memory).  D(x) = sum over i of mix(i << 32 | x_i) mod 2^64, mix the splitmix64 finalizer; equal
 * arrays give equal digests, and pm_digest_host computes the same value for host memory.
 * Synchronous on `stream`. */
int pm_digest(const uint32_t* d_words, uint64_t words, uint32_t count, void* stream, uint64_t* out);
uint64_t pm_digest_host(const uint32_t* words, uint64_t n);

/* Test hook: writes `bits` (PM_DEVICE_* below) into the context's device status word, as a
 * failed device-side check would; the next pm_sync or pm_run then reports PM_ERR_DEVICE and
 * clears the word.  Waits for the context's device work first. */
int pm_test_set_status(pm_context* ctx, uint32_t bits);
#define PM_DEVICE_CRT_BOUND 1u /* fp32 CRT estimate not within 1/4 of an integer (|x| < M/8 violated) */
#define PM_DEVICE_FOLD 2u      /* CRT value above its bound after the folds */
#define PM_DEVICE_WAIT 4u      /* an mbarrier wait of a tensor-core kernel ran out */

/* No reference counterpart (the reference's waits are host-side, solve.cu:814-816): the bounded
 * mbarrier waits of the tensor-core kernels, made to run out.  One block of 64 threads waits
 * with a limit of `limit_clocks` (1 .. 2e9) on an mbarrier that nothing arrives on, as the
 * kernels' waits do (one thread alone, and a warp sharing an abort flag); each must give up and
 * report PM_DEVICE_WAIT in *status_out.  Then the phase is completed and every thread's wait must
 * succeed (bit 8 of *status_out otherwise).  Nothing is in flight while they wait, so the context
 * stays usable.  Synchronous. */
int pm_selftest_wait(int device, uint64_t limit_clocks, uint32_t* status_out);

/* No reference counterpart: the measured ceiling of the NTT's arithmetic.  Runs the NTT's
 * Harvey-Shoup butterfly (two low 32-bit multiplies, one 64-bit product, three adds) on register
 * operands, no memory traffic, over every SM of `device`, and gives the rate in butterflies per
 * second and per clock per SM (at the device's reported SM clock).  The NTT kernels are bound by
 * the integer multiply-add pipe this exercises, so their butterfly rate against this one is their
 * roofline fraction.  PM_ERR_DEVICE if the kernel's checksum differs from a host recomputation.
 * Synchronous; a few milliseconds. */
int pm_butterfly_peak(int device, double* bfly_per_s, double* bfly_per_clk_sm);

#ifdef __cplusplus
}
#endif

#endif /* POLYMULT_B200_H */
