// pm_static_scratch.cu -- pm_run_device_static: the device-resident multiply with its residue
// scratch in a fixed device array compiled into this library, so that the call allocates
// nothing.
//
// Who needs it: callers that cannot call cudaMalloc while they compute.  Examples are a host
// framework that owns the device memory through its own caching allocator (it has reserved the
// free memory, so a cudaMalloc from a library may fail, or force it to give memory back), and
// latency-critical paths where cudaMalloc's implicit device-wide synchronisation is not
// acceptable.  pm_run_device may cudaMalloc (it grows its scratch for larger batches); this
// entry point never does.  The context itself (tables, status word) comes from pm_init, which
// allocates, so such callers create their context once at start-up.
//
// The scratch is `g_residue_scratch`: 16 Mi words (64 MiB), two residue arrays of up to
// kStaticScratchWords / 2 = 8 Mi words each, i.e. K*N <= 8,388,608 (N = 65536 with up to 128
// primes, which covers W = 1747).  Every GPU that loads this library holds those 64 MiB until
// the process exits.  Every call shares the array and it keeps the last call's contents;
// nothing in it has to start at zero (each call overwrites the residues before reading them).
// Calls that overlap on the GPU (different streams or threads, with no ordering between them)
// race on the array and give wrong results: serialise them.
//
// In host code `g_residue_scratch` names a host-side stand-in, not device memory, so it is never
// passed to a kernel.  The device address is looked up once per device, with that device
// current, by cudaGetSymbolAddress, on the first call on that device; make that first call
// before any stream capture.
#include <cstdint>
#include <mutex>
#include <string>

#include "../../include/polymult_b200.h"
#include "pm_context.h"

namespace pm {
int fail(int code, const char* what);
extern thread_local std::string g_last_error;
}  // namespace pm

namespace {

constexpr size_t kStaticScratchWords = size_t(16) << 20;  // 64 MiB
__device__ __align__(256) uint32_t g_residue_scratch[kStaticScratchWords];

constexpr int kMaxDevices = 64;
std::mutex g_lookup_mutex;
uint32_t* g_device_address[kMaxDevices] = {};

// Device address of g_residue_scratch on `device` (which must be current).
cudaError_t scratch_address(int device, uint32_t** out) {
    std::lock_guard<std::mutex> lk(g_lookup_mutex);
    if (!g_device_address[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_residue_scratch);
        if (e != cudaSuccess) return e;
        g_device_address[device] = static_cast<uint32_t*>(p);
    }
    *out = g_device_address[device];
    return cudaSuccess;
}

}  // namespace

extern "C" int pm_run_device_static(pm_context* ctx, const uint32_t* d_a, const uint32_t* d_b, uint32_t* d_c,
                                    void* stream) {
    if (!ctx || !ctx->engine) return pm::fail(PM_ERR_INVALID, "null context");
    if (!d_a || !d_b || !d_c) return pm::fail(PM_ERR_INVALID, "null operand");
    pm::Engine& e = *ctx->engine;
    const size_t words = (size_t)e.plan().K * e.plan().N;
    if (2 * words > kStaticScratchWords) {
        return pm::fail(PM_ERR_INVALID,
                        ("pm_run_device_static: K*N = " + std::to_string(words) + " residue words per operand exceeds the " +
                         std::to_string(kStaticScratchWords / 2) + " of the static scratch; use pm_run_device")
                            .c_str());
    }
    const int dev = e.device();
    if (dev < 0 || dev >= kMaxDevices) return pm::fail(PM_ERR_INVALID, "device index out of range");
    cudaError_t ce = cudaSetDevice(dev);
    if (ce != cudaSuccess) return pm::fail(PM_ERR_CUDA, cudaGetErrorString(ce));
    uint32_t* ra = nullptr;
    ce = scratch_address(dev, &ra);
    if (ce != cudaSuccess)
        return pm::fail(PM_ERR_CUDA, (std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(ce)).c_str());
    try {
        e.run_device_with_scratch(d_a, d_b, d_c, ra, ra + words, static_cast<cudaStream_t>(stream));
    } catch (const std::exception& ex) {
        return pm::fail(PM_ERR_CUDA, ex.what());
    }
    pm::g_last_error.clear();
    return PM_OK;
}
