// pm_static_scratch.cu -- the scratch of pm_run_device_static: the device-resident multiply
// with its residue scratch in a fixed device array compiled into this library, so that the
// call allocates nothing.
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
// before any stream capture.  pm_free forgets the looked-up address of its context's device,
// so the next call looks it up again (after a cudaDeviceReset the old address is stale: free
// every context of a device before resetting it).
#include <cstdint>
#include <mutex>
#include <string>

#include "pm_engine.h"
#include "pm_kernels.cuh"

constexpr size_t kStaticScratchWords = size_t(16) << 20;  // 64 MiB
static __device__ __align__(256) uint32_t g_residue_scratch[kStaticScratchWords];

namespace pm {
namespace {

constexpr int kMaxDevices = 64;
std::mutex g_lookup_mutex;
uint32_t* g_device_address[kMaxDevices] = {};

// Device address of g_residue_scratch on `device` (which must be current).
uint32_t* scratch_address(int device) {
    std::lock_guard<std::mutex> lk(g_lookup_mutex);
    if (!g_device_address[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_residue_scratch);
        if (e != cudaSuccess) throw_cuda(e, "cudaGetSymbolAddress of the static scratch");
        g_device_address[device] = static_cast<uint32_t*>(p);
    }
    return g_device_address[device];
}

}  // namespace

// The body of pm_run_device_static (pm_capi.cpp maps its exceptions to status codes and
// restores the caller's current device).
void run_device_static(Engine& e, const uint32_t* d_a, const uint32_t* d_b, uint32_t* d_c, cudaStream_t stream) {
    const size_t words = (size_t)e.plan().K * e.plan().N;
    if (2 * words > kStaticScratchWords)
        throw InvalidPoint("pm_run_device_static: K*N = " + std::to_string(words) +
                           " residue words per operand exceeds the " + std::to_string(kStaticScratchWords / 2) +
                           " of the static scratch; use pm_run_device");
    const int dev = e.device();
    if (dev < 0 || dev >= kMaxDevices) throw InvalidPoint("device index out of range");
    cuda_check(cudaSetDevice(dev), "cudaSetDevice");
    uint32_t* ra = scratch_address(dev);
    e.run_device_with_scratch(d_a, d_b, d_c, ra, ra + words, stream);
}

void forget_static_scratch_address(int device) {
    if (device < 0 || device >= kMaxDevices) return;
    std::lock_guard<std::mutex> lk(g_lookup_mutex);
    g_device_address[device] = nullptr;
}

}  // namespace pm
