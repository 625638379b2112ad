// k_peak.cu -- the measured ceiling of the NTT's arithmetic: Harvey–Shoup butterflies per second
// on this GPU, with the operands in registers (no memory traffic, no twiddle loads).
//
// Every NTT kernel here is bound by the integer multiply-add pipe, not by HBM: a Shoup
// butterfly is two low 32-bit multiplies and one 64-bit product, and that pipe takes the wide
// product at about 25 per clock per SM against 64 for a low multiply.  This kernel runs the
// exact butterfly of the NTT (bfly_ct_sh, pm_device.cuh) over 16 register values per thread,
// radix-2 stages on four twiddles, so that the NTT kernels' butterfly rates can be set against
// the rate of the butterfly alone.  Each thread also reports a checksum (XOR of its values
// reduced mod p), which the host recomputes for thread 0 to confirm the work was done.
#include "pm_engine.h"
#include "pm_kernels.cuh"

namespace pm {
namespace {

constexpr int PEAK_ITER = 256;     // rounds of 4 stages x 8 butterflies per thread
constexpr int PEAK_THREADS = 512;
constexpr int PEAK_BLOCKS_PER_SM = 2;

__global__ void __launch_bounds__(PEAK_THREADS) k_bfly_peak(Tw2 w0, Tw2 w1, Tw2 w2, Tw2 w3, uint32_t p,
                                                            uint32_t* __restrict__ out) {
    uint32_t v[16];
    const uint32_t gt = blockIdx.x * blockDim.x + threadIdx.x;
#pragma unroll
    for (int e = 0; e < 16; ++e) v[e] = (gt * 16u + (uint32_t)e) * 2654435761u % (4u * p);
    const Tw2 w[4] = {w0, w1, w2, w3};
    for (int it = 0; it < PEAK_ITER; ++it) {
#pragma unroll
        for (int st = 0; st < 4; ++st) {
#pragma unroll
            for (int e = 0; e < 16; ++e) {
                if (e & (1 << st)) continue;
                bfly_ct_sh(v[e], v[e + (1 << st)], w[st], p);
            }
        }
    }
    uint32_t r = 0;
#pragma unroll
    for (int e = 0; e < 16; ++e) r ^= v[e] % p;
    out[gt] = r;
}

}  // namespace

// Host side of pm_butterfly_peak: butterflies per second over the whole GPU and per clock per
// SM (from the SM clock the device reports), and whether thread 0's checksum matches a host
// recomputation of the same butterflies.
void butterfly_peak(int device, double* per_s, double* per_clk_sm, bool* checked) {
    cuda_check(cudaSetDevice(device), "cudaSetDevice");
    int sms = 0, clk_khz = 0;
    cuda_check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "attribute");
    cuda_check(cudaDeviceGetAttribute(&clk_khz, cudaDevAttrClockRate, device), "attribute");
    const uint32_t p = 1073479681u;  // a prime below 2^30
    Tw2 w[4];
    for (int t = 0; t < 4; ++t) {
        const uint32_t x = (uint32_t)((123456789ull * (uint64_t)(t + 3)) % p);
        w[t] = Tw2{x, (uint32_t)(((unsigned __int128)x << 32) / p)};
    }
    const int blocks = sms * PEAK_BLOCKS_PER_SM;
    const size_t nthreads = (size_t)blocks * PEAK_THREADS;
    uint32_t* d_out = nullptr;
    cuda_check(cudaMalloc(&d_out, nthreads * 4), "cudaMalloc");
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    float ms = 0.f;
    uint32_t r0 = 0;
    try {
        cuda_check(cudaEventCreate(&e0), "event");
        cuda_check(cudaEventCreate(&e1), "event");
        k_bfly_peak<<<blocks, PEAK_THREADS>>>(w[0], w[1], w[2], w[3], p, d_out);  // warm-up
        cuda_check(cudaEventRecord(e0), "record");
        const int reps = 5;
        for (int r = 0; r < reps; ++r) k_bfly_peak<<<blocks, PEAK_THREADS>>>(w[0], w[1], w[2], w[3], p, d_out);
        cuda_check(cudaEventRecord(e1), "record");
        cuda_check(cudaEventSynchronize(e1), "sync");
        cuda_check(cudaGetLastError(), "launch k_bfly_peak");
        cuda_check(cudaEventElapsedTime(&ms, e0, e1), "elapsed");
        ms /= reps;
        cuda_check(cudaMemcpy(&r0, d_out, 4, cudaMemcpyDeviceToHost), "D2H");
    } catch (...) {
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        cudaFree(d_out);
        throw;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(d_out);
    const double bfly = (double)nthreads * PEAK_ITER * 32.0;
    *per_s = bfly / (ms * 1e-3);
    *per_clk_sm = *per_s / ((double)clk_khz * 1e3 * sms);
    // thread 0 on the host: the same values, butterflies and checksum
    uint32_t v[16];
    for (int e = 0; e < 16; ++e) v[e] = ((uint32_t)e * 2654435761u) % (4u * p);
    for (int it = 0; it < PEAK_ITER; ++it)
        for (int st = 0; st < 4; ++st)
            for (int e = 0; e < 16; ++e) {
                if (e & (1 << st)) continue;
                uint32_t& x = v[e];
                uint32_t& y = v[e + (1 << st)];
                const uint32_t p2 = 2 * p;
                const uint32_t xr = x < p2 ? x : x - p2;
                const uint32_t t = y * w[st].w - (uint32_t)(((uint64_t)y * w[st].wc) >> 32) * p;
                x = xr + t;
                y = xr - t + p2;
            }
    uint32_t r = 0;
    for (int e = 0; e < 16; ++e) r ^= v[e] % p;
    *checked = r == r0;
}

}  // namespace pm
