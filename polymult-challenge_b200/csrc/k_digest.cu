// k_digest.cu -- a 64-bit digest of result arrays, computed where they are.
//
// D(x) = sum_i mix(i << 32 | x_i) mod 2^64 over the words x_i of one array, with mix the
// splitmix64 finalizer (Steele, Lea and Flood, "Fast splittable pseudorandom number generators",
// 2014).  A sum of per-position hashes is order-free, so the device form reduces it in any order
// with 64-bit atomic adds and the host form (digest_host) gives the same value.  It lets a caller
// check every result of a run -- the server's requests, whose host result buffers a long stream
// reuses -- against expected values without copying the results back.
#include "pm_kernels.cuh"

namespace pm {

__host__ __device__ inline uint64_t digest_mix(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// grid (blocks, count): array z = blockIdx.y of `words` words; out[z] must start at zero
__global__ void __launch_bounds__(256) k_digest(const uint32_t* __restrict__ x, uint64_t words,
                                                unsigned long long* __restrict__ out) {
    const uint32_t* xz = x + (size_t)blockIdx.y * words;
    uint64_t acc = 0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < words; i += (uint64_t)gridDim.x * blockDim.x)
        acc += digest_mix((i << 32) | __ldg(xz + i));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(out + blockIdx.y, (unsigned long long)acc);
}

void launch_digest(const uint32_t* x, uint64_t words, uint32_t count, uint64_t* out_dev, cudaStream_t s) {
    if (count == 0) return;
    cudaError_t e = cudaMemsetAsync(out_dev, 0, (size_t)count * 8, s);
    if (e != cudaSuccess) throw_cuda(e, "digest clear");
    const uint64_t per_block = 256 * 16;
    const unsigned blocks = (unsigned)std::min<uint64_t>(1024, (words + per_block - 1) / per_block);
    e = launch_kernel(k_digest, dim3(std::max(1u, blocks), count), dim3(256), 0, s, false, x, words,
                      reinterpret_cast<unsigned long long*>(out_dev));
    if (e != cudaSuccess) throw_cuda(e, "launch k_digest");
}

uint64_t digest_host(const uint32_t* x, uint64_t words) {
    uint64_t acc = 0;
    for (uint64_t i = 0; i < words; ++i) acc += digest_mix((i << 32) | x[i]);
    return acc;
}

}  // namespace pm
