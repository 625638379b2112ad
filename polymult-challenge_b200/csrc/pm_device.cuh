// pm_device.cuh -- device-side parameters and modular arithmetic shared by every kernel.
//
// Residue arithmetic modulo p < 2^30 with R = 2^32:
//   * Montgomery-Shoup product by a constant w held in Montgomery form (w R mod p) with its
//     companion wc = w p^-1 mod 2^32: three integer multiplies, result in (0, 2p) for any
//     32-bit multiplicand.  It replaces the reference's REDC-based mont_mul
//     (solve.cu:123-130), which needs a 64-bit product and a wide add for every butterfly.
//   * Harvey's lazy butterflies: forward values stay in [0, 4p), inverse values in [0, 2p),
//     because 4p < 2^32.  The reference reduces to [0, p) after every butterfly
//     (solve.cu:131-138, 230-241).
#pragma once

#include <cstdint>

namespace pm {

// Device status word bits (read back by the host after a run).
enum : uint32_t {
    DEV_ERR_CRT_BOUND = 1u,   // fp32 CRT estimate not within 1/4 of an integer (|x| < M/8 violated)
    DEV_ERR_FOLD = 2u,        // the CRT value had bits above 2^W after its folds (outside its bound)
    DEV_ERR_WAIT = 4u,        // an mbarrier wait hit its iteration limit
};

// Per-point device view of the plan.  POD, passed by value.
struct DevPlan {
    uint32_t N, nrows, ncols;
    int logN, w1, w2;
    int K, KP, L, W;
    int D, DP;                // 24-bit digits of a W-bit value (DP: rounded up to a multiple of 4)
    int fold_count;           // CRT folds z -> (z mod 2^W) + (z >> W) delta before the final -q
    int Kr;                   // primes of the residue arrays R[batch][Kr][N] (K except in a prime block)
    uint64_t delta;
    const uint32_t* p;        // [KP]
    const uint32_t* pinv;     // [KP] p^-1 mod 2^32
    const uint32_t* crt_c;    // [KP]
    const uint32_t* crt_cc;   // [KP]
    const float* rcp;         // [KP]
    const uint2* tw;          // [K][N] {psi^bitrev(k), floor(psi^bitrev(k) 2^32 / p)} (Shoup form)
    const uint32_t* dec24;    // [DP][KP] 2^(24 d) R mod p_j
    const uint32_t* crt24;    // [K+1][DP] 24-bit digits of Q_j = (M/p_j) mod q; row K: of T_1
    const uint32_t* t1;       // [L] T_1 = (-M) mod q
    const uint32_t* q;        // [L]
    const uint8_t* dec_b;     // tensor-core decomposition B operand (canonical image)
    const uint8_t* dec_b_ra;  // the same, constants times gamma_j = crt_c_j 2^-32 (operand RA)
    const uint8_t* crt_b;     // tensor-core CRT B operand (canonical image)
    int crt_kv;               // CRT K-byte column of v (B column: the bytes of T_1)
    int dec_nrows, dec_kbytes;
    int crt_nrows, crt_kbytes;
    uint32_t* status;         // device status word
    long long wait_clocks;    // limit of every mbarrier wait of the tcgen05 and TMA kernels (2e9 clocks, ~1 s)
    int col_tma;              // host-side choice: column passes of 64-column tiles take the TMA kernel
};

// A chunk of coefficient positions: all rows x `cw` columns starting at `col0`, stored
// row-major as [row][column-in-chunk][limb].  With col0 = 0 and cw = ncols this is the
// natural [N][L] layout.  Position pos maps to coefficient n = (pos / cw) * ncols + col0 + pos % cw.
struct ChunkMap {
    uint32_t col0, cw;
    int lcw;  // log2(cw)
};

// Prime blocks of one result-byte block of the tensor-core CRT, accumulated in TMEM within one
// launch: block q holds primes j0[q] .. j0[q] + k[q] (kp[q] padded, kb[q] K bytes, B image b[q]
// of this byte block), each tile's MMAs over the blocks in turn.  n = 0: one block, the
// launch's DevPlan.
struct CrtPrimeBlocks {
    static constexpr int MAX = 8;
    int n;
    int j0[MAX], k[MAX], kp[MAX], kb[MAX];
    const unsigned char* b[MAX];
};

__device__ __forceinline__ uint32_t chunk_pos_to_n(const DevPlan& P, const ChunkMap& C, uint32_t pos) {
    return ((pos >> C.lcw) << P.w2) + C.col0 + (pos & (C.cw - 1));
}

// x * w * 2^-32 mod p in (0, 2p); w < p in Montgomery form, wc = w * p^-1 mod 2^32.
__device__ __forceinline__ uint32_t mul_ms(uint32_t x, uint32_t w, uint32_t wc, uint32_t p) {
    const uint32_t m = x * wc;
    return __umulhi(x, w) - __umulhi(m, p) + p;
}

// a * b * 2^-32 mod p in (0, 2p); requires a * b < p * 2^32.  The product a * b is formed once
// as a 64-bit value (one wide multiply for both halves), which measured 1.5% faster in the
// row pass, whose integer multiply-add pipe is the binding one, than a low and a high multiply.
__device__ __forceinline__ uint32_t mont_mul(uint32_t a, uint32_t b, uint32_t p, uint32_t pinv) {
    const uint64_t t = (uint64_t)a * b;
    const uint32_t m = (uint32_t)t * pinv;
    return (uint32_t)(t >> 32) - __umulhi(m, p) + p;
}

// t * 2^-32 mod p in (0, 2p) for a 64-bit t < p * 2^32 (the high product from one 64-bit
// multiply, as in mont_mul).
__device__ __forceinline__ uint32_t redc64(uint64_t t, uint32_t p, uint32_t pinv) {
    const uint32_t m = (uint32_t)t * pinv;
    return (uint32_t)(t >> 32) - (uint32_t)(((uint64_t)m * p) >> 32) + p;
}

// [0, 2m) -> [0, m) (also [0, 4p) -> [0, 2p) with m = 2p): unsigned min of x and x - m (one
// fused add-and-min instruction on this architecture).
__device__ __forceinline__ uint32_t red_once(uint32_t x, uint32_t m) { return min(x, x - m); }

// A twiddle in Shoup form: w < p and wc = floor(w 2^32 / p).
struct Tw2 {
    uint32_t w, wc;
};

// Shoup product: x * w mod p in [0, 2p) for any x < 2^32, w < p plain and wsh = floor(w 2^32 / p)
// (the quotient estimate umulhi(x, wsh) is at most one below floor(x w / p)).
__device__ __forceinline__ uint32_t mul_sh(uint32_t x, uint32_t w, uint32_t wsh, uint32_t p) {
    return x * w - (uint32_t)(((uint64_t)x * wsh) >> 32) * p;
}

// Cooley-Tukey butterfly with a Shoup twiddle {w, wsh}: x, y in [0, 4p) -> [0, 4p).
// Three multiplies (one high) and three adds / one fused add-and-min.
__device__ __forceinline__ void bfly_ct_sh(uint32_t& x, uint32_t& y, Tw2 w, uint32_t p) {
    const uint32_t p2 = 2 * p;
    const uint32_t xr = red_once(x, p2);
    const uint32_t t = mul_sh(y, w.w, w.wc, p);
    x = xr + t;
    y = xr - t + p2;
}

// Gentleman-Sande (inverse) butterfly with the mirrored Shoup twiddle: x, y in [0, 2p) ->
// x + y, (y - x) w in [0, 2p).  (x - y) psi^-b = (y - x) psi^b' with b + b' = N.
__device__ __forceinline__ void bfly_gs_sh(uint32_t& x, uint32_t& y, Tw2 w, uint32_t p) {
    const uint32_t p2 = 2 * p;
    const uint32_t s = x + y;
    const uint32_t d = y - x + p2;
    x = red_once(s, p2);
    y = mul_sh(d, w.w, w.wc, p);
}

// Programmatic dependent launch.  A kernel launched with programmatic stream serialization may
// start while the kernel before it in the stream is still running.  pdl_wait() returns once
// that kernel has completed and its memory operations are visible (at once after an ordinary
// launch), so a kernel touches only shared memory, TMEM and the plan's constant tables before
// it.  pdl_trigger() lets the next kernel's blocks launch, so that their prologues overlap this
// kernel's tail; it takes effect once every block of this grid has called it or exited.
// Kernels that allocate TMEM call it only after their own allocation: a dependent block on the
// same SM could otherwise hold the columns while it waits for this kernel to finish.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

__device__ __forceinline__ void flag_error(uint32_t* status, uint32_t bit) {
    if (status) atomicOr(status, bit);
}

}  // namespace pm
