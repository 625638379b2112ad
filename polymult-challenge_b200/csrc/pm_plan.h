// pm_plan.h -- host-side precompute for one (N, W, q) point: RNS primes, twiddle tables,
// the constants of the plain (CUDA-core) GEMMs, the byte-sliced operand images of the
// tensor-core GEMMs, and the bound that fixes the CRT's fold count.  Pure C++ (no CUDA), so
// the host logic is testable on a machine without a GPU.
//
// Replaces the reference's precompute() (solve.cu:869-1020) with a different design:
//   * primes p < 2^30 with p == 1 (mod 2 max(N, 2^16)), found by trial division against a
//     sieve of the primes below 2^15: below 2^30, 4p < 2^32, so every NTT stage keeps its values
//     lazily in [0, 4p) (Harvey butterflies), and one prime list serves every N <= 2^16, which
//     the batched path relies on;
//   * psi from a quadratic non-residue (the 2-power part of the multiplicative group,
//     Tonelli-Shanks style) instead of a search over candidate generators;
//   * M / p_j by exact division of the bigint M, which gives both (M / p_j) mod p_j and
//     Q_j = (M / p_j) mod q;
//   * the plain GEMMs work on 24-bit digits (the reference's on 16-bit halves).
#pragma once

#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace pm {

// Thrown for an invalid point; the C ABI maps it to PM_ERR_INVALID (the reference throws
// std::runtime_error from precompute for the same conditions, solve.cu:873-913).
struct InvalidPoint : std::runtime_error {
    explicit InvalidPoint(const std::string& s) : std::runtime_error(s) {}
};

// Shape of the byte-sliced tensor-core GEMMs (UMMA K-major, no-swizzle canonical layout:
// core matrices of 8 rows x 16 bytes, LBO = 128 B between K-adjacent core matrices,
// SBO = 8 * k_bytes between 8-row groups).
struct GemmShape {
    int n_rows = 0;    // UMMA N (rows of the K-major B operand), multiple of 16
    int k_bytes = 0;   // UMMA K in bytes, multiple of 32
    size_t b_bytes() const { return (size_t)n_rows * k_bytes; }
};

// Bits per digit of the plain GEMMs.  A 30-bit factor times a 24-bit digit is below 2^54, so
// up to 1023 such products sum exactly in 64 bits.
constexpr int kDigitBits = 24;

struct Plan {
    // point
    uint32_t N = 0, W = 0, L = 0;
    int logN = 0, w1 = 0, w2 = 0;     // 4-step split: nrows = 2^w1 (column pass), ncols = 2^w2
    uint32_t nrows = 1, ncols = 1;
    std::vector<uint32_t> q;          // [L]
    uint64_t delta = 0;               // 2^W - q (< 2^63)

    // RNS
    int K = 0;                        // primes
    int KP = 0;                       // K rounded up to a multiple of 4
    uint64_t prime_step = 0;          // primes are == 1 mod prime_step
    std::vector<uint32_t> p;          // [KP] (padding primes repeat the last one)
    std::vector<uint32_t> pinv;       // [KP] p^-1 mod 2^32
    std::vector<uint32_t> crt_c;      // [KP] N^-1 R^2 (M/p_j)^-1 mod p_j   (R = 2^32)
    std::vector<uint32_t> crt_cc;     // [KP] crt_c * pinv mod 2^32 (Montgomery-Shoup companion)
    std::vector<float> rcp;           // [KP] 1/p_j (0 for padding)

    // twiddles in Shoup form: tw[j][k] = {w, floor(w 2^32 / p_j)}, w = psi_j^bitrev_logN(k) mod p_j,
    // k < N (two words per entry)
    std::vector<uint32_t> tw;         // [K][N][2]

    // plain (CUDA-core) GEMM tables, 24-bit digits: a coefficient is sum_d digit_d 2^(24 d)
    int D = 0;                        // digits of a W-bit value: ceil(W / 24)
    int DP = 0;                       // D rounded up to a multiple of 4
    std::vector<uint32_t> dec24;      // [DP][KP]  2^(24 d) R mod p_j (0 for d >= D)
    std::vector<uint32_t> crt24;      // [K + 1][DP] 24-bit digits of Q_j = (M/p_j) mod q; row K: of T_1
    std::vector<uint32_t> t1;         // [L]  T_1 = (-M) mod q

    // The CRT's value before reduction is below crt_bound (sum over primes of y'_j Q_j with
    // y'_j < 2 p_j, plus v' T_1 with v' < 2K); fold_count folds z -> (z mod 2^W) + (z >> W) delta
    // bring every such value below 2q, after which one conditional subtraction of q finishes.
    std::vector<uint32_t> crt_bound;  // bigint limbs
    int fold_count = 1;

    // tensor-core GEMM tables (canonical smem images, uploaded as-is)
    GemmShape dec_gemm;               // rows (j,t) = 4j+t, K = coefficient bytes
    GemmShape crt_gemm;               // rows = result byte v, K = (j,t) = 4j+t
    std::vector<uint8_t> dec_b;       // dec_gemm.b_bytes()
    std::vector<uint8_t> dec_b_ra;    // dec_b with every constant times gamma_j = crt_c_j 2^-32 mod p_j
    std::vector<uint8_t> crt_b;       // crt_gemm.b_bytes()
    int crt_kv = 0;                   // CRT K-byte column of v (its B column: the bytes of T_1)

    size_t coeff_words() const { return (size_t)N * L; }
    size_t residue_words() const { return (size_t)K * N; }
};

// Builds every table. Throws InvalidPoint for a malformed point.
Plan make_plan(uint32_t N, uint32_t W, uint32_t L, const uint32_t* q);

// Changes the 4-step split to nrows = 2^w1, ncols = 2^(logN - w1).  The tables do not
// depend on the split (twiddles are indexed by the bit-reversed stage position), so any
// w1 with both line lengths in [1, 2^10] gives the same transform.  Throws InvalidPoint.
void set_split(Plan& P, int w1);

// Offset in bytes of element (row, kbyte) inside a K-major no-swizzle canonical tile
// whose rows hold k_bytes bytes.
inline size_t umma_kmajor_offset(int row, int kbyte, int k_bytes) {
    return (size_t)(row >> 3) * (size_t)(8 * k_bytes) + (size_t)(kbyte >> 4) * 128 + (size_t)(row & 7) * 16 +
           (size_t)(kbyte & 15);
}

// Host-side self-checks of a plan (used by tests through the C ABI): returns an empty
// string when every check passes, else a description of the first failure.
std::string check_plan(const Plan& P);

}  // namespace pm
