// pm_plan.cpp -- host precompute for one point (see pm_plan.h).
//
// What it must produce, and the reference function each piece stands in for:
//   - point validation and delta = 2^W - q                 (solve.cu:873-897)
//   - the RNS prime list with prod p >= 2^(2W+logN+3)     (solve.cu:899-913)
//   - twiddles psi^bitrev(k) in Shoup form                (solve.cu:934-958)
//   - plain decomposition constants 2^(24d) R mod p       (solve.cu:966 uses 16-bit halves)
//   - CRT constants (M/p_j) mod q and T_1 = (-M) mod q    (solve.cu:969-1007)
// plus the byte-sliced B operands of the two tensor-core GEMMs and the CRT fold bound, which
// have no reference counterpart.  Every table is built with this file's own arithmetic: a small
// bigint type `Nat`, primes by trial division against a sieve, psi from a quadratic non-residue,
// inverses by the extended Euclidean algorithm, p^-1 mod 2^32 by Hensel lifting.
#include "pm_plan.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>

namespace pm {
namespace {

using u32 = uint32_t;
using u64 = uint64_t;

// ---------------------------------------------------------------------------------------
// Unsigned bigints: little-endian u32 limbs with no high zero limbs (zero = no limbs).
// ---------------------------------------------------------------------------------------
struct Nat {
    std::vector<u32> d;
    Nat() = default;
    explicit Nat(u64 v) {
        for (; v; v >>= 32) d.push_back((u32)v);
    }
    Nat(const u32* p, size_t n) : d(p, p + n) { trim(); }
    void trim() {
        while (!d.empty() && d.back() == 0) d.pop_back();
    }
    bool is_zero() const { return d.empty(); }
    u32 limb(size_t i) const { return i < d.size() ? d[i] : 0u; }
    int bits() const { return d.empty() ? 0 : 32 * (int)(d.size() - 1) + 32 - __builtin_clz(d.back()); }
    // the value as exactly n limbs (n >= the limb count)
    std::vector<u32> limbs(size_t n) const {
        std::vector<u32> r(n, 0);
        std::copy(d.begin(), d.begin() + std::min(n, d.size()), r.begin());
        return r;
    }
};

int cmp(const Nat& a, const Nat& b) {
    if (a.d.size() != b.d.size()) return a.d.size() < b.d.size() ? -1 : 1;
    for (size_t i = a.d.size(); i-- > 0;)
        if (a.d[i] != b.d[i]) return a.d[i] < b.d[i] ? -1 : 1;
    return 0;
}

Nat add(const Nat& a, const Nat& b) {
    Nat r;
    const size_t n = std::max(a.d.size(), b.d.size());
    r.d.resize(n + 1);
    u64 c = 0;
    for (size_t i = 0; i < n; ++i) {
        c += (u64)a.limb(i) + b.limb(i);
        r.d[i] = (u32)c;
        c >>= 32;
    }
    r.d[n] = (u32)c;
    r.trim();
    return r;
}

// a - b for a >= b
Nat sub(const Nat& a, const Nat& b) {
    Nat r;
    r.d.resize(a.d.size());
    u64 borrow = 0;
    for (size_t i = 0; i < a.d.size(); ++i) {
        const u64 t = (u64)a.d[i] - b.limb(i) - borrow;
        r.d[i] = (u32)t;
        borrow = t >> 63;
    }
    r.trim();
    return r;
}

Nat mul_small(const Nat& a, u64 m) {  // m < 2^64
    Nat r;
    r.d.assign(a.d.size() + 2, 0);
    const u32 m0 = (u32)m, m1 = (u32)(m >> 32);
    for (size_t i = 0; i < a.d.size(); ++i) {
        u64 t = (u64)a.d[i] * m0 + r.d[i];
        r.d[i] = (u32)t;
        u64 c = t >> 32;
        t = (u64)a.d[i] * m1 + r.d[i + 1] + c;
        r.d[i + 1] = (u32)t;
        c = t >> 32;
        for (size_t k = i + 2; c; ++k) {
            t = (u64)r.d[k] + c;
            r.d[k] = (u32)t;
            c = t >> 32;
        }
    }
    r.trim();
    return r;
}

Nat pow2(int e) {
    Nat r;
    r.d.assign((size_t)e / 32 + 1, 0);
    r.d.back() = 1u << (e % 32);
    return r;
}

// a mod 2^n and a >> n
Nat low_part(const Nat& a, int n) {
    Nat r;
    const size_t full = (size_t)n / 32;
    r.d.assign(a.d.begin(), a.d.begin() + std::min(a.d.size(), full + 1));
    if (r.d.size() > full) r.d[full] &= (n % 32) ? (1u << (n % 32)) - 1u : 0u;
    r.trim();
    return r;
}
Nat high_part(const Nat& a, int n) {
    Nat r;
    const size_t w = (size_t)n / 32;
    const int b = n % 32;
    for (size_t i = w; i < a.d.size(); ++i) {
        const u64 two = (u64)a.d[i] | ((u64)a.limb(i + 1) << 32);
        r.d.push_back((u32)(two >> b));
    }
    r.trim();
    return r;
}

// divides a by m in place (from the top limb down); returns the remainder
u32 div_small(Nat& a, u32 m) {
    u64 rem = 0;
    for (size_t i = a.d.size(); i-- > 0;) {
        const u64 cur = (rem << 32) | a.d[i];
        a.d[i] = (u32)(cur / m);
        rem = cur % m;
    }
    a.trim();
    return (u32)rem;
}
u32 mod_small(const Nat& a, u32 m) {
    Nat t = a;
    return div_small(t, m);
}

// x mod q for q = 2^W - delta: 2^W == delta (mod q), so x == (x mod 2^W) + (x >> W) delta;
// repeat until x < 2^W, then subtract q while x >= q.
Nat reduce_mod_q(Nat x, const Nat& q, int W, u64 delta) {
    while (x.bits() > W) x = add(low_part(x, W), mul_small(high_part(x, W), delta));
    while (cmp(x, q) >= 0) x = sub(x, q);
    return x;
}

// x mod q by binary long division (independent of the fold above; used by the self-check)
Nat long_mod(const Nat& x, const Nat& q) {
    Nat r;
    for (int b = x.bits() - 1; b >= 0; --b) {
        r = add(r, r);
        if ((x.d[b / 32] >> (b % 32)) & 1u) r = add(r, Nat(1));
        if (cmp(r, q) >= 0) r = sub(r, q);
    }
    return r;
}

// ---------------------------------------------------------------------------------------
// Modular arithmetic on primes below 2^30
// ---------------------------------------------------------------------------------------
u64 mulmod(u64 a, u64 b, u64 m) { return a * b % m; }  // a, b < m < 2^32

// x^e mod m, left-to-right over the bits of e
u64 expmod(u64 x, u64 e, u64 m) {
    u64 r = 1 % m;
    x %= m;
    for (int b = 63; b >= 0; --b) {
        r = mulmod(r, r, m);
        if ((e >> b) & 1u) r = mulmod(r, x, m);
    }
    return r;
}

// a^-1 mod m (gcd(a, m) = 1) by the extended Euclidean algorithm
u64 invmod(u64 a, u64 m) {
    int64_t r0 = (int64_t)m, r1 = (int64_t)(a % m), s0 = 0, s1 = 1;
    while (r1 != 0) {
        const int64_t qt = r0 / r1;
        int64_t t = r0 - qt * r1;
        r0 = r1;
        r1 = t;
        t = s0 - qt * s1;
        s0 = s1;
        s1 = t;
    }
    if (r0 != 1) throw InvalidPoint("internal: no modular inverse");
    return (u64)(s0 < 0 ? s0 + (int64_t)m : s0);
}

// p^-1 mod 2^32 for odd p, one bit at a time (Hensel lifting): x p == 1 (mod 2^(b+1)) after bit b
u32 inv_mod_2_32(u32 p) {
    u32 x = 1;
    for (int b = 1; b < 32; ++b)
        if (((u32)(p * x) >> b) & 1u) x |= 1u << b;
    return x;
}

// primes below 2^15 (sieve of Eratosthenes): enough to decide primality below 2^30
const std::vector<u32>& small_primes() {
    static const std::vector<u32> list = [] {
        const u32 lim = 1u << 15;
        std::vector<bool> composite(lim, false);
        std::vector<u32> out;
        for (u32 i = 2; i < lim; ++i) {
            if (composite[i]) continue;
            out.push_back(i);
            for (u32 k = i * i; k < lim; k += i) composite[k] = true;
        }
        return out;
    }();
    return list;
}

bool prime_below_2_30(u32 n) {
    if (n < 2) return false;
    for (u32 s : small_primes()) {
        if ((u64)s * s > n) break;
        if (n % s == 0) return false;
    }
    return true;
}

// Deterministic Miller-Rabin with bases 2, 3, 5, 7 (exact below 3,215,031,751); the
// self-check's independent primality test.
bool miller_rabin(u32 n) {
    if (n < 2) return false;
    for (u32 s : {2u, 3u, 5u, 7u})
        if (n % s == 0) return n == s;
    u32 d = n - 1;
    int r = 0;
    while ((d & 1u) == 0) {
        d >>= 1;
        ++r;
    }
    for (u32 a : {2u, 3u, 5u, 7u}) {
        u64 x = expmod(a, d, n);
        if (x == 1 || x == n - 1) continue;
        bool witness = true;
        for (int i = 1; i < r && witness; ++i) {
            x = mulmod(x, x, n);
            if (x == n - 1) witness = false;
        }
        if (witness) return false;
    }
    return true;
}

// A primitive 2N-th root of unity mod p (p == 1 mod 2N, N a power of two): with
// p - 1 = 2^e m (m odd) and z a quadratic non-residue, z^m has order exactly 2^e; squaring it
// e - logN - 1 times leaves order 2^(logN + 1) = 2N.
u32 root_of_order_2n(u32 p, int logN) {
    const u32 pm1 = p - 1;
    const int e = __builtin_ctz(pm1);
    const u32 m = pm1 >> e;
    u32 z = 2;
    while (expmod(z, pm1 / 2, p) != pm1) ++z;  // Euler's criterion
    u64 g = expmod(z, m, p);
    for (int i = 0; i < e - (logN + 1); ++i) g = mulmod(g, g, p);
    return (u32)g;
}

int round_up(int x, int m) { return (x + m - 1) / m * m; }

// The value the device's fold sequence leaves from any z <= zmax (see Plan::fold_count):
// the largest result of one fold z -> (z mod 2^W) + (z >> W) delta over z <= zmax.
Nat fold_max(const Nat& zmax, int W, u64 delta) {
    const Nat hi = high_part(zmax, W);
    if (hi.is_zero()) return zmax;
    const Nat lo_all = sub(pow2(W), Nat(1));  // a smaller high part leaves the low part free
    const Nat a = add(lo_all, mul_small(sub(hi, Nat(1)), delta));
    const Nat b = add(low_part(zmax, W), mul_small(hi, delta));
    return cmp(a, b) >= 0 ? a : b;
}

// The device's reduction of z (zmax-bounded) restated on bigints: `folds` folds of at most 64
// high bits each, then q subtracted iff z + delta reaches 2^W.
Nat device_reduce(Nat z, int folds, int W, u64 delta) {
    for (int f = 0; f < folds; ++f) {
        const Nat hi = low_part(high_part(z, W), 64);
        z = add(low_part(z, W), mul_small(hi, delta));
    }
    const Nat t = add(z, Nat(delta));
    return t.bits() > W ? low_part(t, W) : z;
}

}  // namespace

Plan make_plan(uint32_t N, uint32_t W, uint32_t L, const uint32_t* qlimbs) {
    Plan P;
    if (N == 0 || (N & (N - 1)) != 0) throw InvalidPoint("N is not a power of two");
    if (N > (1u << 20)) throw InvalidPoint("N is above 2^20");
    if (W < 2 || L != (W + 31) / 32) throw InvalidPoint("L does not equal ceil(W / 32)");
    if (!qlimbs) throw InvalidPoint("no q given");
    P.N = N;
    P.W = W;
    P.L = L;
    P.q.assign(qlimbs, qlimbs + L);
    const Nat q(qlimbs, L);
    if ((P.q[0] & 1u) == 0) throw InvalidPoint("q is even");
    if (q.bits() > (int)W) throw InvalidPoint("q is not below 2^W");
    // delta = 2^W - q drives the CRT's fold: it must fit 63 bits and leave q above 2^(W-1),
    // so that q has exactly L limbs and a fold always shrinks the value
    const Nat dl = sub(pow2((int)W), q);
    if (dl.bits() > 63 || dl.bits() >= (int)W) throw InvalidPoint("q is too far below 2^W (delta needs < 2^63 and q > 2^(W-1))");
    P.delta = (u64)dl.limb(0) | ((u64)dl.limb(1) << 32);
    P.logN = __builtin_ctz(N);
    P.w1 = P.logN / 2;
    P.w2 = P.logN - P.w1;
    P.nrows = 1u << P.w1;
    P.ncols = 1u << P.w2;

    // RNS primes below 2^30, == 1 mod step, largest first, until M = prod p >= 2^need: then
    // |x| < M/8 holds for every exact negacyclic product coefficient (|x| < N q^2 < 2^(2W+logN))
    const u64 step = 2ull * std::max<u32>(N, 1u << 16);
    P.prime_step = step;
    const int need = 2 * (int)W + P.logN + 3;
    Nat M(1);
    std::vector<u32> primes;
    for (u64 k = ((1ull << 30) - 1) / step; k >= 1 && M.bits() <= need; --k) {
        const u32 cand = (u32)(1 + k * step);
        if (prime_below_2_30(cand)) {
            primes.push_back(cand);
            M = mul_small(M, cand);
        }
    }
    if (M.bits() <= need) throw InvalidPoint("too few NTT primes below 2^30 for this point");
    const int K = (int)primes.size();
    P.K = K;
    P.KP = round_up(K, 4);
    const int KP = P.KP;

    // per prime: Montgomery inverse, twiddles, CRT factor; M / p_j by exact division
    P.p.assign(KP, primes.back());
    P.pinv.assign(KP, 0);
    P.crt_c.assign(KP, 0);
    P.crt_cc.assign(KP, 0);
    P.rcp.assign(KP, 0.f);
    P.tw.assign((size_t)K * N * 2, 0);
    std::vector<u32> rev(N, 0), pw(N, 1);
    for (u32 k = 1; k < N; ++k) rev[k] = (rev[k >> 1] >> 1) | ((k & 1u) << (P.logN - 1));
    std::vector<Nat> Q(K);  // (M / p_j) mod q
    for (int j = 0; j < KP; ++j) {
        const u32 pj = j < K ? primes[j] : primes.back();
        P.p[j] = pj;
        P.pinv[j] = inv_mod_2_32(pj);
        if (j >= K) continue;
        P.rcp[j] = 1.0f / (float)pj;
        const u64 psi = root_of_order_2n(pj, P.logN);
        for (u32 e = 1; e < N; ++e) pw[e] = (u32)mulmod(pw[e - 1], psi, pj);
        u32* tw = P.tw.data() + (size_t)j * N * 2;
        for (u32 k = 0; k < N; ++k) {
            const u64 w = pw[rev[k]];
            tw[2 * k] = (u32)w;
            tw[2 * k + 1] = (u32)((w << 32) / pj);
        }
        Nat Mj = M;
        if (div_small(Mj, pj) != 0) throw InvalidPoint("internal: M not divisible by its prime");
        const u64 mj_mod_p = mod_small(Mj, pj);
        const u64 r = (1ull << 32) % pj;
        const u64 c = mulmod(mulmod(invmod(N % pj, pj), mulmod(r, r, pj), pj), invmod(mj_mod_p, pj), pj);
        P.crt_c[j] = (u32)c;
        P.crt_cc[j] = (u32)c * P.pinv[j];
        Q[j] = reduce_mod_q(Mj, q, (int)W, P.delta);
    }
    const Nat Mq = reduce_mod_q(M, q, (int)W, P.delta);
    const Nat T1 = Mq.is_zero() ? Nat() : sub(q, Mq);
    P.t1 = T1.limbs(L);

    // plain GEMM tables on 24-bit digits
    P.D = ((int)W + kDigitBits - 1) / kDigitBits;
    P.DP = round_up(P.D, 4);
    P.dec24.assign((size_t)P.DP * KP, 0);
    for (int j = 0; j < K; ++j) {
        u64 c = (1ull << 32) % primes[j];  // 2^(24 d) R mod p, d = 0, 1, ...
        const u64 step24 = (1ull << kDigitBits) % primes[j];
        for (int d = 0; d < P.D; ++d, c = mulmod(c, step24, primes[j])) P.dec24[(size_t)d * KP + j] = (u32)c;
    }
    P.crt24.assign((size_t)(K + 1) * P.DP, 0);
    auto put_digits = [&](const Nat& x, u32* row) {
        for (int d = 0; d < P.D; ++d) {
            const int b0 = kDigitBits * d;
            const u64 two = (u64)x.limb(b0 / 32) | ((u64)x.limb(b0 / 32 + 1) << 32);
            row[d] = (u32)(two >> (b0 % 32)) & ((1u << kDigitBits) - 1u);
        }
    };
    for (int j = 0; j < K; ++j) put_digits(Q[j], P.crt24.data() + (size_t)j * P.DP);
    put_digits(T1, P.crt24.data() + (size_t)K * P.DP);

    // the CRT value before reduction: sum_j y'_j Q_j + v' T_1 with y'_j < 2 p_j and v' <= 2K,
    // Q_j and T_1 below q, so z < (2 sum_j p_j + 2K + 1) q =: crt_bound
    u64 psum = 0;
    for (int j = 0; j < K; ++j) psum += primes[j];
    const Nat bound = mul_small(q, 2 * psum + 2 * (u64)K + 1);
    P.crt_bound = bound.d;
    if (bound.bits() > (int)W + 64 || bound.bits() > 32 * ((int)L + 3))
        throw InvalidPoint("internal: CRT value outside the fold's 64-bit window");
    const Nat two_q = add(q, q);
    Nat zmax = sub(bound, Nat(1));
    int folds = 0;
    while (cmp(zmax, two_q) >= 0) {
        if (++folds > 64) throw InvalidPoint("delta too large for the CRT's fold");
        zmax = fold_max(zmax, (int)W, P.delta);
    }
    P.fold_count = folds;

    // tensor-core decomposition operand B: row 4j+t, K-byte s -> byte t of 2^(8s) R mod p_j
    P.dec_gemm.n_rows = 4 * KP;
    P.dec_gemm.k_bytes = round_up(4 * (int)L, 32);
    P.dec_b.assign(P.dec_gemm.b_bytes(), 0);
    P.dec_b_ra.assign(P.dec_gemm.b_bytes(), 0);
    for (int j = 0; j < K; ++j) {
        // gamma_j = crt_c_j 2^-32 mod p_j: the factor the CRT applies to every residue x_j of the
        // inverse transform (y_j = x_j gamma_j).  The transform is linear over Z_p, so scaling one
        // operand's residues by gamma_j makes the inverse transform deliver y_j itself; dec_b_ra
        // decomposes the operand whose transform the fused row pass reads (RA) that way.
        const u64 pj = primes[j];
        const u64 gamma = mulmod(P.crt_c[j], invmod((1ull << 32) % pj, pj), pj);
        u64 c = (1ull << 32) % pj;  // 2^(8 s) R mod p, s = 0, 1, ...
        for (int s = 0; s < 4 * (int)L; ++s, c = mulmod(c, 256, pj)) {
            const u32 cg = (u32)mulmod(c, gamma, pj);
            for (int t = 0; t < 4; ++t) {
                const size_t off = umma_kmajor_offset(4 * j + t, s, P.dec_gemm.k_bytes);
                P.dec_b[off] = (uint8_t)(c >> (8 * t));
                P.dec_b_ra[off] = (uint8_t)(cg >> (8 * t));
            }
        }
    }

    // tensor-core CRT operand B: row v (result byte), K-byte 4j+t -> byte (v - t) of Q_j; K-byte
    // crt_kv = 4K (the first padding byte, or one past the primes) -> byte v of T_1 = (-M) mod q,
    // against the A column that holds v (<= K < 256), so that the MMA adds v T_1 itself
    P.crt_gemm.n_rows = round_up(4 * (int)L + 3, 16);
    P.crt_kv = 4 * K;
    P.crt_gemm.k_bytes = round_up(std::max(4 * KP, P.crt_kv + 1), 32);
    P.crt_b.assign(P.crt_gemm.b_bytes(), 0);
    for (int j = 0; j < K; ++j) {
        const std::vector<u32> qj = Q[j].limbs(L);
        for (int byte = 0; byte < 4 * (int)L; ++byte) {
            const uint8_t b8 = (uint8_t)(qj[byte / 4] >> (8 * (byte % 4)));
            for (int t = 0; t < 4; ++t) P.crt_b[umma_kmajor_offset(byte + t, 4 * j + t, P.crt_gemm.k_bytes)] = b8;
        }
    }
    for (int v = 0; v < 4 * (int)L; ++v)
        P.crt_b[umma_kmajor_offset(v, P.crt_kv, P.crt_gemm.k_bytes)] = (uint8_t)(P.t1[v / 4] >> (8 * (v % 4)));
    return P;
}

std::string check_plan(const Plan& P) {
    const int K = P.K, W = (int)P.W;
    const Nat q(P.q.data(), P.L);
    Nat M(1);
    for (int j = 0; j < K; ++j) {
        const u32 p = P.p[j];
        if (!miller_rabin(p) || p >= (1u << 30) || (p - 1) % P.prime_step != 0) return "bad prime";
        if ((u32)(p * P.pinv[j]) != 1u) return "bad p^-1 mod 2^32";
        const u32* tw = P.tw.data() + (size_t)j * P.N * 2;
        if (tw[0] != 1) return "tw[0] is not 1";
        if (P.N >= 2) {  // tw[1] = psi^(N/2): its square is -1
            const u64 w = tw[2];
            if (w * w % p != p - 1) return "psi^(N/2) squared is not -1";
        }
        for (u32 k = 0; k < P.N; k += 1 + P.N / 64)  // Shoup companions
            if (tw[2 * k] >= p || tw[2 * k + 1] != (u32)(((u64)tw[2 * k] << 32) / p)) return "bad Shoup twiddle";
        for (int d = 0; d < P.D; ++d)  // plain decomposition constants
            if (P.dec24[(size_t)d * P.KP + j] != (u32)expmod(2, 24ull * d + 32, p)) return "bad digit constant";
        M = mul_small(M, p);
    }
    if (M.bits() <= 2 * W + P.logN + 3) return "M too small";

    // the fold sequence on its worst case and on a value that is all ones below the bound
    const Nat bound(P.crt_bound.data(), P.crt_bound.size());
    for (const Nat& z : {sub(bound, Nat(1)), low_part(sub(bound, Nat(1)), W + 1), Nat(P.delta)}) {
        const Nat got = device_reduce(z, P.fold_count, W, P.delta);
        if (cmp(got, q) >= 0 || cmp(got, long_mod(z, q)) != 0) return "fold sequence does not reduce its bound";
    }

    // CRT reconstruction through the plain tables on random |X| < M/8: residues -> y_j -> fp32 v
    // -> z = sum y_j Q_j + v T_1 (Q_j and T_1 from their 24-bit digits) -> the device's folds
    std::mt19937_64 rng(12345 + P.N + P.W);
    const int xbits = M.bits() - 4;
    for (int trial = 0; trial < 16; ++trial) {
        Nat X;
        X.d.resize((size_t)(xbits + 31) / 32);
        for (auto& w : X.d) w = (u32)rng();
        if (xbits % 32) X.d.back() &= (1u << (xbits % 32)) - 1u;
        X.trim();
        const bool neg = trial & 1;
        Nat want = long_mod(X, q);
        if (neg && !want.is_zero()) want = sub(q, want);
        Nat z;
        float s = 0.f;
        auto from_digits = [&](const u32* row) {
            Nat v;
            for (int d = P.D - 1; d >= 0; --d) v = add(mul_small(v, 1ull << kDigitBits), Nat(row[d]));
            return v;
        };
        for (int j = 0; j < K; ++j) {
            const u32 p = P.p[j];
            u64 xr = mod_small(X, p);
            if (neg) xr = (p - xr) % p;
            Nat Mj = M;
            div_small(Mj, p);
            const u32 y = (u32)mulmod(xr, invmod(mod_small(Mj, p), p), p);
            s = std::fma((float)y, P.rcp[j], s);
            z = add(z, mul_small(from_digits(P.crt24.data() + (size_t)j * P.DP), y));
        }
        const float v = std::nearbyint(s);
        if (std::fabs(s - v) > 0.25f) return "fp32 CRT estimate outside its bound";
        z = add(z, mul_small(from_digits(P.crt24.data() + (size_t)K * P.DP), (u64)v));
        if (cmp(z, bound) >= 0) return "CRT value above its bound";
        if (cmp(device_reduce(z, P.fold_count, W, P.delta), want) != 0) return "CRT reconstruction mismatch";
    }
    return "";
}

void set_split(Plan& P, int w1) {
    const int w2 = P.logN - w1;
    if (w1 < 0 || w2 < 0 || w1 > 10 || w2 > 10 || (P.logN > 0 && w2 < 1))
        throw InvalidPoint("4-step split out of range: w1 = " + std::to_string(w1) + " for logN = " +
                           std::to_string(P.logN));
    P.w1 = w1;
    P.w2 = w2;
    P.nrows = 1u << w1;
    P.ncols = 1u << w2;
}

}  // namespace pm
