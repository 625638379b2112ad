// pm_plan.cpp -- host precompute for one point (see pm_plan.h).
//
// What it must produce, and the reference function each piece replaces:
//   - point validation and delta = 2^W - q                 (solve.cu:873-897)
//   - the RNS prime list with prod p > 2^(2W+logN+3)      (solve.cu:899-913)
//   - Montgomery twiddles psi^bitrev(k) R mod p           (solve.cu:934-958)
//   - decomposition constants 2^(16h) R mod p             (solve.cu:966)
//   - CRT constants (M/p_j) mod q and (-vM) mod q         (solve.cu:969-1007)
// plus the byte-sliced B operands of the two tensor-core GEMMs, which have no reference
// counterpart.
#include "pm_plan.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>

namespace pm {
namespace {

using u32 = uint32_t;
using u64 = uint64_t;
using Big = std::vector<u32>;

u32 powmod(u64 b, u64 e, u32 m) {
    u64 r = 1 % m;
    b %= m;
    while (e) {
        if (e & 1) r = r * b % m;
        b = b * b % m;
        e >>= 1;
    }
    return (u32)r;
}

bool is_prime32(u32 n) {
    if (n < 2) return false;
    for (u32 sp : {2u, 3u, 5u, 7u, 11u, 13u, 17u, 19u, 23u, 29u, 31u, 37u})
        if (n % sp == 0) return n == sp;
    u32 d = n - 1;
    int s = 0;
    while (!(d & 1)) {
        d >>= 1;
        ++s;
    }
    for (u32 a : {2u, 7u, 61u}) {  // deterministic for n < 4,759,123,141
        u64 x = powmod(a, d, n);
        if (x == 1 || x == n - 1) continue;
        bool comp = true;
        for (int r = 1; r < s && comp; ++r) {
            x = x * x % n;
            comp = x != n - 1;
        }
        if (comp) return false;
    }
    return true;
}

int bitlen(const Big& x) {
    for (int i = (int)x.size() - 1; i >= 0; --i)
        if (x[i]) return 32 * i + 32 - __builtin_clz(x[i]);
    return 0;
}

void trim(Big& x) {
    while (x.size() > 1 && x.back() == 0) x.pop_back();
}

Big mul_small(const Big& x, u32 m) {
    Big r(x.size() + 1, 0);
    u64 c = 0;
    for (size_t i = 0; i < x.size(); ++i) {
        u64 t = (u64)x[i] * m + c;
        r[i] = (u32)t;
        c = t >> 32;
    }
    r[x.size()] = (u32)c;
    trim(r);
    return r;
}

Big add(const Big& a, const Big& b) {
    Big r(std::max(a.size(), b.size()) + 1, 0);
    u64 c = 0;
    for (size_t i = 0; i < r.size(); ++i) {
        u64 t = c + (i < a.size() ? a[i] : 0) + (i < b.size() ? b[i] : 0);
        r[i] = (u32)t;
        c = t >> 32;
    }
    trim(r);
    return r;
}

int cmp(const Big& a, const Big& b) {
    size_t n = std::max(a.size(), b.size());
    for (size_t i = n; i-- > 0;) {
        u32 x = i < a.size() ? a[i] : 0, y = i < b.size() ? b[i] : 0;
        if (x != y) return x < y ? -1 : 1;
    }
    return 0;
}

Big sub(const Big& a, const Big& b) {  // a >= b
    Big r(a.size(), 0);
    u64 br = 0;
    for (size_t i = 0; i < a.size(); ++i) {
        u64 t = (u64)a[i] - (i < b.size() ? b[i] : 0) - br;
        r[i] = (u32)t;
        br = (t >> 63) & 1;
    }
    trim(r);
    return r;
}

Big shr(const Big& x, int bits) {
    const int wl = bits / 32, wb = bits % 32;
    if ((int)x.size() <= wl) return Big{0};
    Big r(x.size() - wl, 0);
    for (size_t i = 0; i < r.size(); ++i) {
        u64 lo = x[i + wl], hi = i + wl + 1 < x.size() ? x[i + wl + 1] : 0;
        r[i] = wb ? (u32)((lo >> wb) | (hi << (32 - wb))) : (u32)lo;
    }
    trim(r);
    return r;
}

Big low_bits(const Big& x, int bits) {
    const int wl = bits / 32, wb = bits % 32;
    Big r(x.begin(), x.begin() + std::min<size_t>(x.size(), wl + 1));
    if ((int)r.size() > wl) r[wl] = wb ? (r[wl] & ((1u << wb) - 1u)) : 0u;
    trim(r);
    return r;
}

// x mod q with 2^W == delta (mod q); any x.
Big mod_q(Big x, const Plan& P) {
    const Big q(P.q.begin(), P.q.end());
    const Big d{(u32)P.delta, (u32)(P.delta >> 32)};
    for (int guard = 0; guard < 100000; ++guard) {
        Big hi = shr(x, (int)P.W);
        if (bitlen(hi) == 0) break;
        Big lo = low_bits(x, (int)P.W);
        // hi * delta
        Big prod(hi.size() + 2, 0);
        for (size_t i = 0; i < hi.size(); ++i) {
            u64 c = 0;
            for (size_t k = 0; k < 2; ++k) {
                u64 t = (u64)hi[i] * d[k] + prod[i + k] + c;
                prod[i + k] = (u32)t;
                c = t >> 32;
            }
            for (size_t k = i + 2; c && k < prod.size(); ++k) {
                u64 t = (u64)prod[k] + c;
                prod[k] = (u32)t;
                c = t >> 32;
            }
        }
        trim(prod);
        x = add(lo, prod);
    }
    while (cmp(x, q) >= 0) x = sub(x, q);
    x.resize(P.L, 0);
    return x;
}

u32 big_mod_small(const Big& x, u32 p) {
    u64 r = 0;
    for (size_t i = x.size(); i-- > 0;) r = ((r << 32) | x[i]) % p;
    return (u32)r;
}

u32 bitrev(u32 k, int bits) {
    u32 r = 0;
    for (int b = 0; b < bits; ++b) r |= ((k >> b) & 1u) << (bits - 1 - b);
    return r;
}

int round_up(int x, int m) { return (x + m - 1) / m * m; }

}  // namespace

Plan make_plan(uint32_t N, uint32_t W, uint32_t L, const uint32_t* qlimbs) {
    Plan P;
    if (N == 0 || (N & (N - 1)) != 0) throw InvalidPoint("N must be a power of two");
    if (N > (1u << 20)) throw InvalidPoint("N above 2^20 is not supported");
    if (W < 2 || L != (W + 31) / 32) throw InvalidPoint("inconsistent W / L (L must be ceil(W/32))");
    if (!qlimbs) throw InvalidPoint("q is null");
    P.N = N;
    P.W = W;
    P.L = L;
    P.q.assign(qlimbs, qlimbs + L);
    const Big qb(P.q.begin(), P.q.end());
    const int qbits = bitlen(qb);
    if (qbits > (int)W || qbits < 2 || !(P.q[0] & 1u)) throw InvalidPoint("q out of range (odd, < 2^W)");
    if (qbits <= 32 * ((int)L - 1)) throw InvalidPoint("q top limb is zero");
    while ((1u << P.logN) < N) ++P.logN;
    P.w1 = P.logN / 2;
    P.w2 = P.logN - P.w1;
    P.nrows = 1u << P.w1;
    P.ncols = 1u << P.w2;

    // delta = 2^W - q; the CRT reduction folds with 2^W == delta and needs delta < 2^63
    Big two_w(L + 1, 0);
    two_w[W / 32] |= 1u << (W % 32);
    Big dl = sub(two_w, qb);
    P.delta_bits = bitlen(dl);
    if (P.delta_bits > 63 || P.delta_bits > (int)W - 1)
        throw InvalidPoint("q too far below 2^W: delta = 2^W - q must be < 2^63 and < 2^(W-1)");
    P.delta = (u64)dl[0] | (dl.size() > 1 ? (u64)dl[1] << 32 : 0);

    // RNS primes: p < 2^30, p == 1 mod step, descending, until M >= 2^(2W + logN + 3) > 8 N q^2
    const u64 step = 2ull * std::max<u32>(N, 1u << 16);
    P.prime_step = step;
    const int need = 2 * (int)W + P.logN + 3;
    Big M{1};
    std::vector<u32> primes;
    for (u64 k = ((1ull << 30) - 2) / step; k >= 1 && bitlen(M) - 1 < need; --k) {
        const u64 p = 1 + k * step;
        if (p < (1ull << 30) && is_prime32((u32)p)) {
            primes.push_back((u32)p);
            M = mul_small(M, (u32)p);
        }
    }
    if (bitlen(M) - 1 < need) throw InvalidPoint("not enough NTT primes below 2^30 for this point");
    const int K = (int)primes.size();
    P.K = K;
    P.KP = round_up(K, 4);
    const int KP = P.KP;

    P.p.assign(KP, primes.back());
    P.pinv.assign(KP, 0);
    P.crt_c.assign(KP, 0);
    P.crt_cc.assign(KP, 0);
    P.rcp.assign(KP, 0.f);
    P.tw.assign((size_t)K * N * 2, 0);
    std::vector<u32> pw(N);
    for (int j = 0; j < KP; ++j) {
        const u32 p = j < K ? primes[j] : primes.back();
        P.p[j] = p;
        u32 inv = p;  // Newton: p * inv == 1 mod 2^32
        for (int it = 0; it < 5; ++it) inv *= 2u - p * inv;
        P.pinv[j] = inv;
        if (j >= K) continue;
        P.rcp[j] = 1.0f / (float)p;
        u32 psi = 0;
        for (u32 g = 2;; ++g) {
            const u32 x = powmod(g, (p - 1) / (2ull * N), p);
            if (powmod(x, N, p) == p - 1) {
                psi = x;
                break;
            }
        }
        pw[0] = 1;
        for (u32 e = 1; e < N; ++e) pw[e] = (u32)((u64)pw[e - 1] * psi % p);
        u32* tw = P.tw.data() + (size_t)j * N * 2;
        for (u32 k = 0; k < N; ++k) {
            const u64 w = pw[bitrev(k, P.logN)];
            tw[2 * k] = (u32)w;
            tw[2 * k + 1] = (u32)((w << 32) / p);
        }
        u64 mp = 1;  // (M / p_j) mod p_j
        for (int i = 0; i < K; ++i)
            if (i != j) mp = mp * (primes[i] % p) % p;
        const u64 R = (1ull << 32) % p;
        const u64 c = (u64)powmod(N % p, p - 2, p) * (R * R % p) % p * powmod(mp, p - 2, p) % p;
        P.crt_c[j] = (u32)c;
        P.crt_cc[j] = (u32)c * inv;
    }

    // plain decomposition constants 2^(16h) R mod p
    P.HP = round_up(2 * (int)L, 4);
    P.dec16.assign((size_t)2 * L * KP, 0);
    for (int h = 0; h < 2 * (int)L; ++h)
        for (int j = 0; j < K; ++j) P.dec16[(size_t)h * KP + j] = powmod(2, 16ull * h + 32, primes[j]);

    // CRT constants: Q_j = prod_{i != j} p_i mod q; T_v = (-v M) mod q
    std::vector<Big> Q(K);
    for (int j = 0; j < K; ++j) {
        Big acc{1};
        for (int i = 0; i < K; ++i)
            if (i != j) acc = mod_q(mul_small(acc, primes[i]), P);
        Q[j] = mod_q(acc, P);
    }
    P.qh16.assign((size_t)KP * P.HP, 0);
    for (int j = 0; j < K; ++j)
        for (int l = 0; l < (int)L; ++l) {
            P.qh16[(size_t)j * P.HP + 2 * l] = (uint16_t)(Q[j][l] & 0xFFFFu);
            P.qh16[(size_t)j * P.HP + 2 * l + 1] = (uint16_t)(Q[j][l] >> 16);
        }
    const Big Mq = mod_q(M, P);
    P.tneg.assign((size_t)(K + 1) * L, 0);
    for (int v = 1; v <= K; ++v) {
        Big vm = mod_q(mul_small(Mq, (u32)v), P);
        if (bitlen(vm) == 0) continue;
        Big t = sub(qb, vm);
        t.resize(L, 0);
        std::copy(t.begin(), t.end(), P.tneg.begin() + (size_t)v * L);
    }

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
        const u64 p = primes[j];
        const u64 gamma = (u64)P.crt_c[j] * powmod((1ull << 32) % p, p - 2, p) % p;
        for (int s = 0; s < 4 * (int)L; ++s) {
            const u32 c = powmod(2, 8ull * s + 32, primes[j]);
            const u32 cg = (u32)((u64)c * gamma % p);
            for (int t = 0; t < 4; ++t) {
                P.dec_b[umma_kmajor_offset(4 * j + t, s, P.dec_gemm.k_bytes)] = (uint8_t)(c >> (8 * t));
                P.dec_b_ra[umma_kmajor_offset(4 * j + t, s, P.dec_gemm.k_bytes)] = (uint8_t)(cg >> (8 * t));
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
    for (int j = 0; j < K; ++j)
        for (int t = 0; t < 4; ++t)
            for (int v = t; v < t + 4 * (int)L; ++v) {
                const int byte = v - t;
                const uint8_t qb8 = (uint8_t)(Q[j][byte / 4] >> (8 * (byte % 4)));
                P.crt_b[umma_kmajor_offset(v, 4 * j + t, P.crt_gemm.k_bytes)] = qb8;
            }
    for (int v = 0; v < 4 * (int)L; ++v)
        P.crt_b[umma_kmajor_offset(v, P.crt_kv, P.crt_gemm.k_bytes)] =
            (uint8_t)(P.tneg[(size_t)L + v / 4] >> (8 * (v % 4)));
    return P;
}

std::string check_plan(const Plan& P) {
    const int K = P.K;
    const Big qb(P.q.begin(), P.q.end());
    Big M{1};
    for (int j = 0; j < K; ++j) {
        const u32 p = P.p[j];
        if (!is_prime32(p) || p >= (1u << 30) || (p - 1) % P.prime_step != 0) return "bad prime";
        if ((u32)(p * P.pinv[j]) != 1u) return "bad p^-1 mod 2^32";
        const u32* tw = P.tw.data() + (size_t)j * P.N * 2;
        if (tw[0] != 1) return "tw[0] is not 1";
        if (P.N >= 2) {  // tw[1] = psi^(N/2): its square is -1
            const u64 w = tw[2];
            if (w * w % p != p - 1) return "psi^(N/2) squared is not -1";
        }
        for (u32 k = 0; k < P.N; k += 1 + P.N / 64)  // Shoup companions
            if (tw[2 * k] >= p || tw[2 * k + 1] != (u32)(((u64)tw[2 * k] << 32) / p)) return "bad Shoup twiddle";
        M = mul_small(M, p);
    }
    if (bitlen(M) - 1 < 2 * (int)P.W + P.logN + 3) return "M too small";

    // CRT reconstruction model on random |X| < M/8: residues -> y_j -> fp32 v -> sum y_j Q_j + T_v
    std::mt19937_64 rng(12345 + P.N + P.W);
    const int xbits = bitlen(M) - 4;
    for (int trial = 0; trial < 16; ++trial) {
        Big X((xbits + 31) / 32, 0);
        for (auto& w : X) w = (u32)rng();
        if (xbits % 32) X.back() &= (1u << (xbits % 32)) - 1u;
        trim(X);
        const bool neg = trial & 1;
        // expected X mod q
        Big xq = mod_q(X, P);
        if (neg && bitlen(xq)) xq = sub(qb, xq);
        xq.resize(P.L, 0);
        Big acc{0};
        float s = 0.f;
        for (int j = 0; j < K; ++j) {
            const u32 p = P.p[j];
            u64 xr = big_mod_small(X, p);
            if (neg) xr = (p - xr) % p;
            u64 mp = 1;
            for (int i = 0; i < K; ++i)
                if (i != j) mp = mp * (P.p[i] % p) % p;
            const u32 y = (u32)(xr * powmod(mp, p - 2, p) % p);
            s = std::fma((float)y, P.rcp[j], s);
            Big Qj(P.L);
            for (u32 l = 0; l < P.L; ++l)
                Qj[l] = (u32)P.qh16[(size_t)j * P.HP + 2 * l] | ((u32)P.qh16[(size_t)j * P.HP + 2 * l + 1] << 16);
            trim(Qj);
            Big term(Qj.size() + 1, 0);
            u64 c = 0;
            for (size_t l = 0; l < Qj.size(); ++l) {
                u64 t = (u64)Qj[l] * y + c;
                term[l] = (u32)t;
                c = t >> 32;
            }
            term[Qj.size()] = (u32)c;
            trim(term);
            acc = add(acc, term);
        }
        const float v = std::nearbyint(s);
        if (std::fabs(s - v) > 0.25f) return "fp32 CRT estimate outside its bound";
        Big T(P.tneg.begin() + (size_t)v * P.L, P.tneg.begin() + (size_t)(v + 1) * P.L);
        trim(T);
        Big got = mod_q(add(acc, T), P);
        if (got != xq) return "CRT reconstruction mismatch";
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
