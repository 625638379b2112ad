/*
 * rns_oracle.c -- CPU oracle for c = a*b mod (X^N + 1, q).  TEST INFRASTRUCTURE ONLY.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU legs load the shared object built
 * from this file, and only as the checker; the product (the CUDA library) never does.
 *
 * A plain-C restatement of the reference's method (TrivialError/polymult-challenge,
 * solve.cu), written for clarity rather than speed:
 *   - RNS primes: the largest p < 2^31 with p == 1 (mod 2N), taken in descending order
 *     until sum log2 p >= 2W + logN + 3, i.e. M = prod p > 8 N q^2  (solve.cu:899-913);
 *   - delta = 2^W - q, required < 2^63 and < 2^(W-1)               (solve.cu:883-897);
 *   - residues a_n mod p_j                                          (solve.cu:147-202);
 *   - per prime: psi-merged negacyclic NTT, Cooley-Tukey forward, pointwise product,
 *     Gentleman-Sande inverse, N^-1 scale                           (solve.cu:204-378);
 *   - exact CRT straight to mod q: y_j = x_j (M/p_j)^-1 mod p_j, v = round(sum y_j/p_j),
 *     c = sum_j y_j [(M/p_j) mod q] + [(-vM) mod q], reduced with 2^W == delta (mod q)
 *     and one conditional subtraction                                (solve.cu:380-501).
 * The transform here is one full-length NTT per prime (the 4-step column/row split of the
 * reference computes the same transform); v is estimated in double precision and checked
 * to lie within 1/4 of an integer.
 *
 * Parity pin: tests/test_oracle.py checks this oracle against the golden fixtures made
 * from the reference's own tests/oracle.py.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef uint32_t u32;
typedef uint64_t u64;
typedef unsigned __int128 u128;

static u32 pow_mod(u64 b, u64 e, u32 m) {
    u64 r = 1 % m;
    b %= m;
    while (e) {
        if (e & 1) r = r * b % m;
        b = b * b % m;
        e >>= 1;
    }
    return (u32)r;
}

/* Deterministic Miller-Rabin for 32-bit n (witnesses 2, 7, 61). */
static int is_prime_u32(u32 n) {
    static const u32 small[] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};
    if (n < 2) return 0;
    for (unsigned i = 0; i < sizeof small / sizeof small[0]; ++i)
        if (n % small[i] == 0) return n == small[i];
    u32 d = n - 1;
    int s = 0;
    while (!(d & 1)) { d >>= 1; ++s; }
    static const u32 wit[] = {2, 7, 61};
    for (int w = 0; w < 3; ++w) {
        u64 x = pow_mod(wit[w], d, n);
        if (x == 1 || x == n - 1) continue;
        int composite = 1;
        for (int r = 1; r < s; ++r) {
            x = x * x % n;
            if (x == n - 1) { composite = 0; break; }
        }
        if (composite) return 0;
    }
    return 1;
}

static int bit_length(const u32* x, int n) {
    for (int i = n - 1; i >= 0; --i)
        if (x[i]) return 32 * i + 32 - __builtin_clz(x[i]);
    return 0;
}

/* z (zl limbs) := z mod q using 2^W == delta (mod q); z must have zl >= L + 3 limbs. */
static void fold_mod_q(u32* z, int zl, int W, u64 delta, const u32* q, int L) {
    const int wl = W / 32, wb = W % 32;
    for (int guard = 0; guard < 64; ++guard) {
        /* hi = z >> W, as up to 4 limbs (callers keep z < 2^(W+128)) */
        u32 hi[4] = {0, 0, 0, 0};
        int any = 0;
        for (int k = 0; k < 4; ++k) {
            int src = wl + k;
            u64 lo = src < zl ? z[src] : 0, up = src + 1 < zl ? z[src + 1] : 0;
            hi[k] = wb ? (u32)((lo >> wb) | (up << (32 - wb))) : (u32)lo;
            any |= hi[k] != 0;
        }
        if (!any) break;
        z[wl] = wb ? (z[wl] & ((1u << wb) - 1u)) : 0u;
        for (int k = wl + 1; k < zl; ++k) z[k] = 0;
        /* z += hi * delta */
        u32 d[2] = {(u32)delta, (u32)(delta >> 32)};
        u32 prod[6] = {0, 0, 0, 0, 0, 0};
        for (int i = 0; i < 4; ++i) {
            u64 carry = 0;
            for (int j = 0; j < 2; ++j) {
                u64 t = (u64)hi[i] * d[j] + prod[i + j] + carry;
                prod[i + j] = (u32)t;
                carry = t >> 32;
            }
            for (int k = i + 2; carry && k < 6; ++k) {
                u64 t = (u64)prod[k] + carry;
                prod[k] = (u32)t;
                carry = t >> 32;
            }
        }
        u64 carry = 0;
        for (int k = 0; k < zl; ++k) {
            u64 t = (u64)z[k] + (k < 6 ? prod[k] : 0) + carry;
            z[k] = (u32)t;
            carry = t >> 32;
        }
    }
    /* z < 2^W = q + delta < 2q: at most one subtraction */
    int ge = 1;
    for (int k = zl - 1; k >= 0; --k) {
        u32 qk = k < L ? q[k] : 0;
        if (z[k] != qk) { ge = z[k] > qk; break; }
    }
    if (ge) {
        u64 borrow = 0;
        for (int k = 0; k < zl; ++k) {
            u64 t = (u64)z[k] - (k < L ? q[k] : 0) - borrow;
            z[k] = (u32)t;
            borrow = (t >> 63) & 1;
        }
    }
}

/* r := (x * m) mod q, x and r with L limbs (scratch of L+4 limbs). */
static void mul_small_mod_q(u32* r, const u32* x, u32 m, int W, u64 delta, const u32* q, int L) {
    u32* z = (u32*)calloc((size_t)L + 4, 4);
    u64 carry = 0;
    for (int k = 0; k < L; ++k) {
        u64 t = (u64)x[k] * m + carry;
        z[k] = (u32)t;
        carry = t >> 32;
    }
    z[L] = (u32)carry;
    fold_mod_q(z, L + 4, W, delta, q, L);
    memcpy(r, z, (size_t)L * 4);
    free(z);
}

static void ntt_forward(u32* x, u32 N, int logN, const u32* tw, u32 p) {
    u32 half = N, groups = 1;
    while (groups < N) {
        half >>= 1;
        for (u32 g = 0; g < groups; ++g) {
            const u64 w = tw[groups + g];
            for (u32 j = 2 * g * half; j < 2 * g * half + half; ++j) {
                u32 u = x[j], v = (u32)(x[j + half] * w % p);
                x[j] = (u32)(((u64)u + v) % p);
                x[j + half] = (u32)(((u64)u + p - v) % p);
            }
        }
        groups <<= 1;
    }
    (void)logN;
}

static void ntt_inverse(u32* x, u32 N, const u32* itw, u32 p) {
    u32 half = 1, groups = N >> 1;
    while (groups >= 1) {
        for (u32 g = 0; g < groups; ++g) {
            const u64 w = itw[groups + g];
            for (u32 j = 2 * g * half; j < 2 * g * half + half; ++j) {
                u32 u = x[j], v = x[j + half];
                x[j] = (u32)(((u64)u + v) % p);
                x[j + half] = (u32)((((u64)u + p - v) % p) * w % p);
            }
        }
        half <<= 1;
        groups >>= 1;
    }
}

/*
 * Returns 0 on success; negative on an invalid point:
 *  -1 N not a power of two, -2 L != ceil(W/32), -3 q out of range, -4 delta too large,
 *  -5 not enough primes, -6 CRT estimate outside its exactness bound, -7 out of memory.
 */
int orc_negacyclic_mul(u32 N, u32 W, u32 L, const u32* q, const u32* a, const u32* b, u32* c) {
    if (N == 0 || (N & (N - 1))) return -1;
    if (W < 2 || L != (W + 31) / 32) return -2;
    if (bit_length(q, (int)L) > (int)W || !(q[0] & 1) || bit_length(q, (int)L) <= 32 * ((int)L - 1)) return -3;
    int logN = 0;
    while ((1u << logN) < N) ++logN;

    /* delta = 2^W - q (solve.cu:883-897) */
    u32* two_w = (u32*)calloc((size_t)L + 1, 4);
    two_w[W / 32] |= 1u << (W % 32);
    {
        u64 borrow = 0;
        for (u32 k = 0; k <= L; ++k) {
            u64 t = (u64)two_w[k] - (k < L ? q[k] : 0) - borrow;
            two_w[k] = (u32)t;
            borrow = (t >> 63) & 1;
        }
    }
    int dbits = bit_length(two_w, (int)L + 1);
    if (dbits > 63 || dbits > (int)W - 1) { free(two_w); return -4; }
    const u64 delta = (u64)two_w[0] | (L > 1 ? (u64)two_w[1] << 32 : 0);
    free(two_w);

    /* primes (solve.cu:899-913) */
    const double need = 2.0 * W + logN + 3;
    const u64 step = 2ull * N;
    u32* primes = (u32*)malloc(4096 * sizeof(u32));
    int K = 0;
    double bits = 0;
    for (u64 k = ((1ull << 31) - 2) / step; k >= 1 && bits < need + 1e-6 && K < 4096; --k) {
        u64 p = 1 + k * step;
        if (p < (1ull << 31) && is_prime_u32((u32)p)) {
            primes[K++] = (u32)p;
            bits += log2((double)p);
        }
    }
    if (bits < need + 1e-6) { free(primes); return -5; }

    u32* res = (u32*)malloc((size_t)K * N * 4);      /* x_j per prime, then y_j */
    u32* Qj = (u32*)malloc((size_t)K * L * 4);       /* (M/p_j) mod q */
    u32* Tv = (u32*)calloc((size_t)(K + 1) * L, 4);  /* (-v M) mod q */
    int err = 0;
    if (!res || !Qj || !Tv) { err = -7; goto done; }

#pragma omp parallel for schedule(dynamic)
    for (int j = 0; j < K; ++j) {
        const u32 p = primes[j];
        u32* ra = (u32*)malloc((size_t)N * 4);
        u32* rb = res + (size_t)j * N;
        u32* tw = (u32*)malloc((size_t)N * 4);
        u32* itw = (u32*)malloc((size_t)N * 4);
        /* limb weights 2^(32l) mod p */
        u32* wl = (u32*)malloc((size_t)L * 4);
        for (u32 l = 0; l < L; ++l) wl[l] = pow_mod(2, 32ull * l, p);
        for (u32 n = 0; n < N; ++n) {
            u128 sa = 0, sb = 0;
            for (u32 l = 0; l < L; ++l) {
                sa += (u128)a[(size_t)n * L + l] * wl[l];
                sb += (u128)b[(size_t)n * L + l] * wl[l];
            }
            ra[n] = (u32)(sa % p);
            rb[n] = (u32)(sb % p);
        }
        /* psi: a primitive 2N-th root of unity mod p */
        u32 psi = 0;
        for (u32 g = 2;; ++g) {
            u32 x = pow_mod(g, (p - 1) / step, p);
            if (pow_mod(x, N, p) == p - 1) { psi = x; break; }
        }
        const u32 ipsi = pow_mod(psi, p - 2, p);
        for (u32 k = 0; k < N; ++k) {
            u32 r = 0;
            for (int bb = 0; bb < logN; ++bb) r |= ((k >> bb) & 1u) << (logN - 1 - bb);
            tw[k] = pow_mod(psi, r, p);
            itw[k] = pow_mod(ipsi, r, p);
        }
        ntt_forward(ra, N, logN, tw, p);
        ntt_forward(rb, N, logN, tw, p);
        for (u32 n = 0; n < N; ++n) rb[n] = (u32)((u64)ra[n] * rb[n] % p);
        ntt_inverse(rb, N, itw, p);
        /* y_j = x_j * N^-1 * (M/p_j)^-1 mod p_j */
        u64 mp = 1;
        for (int i = 0; i < K; ++i)
            if (i != j) mp = mp * (primes[i] % p) % p;
        const u64 scale = (u64)pow_mod(N % p, p - 2, p) * pow_mod(mp, p - 2, p) % p;
        for (u32 n = 0; n < N; ++n) rb[n] = (u32)(rb[n] * scale % p);
        free(ra); free(tw); free(itw); free(wl);
    }

    /* Q_j = prod_{i != j} p_i mod q;  T_v = (-v M) mod q  */
    {
        u32* acc = (u32*)malloc((size_t)L * 4);
        for (int j = 0; j < K; ++j) {
            memset(acc, 0, (size_t)L * 4);
            acc[0] = 1;
            for (int i = 0; i < K; ++i)
                if (i != j) mul_small_mod_q(acc, acc, primes[i], (int)W, delta, q, (int)L);
            memcpy(Qj + (size_t)j * L, acc, (size_t)L * 4);
        }
        u32* Mq = (u32*)calloc(L, 4);
        Mq[0] = 1;
        for (int i = 0; i < K; ++i) mul_small_mod_q(Mq, Mq, primes[i], (int)W, delta, q, (int)L);
        for (int v = 1; v <= K; ++v) {
            mul_small_mod_q(acc, Mq, (u32)v, (int)W, delta, q, (int)L);   /* v M mod q */
            int zero = 1;
            for (u32 l = 0; l < L; ++l) zero &= acc[l] == 0;
            if (!zero) {
                u64 borrow = 0;
                for (u32 l = 0; l < L; ++l) {
                    u64 t = (u64)q[l] - acc[l] - borrow;
                    Tv[(size_t)v * L + l] = (u32)t;
                    borrow = (t >> 63) & 1;
                }
            }
        }
        free(acc);
        free(Mq);
    }

    /* CRT per coefficient (solve.cu:384-501) */
#pragma omp parallel for schedule(static)
    for (long long n = 0; n < (long long)N; ++n) {
        const int zl = (int)L + 6;
        u32 z[zl];
        memset(z, 0, sizeof z);
        long double s = 0;
        for (int j = 0; j < K; ++j) {
            const u32 y = res[(size_t)j * N + n];
            s += (long double)y / primes[j];
            const u32* Q = Qj + (size_t)j * L;
            u64 carry = 0;
            for (u32 l = 0; l < L; ++l) {
                u64 t = (u64)Q[l] * y + z[l] + carry;
                z[l] = (u32)t;
                carry = t >> 32;
            }
            for (int l = (int)L; carry && l < zl; ++l) {
                u64 t = (u64)z[l] + carry;
                z[l] = (u32)t;
                carry = t >> 32;
            }
        }
        const long double vr = floorl(s + 0.5L);
        if (fabsl(s - vr) > 0.25L) {
#pragma omp atomic write
            err = -6;
        }
        const int v = (int)vr;
        u64 carry = 0;
        for (int l = 0; l < zl; ++l) {
            u64 t = (u64)z[l] + (l < (int)L ? Tv[(size_t)v * L + l] : 0) + carry;
            z[l] = (u32)t;
            carry = t >> 32;
        }
        fold_mod_q(z, zl, (int)W, delta, q, (int)L);
        memcpy(c + (size_t)n * L, z, (size_t)L * 4);
    }

done:
    free(res); free(Qj); free(Tv); free(primes);
    return err;
}

/* Number of RNS primes the reference's rule selects for (N, W); for reporting. */
int orc_prime_count(u32 N, u32 W) {
    int logN = 0;
    while ((1u << logN) < N) ++logN;
    const double need = 2.0 * W + logN + 3;
    const u64 step = 2ull * N;
    int K = 0;
    double bits = 0;
    for (u64 k = ((1ull << 31) - 2) / step; k >= 1 && bits < need + 1e-6; --k) {
        u64 p = 1 + k * step;
        if (p < (1ull << 31) && is_prime_u32((u32)p)) { ++K; bits += log2((double)p); }
    }
    return bits < need + 1e-6 ? -1 : K;
}
