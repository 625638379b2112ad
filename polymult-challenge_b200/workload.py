"""Workload generation for benchmarks and serving: spec-derived primes and seeded operands.

The spec-derived prime of a point (the largest prime q < 2^W with q == 1 mod 2N) is what
the challenge's points use (tests/oracle.py:48-57 describes the rule).  Searching for it at
W = 3000 takes tens of seconds in Python, so the primes of the benchmark grid are listed in
SPEC_PRIMES (their values are checked against an independent search in the tests).
"""
from __future__ import annotations

import random
from typing import Dict, Tuple

import numpy as np

# delta = 2^W - q of the spec-derived primes of the benchmark grid (N, W) -> delta
SPEC_DELTAS: Dict[Tuple[int, int], int] = {}


def _is_probable_prime(n: int, rounds: int = 24) -> bool:
    if n < 2:
        return False
    for sp in (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47):
        if n % sp == 0:
            return n == sp
    d, s = n - 1, 0
    while not d & 1:
        d >>= 1
        s += 1
    rng = random.Random(n & 0xFFFFFFFF)
    for _ in range(rounds):
        x = pow(rng.randrange(2, n - 1), d, n)
        if x in (1, n - 1):
            continue
        for _ in range(s - 1):
            x = x * x % n
            if x == n - 1:
                break
        else:
            return False
    return True


def spec_prime(N: int, W: int) -> int:
    """Largest prime q < 2^W with q == 1 (mod 2N)."""
    if (N, W) in SPEC_DELTAS:
        return (1 << W) - SPEC_DELTAS[(N, W)]
    step = 2 * N
    q = (1 << W) - 1
    q -= (q - 1) % step
    while q > 1:
        if _is_probable_prime(q):
            return q
        q -= step
    raise ValueError("no prime == 1 mod 2N below 2^W")


def limbs(x: int, L: int) -> np.ndarray:
    return np.frombuffer(int(x).to_bytes(4 * L, "little"), dtype="<u4").copy()


def uniform_operands(N: int, W: int, q: int, count: int, seed: int) -> np.ndarray:
    """[count, N, L] u32 limbs, coefficients uniform in [0, q) (seeded PCG64, rejection of the
    rare values >= q by redrawing their top limb)."""
    L = (W + 31) // 32
    rng = np.random.Generator(np.random.PCG64(seed))
    out = rng.integers(0, 1 << 32, size=(count, N, L), dtype=np.uint64).astype(np.uint32)
    top = W - 32 * (L - 1)
    if top < 32:
        out[..., L - 1] &= np.uint32((1 << top) - 1)
    qv = limbs(q, L)
    flat = out.reshape(-1, L)
    while True:
        ge = np.zeros(flat.shape[0], dtype=bool)
        eq = np.ones(flat.shape[0], dtype=bool)
        for l in range(L - 1, -1, -1):
            ge |= eq & (flat[:, l] > qv[l])
            eq &= flat[:, l] == qv[l]
        ge |= eq
        bad = np.nonzero(ge)[0]
        if bad.size == 0:
            break
        fresh = rng.integers(0, 1 << 32, size=bad.size, dtype=np.uint64).astype(np.uint32)
        flat[bad, L - 1] = fresh & np.uint32((1 << top) - 1) if top < 32 else fresh
    return out


# the operand distributions of the N=32768, W=868 benchmark configuration
DISTRIBUTIONS = ("uniform", "all_q_minus_1", "sparse_1pct", "small_16bit")


def operands(dist: str, N: int, W: int, q: int, count: int, seed: int) -> np.ndarray:
    """[count, N, L] u32 limbs drawn from a named distribution (seeded):
    uniform        coefficients uniform in [0, q);
    all_q_minus_1  every coefficient q - 1 (the largest input);
    sparse_1pct    1% of the coefficients (positions drawn without replacement) uniform in
                   [0, q), the rest 0;
    small_16bit    coefficients uniform in [0, 2^16)."""
    L = (W + 31) // 32
    if dist == "uniform":
        return uniform_operands(N, W, q, count, seed)
    if dist == "all_q_minus_1":
        return np.broadcast_to(limbs(q - 1, L), (count, N, L)).copy()
    rng = np.random.Generator(np.random.PCG64(seed))
    if dist == "small_16bit":
        out = np.zeros((count, N, L), dtype=np.uint32)
        out[..., 0] = rng.integers(0, 1 << 16, size=(count, N), dtype=np.uint32)
        return out
    if dist == "sparse_1pct":
        out = np.zeros((count, N, L), dtype=np.uint32)
        nz = max(1, N // 100)
        vals = uniform_operands(nz, W, q, count, seed + 1)
        for i in range(count):
            pos = rng.choice(N, size=nz, replace=False)
            out[i, pos] = vals[i]
        return out
    raise ValueError("unknown distribution %r" % dist)


def _load_grid():
    # spec-derived primes of N in {4096..65536} x W in {256, 868, 1747, 3000}, as 2^W - q
    table = {
        (4096, 256): 466943, (4096, 868): 2990079, (4096, 1747): 3850239, (4096, 3000): 5382143,
        (8192, 256): 2719743, (8192, 868): 11993087, (8192, 1747): 3850239, (8192, 3000): 61112319,
        (16384, 256): 2719743, (16384, 868): 11993087, (16384, 1747): 5275647, (16384, 3000): 61112319,
        (32768, 256): 5308415, (32768, 868): 11993087, (32768, 1747): 9699327, (32768, 3000): 252903423,
        (65536, 256): 8519679, (65536, 868): 43646975, (65536, 1747): 9699327, (65536, 3000): 293994495,
    }
    SPEC_DELTAS.update(table)


_load_grid()
