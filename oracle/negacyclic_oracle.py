"""CPU oracle for the negacyclic product c = a*b mod (X^N + 1, q).

TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and bench.py's
cpu_baseline / reference leg may import this module, and only as the checker.
The product path (the CUDA library) never calls it.

This file restates, in its own code, the reference's independent Python bigint
checker (tests/oracle.py of TrivialError/polymult-challenge):

  * spec prime q: the largest prime below 2^W with q == 1 (mod 2N)
    (tests/oracle.py:48-57), with a Miller-Rabin test (tests/oracle.py:22-45);
  * a primitive 2N-th root of unity psi mod q (tests/oracle.py:60-67);
  * the negacyclic product through a psi-merged NTT computed directly mod q,
    Cooley-Tukey forward and Gentleman-Sande inverse (tests/oracle.py:78-128);
  * schoolbook negacyclic multiplication for cross-checks (tests/oracle.py:131-140);
  * the limb layout, L little-endian u32 limbs per coefficient (tests/oracle.py:143-153,
    fherma.h:31-40);
  * the seeded case generator and its operand modes (tests/oracle.py:156-195), plus the
    two extra distributions the benchmark configurations name (1% sparse, < 2^16);
  * the point-directory layout main.cpp reads and writes (main.cpp:8-12, 137-209).

Parity pin: tests/golden/ holds fixtures produced by importing the reference's own
tests/oracle.py (script: tests/golden/make_golden.py); tests/test_oracle.py checks this
module against them.
"""
from __future__ import annotations

import hashlib
import json
import os
import random
from typing import List, Sequence, Tuple

import numpy as np

# ----------------------------------------------------------------------------------
# primes and roots (tests/oracle.py:22-67)
# ----------------------------------------------------------------------------------

_SMALL_PRIMES = (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37)


def is_probable_prime(n: int, rounds: int = 32) -> bool:
    """Miller-Rabin with fixed-seed witnesses (tests/oracle.py:22-45)."""
    if n < 2:
        return False
    for sp in _SMALL_PRIMES:
        if n % sp == 0:
            return n == sp
    d, s = n - 1, 0
    while not d & 1:
        d >>= 1
        s += 1
    wit = random.Random(0xC0FFEE)
    for _ in range(rounds):
        x = pow(wit.randrange(2, n - 1), d, n)
        if x == 1 or x == n - 1:
            continue
        for _ in range(s - 1):
            x = x * x % n
            if x == n - 1:
                break
        else:
            return False
    return True


def spec_prime(N: int, W: int) -> int:
    """Largest prime q < 2^W with q == 1 (mod 2N) (tests/oracle.py:48-57)."""
    step = 2 * N
    cand = (1 << W) - 1
    cand -= (cand - 1) % step          # largest value == 1 (mod 2N) not above 2^W - 1
    while cand > 1:
        if is_probable_prime(cand):
            return cand
        cand -= step
    raise ValueError("no prime == 1 mod 2N below 2^W")


def psi_root(q: int, N: int) -> int:
    """Smallest-generator primitive 2N-th root of unity mod q (tests/oracle.py:60-67)."""
    e = (q - 1) // (2 * N)
    for g in range(2, 10000):
        x = pow(g, e, q)
        if pow(x, N, q) == q - 1:
            return x
    raise ValueError("no primitive 2N-th root found")


# ----------------------------------------------------------------------------------
# negacyclic products (tests/oracle.py:70-140)
# ----------------------------------------------------------------------------------

def _bitrev_table(logn: int) -> List[int]:
    rev = [0] * (1 << logn)
    for k in range(1, 1 << logn):
        rev[k] = (rev[k >> 1] >> 1) | ((k & 1) << (logn - 1))
    return rev


def negacyclic_mul(a: Sequence[int], b: Sequence[int], q: int, N: int) -> List[int]:
    """c = a*b mod (X^N+1, q) by a psi-merged NTT directly mod q (tests/oracle.py:78-128).

    Forward: Cooley-Tukey, natural order in, bit-reversed order out, twiddle of stage
    with m groups, group i = psi^bitrev(m+i).  Inverse: Gentleman-Sande with
    psi^-bitrev(m+i), then the N^-1 scale.
    """
    if N == 1:
        return [a[0] * b[0] % q]
    logn = N.bit_length() - 1
    psi = psi_root(q, N)
    ipsi = pow(psi, q - 2, q)
    rev = _bitrev_table(logn)
    pw, ipw = [1] * N, [1] * N
    for i in range(1, N):
        pw[i] = pw[i - 1] * psi % q
        ipw[i] = ipw[i - 1] * ipsi % q
    fw = [pw[rev[k]] for k in range(N)]
    iw = [ipw[rev[k]] for k in range(N)]

    def forward(x):
        x = [v % q for v in x]
        half = N
        groups = 1
        while groups < N:
            half >>= 1
            for g in range(groups):
                w = fw[groups + g]
                base = 2 * g * half
                for j in range(base, base + half):
                    u, v = x[j], x[j + half] * w % q
                    x[j], x[j + half] = (u + v) % q, (u - v) % q
            groups <<= 1
        return x

    def inverse(x):
        x = list(x)
        half = 1
        groups = N >> 1
        while groups >= 1:
            for g in range(groups):
                w = iw[groups + g]
                base = 2 * g * half
                for j in range(base, base + half):
                    u, v = x[j], x[j + half]
                    x[j], x[j + half] = (u + v) % q, (u - v) * w % q
            half <<= 1
            groups >>= 1
        ninv = pow(N, q - 2, q)
        return [v * ninv % q for v in x]

    fa, fb = forward(a), forward(b)
    return inverse([u * v % q for u, v in zip(fa, fb)])


def negacyclic_mul_schoolbook(a: Sequence[int], b: Sequence[int], q: int, N: int) -> List[int]:
    """O(N^2) negacyclic product mod q (tests/oracle.py:131-140); small N only."""
    acc = [0] * N
    for i, ai in enumerate(a):
        if not ai:
            continue
        for j, bj in enumerate(b):
            k = i + j
            if k < N:
                acc[k] += ai * bj
            else:
                acc[k - N] -= ai * bj
    return [v % q for v in acc]


# ----------------------------------------------------------------------------------
# limb layout (tests/oracle.py:143-153; fherma.h:31-40)
# ----------------------------------------------------------------------------------

def pack_limbs(values: Sequence[int], L: int) -> np.ndarray:
    """Coefficients -> [len(values), L] little-endian u32 limbs."""
    nbytes = 4 * L
    raw = b"".join(int(v).to_bytes(nbytes, "little") for v in values)
    return np.frombuffer(raw, dtype="<u4").reshape(len(values), L).copy()


def unpack_limbs(limbs: np.ndarray) -> List[int]:
    """[N, L] u32 limbs -> Python ints."""
    arr = np.ascontiguousarray(limbs, dtype="<u4")
    n = arr.shape[0]
    raw = arr.tobytes()
    step = 4 * arr.shape[1]
    return [int.from_bytes(raw[k * step:(k + 1) * step], "little") for k in range(n)]


def limbs_of(x: int, L: int) -> np.ndarray:
    return pack_limbs([x], L)[0]


# ----------------------------------------------------------------------------------
# case generation (tests/oracle.py:156-195)
# ----------------------------------------------------------------------------------

REFERENCE_MODES = ("random", "max", "zero", "sparse", "small")
EXTRA_MODES = ("sparse1pct", "small16")
MIXED_CYCLE = ("random", "max", "sparse", "small")


def case_rng(s: int, N: int, W: int) -> random.Random:
    """Per-case generator seed of the reference (tests/oracle.py:180)."""
    return random.Random(1000 + 7919 * s + N + W)


def case_operands(mode: str, rng: random.Random, q: int, N: int) -> Tuple[List[int], List[int]]:
    """Operands of one case.

    The five reference modes draw from `rng` in the same order as tests/oracle.py:156-169,
    so a case generated here is byte-identical to the reference's.  `sparse1pct` (1% of the
    coefficients nonzero, uniform in [0,q)) and `small16` (uniform below 2^16) are the two
    further distributions of the N=32768/W=868 benchmark configuration.
    """
    if mode == "max":
        return [q - 1] * N, [q - 1] * N
    if mode == "zero":
        return [0] * N, [0] * N
    if mode == "sparse":
        a, b = [0] * N, [0] * N
        for _ in range(3):
            a[rng.randrange(N)] = rng.randrange(q)
            b[rng.randrange(N)] = rng.randrange(q)
        return a, b
    if mode == "small":
        a = [rng.randrange(3) for _ in range(N)]
        b = [q - 1 - rng.randrange(3) for _ in range(N)]
        return a, b
    if mode == "random":
        a = [rng.randrange(q) for _ in range(N)]
        b = [rng.randrange(q) for _ in range(N)]
        return a, b
    if mode == "sparse1pct":
        nz = max(1, N // 100)
        a, b = [0] * N, [0] * N
        for idx in rng.sample(range(N), nz):
            a[idx] = rng.randrange(q)
        for idx in rng.sample(range(N), nz):
            b[idx] = rng.randrange(q)
        return a, b
    if mode == "small16":
        a = [rng.randrange(1 << 16) for _ in range(N)]
        b = [rng.randrange(1 << 16) for _ in range(N)]
        return a, b
    raise ValueError("unknown operand mode %r" % mode)


def case_mode(s: int, mode: str) -> str:
    return MIXED_CYCLE[s % len(MIXED_CYCLE)] if mode == "mixed" else mode


def sha256_hex(arr: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(arr, dtype="<u4").tobytes()).hexdigest()


def uniform_limbs(N: int, W: int, q: int, seed: int) -> np.ndarray:
    """Fast seeded uniform [0,q) operand as [N, L] limbs (numpy PCG64 + rejection).

    For benchmark-size inputs where the reference's random.Random stream is too slow to
    reproduce; q = 2^W - delta with tiny delta, so rejection almost never fires.
    """
    L = (W + 31) // 32
    rng = np.random.Generator(np.random.PCG64(seed))
    out = rng.integers(0, 1 << 32, size=(N, L), dtype=np.uint64).astype(np.uint32)
    top_bits = W - 32 * (L - 1)
    if top_bits < 32:
        out[:, L - 1] &= np.uint32((1 << top_bits) - 1)
    qv = limbs_of(q, L)
    # rows >= q: compare from the top limb down
    ge = np.ones(N, dtype=bool)
    eq = np.ones(N, dtype=bool)
    for l in range(L - 1, -1, -1):
        gt_l = out[:, l] > qv[l]
        lt_l = out[:, l] < qv[l]
        ge = np.where(eq & gt_l, True, np.where(eq & lt_l, False, ge))
        eq &= out[:, l] == qv[l]
    for r in np.nonzero(ge)[0]:  # a row >= q has probability ~ delta / 2^W: fold it back below q
        out[r] = limbs_of(unpack_limbs(out[r:r + 1])[0] - q, L)
    return out


# ----------------------------------------------------------------------------------
# point directories (main.cpp:8-12, 137-209; tests/oracle.py:172-195)
# ----------------------------------------------------------------------------------

def write_point_dir(root: str, N: int, W: int, q: int, cases: Sequence[Tuple[np.ndarray, np.ndarray]],
                    expected: Sequence[np.ndarray] = ()) -> None:
    """Writes manifest.json, point/q.bin and cases/NNNNNN/{a,b}.bin (+ expected/NNNNNN/c.bin)."""
    L = (W + 31) // 32
    os.makedirs(os.path.join(root, "point"), exist_ok=True)
    limbs_of(q, L).astype("<u4").tofile(os.path.join(root, "point", "q.bin"))
    for s, (a, b) in enumerate(cases):
        d = os.path.join(root, "cases", "%06d" % s)
        os.makedirs(d, exist_ok=True)
        np.ascontiguousarray(a, dtype="<u4").tofile(os.path.join(d, "a.bin"))
        np.ascontiguousarray(b, dtype="<u4").tofile(os.path.join(d, "b.bin"))
    for s, c in enumerate(expected):
        d = os.path.join(root, "expected", "%06d" % s)
        os.makedirs(d, exist_ok=True)
        np.ascontiguousarray(c, dtype="<u4").tofile(os.path.join(d, "c.bin"))
    with open(os.path.join(root, "manifest.json"), "w") as f:
        json.dump({"point": {"N": N, "W": W, "L": L}, "N": N, "W": W, "L": L, "cases": len(cases)}, f)


def read_result(root: str, s: int, N: int, L: int) -> np.ndarray:
    return np.fromfile(os.path.join(root, "out", "%06d" % s, "c.bin"), dtype="<u4").reshape(N, L)
