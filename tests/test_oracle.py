"""CPU: pins the oracle to the reference's own outputs (tests/golden, made by importing the
reference's tests/oracle.py) and cross-checks the three CPU checkers against each other.
Mirrors the reference's test strategy: bigint NTT vs schoolbook (tests/oracle.py:231-239),
byte-exact comparison of c.bin (tests/oracle.py:198-228), the run_emu.sh point set."""
import ctypes
import os
import random

import numpy as np
import pytest

from conftest import c_oracle_mul, orc, raw_case, ref_emu_path, regen_case, sha


def _points(golden, max_words=None):
    for pt in golden["points"]:
        if max_words is None or pt["N"] * pt["L"] <= max_words:
            yield pt


def test_generator_is_byte_identical_to_reference(golden):
    """a.bin / b.bin regenerated here hash to what the reference's generator wrote."""
    for pt in _points(golden):
        for case in pt["cases"]:
            a, b, _ = regen_case(pt, case)
            assert sha(a) == case["a_sha256"], (pt["N"], pt["W"], case)
            assert sha(b) == case["b_sha256"], (pt["N"], pt["W"], case)


def test_python_oracle_matches_raw_golden(golden):
    n = 0
    for pt in golden["points"]:
        q = int(pt["q_hex"], 16)
        for case in pt["cases"]:
            if "raw" not in case:
                continue
            a, b, c = raw_case(case)
            got = orc.negacyclic_mul(orc.unpack_limbs(a), orc.unpack_limbs(b), q, pt["N"])
            assert got == orc.unpack_limbs(c), (pt["N"], pt["W"], case["s"])
            n += 1
    assert n >= 10


def test_python_oracle_matches_golden_hashes(golden):
    for pt in _points(golden, max_words=64 * 1024):
        q = int(pt["q_hex"], 16)
        for case in pt["cases"]:
            a, b, _ = regen_case(pt, case)
            c = orc.negacyclic_mul(orc.unpack_limbs(a), orc.unpack_limbs(b), q, pt["N"])
            assert sha(orc.pack_limbs(c, pt["L"])) == case["c_sha256"], (pt["N"], pt["W"], case["s"])


def test_ntt_oracle_agrees_with_schoolbook():
    rng = random.Random(5)
    for N, W in [(1, 8), (2, 16), (4, 20), (8, 33), (16, 64), (32, 100), (64, 32), (128, 256)]:
        q = orc.spec_prime(N, W)
        for _ in range(3):
            a = [rng.randrange(q) for _ in range(N)]
            b = [rng.randrange(q) for _ in range(N)]
            assert orc.negacyclic_mul(a, b, q, N) == orc.negacyclic_mul_schoolbook(a, b, q, N)


def test_spec_prime_matches_golden(golden):
    for g in golden["grid_primes"]:
        if g["W"] > 1747:
            continue  # W=3000 searches take tens of seconds; the hex values are pinned in golden.json
        assert orc.spec_prime(g["N"], g["W"]) == int(g["q_hex"], 16)
    for pt in golden["points"]:
        if pt["W"] <= 1747:
            assert orc.spec_prime(pt["N"], pt["W"]) == int(pt["q_hex"], 16)


def test_c_oracle_matches_golden_all_points(golden):
    """The C restatement of the reference's RNS method, on every golden point incl. the
    N=32768/W=868 and N=65536/W=1747 configurations."""
    for pt in golden["points"]:
        q = int(pt["q_hex"], 16)
        for case in pt["cases"]:
            a, b, _ = regen_case(pt, case)
            c = c_oracle_mul(pt["N"], pt["W"], q, a, b)
            assert sha(c) == case["c_sha256"], (pt["N"], pt["W"], case["s"], case["mode"])


@pytest.mark.skipif(ref_emu_path() is None, reason="oracle/_ref not built (reference tree absent)")
def test_reference_emulator_matches_golden(golden):
    """The reference's own solve.cu (CPU-emulator build) reproduces the golden outputs."""
    lib = ctypes.CDLL(ref_emu_path())
    lib.ref_init.restype = ctypes.c_void_p
    lib.ref_init.argtypes = [ctypes.c_uint32] * 3 + [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int]
    lib.ref_run.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32] + [ctypes.c_void_p] * 3 + \
        [ctypes.c_char_p, ctypes.c_int]
    lib.ref_free.argtypes = [ctypes.c_void_p]
    err = ctypes.create_string_buffer(256)
    for pt in _points(golden, max_words=300 * 1024):
        N, W, L = pt["N"], pt["W"], pt["L"]
        qv = orc.limbs_of(int(pt["q_hex"], 16), L)
        st = lib.ref_init(N, W, L, qv.ctypes.data, err, 256)
        assert st, err.value
        try:
            for case in pt["cases"]:
                a, b, _ = regen_case(pt, case)
                c = np.zeros_like(a)
                assert lib.ref_run(st, N, L, a.ctypes.data, b.ctypes.data, c.ctypes.data, err, 256) == 0, err.value
                assert sha(c) == case["c_sha256"], (N, W, case["s"])
        finally:
            lib.ref_free(st)


def test_point_dir_roundtrip(tmp_path, golden):
    """The oracle writes the point-directory layout main.cpp reads (main.cpp:8-12)."""
    pt = next(p for p in golden["points"] if p["N"] == 64 and p["W"] == 32)
    cases = [regen_case(pt, c)[:2] for c in pt["cases"]]
    orc.write_point_dir(str(tmp_path), pt["N"], pt["W"], int(pt["q_hex"], 16), cases)
    m = open(os.path.join(tmp_path, "manifest.json")).read()
    assert '"N": 64' in m and '"cases": 4' in m
    a0 = np.fromfile(os.path.join(tmp_path, "cases", "000000", "a.bin"), dtype="<u4").reshape(64, 1)
    assert sha(a0) == pt["cases"][0]["a_sha256"]


def test_uniform_limbs_in_range():
    q = orc.spec_prime(256, 100)
    x = orc.uniform_limbs(256, 100, q, seed=3)
    vals = orc.unpack_limbs(x)
    assert all(0 <= v < q for v in vals) and len(set(vals)) == 256


def test_workload_spec_primes_match_reference(golden):
    """The package's embedded spec primes (used by bench.py and serving) are the reference's."""
    import workload
    for g in golden["grid_primes"]:
        assert workload.spec_prime(g["N"], g["W"]) == int(g["q_hex"], 16)
    q = workload.spec_prime(256, 100)
    x = workload.uniform_operands(256, 100, q, 2, seed=9)
    vals = [int.from_bytes(x[i, n].tobytes(), "little") for i in range(2) for n in range(256)]
    assert all(v < q for v in vals)
