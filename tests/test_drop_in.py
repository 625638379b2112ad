"""The drop-in as the platform builds it: the reference's own harness main.cpp and fherma.h,
unchanged, compiled and linked against libpolymult_b200.so (oracle/_ref/harness_b200, built by
`make -C oracle` where the reference tree is present, as the recipe in INTEGRATION.md does with
CMake).  The harness binds fherma_init / fherma_run / fherma_free (main.cpp:156, 183, 206;
fherma.toml:7-10) and must find them in our library.

CPU test: the binary exists and resolves every fherma symbol against our library.  GPU test: it
answers a point directory, and every c.bin equals both the oracle's expected value and what the
reference's own solve.cu (CPU-emulator build, oracle/_ref/solution_emu) writes for the same
directory; results.json has the same schema."""
import json
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import ORACLE, orc

HARNESS = os.path.join(ORACLE, "_ref", "harness_b200")
REF_EMU = os.path.join(ORACLE, "_ref", "solution_emu")


def _need(path):
    if not os.path.exists(path):
        pytest.fail("%s is missing: build it with `make -C oracle` where the reference tree is present" % path)
    return path


def test_harness_links_our_library():
    r = subprocess.run(["ldd", _need(HARNESS)], capture_output=True, text=True)
    assert r.returncode == 0 and "libpolymult_b200.so" in r.stdout and "not found" not in r.stdout, r.stdout
    # the harness's undefined fherma symbols are exactly what our library defines
    und = subprocess.run(["nm", "-DC", "--undefined-only", HARNESS], capture_output=True, text=True).stdout
    for sym in ("fherma_init(fherma::Point const&)", "fherma_run(void*, fherma::Inputs const&)", "fherma_free(void*)"):
        assert sym in und, sym
    r = subprocess.run([HARNESS], capture_output=True, text=True)
    assert r.returncode != 0  # usage without a directory


def _point(root, N, W, modes):
    q = orc.spec_prime(N, W)
    L = (W + 31) // 32
    cases, expect = [], []
    for s, mode in enumerate(modes):
        rng = orc.case_rng(s, N, W)
        a, b = orc.case_operands(mode, rng, q, N)
        cases.append((orc.pack_limbs(a, L), orc.pack_limbs(b, L)))
        expect.append(orc.pack_limbs(orc.negacyclic_mul(a, b, q, N), L))
    orc.write_point_dir(root, N, W, q, cases, expect)
    return L, expect


@pytest.mark.gpu
@pytest.mark.parametrize("N,W,modes", [(4096, 256, ["random", "max", "sparse", "small"]),
                                       (2048, 868, ["random", "max"]),
                                       (64, 32, ["random", "max"])])
def test_reference_harness_on_our_library(tmp_path, N, W, modes):
    root = str(tmp_path / "point")
    L, expect = _point(root, N, W, modes)
    r = subprocess.run([_need(HARNESS), root], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    res = json.load(open(os.path.join(root, "out", "results.json")))
    assert all(c["status"] == "ok" for c in res["cases"]), res
    for s, c in enumerate(expect):
        assert np.array_equal(orc.read_result(root, s, N, L), c), "case %d differs from the oracle" % s
    # the reference's own implementation (CPU-emulator build) on the same directory
    other = str(tmp_path / "point_ref")
    shutil.copytree(root, other, ignore=shutil.ignore_patterns("out"))
    r = subprocess.run([_need(REF_EMU), other], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    for s in range(len(expect)):
        ours = open(os.path.join(root, "out", "%06d" % s, "c.bin"), "rb").read()
        theirs = open(os.path.join(other, "out", "%06d" % s, "c.bin"), "rb").read()
        assert ours == theirs, "case %d: c.bin differs from the reference's" % s
    ref_res = json.load(open(os.path.join(other, "out", "results.json")))
    assert set(ref_res) == set(res) and set(ref_res["cases"][0]) == set(res["cases"][0])
