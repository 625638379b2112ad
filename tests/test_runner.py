"""The point-directory runner (lib/polymult_solution): the challenge harness's directory format
(manifest.json, point/q.bin, cases/NNNNNN/{a,b}.bin -> out/NNNNNN/c.bin, out/results.json).

CPU tests: usage and error exits.  GPU tests: a point directory written by the oracle's point
writer is answered bit-exactly, results.json has the harness's schema, and the reference's own
harness (its solve.cu in CPU-emulator form, oracle/_ref/solution_emu) writes the same c.bin
files for the same directory."""
import json
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import PKG, ORACLE, orc

RUNNER = os.path.join(PKG, "lib", "polymult_solution")


def _runner():
    if not os.path.exists(RUNNER):
        subprocess.run(["python", os.path.join(PKG, "build.py")], check=True)
    return RUNNER


def test_runner_usage_and_missing_directory(tmp_path):
    r = subprocess.run([_runner()], capture_output=True, text=True)
    assert r.returncode == 2 and "usage" in r.stderr
    r = subprocess.run([_runner(), str(tmp_path / "nope")], capture_output=True, text=True)
    assert r.returncode == 1 and "manifest.json" in r.stderr


def _point(tmp_path, N, W, modes):
    q = orc.spec_prime(N, W)
    L = (W + 31) // 32
    cases, expect = [], []
    for s, mode in enumerate(modes):
        rng = orc.case_rng(s, N, W)
        a, b = orc.case_operands(mode, rng, q, N)
        cases.append((orc.pack_limbs(a, L), orc.pack_limbs(b, L)))
        expect.append(orc.pack_limbs(orc.negacyclic_mul(a, b, q, N), L))
    root = str(tmp_path / "point")
    orc.write_point_dir(root, N, W, q, cases, expect)
    return root, q, L, expect


@pytest.mark.gpu
def test_runner_answers_point_directory(tmp_path):
    N, W = 1024, 256
    root, q, L, expect = _point(tmp_path, N, W, ["random", "max", "sparse", "small"])
    r = subprocess.run([_runner(), root], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    res = json.load(open(os.path.join(root, "out", "results.json")))
    assert res["init_s"] > 0
    assert [c["i"] for c in res["cases"]] == list(range(4))
    assert all(c["status"] == "ok" and c["seconds"] > 0 for c in res["cases"])
    for s, c in enumerate(expect):
        assert np.array_equal(orc.read_result(root, s, N, L), c), s
    ref = os.path.join(ORACLE, "_ref", "solution_emu")
    if os.path.exists(ref):  # the reference's own harness + solve.cu on the same directory
        other = str(tmp_path / "point_ref")
        shutil.copytree(root, other, ignore=shutil.ignore_patterns("out"))
        r = subprocess.run([ref, other], capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr
        for s in range(len(expect)):
            a = open(os.path.join(root, "out", "%06d" % s, "c.bin"), "rb").read()
            b = open(os.path.join(other, "out", "%06d" % s, "c.bin"), "rb").read()
            assert a == b, s
        ref_res = json.load(open(os.path.join(other, "out", "results.json")))
        assert set(ref_res) == set(res) and set(ref_res["cases"][0]) == set(res["cases"][0])


@pytest.mark.gpu
def test_runner_records_a_crashed_case(tmp_path):
    N, W = 64, 100
    root, q, L, expect = _point(tmp_path, N, W, ["random", "random"])
    # truncate case 1's b.bin: the harness records that case as crashed and goes on
    with open(os.path.join(root, "cases", "000001", "b.bin"), "r+b") as f:
        f.truncate(12)
    r = subprocess.run([_runner(), root], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    res = json.load(open(os.path.join(root, "out", "results.json")))
    assert res["cases"][0]["status"] == "ok"
    assert res["cases"][1]["status"] == "crashed" and res["cases"][1]["seconds"] is None
    assert "b.bin" in res["cases"][1]["note"]
    assert np.array_equal(orc.read_result(root, 0, N, L), expect[0])
