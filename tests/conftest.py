"""Shared test setup: the `gpu` marker, import paths, golden fixtures, case regeneration."""
import hashlib
import json
import os
import subprocess
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "polymult-challenge_b200")
ORACLE = os.path.join(REPO, "oracle")
GOLDEN = os.path.join(REPO, "tests", "golden")
for p in (PKG, ORACLE):
    if p not in sys.path:
        sys.path.insert(0, p)

import negacyclic_oracle as orc  # noqa: E402


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 and the built CUDA library")


def load_golden():
    with open(os.path.join(GOLDEN, "golden.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def golden():
    return load_golden()


def sha(arr) -> str:
    return hashlib.sha256(np.ascontiguousarray(arr, dtype="<u4").tobytes()).hexdigest()


def regen_case(point, case):
    """Re-creates a golden case's operands with the oracle's generator (byte-identical to
    the reference's tests/oracle.py for its modes)."""
    N, W, L = point["N"], point["W"], point["L"]
    q = int(point["q_hex"], 16)
    rng = orc.case_rng(case["s"], N, W)
    a, b = orc.case_operands(case["mode"], rng, q, N)
    return orc.pack_limbs(a, L), orc.pack_limbs(b, L), q


def raw_case(case):
    d = np.load(os.path.join(GOLDEN, case["raw"]))
    return d["a"], d["b"], d["c"]


_built = {}


def ensure_oracle_built():
    """Builds oracle/_build/librns_oracle.so (and oracle/_ref when the reference tree exists)."""
    if "oracle" not in _built:
        so = os.path.join(ORACLE, "_build", "librns_oracle.so")
        if not os.path.exists(so):
            subprocess.run(["make", "-s", "-C", ORACLE], check=True)
        _built["oracle"] = so
    return _built["oracle"]


def c_oracle():
    import ctypes
    lib = ctypes.CDLL(ensure_oracle_built())
    lib.orc_negacyclic_mul.argtypes = [ctypes.c_uint32] * 3 + [ctypes.c_void_p] * 4
    lib.orc_negacyclic_mul.restype = ctypes.c_int
    return lib


def c_oracle_mul(N, W, q, a, b):
    L = (W + 31) // 32
    qv = orc.limbs_of(q, L)
    c = np.zeros((N, L), dtype=np.uint32)
    a = np.ascontiguousarray(a, dtype=np.uint32)
    b = np.ascontiguousarray(b, dtype=np.uint32)
    rc = c_oracle().orc_negacyclic_mul(N, W, L, qv.ctypes.data, a.ctypes.data, b.ctypes.data, c.ctypes.data)
    assert rc == 0, "C oracle returned %d" % rc
    return c


def ref_emu_path():
    p = os.path.join(ORACLE, "_ref", "libref_emu.so")
    return p if os.path.exists(p) else None


def ensure_library():
    """The CUDA library must exist for GPU tests; build it in-tree if it is missing."""
    import polymult
    if not os.path.exists(polymult.LIB_PATH):
        subprocess.run([sys.executable, os.path.join(PKG, "build.py")], check=True)
    return polymult.load()
