#!/usr/bin/env python3
"""Generates the golden fixtures in this directory from the reference's OWN checker.

Run where the reference is checked out: by default a directory named `reference` beside
this repository; POLYMULT_REFERENCE names another.  It imports the reference's tests/oracle.py unchanged and uses
its spec-prime search, case generator and bigint negacyclic NTT to produce, per point:

  * q (hex) and delta = 2^W - q;
  * for each case: operand mode, seed index, sha256 of a.bin / b.bin / c.bin exactly as
    the reference writes them (tests/oracle.py:172-195);
  * for tiny points, the raw a/b/c limbs in raw/<N>_<W>_<s>.npz.

The points are the reference's own regression set (tests/run_emu.sh:20-33) plus the
benchmark configurations (N=4096/W=256; N=32768/W=868 in four distributions;
N=65536/W=1747) and the spec primes of the batched N x W grid.

    python tests/golden/make_golden.py            # everything (about 10 minutes)
    python tests/golden/make_golden.py --quick    # skip the two largest points
"""
import argparse
import hashlib
import importlib.util
import json
import multiprocessing as mp
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get("POLYMULT_REFERENCE",
                     os.path.normpath(os.path.join(HERE, "..", "..", "..", "reference")))

# (N, W, cases, mode) — tests/run_emu.sh:20-33, then the benchmark configurations.
POINTS = [
    (64, 32, 4, "mixed"),
    (16, 33, 4, "mixed"),
    (2, 40, 2, "mixed"),
    (1, 64, 2, "mixed"),
    (1024, 512, 4, "mixed"),
    (256, 1747, 4, "mixed"),
    (4096, 100, 2, "mixed"),
    (8192, 256, 4, "mixed"),
    (2048, 868, 2, "mixed"),
    (512, 4000, 2, "mixed"),
    (4096, 256, 1, "random"),                    # configuration: plain method, small
    (32768, 868, 4, "bench4"),                   # configuration: four distributions
    (65536, 1747, 1, "random"),                  # configuration: the ranked point
]
BENCH4 = ("random", "max", "sparse1pct", "small16")
GRID_N = (4096, 8192, 16384, 32768, 65536)
GRID_W = (256, 868, 1747, 3000)
RAW_LIMIT_WORDS = 4096       # raw limbs stored for points with N*L <= this


def load_reference_oracle():
    path = os.path.join(REF, "tests", "oracle.py")
    spec = importlib.util.spec_from_file_location("reference_oracle", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def load_own_generator():
    sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
    import negacyclic_oracle
    return negacyclic_oracle


def sha(raw: bytes) -> str:
    return hashlib.sha256(raw).hexdigest()


def one_point(args):
    N, W, cases, mode = args
    ref = load_reference_oracle()
    own = load_own_generator()
    L = (W + 31) // 32
    t0 = time.time()
    q = ref.negacyclic_prime(N, W)
    entry = {"N": N, "W": W, "L": L, "q_hex": "%x" % q, "delta": (1 << W) - q, "cases": []}
    for s in range(cases):
        if mode == "bench4":
            m = BENCH4[s % len(BENCH4)]
        elif mode == "mixed":
            m = ["random", "max", "sparse", "small"][s % 4]
        else:
            m = mode
        rng = ref.random.Random(1000 + 7919 * s + N + W)     # tests/oracle.py:180
        if m in ("sparse1pct", "small16"):
            a, b = own.case_operands(m, rng, q, N)             # distributions the reference lacks
        else:
            a, b = ref.operands(m, rng, q, N)                  # tests/oracle.py:156-169
        c = ref.negacyclic_ntt_mul(a, b, q, N)                 # tests/oracle.py:78-128
        ra, rb, rc = ref.pack(a, L), ref.pack(b, L), ref.pack(c, L)
        case = {"s": s, "mode": m, "a_sha256": sha(ra), "b_sha256": sha(rb), "c_sha256": sha(rc)}
        if N * L <= RAW_LIMIT_WORDS:
            fn = "%d_%d_%d.npz" % (N, W, s)
            np.savez_compressed(os.path.join(HERE, "raw", fn),
                                a=np.frombuffer(ra, "<u4").reshape(N, L),
                                b=np.frombuffer(rb, "<u4").reshape(N, L),
                                c=np.frombuffer(rc, "<u4").reshape(N, L))
            case["raw"] = "raw/" + fn
        entry["cases"].append(case)
    entry["gen_seconds"] = round(time.time() - t0, 1)
    return entry


def grid_prime(args):
    N, W = args
    ref = load_reference_oracle()
    q = ref.negacyclic_prime(N, W)
    return {"N": N, "W": W, "q_hex": "%x" % q, "delta": (1 << W) - q}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--quick", action="store_true")
    ap.add_argument("--jobs", type=int, default=os.cpu_count())
    args = ap.parse_args()
    os.makedirs(os.path.join(HERE, "raw"), exist_ok=True)
    pts = [p for p in POINTS if not (args.quick and p[0] >= 32768)]
    ctx = mp.get_context("spawn")
    with ctx.Pool(args.jobs) as pool:
        points = pool.map(one_point, sorted(pts, key=lambda p: -p[0] * p[1]))
        grid = pool.map(grid_prime, [(n, w) for n in GRID_N for w in GRID_W])
    ref = load_reference_oracle()
    ref.selftest()                                              # tests/oracle.py:231-239
    points.sort(key=lambda e: (e["N"], e["W"]))
    out = {"generator": "tests/golden/make_golden.py (imports the reference's tests/oracle.py)",
           "points": points, "grid_primes": grid}
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(out, f, indent=1)
    print("wrote %d points, %d grid primes" % (len(points), len(grid)))


if __name__ == "__main__":
    main()
