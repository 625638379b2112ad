#!/usr/bin/env python3
"""Builds libpolymult_b200.so in-tree for sm_100a (B200) with nvcc.

    python polymult-challenge_b200/build.py [--force] [--verbose]

Every .cu / .cpp under csrc/ is compiled with
    -gencode arch=compute_100a,code=sm_100a -lineinfo -O3 -Xptxas -v
and linked (shared cudart) into polymult-challenge_b200/lib/libpolymult_b200.so; the
point-directory runner runner/polymult_solution.cpp is linked against it into
lib/polymult_solution.  The ptxas
resource report (registers, spills, shared memory per kernel) goes to lib/ptxas.log.
"""
import argparse
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
OBJDIR = os.path.join(HERE, "_build")
LIB = os.path.join(LIBDIR, "libpolymult_b200.so")
RUNNER_SRC = os.path.join(HERE, "runner", "polymult_solution.cpp")
RUNNER = os.path.join(LIBDIR, "polymult_solution")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
          "-I" + CSRC, "-I" + os.path.join(HERE, "..", "include")]


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    inc = os.path.join(HERE, "..", "include")
    hs += [os.path.join(inc, f) for f in os.listdir(inc) if f.endswith(".h")]
    return hs


def compile_one(src, verbose):
    obj = os.path.join(OBJDIR, os.path.basename(src) + ".o")
    cmd = [NVCC] + ARCH + COMMON + ["-Xptxas", "-v", "-c", src, "-o", obj]
    if src.endswith(".cpp"):
        cmd = [NVCC] + ARCH + COMMON + ["-x", "cu", "-c", src, "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed on %s:\n%s%s" % (src, r.stdout, r.stderr))
    return obj, r.stderr


def up_to_date():
    if not os.path.exists(LIB):
        return False
    if not os.path.exists(RUNNER):
        return False
    t = min(os.path.getmtime(LIB), os.path.getmtime(RUNNER))
    return all(os.path.getmtime(f) < t for f in sources() + headers() + [__file__, RUNNER_SRC])


def build(force=False, verbose=False):
    if not force and up_to_date():
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    os.makedirs(OBJDIR, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        results = list(ex.map(lambda s: compile_one(s, verbose), sources()))
    objs = [o for o, _ in results]
    with open(os.path.join(LIBDIR, "ptxas.log"), "w") as f:
        for (_, log), src in zip(results, sources()):
            f.write("== %s\n%s\n" % (os.path.basename(src), log))
    cmd = [NVCC] + ARCH + ["-shared", "-cudart", "shared", "-o", LIB] + objs + \
        ["-Xlinker", "-rpath,/usr/local/cuda/lib64", "-lpthread"]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed:\n%s%s" % (r.stdout, r.stderr))
    # the point-directory runner, linked against the library (found next to it at run time)
    cmd = ["g++", "-O2", "-std=c++17", "-I" + os.path.join(HERE, "..", "include"), RUNNER_SRC, "-o", RUNNER,
           "-L" + LIBDIR, "-lpolymult_b200", "-Wl,-rpath,$ORIGIN", "-Wl,-rpath,/usr/local/cuda/lib64"]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("runner build failed:\n%s%s" % (r.stdout, r.stderr))
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    try:
        print(build(a.force, a.verbose))
    except RuntimeError as e:
        print(e, file=sys.stderr)
        sys.exit(1)
