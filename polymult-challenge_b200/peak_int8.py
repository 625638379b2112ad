#!/usr/bin/env python3
"""Measured int8 tensor-core peak of this GPU: the denominator for the tcgen05 kernels'
tensor-pipe rates (the decomposition and the CRT are int8 GEMMs, kind::i8).

    python polymult-challenge_b200/peak_int8.py [--size 8192] [--seconds 2]

cuBLAS's int8 GEMM (torch._int_mm: int8 x int8 -> int32, a row-major, b column-major) on
square M = N = K = size operands, timed with CUDA events on the current stream after warm-up.
burst: the best of 10 single GEMMs; sustained: a loop of about `seconds` seconds (the power cap
settles there). Prints one JSON line in TOPS (10^12 int8 multiply-adds x 2 per second).
"""
import argparse
import json


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--size", type=int, default=8192)
    ap.add_argument("--seconds", type=float, default=2.0)
    args = ap.parse_args()
    import torch

    n = args.size
    g = torch.Generator(device="cuda").manual_seed(7)
    a = torch.randint(-128, 128, (n, n), dtype=torch.int8, device="cuda", generator=g)
    b = torch.randint(-128, 128, (n, n), dtype=torch.int8, device="cuda", generator=g).t()  # column-major
    ops = 2.0 * n * n * n
    for _ in range(5):
        torch._int_mm(a, b)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    best = float("inf")
    for _ in range(10):
        e0.record()
        torch._int_mm(a, b)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1000.0)
    reps = max(1, int(args.seconds / best))
    e0.record()
    for _ in range(reps):
        torch._int_mm(a, b)
    e1.record()
    e1.synchronize()
    sustained = e0.elapsed_time(e1) / 1000.0 / reps
    # exactness spot check of the library GEMM on a corner block
    k = 64
    ref = (a[:k].to(torch.int32).cpu() @ b[:, :k].to(torch.int32).cpu())
    ok = bool(torch.equal(torch._int_mm(a, b)[:k, :k].cpu(), ref))
    print(json.dumps({"int8_tops_burst": round(ops / best / 1e12, 1), "int8_tops_sustained": round(ops / sustained / 1e12, 1),
                      "size": n, "sustained_reps": reps, "method": "torch._int_mm (cuBLAS int8 GEMM), CUDA events",
                      "device": torch.cuda.get_device_name(0), "corner_block_exact": ok}))


if __name__ == "__main__":
    main()
