#!/usr/bin/env python3
"""One device-resident multiply group at a chosen point, for profiling under ncu.

    python polymult-challenge_b200/profile_case.py [--N 65536] [--W 1747] [--gemm tensor] [--count 1] [--host 0]

pm_init runs one warm-up multiply through the chunked host pipeline first (the input
column chunks launch the decomposition and column-pass kernels once per chunk, the output
chunks the inverse column pass and CRT once per chunk; the row passes launch once each), then
this script runs `count` multiplies through pm_run_device and checks the device status.
Select the device-resident launch of a kernel with ncu's -k / -s (skip the warm-up launches):
    ncu --set full --clock-control none -k regex:k_crt_tc -s 20 -c 1 python .../profile_case.py
--host H then runs H multiplies through pm_run (host operands, the chunked PCIe pipeline;
--pinned puts them in page-locked memory, which pm_run copies directly; --tune runs the
chunk-schedule autotuner for that kind of call first); with
POLYMULT_PROFILE=1 in the environment each call prints its host and device timeline.
"""
import argparse
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--N", type=int, default=65536)
    ap.add_argument("--W", type=int, default=1747)
    ap.add_argument("--gemm", default="tensor")
    ap.add_argument("--count", type=int, default=1)
    ap.add_argument("--host", type=int, default=0)
    ap.add_argument("--pinned", action="store_true", help="host operands and result in page-locked memory")
    ap.add_argument("--tune", action="store_true", help="tune the host pipeline's chunk schedule first")
    a = ap.parse_args()
    import numpy as np
    import torch
    import polymult
    import workload
    L = (a.W + 31) // 32
    q = workload.spec_prime(a.N, a.W)
    ops = workload.uniform_operands(a.N, a.W, q, 2 * a.count, seed=5)
    da = torch.from_numpy(np.ascontiguousarray(ops[:a.count]).view(np.int32)).cuda()
    db = torch.from_numpy(np.ascontiguousarray(ops[a.count:]).view(np.int32)).cuda()
    dc = torch.zeros_like(da)
    with polymult.Multiplier(a.N, a.W, workload.limbs(q, L), gemm=a.gemm) as m:
        info = m.info()
        m.multiply_device(da.data_ptr(), db.data_ptr(), dc.data_ptr(), a.count,
                          torch.cuda.current_stream().cuda_stream)
        m.sync()
        if a.host and a.tune:
            print("schedule", m.tune_pipeline(3, pinned=a.pinned))
        if a.host:
            if a.pinned:
                def buf():
                    return torch.empty((a.N, L), dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)
                a0, b0, out = buf(), buf(), buf()
                a0[:] = ops[0]
                b0[:] = ops[a.count]
            else:
                a0 = np.ascontiguousarray(ops[0])
                b0 = np.ascontiguousarray(ops[a.count])
                out = np.empty((a.N, L), dtype=np.uint32)
            for _ in range(a.host):
                m.multiply(a0, b0, out)
            if not np.array_equal(out, dc[0].cpu().numpy().view(np.uint32)):
                raise SystemExit("host and device paths differ")
    print("ok N=%d W=%d K=%d gemm=%s count=%d input chunks/operand=%s" % (
        a.N, a.W, info["K"], info["gemm"], a.count, "see pm_info"))


if __name__ == "__main__":
    main()
