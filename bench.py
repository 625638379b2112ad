#!/usr/bin/env python3
"""Throughput of the negacyclic multiply c = a*b mod (X^N+1, q) at N=65536, W=1747 (L=55),
bit-exact, on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--gemm tensor|plain]
    python bench.py --profile-case [--N 65536 --W 1747 --gemm tensor --count 8 --host 0 ...]
    python bench.py --peak-int8 [--size 8192 --seconds 2]
    python bench.py --peak-butterfly

One step = one device-resident pass over a batch of BATCH multiplications whose operands
are already in HBM (inputs 2 x BATCH x 14.4 MB > the 126 MB L2, so no flush is needed).
Rank 0 prints one JSON line:
  value       whole-job device-resident mults/s (tensor-core form unless --gemm plain),
              CUDA events on the launching stream, max over ranks;
  plain_value the same with the CUDA-core (plain int32) GEMM form, measured in the same run;
  e2e         mults/s through the reference-facing call pm_run (fherma_run's C ABI) with
              operands and result in pinned host memory, host<->device copies inside the timed
              region, plus p50/p99 latency of that call; e2e.pageable: the same with pageable
              buffers (the reference harness's case, staged through the host pool);
  roofline    the dominant kernel's algorithmic bytes / its CUDA-event time vs measured HBM, on
              launches of BATCH multiplies as in the timed region;
  configs     the other benchmark configurations: N=4096/W=256 and N=32768/W=868 in four operand
              distributions, device-resident (tensor and plain forms) and end to end, each
              checked against the reference's CPU path;
  reference_gpu the reference's own GPU build (solve.cu + its harness, nvcc for sm_100a) on a
              point directory of the ranked point, beside this library's runner on the same one;
  serving     continuous batching over a sweep of offered rates, every result checked;
  batched     256 uneven multiplications in one CUDA-graph launch;
  cpu_baseline the reference's own solve.cu (CPU-emulator build) on host cores.
Multi-GPU: every rank multiplies its own batch (independent multiplications, no exchange):
"scaling": "weak".
--impl reference times the reference's CPU implementation alone (rank 0).
--profile-case runs one small device-resident group at a chosen point (for ncu: select its
launches with -k / -s / -c); --peak-int8 measures cuBLAS's int8 GEMM rate (the tensor-pipe
denominator of the tcgen05 kernels).
"""
import argparse
import ctypes
import datetime
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(REPO, "polymult-challenge_b200")
ORACLE = os.path.join(REPO, "oracle")
REF_GPU = os.path.join(REPO, "baseline", "_ref", "solution_gpu")
RUNNER = os.path.join(PKG, "lib", "polymult_solution")
sys.path.insert(0, PKG)

N_RANK, W_RANK = 65536, 1747
BATCH = 32
METRIC = "mults/s at N=65536 W=1747 (bit-exact): tensor-core+batched vs plain; p99 ms"
L2_BYTES = 126 * 10**6


def headline_config():
    """The `config` both arms print (the driver compares them)."""
    return {"workload": "negacyclic multiply c = a*b mod (X^N+1, q), N=65536 W=1747 L=55, q the spec-derived prime, "
                        "a and b uniform in [0, q) (seeded)",
            "N": N_RANK, "W": W_RANK, "L": 55, "parallelism": "replicas (independent multiplications per GPU)",
            "l2": "device-resident inputs larger than L2 (2 x 8 x 14.4 MB per step), no flush"}


# algorithmic HBM bytes of each kernel for ONE multiply (a launch of B multiplies moves B times this):
#   decomposition: N*L*4 in + K*N*4 out; column/row passes: K*N*4 in + out;
#   row pass of both operands (forward rows of a and b, pointwise, inverse rows of b; the
#   device-resident group's "rows_fused" stage, its "rows_a" stage then empty): 2*K*N*4 in +
#   K*N*4 out; CRT: K*N*4 in + N*L*4 out
def stage_bytes(stage, N, L, K):
    rn, cw = K * N * 4, N * L * 4
    return {"dec_a": cw + rn, "dec_b": cw + rn, "cols_a": 2 * rn, "cols_b": 2 * rn, "rows_a": 2 * rn,
            "rows_fused": 3 * rn, "cols_inv": 2 * rn, "crt": rn + cw}[stage]


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--gemm", default="tensor", choices=["tensor", "plain", "auto"])
    ap.add_argument("--batch", type=int, default=BATCH)
    ap.add_argument("--e2e-steps", type=int, default=20)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-batched", action="store_true", help="skip the uneven-batch leg")
    ap.add_argument("--no-configs", action="store_true", help="skip the N=4096 and N=32768 configuration legs")
    ap.add_argument("--no-reference-gpu", action="store_true", help="skip the reference's GPU build leg")
    ap.add_argument("--no-tune-pipeline", action="store_true", help="keep the default host chunk schedule")
    ap.add_argument("--batch-count", type=int, default=256)
    ap.add_argument("--batch-steps", type=int, default=5)
    ap.add_argument("--no-serving", action="store_true", help="skip the serving leg")
    ap.add_argument("--serve-requests", type=int, default=10000, help="requests per offered rate of the sweep")
    ap.add_argument("--serve-rates", default="2500,3500,4500", help="offered rates (requests/s) of the sweep")
    ap.add_argument("--serve-single-rate", type=float, default=600.0,
                    help="offered rate of the unbatched tensor-core comparator (one it sustains)")
    ap.add_argument("--serve-batch", type=int, default=8)
    ap.add_argument("--serve-streams", type=int, default=4)
    ap.add_argument("--serve-pool", type=int, default=64)
    ap.add_argument("--ref-gpu-cases", type=int, default=10)
    # --profile-case / --peak-int8 modes
    ap.add_argument("--profile-case", action="store_true")
    ap.add_argument("--N", type=int, default=N_RANK)
    ap.add_argument("--W", type=int, default=W_RANK)
    ap.add_argument("--count", type=int, default=1)
    ap.add_argument("--host", type=int, default=0)
    ap.add_argument("--pinned", action="store_true")
    ap.add_argument("--tune", action="store_true")
    ap.add_argument("--peak-int8", action="store_true")
    ap.add_argument("--peak-butterfly", action="store_true")
    ap.add_argument("--size", type=int, default=8192)
    ap.add_argument("--seconds", type=float, default=2.0)
    return ap.parse_args()


def measured_peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


class ClockSampler:
    """Samples SM clock and throttle reasons through NVML (read-only) while running."""

    def __init__(self, device_index):
        self.samples, self.reasons = [], set()
        self.max_mhz = None
        self._stop = threading.Event()
        self._ok = False
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(device_index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
            self._ok = True
        except Exception:
            pass

    def _run(self):
        nv = self.nv
        names = {"hw_slowdown": getattr(nv, "nvmlClocksThrottleReasonHwSlowdown", 0x8),
                 "hw_thermal_slowdown": getattr(nv, "nvmlClocksThrottleReasonHwThermalSlowdown", 0x40),
                 "sw_thermal_slowdown": getattr(nv, "nvmlClocksThrottleReasonSwThermalSlowdown", 0x20),
                 "sw_power_cap": getattr(nv, "nvmlClocksThrottleReasonSwPowerCap", 0x4)}
        while not self._stop.is_set():
            try:
                self.samples.append(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM))
                r = nv.nvmlDeviceGetCurrentClocksThrottleReasons(self.h)
                for k, bit in names.items():
                    if r & bit:
                        self.reasons.add(k)
            except Exception:
                pass
            time.sleep(0.005)

    def __enter__(self):
        if self._ok:
            self.t = threading.Thread(target=self._run, daemon=True)
            self.t.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        if self._ok:
            self.t.join()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons), "samples": 0}
        return {"sm_mhz": statistics.median(self.samples), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(self.samples)}


def dist_init():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=180))
    return world, rank, local


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda" if torch.cuda.is_available() else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def pct(sorted_ms, p):
    return sorted_ms[min(len(sorted_ms) - 1, int(p * len(sorted_ms)))]


# ------------------------------------------------------------------------------------------
# CPU legs: the reference's own implementation (oracle/_ref), else the C restatement
# ------------------------------------------------------------------------------------------
class ReferenceCPU:
    """The reference's solve.cu in CPU-emulator form (oracle/_ref/libref_emu.so, its own
    fherma_run behind a C shim), else the C restatement of its RNS method."""

    def __init__(self, N, W, q):
        import numpy as np
        self.N, self.W, self.L = N, W, (W + 31) // 32
        self.qv = np.frombuffer(int(q).to_bytes(4 * self.L, "little"), dtype="<u4").copy()
        so = os.path.join(ORACLE, "_ref", "libref_emu.so")
        self.err = ctypes.create_string_buffer(256)
        if os.path.exists(so):
            lib = ctypes.CDLL(so)
            lib.ref_init.restype = ctypes.c_void_p
            lib.ref_init.argtypes = [ctypes.c_uint32] * 3 + [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int]
            lib.ref_run.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32] + [ctypes.c_void_p] * 3 + \
                [ctypes.c_char_p, ctypes.c_int]
            lib.ref_free.argtypes = [ctypes.c_void_p]
            self.lib, self.kind = lib, "reference"
            self.st = lib.ref_init(N, W, self.L, self.qv.ctypes.data, self.err, 256)
            if not self.st:
                raise RuntimeError("reference init failed: %s" % self.err.value)
        else:
            lib = ctypes.CDLL(os.path.join(ORACLE, "_build", "librns_oracle.so"))
            lib.orc_negacyclic_mul.argtypes = [ctypes.c_uint32] * 3 + [ctypes.c_void_p] * 4
            self.lib, self.kind, self.st = lib, "port", None

    def run(self, a, b, c):
        if self.st:
            rc = self.lib.ref_run(self.st, self.N, self.L, a.ctypes.data, b.ctypes.data, c.ctypes.data, self.err, 256)
            if rc != 0:
                raise RuntimeError("reference run failed: %s" % self.err.value)
        else:
            rc = self.lib.orc_negacyclic_mul(self.N, self.W, self.L, self.qv.ctypes.data, a.ctypes.data, b.ctypes.data,
                                             c.ctypes.data)
            if rc != 0:
                raise RuntimeError("C oracle failed: %d" % rc)

    def multiply(self, a, b):
        import numpy as np
        c = np.zeros((self.N, self.L), dtype=np.uint32)
        self.run(np.ascontiguousarray(a, dtype=np.uint32), np.ascontiguousarray(b, dtype=np.uint32), c)
        return c

    def close(self):
        if self.st:
            self.lib.ref_free(self.st)
            self.st = None


def reference_cpu(N, W, q, a, b, calls, warm):
    """Times fherma_run of the reference's solve.cu (CPU-emulator build). Returns (dict, c)."""
    import numpy as np
    ref = ReferenceCPU(N, W, q)
    c = np.zeros((N, (W + 31) // 32), dtype=np.uint32)
    times = []
    try:
        for i in range(warm + calls):
            t0 = time.perf_counter()
            ref.run(a, b, c)
            dt = time.perf_counter() - t0
            if i >= warm:
                times.append(dt)
    finally:
        ref.close()
    if ref.kind == "reference":
        cores = 1
        sample = ("%d fherma_run call(s) after %d warm-up call(s) of the reference's solve.cu built against its CPU "
                  "emulator pm_emu.h (kernels run on 1 thread; staging pool min(12, cpus-2) threads), N=%d W=%d"
                  % (calls, warm, N, W))
    else:
        cores = os.cpu_count()
        sample = "%d call(s) of the C restatement of the reference's RNS method (OpenMP), N=%d W=%d" % (calls, N, W)
    return {"value": len(times) / sum(times), "unit": "mults/s", "cores": cores, "kind": ref.kind, "sample": sample,
            "host_cpus": os.cpu_count(), "cpu_model": cpu_model(), "seconds_per_call": statistics.median(times)}, c


def run_reference(args):
    world, rank, _ = dist_init()
    if rank != 0:
        return
    import numpy as np
    import workload
    N, W = N_RANK, W_RANK
    q = workload.spec_prime(N, W)
    ops = workload.uniform_operands(N, W, q, 2, seed=7)
    t0 = time.perf_counter()
    cpu, _ = reference_cpu(N, W, q, np.ascontiguousarray(ops[0]), np.ascontiguousarray(ops[1]),
                           calls=args.steps, warm=args.warmup)
    total = time.perf_counter() - t0
    line = {"metric": METRIC, "impl": "reference", "value": cpu["value"], "unit": "mults/s", "n_gpus": 0,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 / cpu["value"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic (uniform in [0,q), seeded)", "config": headline_config(),
            "arm": "the reference's fherma_run (solve.cu + pm_emu.h, CPU form), one call per step on host cores",
            "cpu_baseline": cpu, "e2e": {"value": cpu["value"], "unit": "mults/s", "h2d_bytes_per_step": 0,
                                         "d2h_bytes_per_step": 0},
            "wall_seconds": round(total, 1)}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------------------------------
# our arm
# ------------------------------------------------------------------------------------------
def pcie_bandwidth(torch, nbytes_h2d, nbytes_d2h, reps=5):
    """Pinned cudaMemcpyAsync bandwidth (GB/s) at the call's transfer sizes, CUDA events."""
    out = {}
    for name, n in (("h2d", nbytes_h2d), ("d2h", nbytes_d2h)):
        h = torch.empty(n, dtype=torch.uint8, pin_memory=True)
        d = torch.empty(n, dtype=torch.uint8, device="cuda")
        best = None
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            if name == "h2d":
                d.copy_(h, non_blocking=True)
            else:
                h.copy_(d, non_blocking=True)
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            best = ms if best is None else min(best, ms)
        out[name] = n / (best / 1000.0) / 1e9
    return out


def host_copy_gbs(torch, nbytes, threads=8, reps=5):
    """Host memory copy rate pageable -> page-locked (the pageable call's staging copy) with
    `threads` threads, best of `reps`, in GB/s."""
    import numpy as np
    words = nbytes // 4
    src = np.random.default_rng(3).integers(0, 2**32, size=words, dtype=np.uint32)
    dst = torch.empty(words, dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)
    parts = np.array_split(np.arange(words), threads)

    def work(p):
        np.copyto(dst[p[0]:p[-1] + 1], src[p[0]:p[-1] + 1])
    best = float("inf")
    for _ in range(reps):
        ts = [threading.Thread(target=work, args=(p,)) for p in parts]
        t0 = time.perf_counter()
        for t in ts:
            t.start()
        for t in ts:
            t.join()
        best = min(best, time.perf_counter() - t0)
    return nbytes / best / 1e9


def pcie_floor_ms(bw, N, L):
    return (2 * N * L * 4 / (bw["h2d"] * 1e9) + N * L * 4 / (bw["d2h"] * 1e9)) * 1000


def time_device(torch, m, sets, batch, steps, warm):
    """Device-resident groups: step k multiplies the batch of operand set k % len(sets)."""
    stream = torch.cuda.current_stream()
    for k in range(warm):
        da, db, dc = sets[k % len(sets)]
        m.multiply_device(da.data_ptr(), db.data_ptr(), dc.data_ptr(), batch, stream.cuda_stream)
    m.sync()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for k in range(steps):
        da, db, dc = sets[k % len(sets)]
        m.multiply_device(da.data_ptr(), db.data_ptr(), dc.data_ptr(), batch, stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize()
    m.sync()
    return e0.elapsed_time(e1)


def pinned_words(torch, shape):
    import numpy as np
    return torch.empty(shape, dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)


def e2e_leg(m, a0, b0, out, steps, world, floor_ms, want):
    """End to end through pm_run: per-call wall time, host buffers as given."""
    import numpy as np
    for _ in range(3):
        m.multiply(a0, b0, out)
    lat = []
    barrier(world)
    for _ in range(steps):
        t0 = time.perf_counter()
        m.multiply(a0, b0, out)
        lat.append(time.perf_counter() - t0)
    total_s = max_over_ranks(sum(lat), world)
    lat_ms = sorted(x * 1000 for x in lat)
    p50 = lat_ms[len(lat_ms) // 2]
    N, L = out.shape
    return {"value": world * steps / total_s, "unit": "mults/s", "h2d_bytes_per_step": 2 * N * L * 4,
            "d2h_bytes_per_step": N * L * 4, "p50_ms": round(p50, 4), "p99_ms": round(pct(lat_ms, 0.99), 4),
            "steps": steps, "matches_device_path": bool(np.array_equal(out, want)),
            "p50_over_floor": round(p50 / floor_ms, 3)}


def run_configs(torch, args, local, pending):
    """The other benchmark configurations (one GPU): N=4096/W=256 uniform, and N=32768/W=868
    in four operand distributions.  Per configuration: device-resident mults/s in the tensor and
    plain forms (batches of the engine's group, rotated over operand sets larger than twice L2),
    end-to-end pm_run latency with pinned and pageable buffers against the PCIe floor measured at
    that size.  The first multiply of each timed batch goes into `pending` for the cpu_baseline
    leg, which checks it against the reference's CPU path."""
    import numpy as np
    import polymult
    import workload
    specs = [("c1_N4096_W256_uniform", 4096, 256, "uniform")] + \
        [("c2_N32768_W868_" + d, 32768, 868, d) for d in workload.DISTRIBUTIONS]
    out = {}
    engines = {}
    try:
        for ci, (name, N, W, dist) in enumerate(specs):
            L = (W + 31) // 32
            q = workload.spec_prime(N, W)
            if (N, W) not in engines:
                qv = workload.limbs(q, L)
                mt = polymult.Multiplier(N, W, qv, gemm="tensor", device=local)
                mp = polymult.Multiplier(N, W, qv, gemm="plain", device=local)
                bw = pcie_bandwidth(torch, 2 * N * L * 4, N * L * 4)
                if args.no_tune_pipeline:
                    pipe, pipe_pg = mt.pipeline(pinned=True), mt.pipeline()
                else:
                    pipe, pipe_pg = mt.tune_pipeline(3, pinned=True), mt.tune_pipeline(3)
                engines[(N, W)] = (mt, mp, bw, pipe, pipe_pg)
            mt, mp, bw, pipe, pipe_pg = engines[(N, W)]
            B = min(int(mt.info()["group"]), 32)
            ops = workload.operands(dist, N, W, q, 2 * B, seed=500 + ci)
            a_h, b_h = np.ascontiguousarray(ops[:B]), np.ascontiguousarray(ops[B:])
            per_set = 2 * B * N * L * 4
            nsets = max(2, -(-2 * L2_BYTES // per_set))
            da0 = torch.from_numpy(a_h.view(np.int32)).cuda()
            db0 = torch.from_numpy(b_h.view(np.int32)).cuda()
            sets = [(da0.clone(), db0.clone(), torch.zeros_like(da0)) for _ in range(nsets)]
            steps = max(args.steps, nsets)
            ms_t = time_device(torch, mt, sets, B, steps, max(3, args.warmup))
            ms_p = time_device(torch, mp, sets, B, max(3, nsets), 2)
            res_t = sets[(steps - 1) % nsets][2].cpu().numpy().view(np.uint32)
            # the plain form into a fresh set, compared with the tensor form's timed output
            ct = torch.zeros_like(da0)
            mp.multiply_device(da0.data_ptr(), db0.data_ptr(), ct.data_ptr(), B, torch.cuda.current_stream().cuda_stream)
            mp.sync()
            res_p = ct.cpu().numpy().view(np.uint32)
            want = res_t[0]
            pending[name] = (N, W, q, a_h[0].copy(), b_h[0].copy(), want.copy(), res_p[0].copy())
            floor_ms = pcie_floor_ms(bw, N, L)
            pa, pb, pc = pinned_words(torch, (N, L)), pinned_words(torch, (N, L)), pinned_words(torch, (N, L))
            pa[:] = a_h[0]
            pb[:] = b_h[0]
            e2e_pinned = e2e_leg(mt, pa, pb, pc, args.e2e_steps, 1, floor_ms, want)
            e2e_pageable = e2e_leg(mt, np.ascontiguousarray(a_h[0]), np.ascontiguousarray(b_h[0]),
                                   np.empty((N, L), dtype=np.uint32), args.e2e_steps, 1, floor_ms, want)
            info = mt.info()
            out[name] = {
                "N": N, "W": W, "L": L, "K": info["K"], "distribution": dist, "batch": B, "operand_sets": nsets,
                "tensor_mults_per_s": round(steps * B / (ms_t / 1000.0), 1),
                "plain_mults_per_s": round(max(3, nsets) * B / (ms_p / 1000.0), 1),
                "tensor_over_plain": round((steps * B / ms_t) / (max(3, nsets) * B / ms_p), 3),
                "e2e_pinned": e2e_pinned, "e2e_pageable": e2e_pageable,
                "pcie_floor_ms": round(floor_ms, 4), "pcie_gbs": {k: round(v, 2) for k, v in bw.items()},
                "chunk_schedule_pinned": pipe, "chunk_schedule_pageable": pipe_pg,
                "forms_agree": bool(np.array_equal(res_t, res_p)),
                "matches_reference": None}  # filled in by the cpu_baseline leg
            del sets, da0, db0, ct
    finally:
        for mt, mp, _, _, _ in engines.values():
            mt.close()
            mp.close()
    torch.cuda.empty_cache()
    return out


def write_point_dir(root, N, W, q, a, b, cases):
    """The harness's point directory (main.cpp): manifest.json, point/q.bin and `cases` copies
    (hard links) of the operand pair in cases/NNNNNN/{a,b}.bin."""
    import numpy as np
    L = (W + 31) // 32
    os.makedirs(os.path.join(root, "point"))
    np.frombuffer(int(q).to_bytes(4 * L, "little"), dtype="<u4").tofile(os.path.join(root, "point", "q.bin"))
    first = os.path.join(root, "cases", "000000")
    os.makedirs(first)
    np.ascontiguousarray(a, dtype="<u4").tofile(os.path.join(first, "a.bin"))
    np.ascontiguousarray(b, dtype="<u4").tofile(os.path.join(first, "b.bin"))
    for s in range(1, cases):
        d = os.path.join(root, "cases", "%06d" % s)
        os.makedirs(d)
        for f in ("a.bin", "b.bin"):
            os.link(os.path.join(first, f), os.path.join(d, f))
    with open(os.path.join(root, "manifest.json"), "w") as f:
        json.dump({"point": {"N": N, "W": W, "L": L}, "N": N, "W": W, "L": L, "cases": cases}, f)


def run_point_dir(exe, root, N, L, want, timeout=900):
    """Runs a harness binary on a point directory; per-case fherma_run seconds and whether every
    c.bin equals `want`."""
    import numpy as np
    t0 = time.perf_counter()
    r = subprocess.run([exe, root], capture_output=True, text=True, timeout=timeout)
    wall = time.perf_counter() - t0
    if r.returncode != 0:
        return {"error": "exit %d: %s" % (r.returncode, r.stderr[-300:])}
    res = json.load(open(os.path.join(root, "out", "results.json")))
    secs = [c["seconds"] for c in res["cases"] if c["status"] == "ok"]
    same = len(secs) == len(res["cases"]) and all(
        np.array_equal(np.fromfile(os.path.join(root, "out", "%06d" % c["i"], "c.bin"), dtype="<u4").reshape(N, L), want)
        for c in res["cases"])
    ms = sorted(1000.0 * s for s in secs)
    return {"value": round(len(secs) / sum(secs), 2) if secs else None, "unit": "mults/s",
            "p50_ms": round(ms[len(ms) // 2], 4) if ms else None, "p99_ms": round(pct(ms, 0.99), 4) if ms else None,
            "init_s": round(res["init_s"], 3), "cases": len(res["cases"]), "matches_device_path": bool(same),
            "process_wall_s": round(wall, 1)}


def run_reference_gpu(N, W, q, a, b, want, cases):
    """The reference's own GPU build (baseline/_ref/solution_gpu: its solve.cu and harness
    main.cpp, unmodified, nvcc for sm_100a) on a point directory of `cases` copies of (a, b),
    and this library's point-directory runner on the same directory: fherma_run per call, both
    from pageable std::vectors as the harness passes them."""
    out = {"point": {"N": N, "W": W}, "cases": cases,
           "host_buffers": "pageable std::vector from the harness (main.cpp:183)"}
    if not os.path.exists(REF_GPU):
        out["unavailable"] = "baseline/_ref/solution_gpu not built (make -C oracle with the reference tree present)"
        return out
    L = (W + 31) // 32
    tmp = tempfile.mkdtemp(prefix="polymult_refgpu_")
    try:
        for name, exe in (("reference", REF_GPU), ("ours_runner", RUNNER)):
            root = os.path.join(tmp, name)
            write_point_dir(root, N, W, q, a, b, cases)
            out[name] = run_point_dir(exe, root, N, L, want)
            shutil.rmtree(root, ignore_errors=True)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    out["reference"]["build"] = "solve.cu + main.cpp unmodified, nvcc -O3 -gencode arch=compute_100a,code=sm_100a"
    try:
        out["speedup_p50"] = round(out["reference"]["p50_ms"] / out["ours_runner"]["p50_ms"], 3)
    except (KeyError, TypeError, ZeroDivisionError):
        pass
    return out


BATCH_NS = (4096, 8192, 16384, 32768, 65536)
BATCH_WS = (256, 868, 1747, 3000)


def batched_workload(count=256, seed=4):
    """The uneven batch: `count` multiplications, N and W drawn from a seed; grouped into
    classes of one point each.  Returns [(N, W, count)], sorted by (N, W)."""
    import random
    rng = random.Random(seed)
    draws = [(rng.choice(BATCH_NS), rng.choice(BATCH_WS)) for _ in range(count)]
    cls = {}
    for nw in draws:
        cls[nw] = cls.get(nw, 0) + 1
    return [(N, W, c) for (N, W), c in sorted(cls.items())]


def run_batched(torch, args, local):
    """256 uneven multiplications: one CUDA-graph launch per step (autotuned split and GEMM
    form per class) vs the same multiplications as sequential single calls of the plain form."""
    import numpy as np
    import polymult
    import workload
    classes = batched_workload(args.batch_count)
    stream = torch.cuda.current_stream()
    ks = []
    for i, (N, W, c) in enumerate(classes):
        q = workload.spec_prime(N, W)
        L = (W + 31) // 32
        ops = workload.uniform_operands(N, W, q, 2 * c, seed=9000 + i)
        da = torch.from_numpy(np.ascontiguousarray(ops[:c]).view(np.int32)).cuda()
        db = torch.from_numpy(np.ascontiguousarray(ops[c:]).view(np.int32)).cuda()
        ks.append({"N": N, "W": W, "L": L, "q": q, "count": c, "a": da, "b": db, "c": torch.zeros_like(da)})
    total = sum(k["count"] for k in ks)
    spec = [(k["N"], k["W"], workload.limbs(k["q"], k["L"]), k["count"], k["a"].data_ptr(), k["b"].data_ptr(),
             k["c"].data_ptr()) for k in ks]

    def time_batch(b, steps, warm):
        for _ in range(warm):
            b.run(stream.cuda_stream)
        b.sync()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            b.run(stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize()
        b.sync()
        return e0.elapsed_time(e1) / steps

    out = {"workload": "%d multiplications, N from %s, W from %s (seeded), %d classes, operands in HBM"
                       % (total, list(BATCH_NS), list(BATCH_WS), len(ks)), "classes": len(ks)}
    tune_cache = os.environ.get("POLYMULT_TUNE_CACHE")
    with polymult.Batch(spec, tune=True, device=local) as b:
        ms = time_batch(b, args.batch_steps, 3)
        inf = b.info()
        chosen = [b.class_info(i) for i in range(len(ks))]
    with polymult.Batch(spec, tune=False, device=local) as b:
        ms_default = time_batch(b, args.batch_steps, 3)
    # the same multiplications as sequential single calls of the plain form
    mults = []
    for k in ks:
        m = polymult.Multiplier(k["N"], k["W"], workload.limbs(k["q"], k["L"]), gemm="plain", device=local)
        mults.append(m)
    cw = [k["N"] * k["L"] for k in ks]

    def seq_once():
        for k, m, w in zip(ks, mults, cw):
            for i in range(k["count"]):
                m.multiply_device(k["a"].data_ptr() + 4 * w * i, k["b"].data_ptr() + 4 * w * i,
                                  k["c"].data_ptr() + 4 * w * i, 1, stream.cuda_stream)
    seq_once()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    seq_once()
    e1.record(stream)
    torch.cuda.synchronize()
    ms_seq = e0.elapsed_time(e1)
    for m in mults:
        m.sync()
    # spot check: batch outputs (last written by the sequential plain calls) equal the graph's
    ref = [k["c"].clone() for k in ks]
    with polymult.Batch(spec, tune=True, device=local) as b:
        b.run(stream.cuda_stream)
        b.sync()
    same = all(bool(torch.equal(k["c"], r)) for k, r in zip(ks, ref))
    for m in mults:
        m.close()
    forms = {}
    for c in chosen:
        forms[c["gemm"]] = forms.get(c["gemm"], 0) + 1
    out.update({"value": round(total / (ms / 1000.0), 2), "unit": "mults/s", "ms_per_batch": round(ms, 4),
                "untuned_value": round(total / (ms_default / 1000.0), 2),
                "sequential_plain_value": round(total / (ms_seq / 1000.0), 2),
                "speedup_vs_sequential_plain": round(ms_seq / ms, 3),
                "graph_nodes": inf["graph_nodes"], "kernel_launches": inf["kernel_launches"],
                "streams": inf["streams"], "scratch_gb": round(inf["scratch_bytes"] / 1e9, 3),
                "gemm_forms_chosen": forms, "splits_chosen": sorted({(c["w1"], c["w2"]) for c in chosen}),
                "variants_chosen": {"col_tma": sum(1 for c in chosen if c.get("col_tma")),
                                    "crt_a_in_tmem": sum(1 for c in chosen if c.get("crt_tm")),
                                    "launch_groups": sorted({int(c.get("launch_groups", 1)) for c in chosen})},
                "class_ms": [[k["N"], k["W"], k["count"], c["gemm"], round(c["tuned_ms"], 3)]
                             for k, c in zip(ks, chosen)],
                "matches_sequential_plain": same, "tune_cache": tune_cache or "default"})
    return out


def run_serving(torch, args, local):
    """Poisson request streams at N=65536 W=1747, each request multiplying a fresh operand by one
    of 8 operands resident in NTT form, continuous batching under a 150 GB HBM budget, swept over
    offered rates; beside it the unbatched tensor-core path (one request per batch, one stream) at
    a rate it sustains.  Every served result is checked: the server digests each request's
    output on the device, against the digest of the same product from the single-call path."""
    import numpy as np
    import polymult
    import workload
    N, W = N_RANK, W_RANK
    L = (W + 31) // 32
    q = workload.spec_prime(N, W)
    qv = workload.limbs(q, L)
    res = workload.uniform_operands(N, W, q, 8, seed=77)
    pool = args.serve_pool
    ops = workload.uniform_operands(N, W, q, pool, seed=78)
    rates = [float(x) for x in args.serve_rates.split(",") if x]
    # expected digests of every (operand, resident) pair from the single-call device path
    stream = torch.cuda.current_stream().cuda_stream
    expect = np.zeros((pool, 8), dtype=np.uint64)
    with polymult.Multiplier(N, W, qv, gemm="tensor", device=local) as m:
        da = torch.from_numpy(np.ascontiguousarray(ops).view(np.int32)).cuda()
        dc = torch.zeros_like(da)
        for k in range(8):
            db = torch.from_numpy(np.ascontiguousarray(np.broadcast_to(res[k], ops.shape)).view(np.int32)).cuda()
            m.multiply_device(da.data_ptr(), db.data_ptr(), dc.data_ptr(), pool, stream)
            m.sync()
            expect[:, k] = polymult.digest_device(dc.data_ptr(), N * L, pool)
            del db
        del da, dc
    torch.cuda.empty_cache()
    # the PCIe ceiling of the request stream: 14.4 MB in and 14.4 MB out per request
    bw = pcie_bandwidth(torch, N * L * 4, N * L * 4)
    ceiling = 1.0 / (N * L * 4 / (bw["h2d"] * 1e9))
    out = {"workload": "Poisson arrivals (seeded), N=%d W=%d, 8 resident operands in NTT form, request operands "
                       "from a pool of %d pinned buffers, a ring of 128 pinned result buffers" % (N, W, pool),
           "hbm_budget_gb": 150, "unit": "requests/s",
           "pcie_ceiling_req_per_s": round(ceiling, 1), "pcie_gbs": {k: round(v, 2) for k, v in bw.items()}}

    def leg(rate, n_req, max_batch, streams, gemm, seed):
        rng = np.random.default_rng(seed)
        t = np.cumsum(rng.exponential(1.0 / rate, size=n_req))
        t -= t[0]
        sel = rng.integers(0, 8, size=n_req).astype(np.uint32)
        src = rng.integers(0, pool, size=n_req)
        with polymult.Server(N, W, qv, res, hbm_budget=150 * 10**9, max_batch=max_batch, streams=streams, gemm=gemm,
                             device=local) as srv:
            a = srv.pinned(pool)
            a[:] = ops
            c = srv.pinned(128)
            lat, st, dig = srv.run(t, sel, [a[i] for i in src], [c[i % 128] for i in range(n_req)], digests=True)
        lat_ms = np.sort(lat) * 1000.0
        checked = int(np.sum(dig == expect[src, sel]))
        return {"offered_rate": rate, "requests": n_req, "throughput": round(n_req / st["seconds"], 2),
                "p50_ms": round(float(np.percentile(lat_ms, 50)), 3), "p99_ms": round(float(np.percentile(lat_ms, 99)), 3),
                "mean_ms": round(float(lat_ms.mean()), 3), "batches": st["batches"],
                "mean_batch": round(st["mean_batch"], 2), "peak_inflight": st["peak_inflight"],
                "max_inflight_by_budget": st["max_inflight"], "results_checked": n_req,
                "results_match_single_path": checked == n_req, "mismatches": n_req - checked}

    sweep = [leg(r, args.serve_requests, args.serve_batch, args.serve_streams, "auto", 79 + i)
             for i, r in enumerate(rates)]
    single = leg(args.serve_single_rate, max(500, args.serve_requests // 4), 1, 1, "tensor", 99)
    out.update({"sweep": sweep, "unbatched_tensor": single,
                "all_results_match": all(s["results_match_single_path"] for s in sweep + [single])})
    return out


def run_ours(args):
    import numpy as np
    import torch
    import polymult
    import workload
    world, rank, local = dist_init()
    torch.cuda.set_device(local)
    # torch's CPU thread pool stays at one thread: the host pipeline's staging threads need the
    # cores (the bench does no CPU tensor work)
    torch.set_num_threads(1)
    N, W = N_RANK, W_RANK
    L = (W + 31) // 32
    q = workload.spec_prime(N, W)
    qv = workload.limbs(q, L)
    B = args.batch
    host_a = workload.uniform_operands(N, W, q, B, seed=1000 + rank)
    host_b = workload.uniform_operands(N, W, q, B, seed=2000 + rank)
    da = torch.from_numpy(host_a.view(np.int32)).cuda()
    db = torch.from_numpy(host_b.view(np.int32)).cuda()
    dc = torch.zeros_like(da)
    sets = [(da, db, dc)]

    m = polymult.Multiplier(N, W, qv, gemm=args.gemm, device=local)
    info = m.info()
    # cross-check against the other form on one multiply before timing (outside the timed region)
    other = "plain" if info["gemm"] == "tensor" else "tensor"
    mp = polymult.Multiplier(N, W, qv, gemm=other, device=local)
    dc2 = torch.zeros_like(dc)
    stream = torch.cuda.current_stream().cuda_stream
    m.multiply_device(da.data_ptr(), db.data_ptr(), dc.data_ptr(), 1, stream)
    mp.multiply_device(da.data_ptr(), db.data_ptr(), dc2.data_ptr(), 1, stream)
    m.sync()
    mp.sync()
    forms_agree = bool(torch.equal(dc[0], dc2[0]))

    barrier(world)
    with ClockSampler(local) as clk:
        ms = time_device(torch, m, sets, B, args.steps, args.warmup)
    ms = max_over_ranks(ms, world)
    value = world * args.steps * B / (ms / 1000.0)
    groups_per_step = -(-B // max(1, info["group"]))
    launches = args.steps * groups_per_step * info["launches_per_multiply"]

    plain_steps = max(3, args.steps // 4)
    ms_plain = time_device(torch, mp, [(da, db, dc2)], B, plain_steps, 2)
    ms_plain = max_over_ranks(ms_plain, world)
    plain_value = world * plain_steps * B / (ms_plain / 1000.0)

    # per-kernel times for the roofline, CUDA events on the launching stream: launches of B
    # multiplies each, as in the timed region (and of one multiply, for reference)
    stages = m.time_stages(da.data_ptr(), db.data_ptr(), dc.data_ptr(), B, 5, stream)
    stages1 = m.time_stages(da.data_ptr(), db.data_ptr(), dc.data_ptr(), 1, 5, stream)
    stages_plain = mp.time_stages(da.data_ptr(), db.data_ptr(), dc2.data_ptr(), B, 3, stream)
    dom = max(stages, key=stages.get)
    K = info["K"]
    alg = stage_bytes(dom, N, L, K) * B
    peak, peak_kind = measured_peaks()
    achieved = alg / (stages[dom] / 1000.0) / 1e9
    traffic = None
    pipes = None
    tfile = os.path.join(REPO, "profiles", "traffic_bytes.json")
    if os.path.exists(tfile):
        try:
            tj = json.load(open(tfile))
            tt = tj.get(info["gemm"], {})
            t1 = tt.get(dom)
            # captured on launches of a stated number of multiplies; scaled to B
            if isinstance(t1, dict):
                traffic = int(t1["bytes"] * B / t1.get("multiplies_per_launch", 1))
            elif t1 is not None:
                traffic = int(t1 * B / tt.get("multiplies_per_launch", 1))
            pipes = tj.get("pipes", {}).get(info["gemm"], {}).get(dom)
        except Exception:
            traffic = None
    roofline = {"kernel": dom, "bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "traffic": traffic, "peak_source": peak_kind,
                "algorithmic_bytes": alg, "kernel_ms": round(stages[dom], 4), "multiplies_per_launch": B}
    if pipes:
        # the unit that binds the kernel, from the committed ncu capture (HBM is not it here)
        roofline["binding_pipe"] = pipes
    if dom == "rows_fused":
        # the row pass against the measured rate of its butterfly alone (pm_butterfly_peak): the
        # NTT's own ceiling on this GPU, operands in registers, no memory traffic
        try:
            bp = polymult.butterfly_peak(local)
            w2 = int(info["w2"])
            bf = 3 * K * (N // 2) * w2 * B  # forward rows of a and b, inverse rows of c
            got = bf / (stages[dom] / 1000.0)
            roofline["butterfly"] = {"butterflies_per_launch": bf, "achieved_per_s": round(got, 0),
                                     "peak_per_s": round(bp["bfly_per_s"], 0),
                                     "peak_per_clk_sm": round(bp["bfly_per_clk_sm"], 2),
                                     "frac": round(got / bp["bfly_per_s"], 4)}
        except Exception as e:  # the peak kernel is a measurement aid, not the multiply
            roofline["butterfly"] = {"unavailable": str(e)[:120]}
    whole = {"algorithmic_bytes_per_multiply": (12 * N * L + 24 * K * N), "ms_per_multiply": round(ms / args.steps / B, 5)}
    whole["achieved_gbs"] = round(whole["algorithmic_bytes_per_multiply"] / (whole["ms_per_multiply"] / 1000.0) / 1e9, 1)
    whole["frac_of_hbm"] = round(whole["achieved_gbs"] / peak, 4)

    # end to end through the reference-facing call; the pipeline's chunk schedule chosen by its
    # autotuner first (outside the timed region).  Headline: operands and result in pinned host
    # memory (each column chunk moves by one strided DMA copy, no host staging); beside it the
    # reference harness's case, pageable buffers staged through the host pool.
    # 9 repetitions per candidate: close schedules differ by 1-2%, within the noise of 5
    pipe = m.tune_pipeline(9, pinned=True) if not args.no_tune_pipeline else m.pipeline(pinned=True)
    pipe_pageable = m.tune_pipeline(9) if not args.no_tune_pipeline else m.pipeline()
    bw = pcie_bandwidth(torch, 2 * N * L * 4, N * L * 4)
    floor_ms = pcie_floor_ms(bw, N, L)
    want = dc[0].cpu().numpy().view(np.uint32)
    pa, pb, pc = pinned_words(torch, (N, L)), pinned_words(torch, (N, L)), pinned_words(torch, (N, L))
    pa[:] = host_a[0]
    pb[:] = host_b[0]
    e2e = e2e_leg(m, pa, pb, pc, args.e2e_steps, world, floor_ms, want)
    e2e.update({"host_memory": "pinned", "pcie_gbs": {k: round(v, 2) for k, v in bw.items()},
                "pcie_floor_ms": round(floor_ms, 4), "chunk_schedule": pipe})
    e2e["pageable"] = e2e_leg(m, np.ascontiguousarray(host_a[0]), np.ascontiguousarray(host_b[0]),
                              np.empty((N, L), dtype=np.uint32), args.e2e_steps, world, floor_ms, want)
    e2e["pageable"]["chunk_schedule"] = pipe_pageable
    # beside it, the reference's own schedule (solve.cu:1403-1405: eighths in with narrow heads,
    # sixteenths out with narrow heads and tails: 10 + 10 input and 20 output chunks)
    if not args.no_tune_pipeline:
        m.set_pipeline(8, 16)
        ref_sched = e2e_leg(m, np.ascontiguousarray(host_a[0]), np.ascontiguousarray(host_b[0]),
                            np.empty((N, L), dtype=np.uint32), args.e2e_steps, world, floor_ms, want)
        ref_sched["chunk_schedule"] = m.pipeline()
        e2e["pageable"]["reference_schedule"] = {k: ref_sched[k] for k in ("p50_ms", "p99_ms", "p50_over_floor",
                                                                          "matches_device_path", "chunk_schedule")}
        m.set_pipeline(pipe_pageable["in_body"], pipe_pageable["out_body"])
    # the pageable call's second floor: its host copies (a and b gathered into page-locked
    # staging, c scattered out of it) at the host's measured copy rate with the pool's 8 threads
    hbw = host_copy_gbs(torch, 2 * N * L * 4)
    host_floor = 3 * N * L * 4 / (hbw * 1e9) * 1000
    e2e["pageable"].update({"host_copy_gbs": round(hbw, 1), "host_staging_floor_ms": round(host_floor, 4),
                            "p50_over_host_floor": round(e2e["pageable"]["p50_ms"] / host_floor, 3)})
    m.close()
    mp.close()
    del sets, da, db, dc, dc2
    torch.cuda.synchronize()
    torch.cuda.empty_cache()

    # the legs below describe one GPU: they run in the one-GPU run only (with N > 1 the line
    # carries the replicas' throughput, and the N = 1 line these legs).  The latency-measuring
    # serving leg goes first, with torch's cached blocks released: after the batch leg (GBs of
    # operands in torch's cache, seconds of full load) its p99 measured about twice as high.
    serving = configs = refgpu = batched = cpu = None
    if rank == 0 and world == 1:
        if not args.no_serving:
            serving = run_serving(torch, args, local)
            torch.cuda.empty_cache()
        pending = {}
        if not args.no_configs:
            configs = run_configs(torch, args, local, pending)
        if not args.no_reference_gpu:
            refgpu = run_reference_gpu(N, W, q, host_a[0], host_b[0], want, args.ref_gpu_cases)
        if not args.no_batched:
            batched = run_batched(torch, args, local)
        if world == 1 and not args.no_cpu:
            # cpu_baseline leg: the reference's CPU path timed at the ranked point, and run on the
            # first timed multiply of every configuration as its checker
            cpu, cref = reference_cpu(N, W, q, np.ascontiguousarray(host_a[0]), np.ascontiguousarray(host_b[0]),
                                      calls=2, warm=1)
            cpu["matches_gpu"] = bool(np.array_equal(cref, want))
            for name, (cN, cW, cq, ca, cb, ct, cp) in pending.items():
                ref = ReferenceCPU(cN, cW, cq)
                try:
                    r = ref.multiply(ca, cb)
                finally:
                    ref.close()
                configs[name]["matches_reference"] = bool(np.array_equal(ct, r) and np.array_equal(cp, r))
                configs[name]["reference_kind"] = ref.kind

    if rank == 0:
        line = {"metric": METRIC, "value": round(value, 2), "unit": "mults/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 4),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
                "data": "synthetic (uniform in [0,q), seeded PCG64)", "config": headline_config(),
                "arm": {"K": K, "batch_per_gpu": B, "gemm": info["gemm"], "replicas": world},
                "plain_value": round(plain_value, 2), "tensor_over_plain": round(value / plain_value, 3),
                "forms_agree": forms_agree,
                "stages_ms": {k: round(v, 4) for k, v in stages.items()},
                "stages_ms_one_multiply": {k: round(v, 4) for k, v in stages1.items()},
                "stages_ms_plain": {k: round(v, 4) for k, v in stages_plain.items()},
                "roofline": roofline, "whole_multiply_hbm": whole, "e2e": e2e, "configs": configs,
                "reference_gpu": refgpu, "batched": batched, "serving": serving, "cpu_baseline": cpu,
                "clocks": clk.summary(), "gpu_launches": launches}
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


# ------------------------------------------------------------------------------------------
# measurement modes
# ------------------------------------------------------------------------------------------
def run_profile_case(a):
    """One device-resident group of `count` multiplies at (N, W) through pm_run_device, after
    pm_init's warm-up multiply through the host pipeline; --host H then runs H multiplies through
    pm_run (--pinned: page-locked buffers; --tune: tune that kind of call's schedule first).
    Select the device-resident launch of a kernel with ncu's -k / -s (skip the warm-up's)."""
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
        m.multiply_device(da.data_ptr(), db.data_ptr(), dc.data_ptr(), a.count, torch.cuda.current_stream().cuda_stream)
        m.sync()
        if a.host and a.tune:
            print("schedule", m.tune_pipeline(3, pinned=a.pinned))
        if a.host:
            if a.pinned:
                a0, b0, out = (pinned_words(torch, (a.N, L)) for _ in range(3))
                a0[:] = ops[0]
                b0[:] = ops[a.count]
            else:
                a0, b0 = np.ascontiguousarray(ops[0]), np.ascontiguousarray(ops[a.count])
                out = np.empty((a.N, L), dtype=np.uint32)
            for _ in range(a.host):
                m.multiply(a0, b0, out)
            if not np.array_equal(out, dc[0].cpu().numpy().view(np.uint32)):
                raise SystemExit("host and device paths differ")
    print("ok N=%d W=%d K=%d gemm=%s count=%d" % (a.N, a.W, info["K"], info["gemm"], a.count))


def run_peak_int8(a):
    """cuBLAS's int8 GEMM (torch._int_mm: int8 x int8 -> int32) on square size^3 operands, CUDA
    events: burst = best of 10 single GEMMs, sustained = a loop of about `seconds` (the power cap
    settles there).  One JSON line in TOPS (2 x multiply-adds per second / 10^12)."""
    import torch
    n = a.size
    g = torch.Generator(device="cuda").manual_seed(7)
    x = torch.randint(-128, 128, (n, n), dtype=torch.int8, device="cuda", generator=g)
    y = torch.randint(-128, 128, (n, n), dtype=torch.int8, device="cuda", generator=g).t()  # column-major
    ops = 2.0 * n * n * n
    for _ in range(5):
        torch._int_mm(x, y)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    best = float("inf")
    for _ in range(10):
        e0.record()
        torch._int_mm(x, y)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1000.0)
    reps = max(1, int(a.seconds / best))
    e0.record()
    for _ in range(reps):
        torch._int_mm(x, y)
    e1.record()
    e1.synchronize()
    sustained = e0.elapsed_time(e1) / 1000.0 / reps
    k = 64
    ref = (x[:k].to(torch.int32).cpu() @ y[:, :k].to(torch.int32).cpu())
    ok = bool(torch.equal(torch._int_mm(x, y)[:k, :k].cpu(), ref))
    print(json.dumps({"int8_tops_burst": round(ops / best / 1e12, 1), "int8_tops_sustained": round(ops / sustained / 1e12, 1),
                      "size": n, "sustained_reps": reps, "method": "torch._int_mm (cuBLAS int8 GEMM), CUDA events",
                      "device": torch.cuda.get_device_name(0), "corner_block_exact": ok}))


def run_peak_butterfly(a):
    """The NTT butterfly's rate with operands in registers over every SM (pm_butterfly_peak):
    the ceiling of the NTT kernels, which the integer multiply-add pipe binds.  One JSON line."""
    import torch
    import polymult
    r = polymult.butterfly_peak(0)
    print(json.dumps({"butterflies_per_s": round(r["bfly_per_s"], 0), "butterflies_per_clk_sm": round(r["bfly_per_clk_sm"], 2),
                      "method": "k_bfly_peak: bfly_ct_sh on 16 register values per thread, 2 x 512 threads per SM, "
                                "CUDA events over 5 launches, checksum checked against the host",
                      "device": torch.cuda.get_device_name(0)}))


def main():
    args = parse()
    if args.profile_case:
        run_profile_case(args)
    elif args.peak_butterfly:
        run_peak_butterfly(args)
    elif args.peak_int8:
        run_peak_int8(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
