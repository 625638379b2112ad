"""GPU: pm_run_device_static, the entry point that allocates nothing.

Some callers cannot call cudaMalloc while they compute (a framework whose caching allocator
owns the device memory, a latency-critical path that cannot take cudaMalloc's implicit
synchronisation).  pm_run_device_static serves them with a fixed device array inside the
library as residue scratch.  This test calls it through the C ABI twice in a row, on
different operands, and checks each result bit-exactly (the tolerance of every parity test
here: integer results must be identical) against the existing entry point pm_run_device on
the same operands; and that a point whose residues exceed the static scratch is rejected.

Kept in a file of its own that pytest collects last; it passes alone in a fresh process and
after the other tests.
"""
import ctypes

import numpy as np
import pytest

from conftest import ensure_library

pytestmark = pytest.mark.gpu


def _torch():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def test_static_scratch_entry_matches_device_entry_twice():
    torch = _torch()
    import polymult
    import workload
    lib = ensure_library()
    N, W = 65536, 1747
    L = (W + 31) // 32
    q = workload.spec_prime(N, W)
    ops = workload.uniform_operands(N, W, q, 4, seed=77)
    with polymult.Multiplier(N, W, workload.limbs(q, L), gemm="tensor") as m:
        stream = torch.cuda.current_stream()
        for call in range(2):
            a = torch.from_numpy(np.ascontiguousarray(ops[2 * call]).view(np.int32)).cuda()
            b = torch.from_numpy(np.ascontiguousarray(ops[2 * call + 1]).view(np.int32)).cuda()
            c_static = torch.full_like(a, -1)
            c_ref = torch.zeros_like(a)
            rc = lib.pm_run_device_static(m._h, ctypes.c_void_p(a.data_ptr()), ctypes.c_void_p(b.data_ptr()),
                                          ctypes.c_void_p(c_static.data_ptr()), ctypes.c_void_p(stream.cuda_stream))
            assert rc == polymult.PM_OK, lib.pm_last_error()
            m.multiply_device(a.data_ptr(), b.data_ptr(), c_ref.data_ptr(), 1, stream.cuda_stream)
            m.sync()
            assert torch.equal(c_static, c_ref), "call %d differs from pm_run_device" % call


def test_static_scratch_rejects_oversized_point():
    _torch()
    import polymult
    import workload
    lib = ensure_library()
    N, W = 65536, 3000  # K = 202 primes: 13.2 Mi residue words per operand > 8 Mi
    L = (W + 31) // 32
    q = workload.spec_prime(N, W)
    with polymult.Multiplier(N, W, workload.limbs(q, L), gemm="plain") as m:
        rc = lib.pm_run_device_static(m._h, ctypes.c_void_p(16), ctypes.c_void_p(16), ctypes.c_void_p(16), None)
        assert rc == polymult.PM_ERR_INVALID
        assert b"static scratch" in lib.pm_last_error()
