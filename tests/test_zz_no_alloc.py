"""GPU: pm_run_device_static, the entry point that allocates nothing.

Some callers cannot call cudaMalloc while they compute (a framework whose caching allocator
owns the device memory, a latency-critical path that cannot take cudaMalloc's implicit
synchronisation).  pm_run_device_static serves them with a fixed device array inside the
library as residue scratch.  This test calls it through the C ABI twice in a row, on
different operands, and checks each result bit-exactly (the tolerance of every parity test
here: integer results must be identical) against the existing entry point pm_run_device on
the same operands; that the second call takes no device memory (the free memory the driver
reports does not drop across it); that it leaves the caller's current device as it was; and
that a point whose residues exceed the static scratch is rejected.

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
        # every buffer before the calls, so that only the library could take memory in between
        a = [torch.from_numpy(np.ascontiguousarray(ops[2 * k]).view(np.int32)).cuda() for k in range(2)]
        b = [torch.from_numpy(np.ascontiguousarray(ops[2 * k + 1]).view(np.int32)).cuda() for k in range(2)]
        c_static = [torch.full_like(a[0], -1) for _ in range(2)]
        c_ref = [torch.zeros_like(a[0]) for _ in range(2)]
        torch.cuda.synchronize()
        free_before = None
        for call in range(2):
            if call == 1:
                free_before = torch.cuda.mem_get_info()[0]
            dev_before = torch.cuda.current_device()
            rc = lib.pm_run_device_static(m._h, ctypes.c_void_p(a[call].data_ptr()),
                                          ctypes.c_void_p(b[call].data_ptr()),
                                          ctypes.c_void_p(c_static[call].data_ptr()),
                                          ctypes.c_void_p(stream.cuda_stream))
            assert rc == polymult.PM_OK, lib.pm_last_error()
            assert torch.cuda.current_device() == dev_before
            torch.cuda.synchronize()
            if call == 1:
                assert torch.cuda.mem_get_info()[0] >= free_before, "the second call took device memory"
        assert lib.pm_sync(m._h) == polymult.PM_OK, lib.pm_last_error()
        # the existing entry point on the same operands (it may allocate: after the measurement)
        for call in range(2):
            m.multiply_device(a[call].data_ptr(), b[call].data_ptr(), c_ref[call].data_ptr(), 1, stream.cuda_stream)
        m.sync()
        for call in range(2):
            assert torch.equal(c_static[call], c_ref[call]), "call %d differs from pm_run_device" % call


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
