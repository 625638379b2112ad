"""GPU: failure reporting, driven without a GPU fault.

Every failure here is made on the host, by operands outside the range the kernels' own check
guards, or by a wait that nothing satisfies; none faults, traps or hangs the device, and each
test ends with a normal multiply that must be bit-exact (the context stays usable).
  * the device status word: bits written into it, as a failed device-side check would, make
    pm_sync / pm_run return PM_ERR_DEVICE with the check's message and clear the word;
  * a real device-side check: operands with every limb bit set (beyond q, so the exact product
    leaves the |x| < M/8 window the RNS primes are chosen for) make the CRT's fp32 estimate miss;
    the CRT kernels' own check reports it (the reference has no such check: its CRT would return
    a wrong value silently, solve.cu:440-450);
  * the tensor-core kernels' bounded mbarrier waits, made to run out on a barrier that nothing
    arrives on (pm_selftest_wait);
  * a residue-scratch allocation that fails (host-side injection): PM_ERR_CUDA, then the next
    call allocates again (the engine must not keep claiming the scratch it lost).
"""
import ctypes

import numpy as np
import pytest

from conftest import c_oracle_mul, ensure_library

pytestmark = pytest.mark.gpu


def _torch():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _point(N, W, count, seed):
    import workload
    q = workload.spec_prime(N, W)
    L = (W + 31) // 32
    return q, L, workload.uniform_operands(N, W, q, count, seed=seed)


def _expect(N, W, q, a, b):
    return c_oracle_mul(N, W, q, a, b)


def test_status_word_reports_and_clears():
    _torch()
    import polymult
    import workload
    lib = ensure_library()
    N, W = 4096, 256
    q, L, ops = _point(N, W, 2, seed=31)
    with polymult.Multiplier(N, W, workload.limbs(q, L), gemm="tensor") as m:
        assert lib.pm_test_set_status(m._h, polymult.PM_DEVICE_CRT_BOUND) == polymult.PM_OK
        assert lib.pm_sync(m._h) == polymult.PM_ERR_DEVICE
        assert b"CRT estimate" in lib.pm_last_error()
        assert lib.pm_sync(m._h) == polymult.PM_OK  # cleared by the report
        # pm_run reads the word after its own kernels
        assert lib.pm_test_set_status(m._h, polymult.PM_DEVICE_WAIT | polymult.PM_DEVICE_FOLD) == polymult.PM_OK
        with pytest.raises(polymult.PolymultError) as ei:
            m.multiply(ops[0], ops[1])
        assert ei.value.code == polymult.PM_ERR_DEVICE
        assert "wait timed out" in str(ei.value) and "after folding" in str(ei.value)
        got = m.multiply(ops[0], ops[1])
        assert np.array_equal(got, _expect(N, W, q, ops[0], ops[1]))


@pytest.mark.parametrize("gemm", ["tensor", "plain"])
def test_crt_bound_check_fires_on_operands_beyond_q(gemm):
    _torch()
    import polymult
    import workload
    N, W = 4096, 868  # L = 28: 28 spare bits above W per coefficient
    q, L, ops = _point(N, W, 2, seed=32)
    ones = np.full((N, L), 0xFFFFFFFF, dtype=np.uint32)
    with polymult.Multiplier(N, W, workload.limbs(q, L), gemm=gemm) as m:
        with pytest.raises(polymult.PolymultError) as ei:
            m.multiply(ones, ones)
        assert ei.value.code == polymult.PM_ERR_DEVICE and "CRT estimate" in str(ei.value)
        got = m.multiply(ops[0], ops[1])
        assert np.array_equal(got, _expect(N, W, q, ops[0], ops[1]))


def test_bounded_waits_run_out_and_report():
    _torch()
    import polymult
    import workload
    ensure_library()
    for limit in (1000, 2_000_000):
        st = polymult.wait_selftest(limit)
        assert st & polymult.PM_DEVICE_WAIT, "the wait did not give up (status %#x)" % st
        assert not st & 0x100, "a wait on the completed phase failed (status %#x)" % st
    N, W = 4096, 256
    q, L, ops = _point(N, W, 2, seed=33)
    with polymult.Multiplier(N, W, workload.limbs(q, L), gemm="tensor") as m:
        got = m.multiply(ops[0], ops[1])
        m.sync()
    assert np.array_equal(got, _expect(N, W, q, ops[0], ops[1]))


@pytest.mark.parametrize("skip", [0, 1])
def test_scratch_allocation_failure_then_recovery(skip):
    """skip 0: the first of the two residue arrays fails; skip 1: the second."""
    torch = _torch()
    import polymult
    import workload
    lib = ensure_library()
    N, W, count = 4096, 256, 4
    q, L, ops = _point(N, W, 2 * count, seed=34 + skip)
    a = torch.from_numpy(np.ascontiguousarray(ops[:count]).view(np.int32)).cuda()
    b = torch.from_numpy(np.ascontiguousarray(ops[count:]).view(np.int32)).cuda()
    c = torch.zeros_like(a)
    stream = torch.cuda.current_stream().cuda_stream
    with polymult.Multiplier(N, W, workload.limbs(q, L), gemm="tensor") as m:
        assert m.info()["group"] >= count  # pm_init's warm-up left scratch for one multiply only
        lib.pm_test_fail_scratch_allocs(skip, 1)
        try:
            rc = lib.pm_run_device(m._h, ctypes.c_void_p(a.data_ptr()), ctypes.c_void_p(b.data_ptr()),
                                   ctypes.c_void_p(c.data_ptr()), count, ctypes.c_void_p(stream))
        finally:
            lib.pm_test_fail_scratch_allocs(0, 0)
        assert rc == polymult.PM_ERR_CUDA and b"cudaMalloc residues" in lib.pm_last_error()
        assert m.info()["scratch_bytes"] == 0  # nothing claimed after the failure
        m.multiply_device(a.data_ptr(), b.data_ptr(), c.data_ptr(), count, stream)
        m.sync()
        assert m.info()["scratch_bytes"] > 0
    got = c.cpu().numpy().view(np.uint32)
    for i in range(count):
        assert np.array_equal(got[i], _expect(N, W, q, ops[i], ops[count + i])), "multiply %d" % i
