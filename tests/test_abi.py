"""CPU: the C-ABI library loads, exports every symbol include/polymult_b200.h declares, and its
host-only logic (point validation, prime selection, CRT tables) is right.  No GPU calls."""
import ctypes
import subprocess

import pytest

from conftest import ensure_library, orc


def test_library_exports_every_declared_symbol():
    import polymult
    lib = ensure_library()
    names = polymult.declared_symbols()
    assert {"pm_init", "pm_run", "pm_run_device", "pm_sync", "pm_free", "pm_get_info",
            "pm_last_error", "pm_plan_selfcheck"} <= set(names)
    for n in names:
        assert hasattr(lib, n), n
    out = subprocess.run(["nm", "-D", "--defined-only", polymult.LIB_PATH], capture_output=True, text=True).stdout
    for n in names:
        assert (" T " + n) in out, n


def test_fherma_cxx_symbols_exported():
    """The reference harness binds fherma_init / fherma_run / fherma_free (fherma.toml:7-10)."""
    import polymult
    out = subprocess.run(["nm", "-DC", "--defined-only", polymult.LIB_PATH], capture_output=True, text=True).stdout
    assert "fherma_init(fherma::Point const&)" in out
    assert "fherma_run(void*, fherma::Inputs const&)" in out
    assert "fherma_free(void*)" in out


@pytest.mark.parametrize("N,W", [(1, 64), (2, 40), (16, 33), (64, 32), (256, 1747), (1024, 512), (4096, 256),
                                 (2048, 868), (512, 4000), (32768, 868), (65536, 1747)])
def test_plan_selfcheck_golden_points(golden, N, W):
    import polymult
    pt = next(p for p in golden["points"] if p["N"] == N and p["W"] == W)
    q = orc.limbs_of(int(pt["q_hex"], 16), pt["L"])
    K = polymult.plan_selfcheck(N, W, q)
    # M = prod p > 2^(2W + logN + 3) with p < 2^30
    assert K * 30 >= 2 * W + N.bit_length() - 1 + 3


def test_plan_selfcheck_batched_grid(golden):
    import polymult
    for g in golden["grid_primes"]:
        L = (g["W"] + 31) // 32
        K = polymult.plan_selfcheck(g["N"], g["W"], orc.limbs_of(int(g["q_hex"], 16), L))
        assert K > 0


def _init_error(N, W, L, q_limbs):
    import polymult
    lib = ensure_library()
    q = (ctypes.c_uint32 * max(1, len(q_limbs)))(*q_limbs)
    k = ctypes.c_int32(0)
    rc = lib.pm_plan_selfcheck(N, W, L, ctypes.cast(q, ctypes.c_void_p), ctypes.byref(k))
    return rc, lib.pm_last_error().decode()


def test_invalid_points_rejected():
    import polymult
    q256 = [int(x) for x in orc.limbs_of(orc.spec_prime(64, 256), 8)]
    rc, msg = _init_error(63, 256, 8, q256)
    assert rc == polymult.PM_ERR_INVALID and "power of two" in msg
    rc, msg = _init_error(64, 256, 7, q256[:7])
    assert rc == polymult.PM_ERR_INVALID and "ceil(W / 32)" in msg
    even = list(q256)
    even[0] &= ~1
    rc, msg = _init_error(64, 256, 8, even)
    assert rc == polymult.PM_ERR_INVALID and "q is even" in msg
    small = [12345, 0, 0, 0, 0, 0, 0, 0]   # delta = 2^256 - q far above 2^63
    rc, msg = _init_error(64, 256, 8, small)
    assert rc == polymult.PM_ERR_INVALID and "too far below 2^W" in msg
    big = [0xFFFFFFFF] * 8                 # 2^256 - 1 is not below 2^W... for W = 255
    rc, msg = _init_error(64, 255, 8, big)
    assert rc == polymult.PM_ERR_INVALID and "not below 2^W" in msg
    rc, msg = _init_error(1 << 21, 256, 8, q256)
    assert rc == polymult.PM_ERR_INVALID


def test_python_api_rejects_wrong_sizes():
    import polymult
    with pytest.raises(RuntimeError):
        polymult.fherma_init(64, 256, 7, [1] * 7)


def test_null_arguments():
    import polymult
    lib = ensure_library()
    assert lib.pm_init(64, 256, 8, None, 0, 0, None) == polymult.PM_ERR_INVALID
    assert lib.pm_run(None, None, None, None) == polymult.PM_ERR_INVALID
    assert lib.pm_sync(None) == polymult.PM_ERR_INVALID
    lib.pm_free(None)


def test_batch_server_pipeline_argument_checks():
    """Argument checks of the batch, server and pipeline-tuning entry points, which fail before
    any CUDA call (so they hold on a machine without a GPU)."""
    import polymult
    lib = ensure_library()
    out = ctypes.c_void_p()
    assert lib.pm_batch_init(None, 0, 0, 0, 0, ctypes.byref(out)) == polymult.PM_ERR_INVALID
    one = (polymult.PmBatchClass * 1)()
    assert lib.pm_batch_init(one, 1, 0, 0, 0, None) == polymult.PM_ERR_INVALID
    assert lib.pm_batch_init(one, 1, 7, 0, 0, ctypes.byref(out)) == polymult.PM_ERR_INVALID
    assert lib.pm_batch_init(one, 1, 0, 64, 0, ctypes.byref(out)) == polymult.PM_ERR_INVALID
    assert "unknown flags" in lib.pm_last_error().decode()
    assert lib.pm_batch_run(None, None) == polymult.PM_ERR_INVALID
    assert lib.pm_batch_sync(None) == polymult.PM_ERR_INVALID
    lib.pm_batch_free(None)
    assert lib.pm_server_init(64, 256, 8, None, None, 0, 1 << 30, 4, 2, 0, 0, ctypes.byref(out)) == \
        polymult.PM_ERR_INVALID
    assert "resident" in lib.pm_last_error().decode()
    assert lib.pm_server_run(None, 0, None, None, None, None, None, None, None) == polymult.PM_ERR_INVALID
    lib.pm_server_free(None)
    assert lib.pm_tune_pipeline(None, 3, 0, None) == polymult.PM_ERR_INVALID
    assert lib.pm_tune_pipeline(None, 3, polymult.PIPELINE_PINNED, None) == polymult.PM_ERR_INVALID
    assert lib.pm_get_pipeline(None, 0, None) == polymult.PM_ERR_INVALID
    assert lib.pm_set_pipeline(None, 0, 8, 8) == polymult.PM_ERR_INVALID

