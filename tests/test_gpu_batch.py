"""GPU parity of the batch path (pm_batch_*): many multiplications of uneven points in one
CUDA-graph launch, with explicit and autotuned 4-step splits and GEMM forms.

Every output is compared bit-for-bit with the single-point device path (pm_run_device, whose
parity against the reference's own outputs is tests/test_gpu_parity.py) and, for the small
classes, with the C oracle.  Also: graph replays rewrite their outputs, every valid split of a
point and every kernel variant and launch-group count the tuner chooses from gives the same
bytes, the tuner's cache is written and read back, and line lengths up to
2^10 (N = 2^18 .. 2^20, the three-phase and two-warp-row NTT forms) against the C oracle."""
import os

import numpy as np
import pytest

from conftest import c_oracle_mul, ensure_library, load_golden, orc

pytestmark = pytest.mark.gpu

GOLDEN = {(p["N"], p["W"]): int(p["q_hex"], 16) for p in load_golden()["points"]}


def _torch():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _q(N, W):
    import workload
    if (N, W) in GOLDEN:
        return GOLDEN[(N, W)]
    return workload.spec_prime(N, W)


def _class(torch, N, W, count, seed):
    import workload
    q = _q(N, W)
    L = (W + 31) // 32
    ops = workload.uniform_operands(N, W, q, 2 * max(count, 1), seed=seed)
    da = torch.from_numpy(np.ascontiguousarray(ops[:count]).view(np.int32)).cuda()
    db = torch.from_numpy(np.ascontiguousarray(ops[count:2 * count]).view(np.int32)).cuda()
    dc = torch.zeros_like(da)
    return {"N": N, "W": W, "L": L, "q": q, "count": count, "a": da, "b": db, "c": dc}


def _single(torch, k, gemm="plain"):
    """Outputs of the single-point device path for class k."""
    import polymult
    out = torch.zeros_like(k["a"])
    with polymult.Multiplier(k["N"], k["W"], orc.limbs_of(k["q"], k["L"]), gemm=gemm) as m:
        if k["count"]:
            m.multiply_device(k["a"].data_ptr(), k["b"].data_ptr(), out.data_ptr(), k["count"],
                              torch.cuda.current_stream().cuda_stream)
        m.sync()
    return out.cpu().numpy().view(np.uint32)


def _spec(k, w1=-1):
    return (k["N"], k["W"], orc.limbs_of(k["q"], k["L"]), k["count"], k["a"].data_ptr(), k["b"].data_ptr(),
            k["c"].data_ptr(), w1)


MIXED = [(64, 100, 3), (1024, 256, 2), (4096, 868, 4), (256, 1747, 1), (4096, 3000, 2), (4096, 256, 0),
         (2048, 868, 5), (16, 33, 2), (8192, 256, 3), (65536, 1747, 1)]


@pytest.mark.parametrize("graph", [True, False])
@pytest.mark.parametrize("gemm", ["auto", "plain"])
def test_mixed_batch_matches_single_point_path(gemm, graph):
    torch = _torch()
    import polymult
    ensure_library()
    ks = [_class(torch, N, W, c, seed=100 + i) for i, (N, W, c) in enumerate(MIXED)]
    want = [_single(torch, k) for k in ks]
    with polymult.Batch([_spec(k) for k in ks], gemm=gemm, graph=graph) as b:
        info = b.info()
        assert info["classes"] == len(ks)
        assert (info["graph_nodes"] > 0) == graph
        for rep in range(2):  # a replay must rewrite every output
            for k in ks:
                k["c"].zero_()
            b.run(torch.cuda.current_stream().cuda_stream)
            b.sync()
            for k, w in zip(ks, want):
                got = k["c"].cpu().numpy().view(np.uint32)
                assert np.array_equal(got, w), (k["N"], k["W"], rep)
            if gemm == "plain":
                assert all(b.class_info(i)["gemm"] == "plain" for i in range(len(ks)))


def test_small_classes_against_c_oracle():
    torch = _torch()
    import polymult
    ensure_library()
    ks = [_class(torch, N, W, c, seed=7 + i) for i, (N, W, c) in enumerate([(64, 100, 2), (512, 256, 1), (16, 33, 3)])]
    with polymult.Batch([_spec(k) for k in ks]) as b:
        b.run(torch.cuda.current_stream().cuda_stream)
        b.sync()
    for k in ks:
        a = k["a"].cpu().numpy().view(np.uint32)
        bb = k["b"].cpu().numpy().view(np.uint32)
        got = k["c"].cpu().numpy().view(np.uint32)
        for i in range(k["count"]):
            assert np.array_equal(got[i], c_oracle_mul(k["N"], k["W"], k["q"], a[i], bb[i])), (k["N"], k["W"], i)


# N=16384 and 32768 at w1 = 8 run the TMA column pass with row pitches 2^6 and 2^7
@pytest.mark.parametrize("N,W", [(65536, 1747), (32768, 100), (16384, 256), (4096, 256), (1024, 868), (32, 64)])
def test_every_split_gives_the_same_bytes(N, W):
    torch = _torch()
    import polymult
    ensure_library()
    logN = N.bit_length() - 1
    splits = [w1 for w1 in range(0, 11) if 1 <= logN - w1 <= 10]
    base = _class(torch, N, W, 2, seed=31)
    want = _single(torch, base, gemm="auto")
    ks = []
    for w1 in splits:
        k = dict(base)
        k["c"] = torch.zeros_like(base["a"])
        ks.append((k, w1))
    with polymult.Batch([_spec(k, w1) for k, w1 in ks]) as b:
        for i, (_, w1) in enumerate(ks):
            assert b.class_info(i)["w1"] == w1
        b.run(torch.cuda.current_stream().cuda_stream)
        b.sync()
    for k, w1 in ks:
        assert np.array_equal(k["c"].cpu().numpy().view(np.uint32), want), (N, W, w1)


def test_autotuner_chooses_and_caches(tmp_path, monkeypatch):
    torch = _torch()
    import polymult
    ensure_library()
    cache = tmp_path / "tune.txt"
    monkeypatch.setenv("POLYMULT_TUNE_CACHE", str(cache))
    ks = [_class(torch, N, W, c, seed=50 + i)
          for i, (N, W, c) in enumerate([(4096, 256, 3), (16384, 868, 2), (65536, 1747, 2)])]
    want = [_single(torch, k) for k in ks]
    with polymult.Batch([_spec(k) for k in ks], tune=True) as b:
        chosen = []
        for i, k in enumerate(ks):
            ci = b.class_info(i)
            logN = k["N"].bit_length() - 1
            assert logN // 2 - 1 <= ci["w1"] <= logN // 2 + 1
            assert ci["tuned_ms"] > 0
            assert ci["launch_groups"] in (1, 2, 4) and ci["launch_groups"] <= k["count"]
            assert ci["col_tma"] in (0, 1) and ci["crt_tm"] in (0, 1)
            chosen.append((ci["w1"], ci["gemm_form"], ci["col_tma"], ci["crt_tm"], ci["launch_groups"]))
        for k in ks:
            k["c"].zero_()
        b.run(torch.cuda.current_stream().cuda_stream)
        b.sync()
        for k, w in zip(ks, want):
            assert np.array_equal(k["c"].cpu().numpy().view(np.uint32), w)
    lines = cache.read_text().strip().splitlines()
    assert len(lines) == 3 and all(len(ln.split()) == 10 for ln in lines)
    with polymult.Batch([_spec(k) for k in ks], tune=True) as b2:  # served from the cache
        for i in range(len(ks)):
            ci = b2.class_info(i)
            assert ci["tuned_ms"] == -1.0
            assert (ci["w1"], ci["gemm_form"], ci["col_tma"], ci["crt_tm"], ci["launch_groups"]) == chosen[i]


@pytest.mark.parametrize("col_tma,crt_tm,groups", [(1, 1, 1), (0, 1, 2), (1, 0, 4), (0, 0, 1)])
def test_every_kernel_variant_gives_the_same_bytes(tmp_path, monkeypatch, col_tma, crt_tm, groups):
    """Each variant the tuner can choose -- the column pass by the TMA pipeline or one tile per
    CTA, the CRT's A operand in tensor or shared memory, the class in 1, 2 or 4 launch groups --
    forced through a cache entry, gives the single-point path's bytes.  An entry in the older
    seven-field form is read with the engine's default variants and one launch group."""
    torch = _torch()
    import polymult
    ensure_library()
    cache = tmp_path / "tune.txt"
    monkeypatch.setenv("POLYMULT_TUNE_CACHE", str(cache))
    dev = torch.cuda.get_device_name(0).replace(" ", "_")
    ks = [_class(torch, 65536, 1747, 4, seed=70), _class(torch, 4096, 868, 4, seed=71)]
    want = [_single(torch, k) for k in ks]
    cache.write_text("65536 1747 4 %s 0 8 1.0 %d %d %d\n4096 868 4 %s 0 6 1.0\n"
                     % (dev, col_tma, crt_tm, groups, dev))
    with polymult.Batch([_spec(k) for k in ks], tune=True) as b:
        ci = b.class_info(0)
        assert (ci["w1"], ci["col_tma"], ci["crt_tm"], ci["launch_groups"]) == (8, col_tma, crt_tm, groups)
        assert b.class_info(1)["launch_groups"] == 1
        assert b.info()["kernel_launches"] >= groups * 8
        b.run(torch.cuda.current_stream().cuda_stream)
        b.sync()
        for k, w in zip(ks, want):
            assert np.array_equal(k["c"].cpu().numpy().view(np.uint32), w)


@pytest.mark.parametrize("N,W", [(1 << 17, 64), (1 << 18, 100), (1 << 20, 64)])
def test_long_lines_against_c_oracle(N, W):
    """N = 2^17 .. 2^20: row lines of 2^9 and 2^10 points (three NTT phases; a 1024-point
    row spans two warps) and column lines up to 2^10."""
    torch = _torch()
    import polymult
    ensure_library()
    k = _class(torch, N, W, 1, seed=N + W)
    got = _single(torch, k, gemm="auto")[0]
    a = k["a"].cpu().numpy().view(np.uint32)[0]
    b = k["b"].cpu().numpy().view(np.uint32)[0]
    assert np.array_equal(got, c_oracle_mul(N, W, k["q"], a, b))
