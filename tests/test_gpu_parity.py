"""GPU parity: the CUDA path through the C ABI, bit-exact against the reference's outputs.

Every golden point (the reference's own regression set, tests/run_emu.sh:20-33, plus the
benchmark configurations N=4096/W=256, N=32768/W=868 in four distributions and the ranked
N=65536/W=1747) is run through both entry points (host operands: pm_run, the reference's
fherma_run; device operands: pm_run_device) in both GEMM forms (CUDA-core plain, tcgen05
tensor-core) and compared byte-for-byte with c.bin as the reference's tests/oracle.py wrote
it.  Beyond the golden set: batched device calls, random operands at the ranked point
against the C oracle, repeatability, and a clean device status word after every run (pm_sync);
the status word's failure reports themselves are driven in test_gpu_failures.py."""
import numpy as np
import pytest

from conftest import c_oracle_mul, ensure_library, load_golden, orc, regen_case, sha

pytestmark = pytest.mark.gpu

GOLDEN = load_golden()
POINTS = GOLDEN["points"]
RANKED = [(4096, 256), (32768, 868), (65536, 1747)]


def _q(pt):
    return orc.limbs_of(int(pt["q_hex"], 16), pt["L"])


def _multiplier(pt, gemm):
    import polymult
    ensure_library()
    try:
        return polymult.Multiplier(pt["N"], pt["W"], _q(pt), gemm=gemm)
    except polymult.PolymultError as e:
        if e.code == polymult.PM_ERR_UNSUPPORTED and (pt["N"], pt["W"]) not in RANKED:
            pytest.skip("tensor-core form does not cover N=%d W=%d" % (pt["N"], pt["W"]))
        raise


def _torch():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.mark.parametrize("gemm", ["plain", "tensor"])
@pytest.mark.parametrize("pt", POINTS, ids=["N%d_W%d" % (p["N"], p["W"]) for p in POINTS])
def test_host_path_matches_reference(pt, gemm):
    m = _multiplier(pt, gemm)
    with m:
        assert m.info()["gemm"] == gemm
        for case in pt["cases"]:
            a, b, _ = regen_case(pt, case)
            c = m.multiply(a, b)
            assert sha(c) == case["c_sha256"], (pt["N"], pt["W"], case["s"], case["mode"])
        m.sync()


@pytest.mark.parametrize("gemm", ["plain", "tensor"])
@pytest.mark.parametrize("pt", POINTS, ids=["N%d_W%d" % (p["N"], p["W"]) for p in POINTS])
def test_device_path_matches_reference(pt, gemm):
    torch = _torch()
    m = _multiplier(pt, gemm)
    with m:
        A, B = [], []
        for case in pt["cases"]:
            a, b, _ = regen_case(pt, case)
            A.append(a)
            B.append(b)
        da = torch.from_numpy(np.stack(A).view(np.int32)).cuda()
        db = torch.from_numpy(np.stack(B).view(np.int32)).cuda()
        dc = torch.zeros_like(da)
        s = torch.cuda.current_stream()
        m.multiply_device(da.data_ptr(), db.data_ptr(), dc.data_ptr(), len(A), s.cuda_stream)
        m.sync()
        out = dc.cpu().numpy().view(np.uint32)
        for i, case in enumerate(pt["cases"]):
            assert sha(out[i]) == case["c_sha256"], (pt["N"], pt["W"], case["s"], case["mode"])


@pytest.mark.parametrize("gemm", ["plain", "tensor"])
def test_ranked_point_random_against_c_oracle(gemm):
    """Two fresh uniform cases at N=65536/W=1747 in one device call (two launch groups)."""
    torch = _torch()
    pt = next(p for p in POINTS if (p["N"], p["W"]) == (65536, 1747))
    q = int(pt["q_hex"], 16)
    A = [orc.uniform_limbs(65536, 1747, q, seed=s) for s in (11, 12)]
    B = [orc.uniform_limbs(65536, 1747, q, seed=s) for s in (21, 22)]
    m = _multiplier(pt, gemm)
    with m:
        da = torch.from_numpy(np.stack(A).view(np.int32)).cuda()
        db = torch.from_numpy(np.stack(B).view(np.int32)).cuda()
        dc = torch.zeros_like(da)
        m.multiply_device(da.data_ptr(), db.data_ptr(), dc.data_ptr(), 2, torch.cuda.current_stream().cuda_stream)
        m.sync()
        out = dc.cpu().numpy().view(np.uint32)
    for i in range(2):
        exp = c_oracle_mul(65536, 1747, q, A[i], B[i])
        assert np.array_equal(out[i], exp), i


def test_tensor_and_plain_agree_and_repeat():
    pt = next(p for p in POINTS if (p["N"], p["W"]) == (32768, 868))
    q = int(pt["q_hex"], 16)
    a = orc.uniform_limbs(32768, 868, q, seed=5)
    b = orc.uniform_limbs(32768, 868, q, seed=6)
    with _multiplier(pt, "plain") as mp, _multiplier(pt, "tensor") as mt:
        c1 = mp.multiply(a, b)
        c2 = mt.multiply(a, b)
        c3 = mt.multiply(a, b)
    assert np.array_equal(c1, c2) and np.array_equal(c2, c3)
    assert np.array_equal(c1, c_oracle_mul(32768, 868, q, a, b))


def test_commutative_and_linear():
    """Size-independent properties at the ranked point: a*b == b*a, (a+a')*b == a*b + a'*b."""
    pt = next(p for p in POINTS if (p["N"], p["W"]) == (65536, 1747))
    q = int(pt["q_hex"], 16)
    a = orc.uniform_limbs(65536, 1747, q, seed=31)
    b = orc.uniform_limbs(65536, 1747, q, seed=32)
    with _multiplier(pt, "tensor") as m:
        ab = m.multiply(a, b)
        ba = m.multiply(b, a)
        assert np.array_equal(ab, ba)
        # a' = x^1 * a (negacyclic shift): a'*b must be the shift of a*b
        av = orc.unpack_limbs(a)
        shifted = [(q - av[-1]) % q] + av[:-1]
        sb = m.multiply(orc.pack_limbs(shifted, pt["L"]), b)
    abv = orc.unpack_limbs(ab)
    exp = [(q - abv[-1]) % q] + abv[:-1]
    assert orc.unpack_limbs(sb) == exp


def test_stage_timing_runs_the_device_sequence():
    """pm_time_stages times the device-resident sequence kernel by kernel: every kernel stage
    takes time, a's own row pass is empty (the row pass of both operands covers it), and the
    timed launches leave the exact products in c."""
    torch = _torch()
    import polymult
    pt = next(p for p in POINTS if (p["N"], p["W"]) == (32768, 868))
    q = int(pt["q_hex"], 16)
    A = [orc.uniform_limbs(32768, 868, q, seed=41 + i) for i in range(2)]
    B = [orc.uniform_limbs(32768, 868, q, seed=51 + i) for i in range(2)]
    da = torch.from_numpy(np.stack(A).view(np.int32)).cuda()
    db = torch.from_numpy(np.stack(B).view(np.int32)).cuda()
    dc = torch.zeros_like(da)
    with _multiplier(pt, "tensor") as m:
        st = m.time_stages(da.data_ptr(), db.data_ptr(), dc.data_ptr(), 2, 3, torch.cuda.current_stream().cuda_stream)
        m.sync()
    assert list(st) == list(polymult.STAGES)
    assert st["rows_a"] == 0.0
    assert all(v > 0 for k, v in st.items() if k != "rows_a"), st
    out = dc.cpu().numpy().view(np.uint32)
    for i in range(2):
        assert np.array_equal(out[i], c_oracle_mul(32768, 868, q, A[i], B[i])), i


def test_fherma_python_mirror():
    import polymult
    pt = next(p for p in POINTS if (p["N"], p["W"]) == (4096, 256))
    st = polymult.fherma_init(pt["N"], pt["W"], pt["L"], _q(pt))
    try:
        a, b, _ = regen_case(pt, pt["cases"][0])
        assert sha(polymult.fherma_run(st, a, b)) == pt["cases"][0]["c_sha256"]
        with pytest.raises(RuntimeError):
            polymult.fherma_run(st, a[:-1], b[:-1])
    finally:
        polymult.fherma_free(st)


def test_tuned_pipeline_still_bit_exact():
    """The host pipeline's autotuner (pm_tune_pipeline) only changes the column-chunk schedule:
    results stay byte-identical to the reference's and the schedule is one of the candidates."""
    pt = next(p for p in POINTS if (p["N"], p["W"]) == (32768, 868))
    with _multiplier(pt, "tensor") as m:
        # before tuning the schedule follows the operand size: 3.7 MB per operand -> quarters
        before = m.pipeline()
        assert before["in_body"] == 4 and before["out_body"] == 4 and before["tuned_ms"] == 0
        info = m.tune_pipeline(2)
        assert info["in_body"] in (1, 2, 4, 8, 16) and info["out_body"] in (1, 2, 4, 8, 16) and info["tuned_ms"] > 0
        assert m.pipeline() == info
        # the page-locked schedule is tuned on its own and leaves the staged one alone
        assert m.pipeline(pinned=True)["tuned_ms"] == 0
        pinfo = m.tune_pipeline(2, pinned=True)
        assert pinfo["in_body"] in (1, 2, 3, 4, 5, 8, 16) and pinfo["out_body"] in (1, 2, 3, 4, 5, 8, 16)
        assert pinfo["tuned_ms"] > 0
        assert m.pipeline(pinned=True) == pinfo and m.pipeline() == info
        for case in pt["cases"]:
            a, b, _ = regen_case(pt, case)
            assert sha(m.multiply(a, b)) == case["c_sha256"], (case["s"], case["mode"])
        m.sync()


@pytest.mark.parametrize("shape", [(3, 3), (5, 5), (5, 1), (1, 5), (16, 2)], ids=lambda x: "in%d_out%d" % x)
def test_every_pinned_chunk_shape_is_bit_exact(shape):
    """Each schedule pm_tune_pipeline can choose for page-locked calls, set directly with
    pm_set_pipeline -- the uneven shapes 3 (b in halves and quarters) and 5 (b in 1/2, 1/4,
    1/8, 1/8; c in 1/8, 1/8, 1/4, 1/2) included -- gives the reference's bytes; divisors outside
    the candidates are refused."""
    torch = _torch()
    import polymult
    pt = next(p for p in POINTS if (p["N"], p["W"]) == (65536, 1747))
    with _multiplier(pt, "tensor") as m:
        m.set_pipeline(shape[0], shape[1], pinned=True)
        info = m.pipeline(pinned=True)
        assert (info["in_body"], info["out_body"]) == shape and info["tuned_ms"] == 0
        with pytest.raises(polymult.PolymultError):
            m.set_pipeline(5, 5)  # the uneven shapes are for page-locked calls only
        with pytest.raises(polymult.PolymultError):
            m.set_pipeline(6, 8, pinned=True)
        L = (pt["W"] + 31) // 32
        for case in pt["cases"][:2]:
            a, b, _ = regen_case(pt, case)
            pa, pb, pc = (torch.empty((pt["N"], L), dtype=torch.int32).pin_memory() for _ in range(3))
            pa.numpy().view(np.uint32)[:] = a
            pb.numpy().view(np.uint32)[:] = b
            m.multiply(pa.numpy().view(np.uint32), pb.numpy().view(np.uint32), pc.numpy().view(np.uint32))
            assert sha(pc.numpy().view(np.uint32)) == case["c_sha256"], (shape, case["s"])
        m.sync()


@pytest.mark.parametrize("nw", [(4096, 256), (32768, 868), (65536, 1747)], ids=lambda x: "N%d_W%d" % x)
def test_pinned_host_operands_take_direct_copies(nw):
    """Host operands already in page-locked memory skip the host staging: pm_run moves each
    column chunk with one strided DMA copy in and out.  Every mix of pinned and pageable
    operands and result gives the reference's bytes (narrow chunks of a few columns included
    at N = 4096)."""
    torch = _torch()
    pt = next(p for p in POINTS if (p["N"], p["W"]) == nw)
    N, L = pt["N"], pt["L"]

    def pinned(x=None):
        buf = torch.empty((N, L), dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)
        buf[:] = 0 if x is None else x
        return buf

    with _multiplier(pt, "tensor") as m:
        for case in pt["cases"][:2]:
            a, b, _ = regen_case(pt, case)
            for pa, pb, pc in [(1, 1, 1), (1, 0, 0), (0, 1, 1), (0, 0, 1)]:
                ha = pinned(a) if pa else np.ascontiguousarray(a)
                hb = pinned(b) if pb else np.ascontiguousarray(b)
                hc = pinned() if pc else np.zeros((N, L), dtype=np.uint32)
                m.multiply(ha, hb, hc)
                assert sha(hc) == case["c_sha256"], (case["s"], case["mode"], pa, pb, pc)
        m.sync()


def test_pinned_operands_are_detected(monkeypatch, capfd):
    """The direct-copy path is taken exactly for the page-locked buffers (POLYMULT_PROFILE's
    per-call line names which of a, b and c moved by direct copies)."""
    torch = _torch()
    monkeypatch.setenv("POLYMULT_PROFILE", "1")
    pt = next(p for p in POINTS if (p["N"], p["W"]) == (32768, 868))
    N, L = pt["N"], pt["L"]
    a, b, _ = regen_case(pt, pt["cases"][0])
    pa = torch.empty((N, L), dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)
    pa[:] = a
    with _multiplier(pt, "tensor") as m:
        capfd.readouterr()
        c = m.multiply(pa, np.ascontiguousarray(b))
        err = capfd.readouterr().err
        assert "direct copies a 1 b 0 c 0" in err, err
        assert sha(c) == pt["cases"][0]["c_sha256"]
        m.sync()


def test_wide_points_on_tensor_cores_in_blocks():
    """Above K = 128 primes (W beyond about 1900 bits) one tcgen05 tile no longer holds every
    prime: the decomposition runs in prime blocks and the CRT in (prime block, result-byte block)
    launches that accumulate exact partial integers, finished by one CUDA-core pass.  Bit-exact
    on the reference's W = 4000 golden point and, against the C oracle and the plain form, on a
    W = 3000 point of the batch grid."""
    import workload
    pt = next(p for p in POINTS if p["W"] == 4000)
    with _multiplier(pt, "auto") as m:
        assert m.info()["gemm"] in ("tensor", "mixed")
        for case in pt["cases"]:
            a, b, _ = regen_case(pt, case)
            assert sha(m.multiply(a, b)) == case["c_sha256"], (case["s"], case["mode"])
        m.sync()
    torch = _torch()
    import polymult
    N, W = 4096, 3000
    L = (W + 31) // 32
    q = workload.spec_prime(N, W)
    ops = workload.uniform_operands(N, W, q, 6, seed=17)
    da = torch.from_numpy(np.ascontiguousarray(ops[:3]).view(np.int32)).cuda()
    db = torch.from_numpy(np.ascontiguousarray(ops[3:]).view(np.int32)).cuda()
    outs = {}
    for gemm in ("auto", "plain"):
        with polymult.Multiplier(N, W, workload.limbs(q, L), gemm=gemm) as m:
            outs[gemm] = m.info()["gemm"]
            dc = torch.zeros_like(da)
            m.multiply_device(da.data_ptr(), db.data_ptr(), dc.data_ptr(), 3, torch.cuda.current_stream().cuda_stream)
            m.sync()
            outs[gemm + "_c"] = dc.cpu().numpy().view(np.uint32)
            host = m.multiply(ops[0], ops[3])  # the chunked host pipeline as well
            assert np.array_equal(host, outs[gemm + "_c"][0])
    assert outs["auto"] == "tensor" and outs["plain"] == "plain"
    assert np.array_equal(outs["auto_c"], outs["plain_c"])
    for i in range(3):
        assert np.array_equal(outs["auto_c"][i], c_oracle_mul(N, W, q, ops[i], ops[3 + i])), i


def test_butterfly_peak_matches_the_host():
    """pm_butterfly_peak runs the NTT's Shoup butterfly on register operands over every SM; its
    checksum equals the host's recomputation (else PM_ERR_DEVICE), and the rate is plausible for
    a pipe that takes the 64-bit product at a quarter of the low multiply's rate."""
    _torch()
    import polymult
    ensure_library()
    r = polymult.butterfly_peak(0)
    assert r["bfly_per_s"] > 1e11
    assert 2.0 < r["bfly_per_clk_sm"] < 64.0

