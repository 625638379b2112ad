"""GPU tests of the serving loop (pm_server_*): continuous batching over resident operands.

The tolerance is bit-exact: every result served in a mix of concurrent requests (batched with
requests for other resident operands, several batches in flight) must equal the same request
served alone, and the plain single-point device path (pm_run_device) on the same pair."""
import numpy as np
import pytest

from conftest import ensure_library, load_golden, orc

pytestmark = pytest.mark.gpu

GOLDEN = {(p["N"], p["W"]): int(p["q_hex"], 16) for p in load_golden()["points"]}


def _torch():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _setup(N, W, nres, nreq, seed):
    import workload
    q = GOLDEN.get((N, W)) or workload.spec_prime(N, W)
    L = (W + 31) // 32
    res = workload.uniform_operands(N, W, q, nres, seed=seed)
    reqs = workload.uniform_operands(N, W, q, nreq, seed=seed + 1)
    rng = np.random.default_rng(seed)
    sel = rng.integers(0, nres, size=nreq).astype(np.uint32)
    return q, L, res, reqs, sel


def _alone(torch, N, W, q, L, res, reqs, sel):
    """Each request through the single-point device path."""
    import polymult
    out = np.zeros_like(reqs)
    with polymult.Multiplier(N, W, orc.limbs_of(q, L)) as m:
        for i in range(len(reqs)):
            da = torch.from_numpy(reqs[i:i + 1].view(np.int32)).cuda()
            db = torch.from_numpy(res[sel[i]:sel[i] + 1].view(np.int32)).cuda()
            dc = torch.zeros_like(da)
            m.multiply_device(da.data_ptr(), db.data_ptr(), dc.data_ptr(), 1, torch.cuda.current_stream().cuda_stream)
            m.sync()
            out[i] = dc.cpu().numpy().view(np.uint32)[0]
    return out


def _serve(srv, reqs, sel, t_arrive):
    a = srv.pinned(len(reqs))
    c = srv.pinned(len(reqs))
    a[:] = reqs
    c[:] = 0
    lat, st = srv.run(t_arrive, sel, list(a), list(c))
    return np.array(c), lat, st


@pytest.mark.parametrize("N,W,nres,nreq", [(4096, 256, 3, 40), (2048, 868, 8, 24), (65536, 1747, 8, 12),
                                            (4096, 3000, 4, 16)])
def test_mixed_requests_equal_alone(N, W, nres, nreq):
    torch = _torch()
    import polymult
    ensure_library()
    q, L, res, reqs, sel = _setup(N, W, nres, nreq, seed=N + W)
    want = _alone(torch, N, W, q, L, res, reqs, sel)
    with polymult.Server(N, W, orc.limbs_of(q, L), res, max_batch=4, streams=3) as srv:
        # burst: everything queued at t = 0 -> batches of mixed resident operands in flight together
        got, lat, st = _serve(srv, reqs, sel, np.zeros(nreq))
        assert st["requests"] == nreq and st["batches"] < nreq and st["mean_batch"] > 1
        assert np.all(lat > 0)
        assert np.array_equal(got, want)
        # the same requests one at a time (each alone on the server)
        for i in range(nreq):
            gi, _, sti = _serve(srv, reqs[i:i + 1], sel[i:i + 1], np.zeros(1))
            assert sti["batches"] == 1
            assert np.array_equal(gi[0], want[i]), i
        # Poisson arrivals
        rng = np.random.default_rng(5)
        t = np.cumsum(rng.exponential(1.0 / 4000.0, size=nreq))
        got2, lat2, _ = _serve(srv, reqs, sel, t)
        assert np.array_equal(got2, want)
        assert np.all(lat2 > 0)


def test_hbm_budget_bounds_requests_in_flight():
    torch = _torch()
    import polymult
    ensure_library()
    N, W = 4096, 868
    q, L, res, reqs, sel = _setup(N, W, 2, 16, seed=3)
    want = _alone(torch, N, W, q, L, res, reqs, sel)
    # learn K and the tables' size from a server with room to spare, then budget for 2 requests
    with polymult.Multiplier(N, W, orc.limbs_of(q, L), gemm="auto") as m:
        inf = m.info()
    per_req = (2 * N * L + inf["K"] * N) * 4
    fixed = 2 * inf["K"] * N * 4 + inf["table_bytes"]
    budget = fixed + 2 * per_req + per_req // 2
    with polymult.Server(N, W, orc.limbs_of(q, L), res, hbm_budget=budget, max_batch=8, streams=4) as srv:
        got, _, st = _serve(srv, reqs, sel, np.zeros(len(reqs)))
        assert st["max_inflight"] == 2
        assert st["peak_inflight"] <= 2
        assert np.array_equal(got, want)
    with pytest.raises(polymult.PolymultError) as ei:
        polymult.Server(N, W, orc.limbs_of(q, L), res, hbm_budget=fixed + per_req // 2)
    assert ei.value.code == polymult.PM_ERR_INVALID


def test_result_digests_match_the_results():
    """The server's per-request digests (computed on the device before each result's copy)
    equal the host digest of the result it delivered and of the same product run alone; the
    standalone device digest (pm_digest) agrees with the host one."""
    torch = _torch()
    import polymult
    ensure_library()
    N, W = 4096, 868
    q, L, res, reqs, sel = _setup(N, W, 4, 20, seed=11)
    want = _alone(torch, N, W, q, L, res, reqs, sel)
    with polymult.Server(N, W, orc.limbs_of(q, L), res, max_batch=4, streams=3) as srv:
        a = srv.pinned(len(reqs))
        c = srv.pinned(len(reqs))
        a[:] = reqs
        lat, st, dig = srv.run(np.zeros(len(reqs)), sel, list(a), list(c), digests=True)
        got = np.array(c)
    assert np.array_equal(got, want)
    for i in range(len(reqs)):
        assert int(dig[i]) == polymult.digest_host(got[i]) == polymult.digest_host(want[i]), i
    d = torch.from_numpy(np.ascontiguousarray(want).view(np.int32)).cuda()
    dd = polymult.digest_device(d.data_ptr(), N * L, len(reqs))
    assert [int(x) for x in dd] == [polymult.digest_host(w) for w in want]
    # a one-word change moves the digest
    w2 = want[0].copy()
    w2[N // 2, 3] ^= 1
    assert polymult.digest_host(w2) != polymult.digest_host(want[0])
