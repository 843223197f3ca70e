"""GPU tests of the device Q1 assembler and the continuous-batching server.

Bars: device assembly bit-identical to the host assembler (which is pinned to
the reference); served solves reach the requested relative residual within
+-5% of the oracle's iteration count and within 1e-8 of its solution; a
request's result is bit-identical alone and inside any mix, under any kernel
shape; memory budget, refusals and per-request failures are reported without
disturbing the other requests.
"""
import ctypes as C
import importlib

import numpy as np
import pytest

from pyoracle import control

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pf(b200):
    return b200.Platform(0)


@pytest.fixture(scope="module")
def srv(b200):
    return importlib.import_module("hiflow3_b200.serving")


def within5(got, want):
    return abs(got - want) <= max(1, int(np.ceil(0.05 * want)))


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


@pytest.mark.parametrize("dim,N,kind,coef", [(2, 1, 0, False), (2, 17, 0, True), (2, 33, 1, False),
                                             (2, 9, 1, True), (3, 1, 0, False), (3, 6, 0, True),
                                             (3, 7, 1, False), (3, 5, 1, True)])
def test_q1_assemble_device_bitexact(pf, b200, dim, N, kind, coef):
    import torch
    n, nnz = b200.q1_sizes(dim, N)
    kc = np.exp(np.random.default_rng(3).standard_normal(N ** dim)) if coef else None
    beta = np.array([1.0, 0.5, 0.25])
    row_h, col_h, val_h = b200.q1_assemble(dim, N, kind, kc, 1e-2, beta)
    with pf.on_stream():   # ordered with the library's kernels on the platform's stream
        row = torch.empty(n + 1, dtype=torch.int32, device="cuda")
        col = torch.empty(nnz, dtype=torch.int32, device="cuda")
        val = torch.empty(nnz, dtype=torch.float64, device="cuda")
        rhs = torch.empty(n, dtype=torch.float64, device="cuda")
        kd = torch.from_numpy(kc).cuda() if coef else None
    L = b200.lib()
    pf.check(L.b200la_q1_assemble_device(pf.h, dim, N, kind, _ptr(kd), 1e-2, beta.ctypes.data, _ptr(row),
                                         _ptr(col), _ptr(val)), "q1_assemble_device")
    pf.check(L.b200la_q1_rhs_device(pf.h, 11, dim, N, _ptr(rhs)), "q1_rhs_device")
    pf.sync()
    assert np.array_equal(row.cpu().numpy(), row_h)
    assert np.array_equal(col.cpu().numpy(), col_h)
    assert np.array_equal(val.cpu().numpy().view(np.uint64), val_h.view(np.uint64))
    assert np.array_equal(rhs.cpu().numpy().view(np.uint64), b200.q1_rhs(11, dim, N).view(np.uint64))


def test_serve_cg_vs_oracle(b200, srv, oracle):
    N = 40
    kc = np.exp(0.5 * np.random.default_rng(1).standard_normal(N * N))
    row, col, val = b200.q1_assemble(2, N, 0, kc)
    rhs = b200.q1_rhs(5, 2, N)
    ref = oracle.pcg(row, col, val, rhs, precond=oracle.invdiag(row, col, val),
                     ctl=control(10000, 0.0, 1e-10, 1e6))
    with srv.Server(budget_bytes=1e9, max_slots=64) as s:
        i1 = s.submit(q1=dict(dim=2, N=N, kcell=kc), rhs_seed=5, ctl=(10000, 0.0, 1e-10, 1e6))
        i2 = s.submit(csr=(row, col, val), b=rhs, ctl=(10000, 0.0, 1e-10, 1e6))
        r1, r2 = s.wait(i1), s.wait(i2)
    for r in (r1, r2):
        assert r["status"] == b200.SUCCESS_REL
        assert r["res"] <= 1e-10 * r["res0"]
        assert within5(r["iters"], ref["iters"]), (r["iters"], ref["iters"])
        assert np.linalg.norm(r["x"] - ref["x"]) <= 1e-8 * np.linalg.norm(ref["x"])
    # the device-assembled system and the uploaded host CSR are the same system
    assert r1["iters"] == r2["iters"] and np.array_equal(r1["x"], r2["x"])


def test_serve_mixed_vs_oracle(b200, srv, oracle):
    dim, N = 3, 12
    kc = np.exp(np.random.default_rng(5).standard_normal(N ** dim))
    row, col, val = b200.q1_assemble(dim, N, 0, kc)
    b = b200.q1_rhs(9, dim, N)
    ref = oracle.mpir(row, col, val, b, outer=control(50, 0, 1e-10, 1e6), inner=control(10000, 0, 1e-4, 1e6))
    x64 = oracle.pcg(row, col, val, b, precond=oracle.invdiag(row, col, val),
                     ctl=control(100000, 0.0, 1e-13, 1e6))["x"]
    with srv.Server(budget_bytes=1e9, max_slots=16) as s:
        r = s.wait(s.submit(q1=dict(dim=dim, N=N, kcell=kc), rhs_seed=9, precision=b200.SERVE_MIXED,
                            ctl=(50, 0.0, 1e-10, 1e6), inner=(10000, 0.0, 1e-4, 1e6), max_outer=50))
    assert r["status"] == b200.SUCCESS_REL
    assert r["res"] <= 1e-10 * r["res0"]
    assert abs(r["outer"] - ref["outer"]) <= 1
    assert within5(r["iters"], ref["inner_total"]), (r["iters"], ref["inner_total"])
    assert np.linalg.norm(r["x"] - x64) <= 1e-8 * np.linalg.norm(x64)


def _mix_requests(b200):
    rng = np.random.default_rng(11)
    reqs = []
    for k, (dim, N) in enumerate([(2, 64), (3, 10), (2, 97), (2, 32), (3, 17), (2, 150), (3, 8), (2, 45),
                                  (2, 77), (3, 14)]):
        kc = np.exp(0.5 * rng.standard_normal(N ** dim)) if dim == 2 else None
        reqs.append(dict(q1=dict(dim=dim, N=N, kcell=kc), rhs_seed=100 + k,
                         precision=b200.SERVE_MIXED if k % 3 == 1 else b200.SERVE_F64))
    row, col, val = b200.q1_assemble(2, 50, 0, np.exp(rng.standard_normal(2500)))
    reqs.append(dict(csr=(row, col, val), b=rng.uniform(-1, 1, row.size - 1), precision=b200.SERVE_F64))
    return reqs


def test_serve_alone_vs_mix_bitwise(b200, srv):
    reqs = _mix_requests(b200)
    targets = [0, 1, 5, 10]
    alone = {}
    with srv.Server(budget_bytes=2e9, max_slots=32, warps=4, ctas_per_sm=8, chunks_per_warp=1) as s:
        for t in targets:
            alone[t] = s.wait(s.submit(**reqs[t]))
    with srv.Server(budget_bytes=2e9, max_slots=32, warps=8, ctas_per_sm=4, chunks_per_warp=4,
                    iters_per_round=5, max_active=4) as s:
        ids = [s.submit(**r) for r in reqs]
        mixed = [s.wait(i) for i in ids]
        st = s.stats()
    assert st["completed"] == len(reqs) and st["failed"] == 0
    for t in targets:
        a, m = alone[t], mixed[t]
        assert a["status"] in (b200.SUCCESS_ABS, b200.SUCCESS_REL)
        assert (a["iters"], a["outer"], a["status"]) == (m["iters"], m["outer"], m["status"])
        assert a["res"] == m["res"] and a["res0"] == m["res0"]
        assert np.array_equal(a["x"], m["x"]), t
    for r in mixed:
        assert r["res"] <= 1e-10 * r["res0"]


def test_serve_half_stencil_bitwise(b200, srv, monkeypatch):
    """Q1 Poisson requests stored as half stencils (diagonal and upper half,
    the lower half read from the owning rows) solve to the same bits as with
    the full stencil layout, FP64 and mixed, 2-D and 3-D."""
    reqs = _mix_requests(b200)[:10]
    out = {}
    for half in ("2", "0"):
        monkeypatch.setenv("B200LA_SERVE_HALF", half)
        with srv.Server(budget_bytes=2e9, max_slots=32) as s:
            ids = [s.submit(**r) for r in reqs]
            out[half] = [s.wait(i) for i in ids]
    for a, b in zip(out["2"], out["0"]):
        assert a["status"] in (b200.SUCCESS_ABS, b200.SUCCESS_REL)
        assert (a["iters"], a["outer"], a["status"], a["res"]) == (b["iters"], b["outer"], b["status"], b["res"])
        assert np.array_equal(a["x"], b["x"])


def test_serve_continuous_admission(b200, srv):
    # a long request is running when short ones arrive: they are admitted into
    # the running batch and finish first
    with srv.Server(budget_bytes=2e9, max_slots=32) as s:
        # runs exactly 4000 iterations (no tolerance can be met)
        big = s.submit(q1=dict(dim=2, N=256), rhs_seed=1, ctl=(4000, 0.0, 0.0, 1e300))
        import time
        t0 = time.time()
        while s.stats()["rounds"] < 2 and time.time() - t0 < 30.0:   # the big request is iterating
            time.sleep(0.001)
        small = [s.submit(q1=dict(dim=2, N=40 + k), rhs_seed=2 + k) for k in range(6)]
        rs = [s.wait(i) for i in small]
        rb = s.wait(big)
    assert rb["status"] == b200.FAIL_MAXITS and rb["iters"] == 4000
    assert all(r["status"] == b200.SUCCESS_REL for r in rs)
    assert all(r["t_submit"] > rb["t_ready"] for r in rs)
    assert all(r["t_done"] < rb["t_done"] for r in rs)


def test_serve_budget_and_refusal(b200, srv):
    budget = 1.2e6
    with srv.Server(budget_bytes=budget, max_slots=8) as s:
        with pytest.raises(b200.B200Error) as e:
            s.submit(q1=dict(dim=2, N=256), rhs_seed=1)
        assert e.value.code == 6
        ids = [s.submit(q1=dict(dim=2, N=40 + k), rhs_seed=k) for k in range(10)]
        res = [s.wait(i) for i in ids]
        st = s.stats()
    assert all(r["status"] == b200.SUCCESS_REL for r in res)
    assert st["completed"] == 10 and st["peak_resident_bytes"] <= budget
    # the budget held requests back: some were admitted only after others finished
    t_done = sorted(r["t_done"] for r in res)
    assert any(r["t_admit"] >= t_done[0] for r in res)


def test_serve_failures_are_per_request(b200, srv):
    with srv.Server(budget_bytes=1e9, max_slots=8) as s:
        bad = s.submit(q1=dict(dim=2, N=64), rhs_seed=1, ctl=(5, 0.0, 1e-10, 1e6))
        good = s.submit(q1=dict(dim=2, N=48), rhs_seed=2)
        row = np.array([0, 2, 1], np.int32)   # non-monotone row pointer
        with pytest.raises(b200.B200Error) as e:
            s.submit(csr=(row, np.array([0, 1], np.int32), np.ones(2)), b=np.ones(2))
        assert e.value.code == 5
        rb, rg = s.wait(bad), s.wait(good)
    assert rb["status"] == b200.FAIL_MAXITS and rb["iters"] == 5
    assert rg["status"] == b200.SUCCESS_REL


def test_serve_nan_request_fails_alone(b200, srv):
    """NaN right-hand sides (an FP64 and a mixed request) inside a batch: the
    NaN requests end with FAIL_MAXITS (FP64: at the iteration limit; mixed: no
    outer step starts), and the other requests of the batch converge to the
    same bits as when solved alone."""
    reqs = _mix_requests(b200)[:6]
    with srv.Server(budget_bytes=2e9, max_slots=32) as s:
        alone = [s.wait(s.submit(**r)) for r in reqs]
    bn = b200.q1_rhs(3, 2, 40)
    bn[100] = np.nan
    with srv.Server(budget_bytes=2e9, max_slots=32, iters_per_round=4) as s:
        bad64 = s.submit(q1=dict(dim=2, N=40), b=bn, ctl=(30, 0.0, 1e-10, 1e6))
        ids = [s.submit(**r) for r in reqs]
        badmx = s.submit(q1=dict(dim=2, N=40), b=bn, precision=b200.SERVE_MIXED, max_outer=5)
        rb64, rbmx = s.wait(bad64), s.wait(badmx)
        mixed = [s.wait(i) for i in ids]
    assert rb64["status"] == b200.FAIL_MAXITS and rb64["iters"] == 30
    assert rbmx["status"] == b200.FAIL_MAXITS and rbmx["outer"] == 0
    for a, m in zip(alone, mixed):
        assert a["status"] in (b200.SUCCESS_ABS, b200.SUCCESS_REL)
        assert (a["iters"], a["outer"], a["status"], a["res"]) == (m["iters"], m["outer"], m["status"], m["res"])
        assert np.array_equal(a["x"], m["x"])


def test_serve_long_rows_warp_per_row(b200, srv, oracle):
    # an arrow matrix: row 0 and column 0 dense, so rows are too long for the
    # sliced layout and go through the warp-per-row path
    import scipy.sparse as sp
    n = 400
    A = sp.diags([-np.ones(n - 1), 4.0 * np.ones(n), -np.ones(n - 1)], [-1, 0, 1], format="lil")
    A[0, 1:] = -0.5
    A[1:, 0] = -0.5
    A[0, 0] = float(n)
    A = A.tocsr()
    A.sort_indices()
    row, col, val = A.indptr.astype(np.int32), A.indices.astype(np.int32), A.data.astype(np.float64)
    b = np.random.default_rng(2).uniform(-1, 1, n)
    ref = oracle.pcg(row, col, val, b, precond=oracle.invdiag(row, col, val), ctl=control(10000, 0.0, 1e-10, 1e6))
    with srv.Server(budget_bytes=1e9, max_slots=8) as s:
        r = s.wait(s.submit(csr=(row, col, val), b=b))
        r2 = s.wait(s.submit(csr=(row, col, val), b=b, precision=b200.SERVE_MIXED, ctl=(50, 0.0, 1e-10, 1e6)))
    assert r["status"] == b200.SUCCESS_REL and within5(r["iters"], ref["iters"])
    assert np.linalg.norm(r["x"] - ref["x"]) <= 1e-8 * np.linalg.norm(ref["x"])
    assert r2["status"] == b200.SUCCESS_REL
    assert np.linalg.norm(r2["x"] - ref["x"]) <= 1e-8 * np.linalg.norm(ref["x"])


def test_serve_gmres_nonsymmetric(b200, srv, golden):
    import scipy.sparse as sp
    row, col, val = b200.q1_assemble(2, 32, 1, None, 1e-3, (1.0, 0.5))
    b = golden["gmres2d32_b"]
    A = sp.csr_matrix((val, col, row))
    with srv.Server(budget_bytes=1e9, max_slots=8) as s:
        ids = [s.submit(q1=dict(dim=2, N=32, kind=1, nu=1e-3, beta=(1.0, 0.5)), b=b, method=b200.SERVE_GMRES,
                        gmres_precond=b200.PRECOND_ILU0_LS, ctl=(1000, 0.0, 1e-9, 1e6)),
               s.submit(q1=dict(dim=2, N=40), rhs_seed=3)]
        r, rc = s.wait(ids[0]), s.wait(ids[1])
    assert r["status"] == b200.SUCCESS_REL
    assert within5(r["iters"], int(golden["gmres2d32_iluls_iters"][0])), r["iters"]
    assert np.linalg.norm(b - A @ r["x"]) <= 2e-9 * np.linalg.norm(b)
    assert rc["status"] == b200.SUCCESS_REL
