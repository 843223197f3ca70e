"""GPU parity of the B200 preconditioners and solvers.

Bars: colours, permutations and levels bit-exact with the reference (golden);
preconditioner applies within 1e-12 relative of the oracle; Krylov solves
reach the same relative residual within +-5% of the reference's iteration
count (the counts usually coincide); solutions within 1e-8 relative of the
reference's.
"""
import numpy as np
import pytest

from pyoracle import control

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pf(b200):
    return b200.Platform(0)


def within5(got, want):
    return abs(got - want) <= max(1, int(np.ceil(0.05 * want)))


def test_cg_kat(pf, b200):
    # test/LinearAlgebra/cg.cc:35-91
    row = np.array([0, 3, 6, 9], np.int32)
    col = np.array([0, 1, 2] * 3, np.int32)
    val = np.array([2, -1, 0, -1, 2, -1, 0, -1, 2.0])
    A = b200.CSR_lMatrix.from_csr(pf, row, col, val)
    for P in (None, b200.Preconditioner.Jacobi(pf, A)):
        x = pf.vector(3)
        cg = b200.CG(pf)
        cg.SetupOperator(A)
        cg.SetupPreconditioner(P)
        cg.InitControl(100, 1e-300, 0.0, 1e6)
        cg.Solve(pf.vector([1.0, -2.0, 0.0]), x)
        np.testing.assert_allclose(x.numpy(), [-0.25, -1.5, -0.75], atol=1e-12)
    gm = b200.GMRES(pf, 30)
    gm.SetupOperator(A)
    # the Krylov space is exhausted after 3 steps; the device's summation
    # order leaves a residual of rounding size there, so the absolute stop is
    # set above it
    gm.InitControl(100, 1e-13, 0.0, 1e6)
    x = pf.vector(3)
    gm.Solve(pf.vector([1.0, -2.0, 0.0]), x)
    np.testing.assert_allclose(x.numpy(), [-0.25, -1.5, -0.75], atol=1e-12)


@pytest.mark.parametrize("dim,N", [(2, 32), (3, 12)])
@pytest.mark.parametrize("name", ["none", "jacobi"])
def test_cg_vs_reference(pf, b200, golden, dim, N, name):
    key = f"solve{dim}d{N}"
    row, col, val = b200.q1_assemble(dim, N)
    b = golden[key + "_b"]
    A = b200.CSR_lMatrix.from_csr(pf, row, col, val)
    cg = b200.CG(pf)
    cg.SetupOperator(A)
    if name == "jacobi":
        cg.SetupPreconditioner(b200.Preconditioner.Jacobi(pf, A))
    cg.InitControl(5000, 0.0, 1e-10, 1e6)
    x = pf.vector(len(b))
    st = cg.Solve(pf.vector(b), x, history=5001)
    ref_it = int(golden[f"{key}_{name}_iters"][0])
    assert st == b200.SUCCESS_REL
    assert within5(cg.iter(), ref_it), (cg.iter(), ref_it)
    xr = golden[f"{key}_{name}_x"]
    assert np.linalg.norm(x.numpy() - xr) <= 1e-8 * np.linalg.norm(xr)
    h = golden[f"{key}_{name}_hist"]
    k = min(len(h), len(cg.history))
    np.testing.assert_allclose(cg.history[:k][:10], h[:k][:10], rtol=1e-10)


@pytest.mark.parametrize("dim,N", [(2, 8), (3, 7)])
def test_mcsgs_setup_and_apply(pf, b200, oracle, golden, dim, N):
    key = f"{dim}d{N}_p"
    row, col, val = golden[key + "_row"], golden[key + "_col"], golden[key + "_val"]
    P = b200.Preconditioner.MultiColoringSGS(pf, row, col, val)
    assert np.array_equal(P.perm, golden[key + "_mcsgs_perm"])
    assert np.array_equal(P.block_sizes, golden[key + "_mcsgs_sizes"])
    Ar, Ac, Av = P.A_perm.download()
    assert np.array_equal(Ar, golden[key + "_mcsgs_Arow"]) and np.array_equal(Ac, golden[key + "_mcsgs_Acol"])
    assert np.array_equal(Av, golden[key + "_mcsgs_Aval"])
    r = golden[key + "_x"]
    z = pf.vector(len(r))
    P.ApplyPreconditioner(pf.vector(r), z)
    zr = golden[key + "_mcsgs_z"]
    assert np.max(np.abs(z.numpy() - zr)) <= 1e-12 * np.max(np.abs(zr))


@pytest.mark.parametrize("dim,N", [(2, 32), (3, 12)])
def test_mcsgs_pcg_vs_reference(pf, b200, golden, dim, N):
    key = f"solve{dim}d{N}"
    row, col, val = b200.q1_assemble(dim, N)
    P = b200.Preconditioner.MultiColoringSGS(pf, row, col, val)
    b = golden[key + "_b"][P.perm]
    cg = b200.CG(pf)
    cg.SetupOperator(P.A_perm)
    cg.SetupPreconditioner(P)
    cg.InitControl(5000, 0.0, 1e-8, 1e6)
    x = pf.vector(len(b))
    assert cg.Solve(pf.vector(b), x) == b200.SUCCESS_REL
    ref_it = int(golden[f"{key}_mcsgs_iters"][0])
    assert within5(cg.iter(), ref_it), (cg.iter(), ref_it)
    xr = golden[f"{key}_mcsgs_x"]
    assert np.linalg.norm(x.numpy() - xr) <= 1e-7 * np.linalg.norm(xr)


@pytest.mark.parametrize("syncfree,sweep", [("0", "tickets"), ("1", "tickets"), ("1", "cta"), ("1", "staged")])
@pytest.mark.parametrize("dim,N,tag", [(2, 17, "cd"), (3, 7, "p"), (2, 8, "pk")])
def test_ilu0_ls_apply(pf, b200, golden, dim, N, tag, syncfree, sweep, monkeypatch):
    monkeypatch.setenv("B200LA_SYNCFREE", syncfree)
    monkeypatch.setenv("B200LA_SWEEP", sweep)
    key = f"{dim}d{N}_{tag}"
    row, col, val = golden[key + "_row"], golden[key + "_col"], golden[key + "_val"]
    P = b200.Preconditioner.ILU0(pf, row, col, val, b200.PRECOND_ILU0_LS)
    assert np.array_equal(P.perm, golden[key + "_iluls_perm"])
    assert np.array_equal(P.block_sizes, golden[key + "_iluls_sizes"])
    r = golden[key + "_x"]
    z = pf.vector(len(r))
    for _ in range(3):   # repeated applies (epochs of the sync-free sweep; the ring of the level sweep)
        P.ApplyPreconditioner(pf.vector(r), z)
        zr = golden[key + "_iluls_z"]
        assert np.max(np.abs(z.numpy() - zr)) <= 1e-12 * np.max(np.abs(zr))


def test_ilu0_mc_apply(pf, b200, golden):
    key = "2d17_cd"
    row, col, val = golden[key + "_row"], golden[key + "_col"], golden[key + "_val"]
    P = b200.Preconditioner.ILU0(pf, row, col, val, b200.PRECOND_ILU0_MC)
    assert np.array_equal(P.perm, golden[key + "_ilumc_perm"])
    r = golden[key + "_x"]
    z = pf.vector(len(r))
    P.ApplyPreconditioner(pf.vector(r), z)
    zr = golden[key + "_ilumc_z"]
    assert np.max(np.abs(z.numpy() - zr)) <= 1e-12 * np.max(np.abs(zr))


@pytest.mark.parametrize("syncfree,sweep", [("0", "tickets"), ("1", "tickets"), ("1", "cta"), ("1", "staged")])
def test_gmres_ilu_ls_vs_reference(pf, b200, golden, syncfree, sweep, monkeypatch):
    monkeypatch.setenv("B200LA_SYNCFREE", syncfree)
    monkeypatch.setenv("B200LA_SWEEP", sweep)
    row, col, val = b200.q1_assemble(2, 32, 1, None, 1e-3, (1.0, 0.5))
    P = b200.Preconditioner.ILU0(pf, row, col, val, b200.PRECOND_ILU0_LS)
    b = golden["gmres2d32_b"][P.perm]
    gm = b200.GMRES(pf, 30)
    gm.SetupOperator(P.A_perm)
    gm.SetupPreconditioner(P)
    gm.InitControl(1000, 0.0, 1e-9, 1e6)
    x = pf.vector(len(b))
    assert gm.Solve(pf.vector(b), x) == b200.SUCCESS_REL
    ref_it = int(golden["gmres2d32_iluls_iters"][0])
    assert within5(gm.iter(), ref_it), (gm.iter(), ref_it)
    xr = golden["gmres2d32_iluls_x"]
    assert np.linalg.norm(x.numpy() - xr) <= 1e-7 * np.linalg.norm(xr)


def test_gmres_unpreconditioned_vs_reference(pf, b200, golden):
    row, col, val = b200.q1_assemble(2, 32, 1, None, 1e-3, (1.0, 0.5))
    b = golden["gmres2d32_b"]
    A = b200.CSR_lMatrix.from_csr(pf, row, col, val)
    gm = b200.GMRES(pf, 30)
    gm.SetupOperator(A)
    gm.InitControl(3000, 0.0, 1e-9, 1e6)
    x = pf.vector(len(b))
    assert gm.Solve(pf.vector(b), x) == b200.SUCCESS_REL
    ref_it = int(golden["gmres2d32_none_iters"][0])
    assert within5(gm.iter(), ref_it), (gm.iter(), ref_it)


def test_mpir_vs_oracle(pf, b200, oracle):
    dim, N = 3, 12
    rng = np.random.default_rng(5)
    kc = np.exp(rng.standard_normal(N ** dim))
    row, col, val = b200.q1_assemble(dim, N, 0, kc)
    b = b200.q1_rhs(9, dim, N)
    ref = oracle.mpir(row, col, val, b, outer=control(50, 0, 1e-10, 1e6), inner=control(10000, 0, 1e-4, 1e6))
    A = b200.CSR_lMatrix.from_csr(pf, row, col, val)
    m = b200.MPIR(pf, max_outer=50)
    m.SetupOperator(A)
    m.InitControl(50, 0.0, 1e-10, 1e6)
    m.InitInnerControl(10000, 0.0, 1e-4, 1e6)
    x = pf.vector(len(b))
    assert m.Solve(pf.vector(b), x) == b200.SUCCESS_REL
    assert m.result.res <= 1e-10 * m.result.res0
    assert abs(m.result.outer - ref["outer"]) <= 1
    assert within5(m.result.iters, ref["inner_total"]), (m.result.iters, ref["inner_total"])
    # error against the FP64 oracle solve
    xo = oracle.pcg(row, col, val, b, precond=oracle.invdiag(row, col, val), ctl=control(10000, 0, 1e-12, 1e6))["x"]
    assert np.linalg.norm(x.numpy() - xo) <= 1e-8 * np.linalg.norm(xo)


def test_stop_states(pf, b200):
    row, col, val = b200.q1_assemble(2, 16)
    A = b200.CSR_lMatrix.from_csr(pf, row, col, val)
    b = b200.q1_rhs(1, 2, 16)
    cg = b200.CG(pf)
    cg.SetupOperator(A)
    cg.InitControl(3, 0.0, 1e-12, 1e6)
    x = pf.vector(len(b))
    assert cg.Solve(pf.vector(b), x) == b200.FAIL_MAXITS
    assert cg.iter() == 3
    # zero right-hand side: the absolute test fires at step 0
    cg.InitControl(100, 1e-30, 1e-12, 1e6)
    x = pf.vector(len(b))
    assert cg.Solve(pf.vector(len(b)), x) == b200.SUCCESS_ABS
    assert cg.iter() == 0


def test_nan_rhs_runs_to_the_limit(pf, b200, oracle):
    """A NaN in the right-hand side: every comparison of IterateControl::Check
    (iterate_control.cc:84-110) is false, so CG and GMRES iterate to the
    limit and report FAIL_MAXITS, as the reference and the oracle do; MPIR's
    outer loop does not start and reports no success.  The context stays
    usable afterwards."""
    row, col, val = b200.q1_assemble(2, 16)
    A = b200.CSR_lMatrix.from_csr(pf, row, col, val)
    b = b200.q1_rhs(1, 2, 16)
    bn = b.copy()
    bn[37] = np.nan
    ref = oracle.pcg(row, col, val, bn, precond=oracle.invdiag(row, col, val), ctl=control(25, 0, 1e-10, 1e6))
    cg = b200.CG(pf)
    cg.SetupOperator(A)
    cg.SetupPreconditioner(b200.Preconditioner.Jacobi(pf, A))
    cg.InitControl(25, 0.0, 1e-10, 1e6)
    assert cg.Solve(pf.vector(bn), pf.vector(len(b))) == b200.FAIL_MAXITS == ref["status"]
    assert cg.iter() == 25 == ref["iters"]
    gm = b200.GMRES(pf, 10)
    gm.SetupOperator(A)
    gm.InitControl(40, 0.0, 1e-10, 1e6)
    assert gm.Solve(pf.vector(bn), pf.vector(len(b))) == b200.FAIL_MAXITS
    m = b200.MPIR(pf, max_outer=5)
    m.SetupOperator(A)
    m.InitControl(5, 0.0, 1e-10, 1e6)
    m.InitInnerControl(50, 0.0, 1e-4, 1e6)
    assert m.Solve(pf.vector(bn), pf.vector(len(b))) not in (b200.SUCCESS_ABS, b200.SUCCESS_REL)
    # the same context then solves a clean system
    x = pf.vector(len(b))
    cg.InitControl(1000, 0.0, 1e-10, 1e6)
    assert cg.Solve(pf.vector(b), x) == b200.SUCCESS_REL
    assert np.all(np.isfinite(x.numpy()))


def test_precond_dtype_mismatch_rejected(pf, b200):
    row, col, val = b200.q1_assemble(2, 8)
    A = b200.CSR_lMatrix.from_csr(pf, row, col, val)
    A32 = A.CastFrom(b200.F32)
    P = b200.Preconditioner.Jacobi(pf, A)
    cg = b200.CG(pf)
    cg.SetupOperator(A32)
    cg.SetupPreconditioner(P)
    with pytest.raises(b200.B200Error) as e:
        cg.Solve(pf.vector(len(row) - 1, b200.F32), pf.vector(len(row) - 1, b200.F32))
    assert e.value.code == 1


def test_full_size_spmv_128cubed(pf, b200, oracle):
    """The 3-D 128^3 operator: GPU SpMV against the oracle's at full size."""
    row, col, val = b200.q1_assemble(3, 128)
    n = len(row) - 1
    x = np.random.default_rng(7).uniform(-1, 1, n)
    y_ref = oracle.spmv(row, col, val, x)
    A = b200.CSR_lMatrix.from_csr(pf, row, col, val)
    yv = pf.vector(n)
    A.VectorMult(pf.vector(x), yv)
    sc = np.add.reduceat(np.abs(val) * np.abs(x[col]), row[:-1])
    assert np.all(np.abs(yv.numpy() - y_ref) <= 1e-13 * sc)


def test_full_size_cg_property(pf, b200, oracle):
    """3-D 64^3 Jacobi-CG to 1e-10: the true residual, recomputed by the
    oracle's SpMV, meets the tolerance."""
    row, col, val = b200.q1_assemble(3, 64)
    b = b200.q1_rhs(42, 3, 64)
    A = b200.CSR_lMatrix.from_csr(pf, row, col, val)
    cg = b200.CG(pf)
    cg.SetupOperator(A)
    cg.SetupPreconditioner(b200.Preconditioner.Jacobi(pf, A))
    cg.InitControl(20000, 0.0, 1e-10, 1e6)
    x = pf.vector(len(b))
    assert cg.Solve(pf.vector(b), x) == b200.SUCCESS_REL
    r = b - oracle.spmv(row, col, val, x.numpy())
    assert np.linalg.norm(r) <= 2e-10 * np.linalg.norm(b)


def test_mpir_gmres_ilu_mixed_convdiff(pf, b200):
    """Mixed form of the nonsymmetric configuration: FP32 ILU(0) factors and
    Arnoldi inside FP64 defect correction reach the FP64 stop on the true
    residual and agree with the FP64 GMRES solution."""
    row, col, val = b200.q1_assemble(2, 64, 1, None, 1e-3, (1.0, 0.5))
    bh = b200.q1_rhs(7, 2, 64)
    P64 = b200.Preconditioner.ILU0(pf, row, col, val, b200.PRECOND_ILU0_LS)
    P32 = b200.Preconditioner.ILU0(pf, row, col, val, b200.PRECOND_ILU0_LS, dtype=b200.F32)
    assert np.array_equal(P64.perm, P32.perm)
    bp = bh[P64.perm]
    gm = b200.GMRES(pf, 30)
    gm.SetupOperator(P64.A_perm)
    gm.SetupPreconditioner(P64)
    gm.InitControl(5000, 0.0, 1e-9, 1e6)
    x64 = pf.vector(len(bp))
    assert gm.Solve(pf.vector(bp), x64) == b200.SUCCESS_REL
    m = b200.MPIR(pf, max_outer=30)
    m.SetupOperator(P64.A_perm)
    m.SetupLowPrecisionOperator(P32.A_perm)
    m.SetupInnerGMRES(30, P32)
    m.InitControl(30, 0.0, 1e-9, 1e6)
    m.InitInnerControl(5000, 0.0, 1e-4, 1e6)
    x = pf.vector(len(bp))
    bv = pf.vector(bp)
    assert m.Solve(bv, x) == b200.SUCCESS_REL
    assert m.result.outer >= 2 and m.result.res <= 1e-9 * m.result.res0
    r = pf.vector(len(bp))
    true = np.sqrt(P64.A_perm.Residual(bv, x, r))
    assert true <= 1.0001e-9 * np.linalg.norm(bp)
    xs, xr = x.numpy(), x64.numpy()
    assert np.linalg.norm(xs - xr) <= 1e-6 * np.linalg.norm(xr)


@pytest.mark.parametrize("dim,N,kind", [(2, 160, 1), (3, 26, 0)])
def test_ilu0_level_sweep_beyond_ring(pf, b200, dim, N, kind, monkeypatch):
    """The single-CTA level sweep on operators larger than its shared-memory
    ring (columns read from the ring and from L2) equals the ticketed
    sync-free sweep (and the preconditioned residual test of GMRES)."""
    row, col, val = b200.q1_assemble(dim, N, kind, None, 1e-2, (1.0, 0.5, 0.25))
    n = len(row) - 1
    assert n > 8192
    r = np.random.default_rng(3).uniform(-1, 1, n)
    out = {}
    for sweep in ("tickets", "cta", "staged"):
        monkeypatch.setenv("B200LA_SYNCFREE", "1")
        monkeypatch.setenv("B200LA_SWEEP", sweep)
        P = b200.Preconditioner.ILU0(pf, row, col, val, b200.PRECOND_ILU0_LS)
        z = pf.vector(n)
        for _ in range(2):
            P.ApplyPreconditioner(pf.vector(r[P.perm]), z)
        out[sweep] = z.numpy()
    for sweep in ("cta", "staged"):
        assert np.max(np.abs(out[sweep] - out["tickets"])) <= 1e-11 * np.max(np.abs(out["tickets"]))



@pytest.mark.parametrize("precond", ["none", "jacobi", "mcsgs"])
def test_device_loop_matches_host_batches(pf, b200, monkeypatch, precond):
    """The CG iterations run in a device-side while loop (one graph launch per
    solve; the update kernel sets the loop condition after its Check).  The
    arithmetic is the same as with the host reading the stop state between
    batches, so iterations, residuals and solutions are bitwise equal, also
    for maxits stops and for stops inside a batch."""
    row, col, val = b200.q1_assemble(3, 14)
    b = b200.q1_rhs(5, 3, 14)
    out = {}
    for loop in ("1", "0"):
        monkeypatch.setenv("B200LA_GRAPH_LOOP", loop)
        if precond == "mcsgs":
            P = b200.Preconditioner.MultiColoringSGS(pf, row, col, val)
            A, bb = P.A_perm, b[P.perm]
        else:
            A = b200.CSR_lMatrix.from_csr(pf, row, col, val)
            P = b200.Preconditioner.Jacobi(pf, A) if precond == "jacobi" else None
            bb = b
        res = []
        for maxits, tol in ((100000, 1e-10), (7, 1e-10), (100000, 1e-3)):
            cg = b200.CG(pf)
            cg.SetupOperator(A)
            cg.SetupPreconditioner(P)
            cg.InitControl(maxits, 0.0, tol, 1e6)
            x = pf.vector(len(bb))
            st = cg.Solve(pf.vector(bb), x)
            res.append((st, cg.iter(), cg.result.res, x.numpy()))
        out[loop] = res
    monkeypatch.delenv("B200LA_GRAPH_LOOP")
    for a, c in zip(out["1"], out["0"]):
        assert a[:3] == c[:3]
        assert np.array_equal(a[3], c[3])
    assert out["1"][1][0] == b200.FAIL_MAXITS and out["1"][1][1] == 7


def test_mpir_jacobi_scaling_follows_value_changes(pf, b200):
    """The defect correction keeps the FP32 Jacobi scaling of its FP64
    operator between solves; scaling the operator drops it, so the next
    solve matches one on a freshly built operator bit for bit."""
    row, col, val = b200.q1_assemble(3, 12)
    b = b200.q1_rhs(9, 3, 12)
    n = len(b)
    A = b200.CSR_lMatrix.from_csr(pf, row, col, val)
    mp = b200.MPIR(pf)
    mp.SetupOperator(A)
    mp.InitControl(50, 0.0, 1e-10, 1e6)
    x1 = pf.vector(n)
    assert mp.Solve(pf.vector(b), x1) == b200.SUCCESS_REL
    x1b = pf.vector(n)
    mp.Solve(pf.vector(b), x1b)
    assert np.array_equal(x1.numpy(), x1b.numpy())      # the cached scaling gives the same solve
    A.Scale(3.0)
    x2 = pf.vector(n)
    mp.Solve(pf.vector(b), x2)
    B = b200.CSR_lMatrix.from_csr(pf, row, col, 3.0 * val)
    mq = b200.MPIR(pf)
    mq.SetupOperator(B)
    mq.InitControl(50, 0.0, 1e-10, 1e6)
    x3 = pf.vector(n)
    mq.Solve(pf.vector(b), x3)
    assert np.array_equal(x2.numpy(), x3.numpy())
    assert mp.result.iters == mq.result.iters
