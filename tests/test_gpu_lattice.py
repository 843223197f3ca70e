"""GPU parity of the lattice layout of multicolour preconditioners.

On a parity-coloured structured Q1 grid the multicolour preconditioners keep
their two sweep parts and the coloured operator in an index-free lattice
layout (values by neighbour slot).  These tests build the same preconditioner
with the layout and without it (B200LA_LATTICE=0: CSR sweeps), and check the
applies and SpMVs against each other, against the oracle and against the
reference's goldens, the PCG iteration counts, the FP32 path, value updates
of the coloured operator, and that non-grid operators keep the CSR path.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pf(b200):
    return b200.Platform(0)


def build(b200, pf, row, col, val, lattice, monkeypatch, kind="sgs", dtype=None):
    monkeypatch.setenv("B200LA_LATTICE", "1" if lattice else "0")
    dt = b200.F64 if dtype is None else dtype
    if kind == "sgs":
        P = b200.Preconditioner.MultiColoringSGS(pf, row, col, val, dtype=dt)
    else:
        P = b200.Preconditioner.ILU0(pf, row, col, val, b200.PRECOND_ILU0_MC, dtype=dt)
    monkeypatch.delenv("B200LA_LATTICE")
    return P


@pytest.mark.parametrize("dim,N,field", [(2, 33, False), (3, 12, False), (3, 17, True), (2, 40, True)])
def test_lattice_apply_and_spmv_match_csr(pf, b200, oracle, monkeypatch, dim, N, field):
    kc = None
    if field:
        ncell = N ** dim
        kc = np.exp(np.random.default_rng(N).normal(0.0, 1.0, ncell))
    row, col, val = b200.q1_assemble(dim, N, 0, kc)
    n = len(row) - 1
    Pl = build(b200, pf, row, col, val, True, monkeypatch)
    Pc = build(b200, pf, row, col, val, False, monkeypatch)
    assert Pl.A_perm.info()["storage"] == "lattice"
    assert Pc.A_perm.info()["storage"] != "lattice"
    assert np.array_equal(Pl.perm, Pc.perm)
    rng = np.random.default_rng(7)
    r = rng.uniform(-1, 1, n)
    zl, zc = pf.vector(n), pf.vector(n)
    for _ in range(2):   # the second apply reuses the layout unchanged
        Pl.ApplyPreconditioner(pf.vector(r), zl)
    Pc.ApplyPreconditioner(pf.vector(r), zc)
    a, c = zl.numpy(), zc.numpy()
    assert np.max(np.abs(a - c)) <= 1e-13 * np.max(np.abs(c))
    # against the oracle's MC-SGS (lpreconditioner_mc_sgs.cc restated)
    Po, (Ar, Ac, Av) = oracle.mcsgs_build(row, col, val)
    assert np.array_equal(Po.perm, Pl.perm)
    zo = Po.apply(r)
    assert np.max(np.abs(a - zo)) <= 1e-12 * np.max(np.abs(zo))
    # the coloured operator's SpMV on the lattice layout
    x = rng.uniform(-1, 1, n)
    yl, yc = pf.vector(n), pf.vector(n)
    Pl.A_perm.VectorMult(pf.vector(x), yl)
    Pc.A_perm.VectorMult(pf.vector(x), yc)
    yo = oracle.spmv(Ar, Ac, Av, x)
    scale = oracle.spmv(Ar, Ac, np.abs(Av), np.abs(x))
    assert np.max(np.abs(yl.numpy() - yo) / np.maximum(scale, 1e-300)) <= 1e-13
    assert np.max(np.abs(yl.numpy() - yc.numpy()) / np.maximum(scale, 1e-300)) <= 1e-13


def test_lattice_apply_matches_golden(pf, b200, golden, monkeypatch):
    for dim, N in [(2, 8), (3, 7)]:
        key = f"{dim}d{N}_p"
        row, col, val = golden[key + "_row"], golden[key + "_col"], golden[key + "_val"]
        P = build(b200, pf, row, col, val, True, monkeypatch)
        assert P.A_perm.info()["storage"] == "lattice"
        assert np.array_equal(P.perm, golden[key + "_mcsgs_perm"])
        r = golden[key + "_x"]
        z = pf.vector(len(r))
        P.ApplyPreconditioner(pf.vector(r), z)
        zr = golden[key + "_mcsgs_z"]
        assert np.max(np.abs(z.numpy() - zr)) <= 1e-12 * np.max(np.abs(zr))


@pytest.mark.parametrize("dim,N", [(2, 32), (3, 12)])
def test_lattice_pcg_vs_reference(pf, b200, golden, monkeypatch, dim, N):
    key = f"solve{dim}d{N}"
    row, col, val = b200.q1_assemble(dim, N)
    P = build(b200, pf, row, col, val, True, monkeypatch)
    assert P.A_perm.info()["storage"] == "lattice"
    b = golden[key + "_b"][P.perm]
    cg = b200.CG(pf)
    cg.SetupOperator(P.A_perm)
    cg.SetupPreconditioner(P)
    cg.InitControl(5000, 0.0, 1e-8, 1e6)
    x = pf.vector(len(b))
    assert cg.Solve(pf.vector(b), x) == b200.SUCCESS_REL
    ref_it = int(golden[f"{key}_mcsgs_iters"][0])
    assert abs(cg.iter() - ref_it) <= max(1, int(np.ceil(0.05 * ref_it))), (cg.iter(), ref_it)
    xr = golden[f"{key}_mcsgs_x"]
    assert np.linalg.norm(x.numpy() - xr) <= 1e-7 * np.linalg.norm(xr)


def test_lattice_fp32(pf, b200, monkeypatch):
    row, col, val = b200.q1_assemble(3, 14)
    n = len(row) - 1
    Pl = build(b200, pf, row, col, val, True, monkeypatch, dtype=b200.F32)
    Pc = build(b200, pf, row, col, val, False, monkeypatch, dtype=b200.F32)
    assert Pl.A_perm.info()["storage"] == "lattice"
    r = np.random.default_rng(3).uniform(-1, 1, n)
    zl, zc = pf.vector(n, b200.F32), pf.vector(n, b200.F32)
    Pl.ApplyPreconditioner(pf.vector(r, b200.F32), zl)
    Pc.ApplyPreconditioner(pf.vector(r, b200.F32), zc)
    a, c = zl.numpy().astype(np.float64), zc.numpy().astype(np.float64)
    assert np.max(np.abs(a - c)) <= 1e-5 * np.max(np.abs(c))


def test_lattice_ilu0_mc(pf, b200, monkeypatch):
    """ILU(0) in multicolour order has the operator's pattern, so its factors
    take the lattice layout too."""
    row, col, val = b200.q1_assemble(3, 10)
    n = len(row) - 1
    Pl = build(b200, pf, row, col, val, True, monkeypatch, kind="ilu")
    Pc = build(b200, pf, row, col, val, False, monkeypatch, kind="ilu")
    assert Pl.A_perm.info()["storage"] == "lattice"
    r = np.random.default_rng(5).uniform(-1, 1, n)
    zl, zc = pf.vector(n), pf.vector(n)
    Pl.ApplyPreconditioner(pf.vector(r), zl)
    Pc.ApplyPreconditioner(pf.vector(r), zc)
    assert np.max(np.abs(zl.numpy() - zc.numpy())) <= 1e-12 * np.max(np.abs(zc.numpy()))


def test_lattice_follows_value_updates(pf, b200, oracle, monkeypatch):
    row, col, val = b200.q1_assemble(3, 9)
    n = len(row) - 1
    P = build(b200, pf, row, col, val, True, monkeypatch)
    A = P.A_perm
    assert A.info()["storage"] == "lattice"
    Ar, Ac, Av = A.download()
    x = np.random.default_rng(9).uniform(-1, 1, n)
    y = pf.vector(n)
    A.Scale(2.5)
    A.VectorMult(pf.vector(x), y)
    yo = oracle.spmv(Ar, Ac, Av * 2.5, x)
    assert np.max(np.abs(y.numpy() - yo)) <= 1e-13 * np.max(np.abs(yo))
    newv = np.random.default_rng(2).uniform(-1, 1, len(Av))
    pf.check(b200.lib().b200la_csr_set_values(pf.h, A.h, newv.ctypes.data), "csr_set_values")
    A.VectorMult(pf.vector(x), y)
    yo = oracle.spmv(Ar, Ac, newv, x)
    assert np.max(np.abs(y.numpy() - yo)) <= 1e-13 * np.max(np.abs(yo))


def test_non_grid_operator_keeps_csr(pf, b200, golden, monkeypatch):
    """A convection-diffusion operator in the multicolour ILU(0) is a Q1 grid
    too; an operator whose row 0 is not a grid corner is not."""
    key = "2d17_cd"
    row, col, val = golden[key + "_row"], golden[key + "_col"], golden[key + "_val"]
    # permute the rows and columns at random: no longer lexicographic
    n = len(row) - 1
    import scipy.sparse as sp
    M = sp.csr_matrix((val, col, row), shape=(n, n))
    q = np.random.default_rng(1).permutation(n)
    Mq = M[q][:, q].tocsr()
    Mq.sort_indices()
    P = build(b200, pf, Mq.indptr, Mq.indices, Mq.data, True, monkeypatch)
    assert P.A_perm.info()["storage"] != "lattice"


@pytest.mark.parametrize("kind", ["sgs", "ilu"])
def test_last_colour_fused_step_is_bitwise(pf, b200, monkeypatch, kind):
    """The last colour's backward step (no couplings) runs in the epilogue of
    its forward step: the same roundings as the two separate launches."""
    row, col, val = b200.q1_assemble(3, 13, 0, np.exp(np.random.default_rng(4).normal(0.0, 1.0, 13 ** 3)))
    n = len(row) - 1
    P = build(b200, pf, row, col, val, True, monkeypatch, kind=kind)
    r = np.random.default_rng(8).uniform(-1, 1, n)
    out = []
    for flag in (None, "1"):
        if flag:
            monkeypatch.setenv("B200LA_NOFUSE_LAST", flag)
        z = pf.vector(n)
        P.ApplyPreconditioner(pf.vector(r), z)
        out.append(z.numpy())
    monkeypatch.delenv("B200LA_NOFUSE_LAST")
    assert np.array_equal(out[0].view(np.uint64), out[1].view(np.uint64))


def test_programmatic_launch_sweeps_are_bitwise(pf, b200, monkeypatch):
    """Colour sweeps after the first launch as programmatic dependents (their
    value loads overlap the previous colour; the gathers wait for it): the
    same bits as plain stream order, in a single apply and inside PCG."""
    row, col, val = b200.q1_assemble(3, 16)
    b = b200.q1_rhs(3, 3, 16)
    n = len(row) - 1
    P = build(b200, pf, row, col, val, True, monkeypatch)
    r = np.random.default_rng(6).uniform(-1, 1, n)
    out, keep = [], []
    for flag in ("1", "0"):
        monkeypatch.setenv("B200LA_PDL", flag)
        z = pf.vector(n)
        P.ApplyPreconditioner(pf.vector(r), z)
        cg = b200.CG(pf)
        cg.SetupOperator(P.A_perm)
        cg.SetupPreconditioner(P)
        cg.InitControl(1000, 0.0, 1e-8, 1e6)
        # b and x stay alive: new addresses, so the solver captures a new graph
        x, bv = pf.vector(n), pf.vector(b[P.perm])
        keep += [x, bv]
        assert cg.Solve(bv, x) == b200.SUCCESS_REL
        out.append((z.numpy(), cg.iter(), x.numpy()))
    monkeypatch.delenv("B200LA_PDL")
    assert np.array_equal(out[0][0], out[1][0]) and out[0][1] == out[1][1]
    assert np.array_equal(out[0][2], out[1][2])


def test_temporary_inputs_are_stream_ordered(pf, b200, monkeypatch):
    """A temporary input vector (freed as soon as the call returns, while the
    platform's kernels still read it) is reused by the next allocations only
    in the platform stream's order: applies with a temporary r followed at
    once by new zeroed vectors give the result of a synchronised apply."""
    row, col, val = b200.q1_assemble(3, 40)
    n = len(row) - 1
    P = build(b200, pf, row, col, val, True, monkeypatch)
    r = np.random.default_rng(2).uniform(-1, 1, n)
    rv = pf.vector(r)
    z0 = pf.vector(n)
    P.ApplyPreconditioner(rv, z0)
    ref = z0.numpy()
    for _ in range(8):
        z = pf.vector(n)
        P.ApplyPreconditioner(pf.vector(r), z)
        junk = [pf.vector(n) for _ in range(3)]   # noqa: F841  (allocations right behind the call)
        assert z.numpy().tobytes() == ref.tobytes()
