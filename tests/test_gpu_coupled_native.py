"""The native coupled layer (b200la_comm_* / b200la_coupled_*) on one GPU.

Ranks are host threads with their own contexts on one GPU, joined by a local
communicator (event-ordered device copies, a host barrier): the coupled
product, ghost update, dot and CG are checked against the global ones.  The
NCCL communicator is exercised with one rank (the only NCCL configuration one
GPU allows): every NCCL call of the data path runs, with no peers.
"""
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run_ranks(world, fn):
    out, errs = [None] * world, []

    def body(r):
        try:
            out[r] = fn(r)
        except BaseException as e:   # surfaced below
            errs.append(e)

    th = [threading.Thread(target=body, args=(r,)) for r in range(world)]
    for t in th:
        t.start()
    for t in th:
        t.join(timeout=300)
    if errs:
        raise errs[0]
    return out


def _system(b200, N=40):
    kc = np.exp(np.random.default_rng(1).standard_normal(N * N))
    row, col, val = b200.q1_assemble(2, N, 0, kc)
    return row, col, val, b200.q1_rhs(4, 2, N)


def _global_cg(b200, row, col, val, b, jacobi):
    pf0 = b200.Platform(0)
    A = b200.CSR_lMatrix.from_csr(pf0, row, col, val)
    cg = b200.CG(pf0)
    cg.SetupOperator(A)
    if jacobi:
        cg.SetupPreconditioner(b200.Preconditioner.Jacobi(pf0, A))
    cg.InitControl(5000, 0.0, 1e-10, 1e6)
    x0 = pf0.vector(len(b))
    assert cg.Solve(pf0.vector(b), x0) == b200.SUCCESS_REL
    return cg.iter(), x0.numpy()


def _spmv_np(row, col, val, x):
    import scipy.sparse as sp
    n = len(row) - 1
    return sp.csr_matrix((val, col, row), shape=(n, n)) @ x


@pytest.mark.parametrize("world", [1, 2, 3])
def test_native_coupled_local_ranks(b200, world):
    import importlib
    cp = importlib.import_module("hiflow3_b200.coupled")
    row, col, val, b = _system(b200)
    n = len(row) - 1
    its = {j: _global_cg(b200, row, col, val, b, j) for j in (False, True)}
    part = cp.RowPartition.even(n, world)
    trs = cp.LocalTransport.group(world)
    comms = cp.Comm.local_group(world)
    xv = np.sin(np.arange(n) * 0.11)

    def rank_fn(r):
        pf = b200.Platform(0)
        r0, r1 = part.range(r)
        lr = row[r0:r1 + 1] - row[r0]
        M = cp.NativeCoupledMatrix(pf, comms[r], trs[r], part, r, lr, col[row[r0]:row[r1]], val[row[r0]:row[r1]])
        xc, yc = M.vector(xv[r0:r1]), M.vector()
        for _ in range(3):   # back to back: the exchange buffers are reused
            M.VectorMult(xc, yc)
        y_rows = yc.numpy()
        ghosts = M.UpdateGhost(xc)
        dot = M.Dot(xc, xc)
        sols = {}
        for jac in (False, True):
            x = M.vector()
            st = M.CG(M.vector(b[r0:r1]), x, precond="jacobi" if jac else None, maxits=5000, reltol=1e-10)
            sols[jac] = (st, M.iter, x.numpy())
        gg = M.couplings.ghost_global.copy()
        M.close()
        return r0, y_rows, ghosts, gg, dot, sols

    res = _run_ranks(world, rank_fn)
    y_global = _spmv_np(row, col, val, xv)
    for r0, y_rows, ghosts, gg, dot, sols in res:
        assert np.allclose(y_rows, y_global[r0:r0 + len(y_rows)], rtol=0, atol=1e-12 * np.abs(y_global).max())
        assert np.array_equal(ghosts, xv[gg])
        assert abs(dot - xv @ xv) <= 1e-12 * (xv @ xv)
        for jac in (False, True):
            st, it, x = sols[jac]
            it0, xs = its[jac]
            assert st == b200.SUCCESS_REL
            assert abs(it - it0) <= max(1, 0.05 * it0), (jac, it, it0)
            assert np.linalg.norm(x - xs[r0:r0 + len(x)]) <= 1e-8 * np.linalg.norm(xs)
    # every rank took the same decisions
    assert len({tuple((s[0], s[1]) for s in r[5].values()) for r in res}) == 1
    for c in comms:
        c.close()


def test_native_coupled_nccl_single_rank(b200):
    import importlib
    cp = importlib.import_module("hiflow3_b200.coupled")
    row, col, val, b = _system(b200, 32)
    n = len(row) - 1
    it0, xs = _global_cg(b200, row, col, val, b, True)
    pf = b200.Platform(0)
    uid = cp.Comm.unique_id()
    assert len(uid) == cp.COMM_ID_BYTES
    comm = cp.Comm.nccl(pf, uid, 0, 1)
    assert (comm.rank, comm.size) == (0, 1)
    part = cp.RowPartition.even(n, 1)
    tr = cp.LocalTransport.group(1)[0]
    M = cp.NativeCoupledMatrix(pf, comm, tr, part, 0, row, col, val)
    xv = np.cos(np.arange(n) * 0.3)
    y = M.vector()
    M.VectorMult(M.vector(xv), y)
    yg = _spmv_np(row, col, val, xv)
    assert np.allclose(y.numpy(), yg, rtol=0, atol=1e-12 * np.abs(yg).max())
    assert abs(M.Dot(M.vector(xv), M.vector(xv)) - xv @ xv) <= 1e-12 * (xv @ xv)
    x = M.vector()
    assert M.CG(M.vector(b), x, precond="jacobi", reltol=1e-10) == b200.SUCCESS_REL
    assert abs(M.iter - it0) <= max(1, 0.05 * it0)
    assert np.linalg.norm(x.numpy() - xs) <= 1e-8 * np.linalg.norm(xs)
    M.close()
    comm.close()


def test_native_coupled_rejects_bad_couplings(b200):
    import ctypes as C
    import importlib
    cp = importlib.import_module("hiflow3_b200.coupled")
    pf = b200.Platform(0)
    row, col, val, _ = _system(b200, 8)
    A = b200.CSR_lMatrix.from_csr(pf, row, col, val)
    comms = cp.Comm.local_group(2)
    h = C.c_void_p()
    go = np.array([0, 0, 0], np.int32)
    bo = np.array([0, 1, 1], np.int32)   # a border towards this rank itself
    bi = np.array([0], np.int32)
    rc = b200.lib().b200la_coupled_create(pf.h, comms[0].h, A.h, None, go.ctypes.data, bo.ctypes.data,
                                          bi.ctypes.data, C.byref(h))
    assert rc == b200.ERR_ARG
    bo = np.array([0, 0, 1], np.int32)
    bi = np.array([len(row) - 1], np.int32)   # outside the owned rows
    rc = b200.lib().b200la_coupled_create(pf.h, comms[0].h, A.h, None, go.ctypes.data, bo.ctypes.data,
                                          bi.ctypes.data, C.byref(h))
    assert rc == b200.ERR_ARG
    for c in comms:
        c.close()


@pytest.mark.parametrize("world", [1, 2, 3])
def test_native_coupled_cg_mcsgs_blocks(b200, world):
    """Block-Jacobi with the multicoloured SGS of every rank's diagonal block
    (r gathered into the block's colour order, the sweeps, z scattered back):
    on one rank the single-system MC-SGS PCG's iterations; on two and three
    ranks fewer iterations than Jacobi blocks, the solution, and the same
    decisions on every rank."""
    import importlib
    cp = importlib.import_module("hiflow3_b200.coupled")
    N = 24
    row, col, val = b200.q1_assemble(3, N)
    b = b200.q1_rhs(8, 3, N)
    n = len(row) - 1
    pf0 = b200.Platform(0)
    P = b200.Preconditioner.MultiColoringSGS(pf0, row, col, val)
    cg = b200.CG(pf0)
    cg.SetupOperator(P.A_perm)
    cg.SetupPreconditioner(P)
    cg.InitControl(5000, 0.0, 1e-10, 1e6)
    xp = pf0.vector(n)
    assert cg.Solve(pf0.vector(b[P.perm]), xp) == b200.SUCCESS_REL
    it0 = cg.iter()
    xs = np.empty(n)
    xs[P.perm] = xp.numpy()
    part = cp.RowPartition.even(n, world)
    trs = cp.LocalTransport.group(world)
    comms = cp.Comm.local_group(world)

    def rank_fn(r):
        pf = b200.Platform(0)
        r0, r1 = part.range(r)
        lr = row[r0:r1 + 1] - row[r0]
        M = cp.NativeCoupledMatrix(pf, comms[r], trs[r], part, r, lr, col[row[r0]:row[r1]], val[row[r0]:row[r1]])
        x = M.vector()
        st = M.CG(M.vector(b[r0:r1]), x, precond="mcsgs", maxits=5000, reltol=1e-10)
        out = (r0, st, M.iter, x.numpy())    # before the Jacobi solve overwrites M.iter
        xj = M.vector()
        M.CG(M.vector(b[r0:r1]), xj, precond="jacobi", maxits=5000, reltol=1e-10)
        itj = M.iter
        M.close()
        return out + (itj,)

    res = _run_ranks(world, rank_fn)
    assert len({(st, it) for _, st, it, _, _ in res}) == 1
    for r0, st, it, x, itj in res:
        assert st == b200.SUCCESS_REL
        if world == 1:
            assert abs(it - it0) <= max(1, 0.05 * it0), (it, it0)
        assert it < itj
        assert np.linalg.norm(x - xs[r0:r0 + len(x)]) <= 1e-7 * np.linalg.norm(xs)
    for c in comms:
        c.close()
