"""Row-block distributed objects (hiflow3_2.0_b200/coupled.py).

CPU (gloo, world sizes 2 and 3, spawned processes): the host logic of the
multi-GPU layer -- the row-block split, the couplings set-up (which values
every peer needs) and the peer exchange over torch.distributed -- checked
with host tensors and a numpy product of the local blocks against the global
product.  GPU: the device objects (gather kernel, block SpMVs, coupled CG)
with several ranks as threads sharing one GPU (LocalTransport), against the
single-rank solve.
"""
import os
import sys
import threading

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))


def _spmv_np(row, col, val, x):
    y = np.zeros(len(row) - 1)
    for i in range(len(row) - 1):
        y[i] = val[row[i]:row[i + 1]] @ x[col[row[i]:row[i + 1]]]
    return y


def _system():
    from conftest import load_platform
    b200 = load_platform()
    row, col, val = b200.q1_assemble(2, 9, 1, None, 1e-2, (1.0, 0.5))
    return b200, row, col, val


def _gloo_worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import importlib
        b200, row, col, val = _system()
        cp = importlib.import_module("hiflow3_b200.coupled")
        n = len(row) - 1
        part = cp.RowPartition.even(n, world)
        r0, r1 = part.range(rank)
        lr = row[r0:r1 + 1] - row[r0]
        lc, lv = col[row[r0]:row[r1]], val[row[r0]:row[r1]]
        (rd, cd, vd), (ro, co, vo), ghosts = b200.rowblock_split(lr, lc, lv, n, r0, r1)
        tr = cp.DistTransport()
        cpl = cp.LaCouplings(part, rank, ghosts).setup(tr)
        x = np.cos(np.arange(n) * 0.37)              # the global x, each rank keeps its own part
        xi = torch.from_numpy(x[r0:r1].copy())
        border = xi[torch.from_numpy(cpl.border_indices.astype(np.int64))]
        ghost = torch.zeros(len(ghosts), dtype=torch.float64)
        cp.exchange(tr, cpl, border, ghost)
        y = _spmv_np(rd, cd, vd, x[r0:r1]) + (_spmv_np(ro, co, vo, ghost.numpy()) if len(co) else 0.0)
        dot = tr.allreduce_sum(float(xi @ xi), "cpu")
        q.put((rank, r0, y, ghost.numpy().copy(), ghosts.copy(), dot))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_rowblock_spmv_over_gloo(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 400 + world
    procs = [ctx.Process(target=_gloo_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = [q.get(timeout=180) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    b200, row, col, val = _system()
    n = len(row) - 1
    x = np.cos(np.arange(n) * 0.37)
    y_global = _spmv_np(row, col, val, x)
    for rank, r0, y, ghost, ghosts, dot in got:
        assert np.array_equal(ghost, x[ghosts])                       # every ghost holds the owner's value
        assert np.allclose(y, y_global[r0:r0 + len(y)], rtol=0, atol=1e-13 * np.abs(val).max())
        assert abs(dot - x @ x) <= 1e-12 * (x @ x)


def test_rowblock_split_blocks(b200):
    row, col, val = b200.q1_assemble(2, 6, 0)
    n = len(row) - 1
    r0, r1 = 10, 30
    lr = row[r0:r1 + 1] - row[r0]
    lc, lv = col[row[r0]:row[r1]], val[row[r0]:row[r1]]
    (rd, cd, vd), (ro, co, vo), g = b200.rowblock_split(lr, lc, lv, n, r0, r1)
    assert np.all(np.diff(g) > 0) and not np.any((g >= r0) & (g < r1))
    for i in range(r1 - r0):
        full = dict(zip(lc[lr[i]:lr[i + 1]], lv[lr[i]:lr[i + 1]]))
        got = {c + r0: v for c, v in zip(cd[rd[i]:rd[i + 1]], vd[rd[i]:rd[i + 1]])}
        got.update({g[c]: v for c, v in zip(co[ro[i]:ro[i + 1]], vo[ro[i]:ro[i + 1]])})
        assert got == full


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


@pytest.mark.gpu
@pytest.mark.parametrize("world,remote", [(2, False), (3, False), (2, True), (3, True)])
def test_coupled_cg_ranks_on_one_gpu(b200, world, remote):
    import importlib
    cp = importlib.import_module("hiflow3_b200.coupled")
    row, col, val = b200.q1_assemble(2, 40, 0, np.exp(np.random.default_rng(1).standard_normal(1600)))
    n = len(row) - 1
    b = b200.q1_rhs(4, 2, 40)
    # the single-rank Jacobi-PCG
    pf0 = b200.Platform(0)
    A = b200.CSR_lMatrix.from_csr(pf0, row, col, val)
    cg = b200.CG(pf0)
    cg.SetupOperator(A)
    cg.SetupPreconditioner(b200.Preconditioner.Jacobi(pf0, A))
    cg.InitControl(5000, 0.0, 1e-10, 1e6)
    x0 = pf0.vector(n)
    assert cg.Solve(pf0.vector(b), x0) == b200.SUCCESS_REL
    it0, xs = cg.iter(), x0.numpy()
    part = cp.RowPartition.even(n, world)
    trs = cp.LocalTransport.group(world)

    def rank_fn(r):
        pf = b200.Platform(0)
        r0, r1 = part.range(r)
        lr = row[r0:r1 + 1] - row[r0]
        M = cp.CoupledMatrix(pf, part, r, trs[r], lr, col[row[r0]:row[r1]], val[row[r0]:row[r1]], remote=remote)
        xv = np.sin(np.arange(n) * 0.11)
        # the coupled product equals the global one on this rank's rows
        xc, yc = M.vector(xv[r0:r1]), M.vector()
        M.VectorMult(xc, yc)
        y_rows = yc.numpy()
        solver = cp.CoupledCG(M)
        x = M.vector()
        st = solver.Solve(M.vector(b[r0:r1]), x, maxits=5000, reltol=1e-10)
        return r0, y_rows, st, solver.iter, x.numpy()

    res = _run_ranks(world, rank_fn)
    xv = np.sin(np.arange(n) * 0.11)
    y_global = _spmv_np(row, col, val, xv)
    for r0, y_rows, st, it, x in res:
        assert np.allclose(y_rows, y_global[r0:r0 + len(y_rows)], rtol=0, atol=1e-12 * np.abs(y_global).max())
        assert st == b200.SUCCESS_REL
        assert abs(it - it0) <= max(1, 0.05 * it0), (it, it0)
        assert np.linalg.norm(x - xs[r0:r0 + len(x)]) <= 1e-8 * np.linalg.norm(xs)


@pytest.mark.gpu
@pytest.mark.parametrize("remote", [False, True])
def test_coupled_products_back_to_back_without_host_waits(b200, remote):
    """Twelve coupled products in a row, each feeding the next (x <- 0.1 A x
    on the platform's stream), with no host synchronisation between them: the
    stream-ordered exchange must keep every ghost update behind the pack that
    produced it and ahead of the off-diagonal product that reads it, and no
    border may be repacked before its peers have copied it.  Remote mode: the
    off-diagonal product reads the owners' x directly, after their last write
    and before their next."""
    import importlib
    cp = importlib.import_module("hiflow3_b200.coupled")
    row, col, val = b200.q1_assemble(2, 48, 1, None, 1e-2, (1.0, 0.5))
    n = len(row) - 1
    world, steps = 3, 12
    part = cp.RowPartition.even(n, world)
    trs = cp.LocalTransport.group(world)
    x0 = np.cos(np.arange(n) * 0.23)

    def rank_fn(r):
        pf = b200.Platform(0)
        r0, r1 = part.range(r)
        M = cp.CoupledMatrix(pf, part, r, trs[r], row[r0:r1 + 1] - row[r0], col[row[r0]:row[r1]],
                             val[row[r0]:row[r1]], remote=remote)
        x, y = M.vector(x0[r0:r1]), M.vector()
        for _ in range(steps):
            M.VectorMult(x, y)
            x.CopyFrom(y)
            x.Scale(0.1)
        return r0, x.numpy()

    res = _run_ranks(world, rank_fn)
    xg = x0.copy()
    for _ in range(steps):
        xg = 0.1 * _spmv_np(row, col, val, xg)
    for r0, xr in res:
        assert np.allclose(xr, xg[r0:r0 + len(xr)], rtol=0, atol=1e-11 * np.abs(xg).max())


@pytest.mark.gpu
@pytest.mark.parametrize("world,n_global,w", [(2, 1, 1.0), (3, 2, 0.9)])
def test_coupled_async_jacobi_ranks_on_one_gpu(b200, world, n_global, w):
    """Asynchronous block-Jacobi across thread ranks with the ghost update
    between global iterations: every rank stops on the global residual (the
    same decision on all ranks) and the assembled solution solves the global
    system."""
    import importlib
    cp = importlib.import_module("hiflow3_b200.coupled")
    N = 14
    row, col, val = b200.q1_assemble(2, N, 0, np.exp(np.random.default_rng(7).standard_normal(N * N)))
    n = len(row) - 1
    b = b200.q1_rhs(11, 2, N)
    part = cp.RowPartition.even(n, world)
    trs = cp.LocalTransport.group(world)

    def rank_fn(r):
        pf = b200.Platform(0)
        r0, r1 = part.range(r)
        M = cp.CoupledMatrix(pf, part, r, trs[r], row[r0:r1 + 1] - row[r0], col[row[r0]:row[r1]],
                             val[row[r0]:row[r1]])
        s = cp.CoupledAsyncJacobi(M, n_global=n_global, n_block=4, n_inner=3, w=w)
        x = M.vector()
        st = s.Solve(M.vector(b[r0:r1]), x, maxits=400000, reltol=1e-8)
        return r0, st, s.iter, s.res, s.res0, x.numpy()

    res = _run_ranks(world, rank_fn)
    D = np.zeros((n, n))
    for i in range(n):
        D[i, col[row[i]:row[i + 1]]] += val[row[i]:row[i + 1]]
    xe = np.linalg.solve(D, b)
    x = np.zeros(n)
    for r0, st, it, rn, r0n, xr in res:
        assert st == b200.SUCCESS_REL
        assert it % (n_global * 12) == 0
        assert rn < 1e-8 * r0n
        x[r0:r0 + len(xr)] = xr
    assert len({(st, it) for _, st, it, _, _, _ in res}) == 1
    assert np.linalg.norm(b - D @ x) <= 1e-8 * res[0][4] * 1.0001
    assert np.linalg.norm(x - xe) <= 1e-4 * np.linalg.norm(xe)


@pytest.mark.gpu
def test_enable_peer_access_paths(b200):
    """b200la_enable_peer_access: the same device needs nothing; a device that
    does not exist (or has no peer path) is refused with B200LA_ERR_DEVICE,
    and the calling thread keeps its current device."""
    import torch
    lib = b200.lib()
    assert lib.b200la_enable_peer_access(0, 0) == 0
    missing = torch.cuda.device_count() + 3
    assert lib.b200la_enable_peer_access(0, missing) == 4
    assert torch.cuda.current_device() == 0


@pytest.mark.gpu
@pytest.mark.parametrize("world", [1, 2, 3])
def test_coupled_cg_mcsgs_block_jacobi(b200, world):
    """Coupled CG with the multicoloured SGS of each rank's block (block-Jacobi
    across ranks, as PreconditionerMultiColoring on op.diagonal()).  One rank:
    the same iterations (within 5%) as the single-system MC-SGS PCG on the
    permuted operator.  Every world size: the global solution within 1e-8, and
    fewer iterations than the coupled Jacobi-PCG."""
    import importlib
    cp = importlib.import_module("hiflow3_b200.coupled")
    N = 12
    row, col, val = b200.q1_assemble(3, N, 0, np.exp(np.random.default_rng(2).standard_normal(N ** 3)))
    n = len(row) - 1
    b = b200.q1_rhs(6, 3, N)
    D = np.zeros((n, n))
    for i in range(n):
        D[i, col[row[i]:row[i + 1]]] += val[row[i]:row[i + 1]]
    xe = np.linalg.solve(D, b)
    pf0 = b200.Platform(0)
    P0 = b200.Preconditioner.MultiColoringSGS(pf0, row, col, val)
    cg = b200.CG(pf0)
    cg.SetupOperator(P0.A_perm)
    cg.SetupPreconditioner(P0)
    cg.InitControl(5000, 0.0, 1e-10, 1e6)
    assert cg.Solve(pf0.vector(b[P0.perm]), pf0.vector(n)) == b200.SUCCESS_REL
    it_single = cg.iter()
    part = cp.RowPartition.even(n, world)
    trs = cp.LocalTransport.group(world)

    def rank_fn(r):
        pf = b200.Platform(0)
        r0, r1 = part.range(r)
        M = cp.CoupledMatrix(pf, part, r, trs[r], row[r0:r1 + 1] - row[r0], col[row[r0]:row[r1]],
                             val[row[r0]:row[r1]])
        out = []
        for kind in ("mcsgs", "jacobi"):
            s = cp.CoupledCG(M, precond=kind)
            x = M.vector()
            st = s.Solve(M.vector(b[r0:r1]), x, maxits=5000, reltol=1e-10)
            out.append((st, s.iter, x.numpy()))
        return r0, out

    res = _run_ranks(world, rank_fn)
    x = np.zeros(n)
    for r0, ((st, it, xr), (stj, itj, _)) in res:
        assert st == b200.SUCCESS_REL and stj == b200.SUCCESS_REL
        assert it < itj, (it, itj)
        if world == 1:
            assert abs(it - it_single) <= max(1, 0.05 * it_single), (it, it_single)
        x[r0:r0 + len(xr)] = xr
    assert np.linalg.norm(x - xe) <= 1e-8 * np.linalg.norm(xe)


@pytest.mark.gpu
@pytest.mark.parametrize("world", [1, 2, 3])
def test_coupled_gmres_ranks_on_one_gpu(b200, world):
    """Coupled GMRES(30) on the reference's GMRES case (2-D 32^2 convection-
    diffusion, nu = 1e-3, its right-hand side from the golden fixtures).
    Unpreconditioned it is the global method: the reference's iteration count
    and the single-system GMRES's, within 5%.  With the local blocks' Jacobi
    (block-Jacobi across ranks) it reaches the global solution; with the
    blocks' MC-SGS it does so on a milder case (24^2, nu = 1e-2), since on
    this strongly convective one SGS blocks make a poor right preconditioner
    (GMRES(30) stalls)."""
    import importlib
    cp = importlib.import_module("hiflow3_b200.coupled")
    golden = np.load(os.path.join(ROOT, "tests", "golden", "lmp_golden.npz"))
    N = 32
    row, col, val = b200.q1_assemble(2, N, 1, None, 1e-3, (1.0, 0.5))
    n = len(row) - 1
    b = golden["gmres2d32_b"]
    it_ref = int(golden["gmres2d32_none_iters"][0])
    D = np.zeros((n, n))
    for i in range(n):
        D[i, col[row[i]:row[i + 1]]] += val[row[i]:row[i + 1]]
    xe = np.linalg.solve(D, b)
    pf0 = b200.Platform(0)
    gm = b200.GMRES(pf0, 30)
    gm.SetupOperator(b200.CSR_lMatrix.from_csr(pf0, row, col, val))
    gm.InitControl(3000, 0.0, 1e-9, 1e6)
    assert gm.Solve(pf0.vector(b), pf0.vector(n)) == b200.SUCCESS_REL
    it_single = gm.iter()
    part = cp.RowPartition.even(n, world)
    trs = cp.LocalTransport.group(world)

    def rank_fn(r):
        pf = b200.Platform(0)
        r0, r1 = part.range(r)
        M = cp.CoupledMatrix(pf, part, r, trs[r], row[r0:r1 + 1] - row[r0], col[row[r0]:row[r1]],
                             val[row[r0]:row[r1]])
        out = []
        for kind in ("none", "jacobi"):
            s = cp.CoupledGMRES(M, 30, precond=kind)
            x = M.vector()
            st = s.Solve(M.vector(b[r0:r1]), x, maxits=3000, reltol=1e-9)
            out.append((kind, st, s.iter, x.numpy()))
        # the milder case with MC-SGS blocks
        r0m, r1m = part_m.range(r)
        Mm = cp.CoupledMatrix(pf, part_m, r, trs_m[r], row_m[r0m:r1m + 1] - row_m[r0m], col_m[row_m[r0m]:row_m[r1m]],
                              val_m[row_m[r0m]:row_m[r1m]])
        s = cp.CoupledGMRES(Mm, 30, precond="mcsgs")
        xm = Mm.vector()
        stm = s.Solve(Mm.vector(b_m[r0m:r1m]), xm, maxits=3000, reltol=1e-9)
        return r0, out, (r0m, stm, xm.numpy())

    row_m, col_m, val_m = b200.q1_assemble(2, 24, 1, None, 1e-2, (1.0, 0.5))
    n_m = len(row_m) - 1
    b_m = b200.q1_rhs(8, 2, 24)
    part_m = cp.RowPartition.even(n_m, world)
    trs_m = cp.LocalTransport.group(world)
    res = _run_ranks(world, rank_fn)
    Dm = np.zeros((n_m, n_m))
    for i in range(n_m):
        Dm[i, col_m[row_m[i]:row_m[i + 1]]] += val_m[row_m[i]:row_m[i + 1]]
    xm = np.zeros(n_m)
    for _, _, (r0m, stm, xr) in res:
        assert stm == b200.SUCCESS_REL
        xm[r0m:r0m + len(xr)] = xr
    assert np.linalg.norm(b_m - Dm @ xm) <= 2e-9 * np.linalg.norm(b_m)
    res = [(r0, out) for r0, out, _ in res]
    for kind_i, kind in enumerate(("none", "jacobi")):
        x = np.zeros(n)
        for r0, out in res:
            k, st, it, xr = out[kind_i]
            assert st == b200.SUCCESS_REL, (kind, st)
            if kind == "none":
                assert abs(it - it_single) <= max(1, 0.05 * it_single), (it, it_single)
                assert abs(it - it_ref) <= max(1, 0.05 * it_ref), (it, it_ref)
            x[r0:r0 + len(xr)] = xr
        # the stop test is on the Givens estimate; the true residual agrees closely
        assert np.linalg.norm(b - D @ x) <= 2e-9 * np.linalg.norm(b), kind
        assert np.linalg.norm(x - xe) <= 1e-4 * np.linalg.norm(xe), kind


@pytest.mark.gpu
@pytest.mark.parametrize("world", [1, 2, 3])
def test_coupled_mpir_ranks_on_one_gpu(b200, oracle, world):
    """Mixed-precision defect correction across ranks: FP64 coupled residuals,
    FP32 coupled Jacobi-CG corrections to 1e-4.  It reaches 1e-10 of the first
    residual, the solution agrees with the direct solve within 1e-8, and it
    takes as many corrections (within one) as the oracle's single-system MPIR."""
    import importlib
    from pyoracle import control
    cp = importlib.import_module("hiflow3_b200.coupled")
    N = 12
    kc = np.exp(np.random.default_rng(5).standard_normal(N ** 3))
    row, col, val = b200.q1_assemble(3, N, 0, kc)
    n = len(row) - 1
    b = b200.q1_rhs(9, 3, N)
    ref = oracle.mpir(row, col, val, b, outer=control(50, 0, 1e-10, 1e6), inner=control(10000, 0, 1e-4, 1e6))
    D = np.zeros((n, n))
    for i in range(n):
        D[i, col[row[i]:row[i + 1]]] += val[row[i]:row[i + 1]]
    xe = np.linalg.solve(D, b)
    part = cp.RowPartition.even(n, world)
    trs = cp.LocalTransport.group(world)

    def rank_fn(r):
        pf = b200.Platform(0)
        r0, r1 = part.range(r)
        M = cp.CoupledMatrix(pf, part, r, trs[r], row[r0:r1 + 1] - row[r0], col[row[r0]:row[r1]],
                             val[row[r0]:row[r1]])
        s = cp.CoupledMPIR(M)
        x = M.vector()
        st = s.Solve(M.vector(b[r0:r1]), x, maxits=50, reltol=1e-10, inner=(10000, 0.0, 1e-4, 1e6))
        return r0, st, s.outer, s.res, s.res0, x.numpy()

    res = _run_ranks(world, rank_fn)
    x = np.zeros(n)
    for r0, st, outer, rn, r0n, xr in res:
        assert st == b200.SUCCESS_REL and rn < 1e-10 * r0n
        assert abs(outer - ref["outer"]) <= 1, (outer, ref["outer"])
        x[r0:r0 + len(xr)] = xr
    assert np.linalg.norm(x - xe) <= 1e-8 * np.linalg.norm(xe)


def test_couplings_ghost_owner_and_index():
    """Where every ghost lives (the remote-read tables): its owner from the
    partition, and its number there (global minus the owner's first row); no
    transport is needed for these."""
    import importlib
    from conftest import load_platform
    load_platform()
    cp = importlib.import_module("hiflow3_b200.coupled")
    part = cp.RowPartition([0, 10, 25, 25, 40])          # rank 2 owns nothing
    ghosts = np.array([3, 9, 30, 39], np.int64)         # rank 1's ghosts
    c = cp.LaCouplings(part, 1, ghosts)
    assert c.ghost_owner.tolist() == [0, 0, 3, 3]
    assert c.ghost_index.tolist() == [3, 9, 5, 14]
    assert c.ghost_offsets.tolist() == [0, 2, 2, 2, 4]
    with pytest.raises(ValueError):
        cp.LaCouplings(part, 1, np.array([12], np.int64))   # a ghost this rank owns
    empty = cp.LaCouplings(part, 0, np.zeros(0, np.int64))
    assert empty.ghost_owner.size == 0 and empty.ghost_index.size == 0
