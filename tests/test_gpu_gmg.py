"""Geometric-multigrid level steps (b200la_gmg_*) against a numpy restatement
of lmp/cuda/cuda_gmg_kernel.h (residual, restriction, prolongation update),
with and without an off-diagonal (ghost) block.

The operators come from two levels of the 2-D Q1 Poisson problem: the fine
operator, bilinear prolongation P (fine x coarse) and restriction R = P^T / 4.
The "rank" owns the first half of the fine rows; its diagonal block holds the
owned columns, its off-diagonal block the others (the ghosts, compacted).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TOL = 1e-13   # per row, relative to sum_j |a_ij x_j| (FP64 sums in another order)


@pytest.fixture(scope="module")
def pf(b200):
    return b200.Platform(0)


def dense(row, col, val, m):
    A = np.zeros((len(row) - 1, m))
    for i in range(len(row) - 1):
        for j in range(row[i], row[i + 1]):
            A[i, col[j]] += val[j]
    return A


def to_csr(A):
    row, col, val = [0], [], []
    for i in range(A.shape[0]):
        nz = np.nonzero(A[i])[0]
        col += list(nz)
        val += list(A[i, nz])
        row.append(len(col))
    return np.array(row, np.int32), np.array(col, np.int32), np.array(val)


def prolongation(Nc):
    """Bilinear interpolation from (Nc+1)^2 coarse to (2Nc+1)^2 fine nodes."""
    Pc, Pf = Nc + 1, 2 * Nc + 1
    P = np.zeros((Pf * Pf, Pc * Pc))
    w1 = {0: [(0, 1.0)], 1: [(0, 0.5), (1, 0.5)]}
    for fy in range(Pf):
        for fx in range(Pf):
            for dy, wy in w1[fy % 2]:
                for dx, wx in w1[fx % 2]:
                    P[fy * Pf + fx, (fy // 2 + dy) * Pc + fx // 2 + dx] += wy * wx
    return P


def split(A, own_rows, own_cols):
    """Rows own_rows; diagonal block on own_cols, off-diagonal block on the rest."""
    rest = np.setdiff1d(np.arange(A.shape[1]), own_cols)
    return A[np.ix_(own_rows, own_cols)], A[np.ix_(own_rows, rest)], rest


def check(b200, got, ref, scale):
    assert np.all(np.abs(got - ref) <= TOL * np.maximum(scale, 1e-300)), np.max(np.abs(got - ref) / scale)


@pytest.mark.parametrize("ghost", [False, True])
def test_gmg_level_steps(b200, pf, ghost):
    rng = np.random.default_rng(7)
    Nc = 8
    row, col, val = b200.q1_assemble(2, 2 * Nc)
    n = len(row) - 1
    A = dense(row, col, val, n)
    P = prolongation(Nc)
    R = P.T / 4.0
    nc = P.shape[1]
    own_f = np.arange(n // 2) if ghost else np.arange(n)
    own_c = np.arange(nc // 2) if ghost else np.arange(nc)
    Ad, Ao, gA = split(A, own_f, own_f)
    Rd, Ro, gR = split(R, own_c, own_f)
    Pd, Po, gP = split(P, own_f, own_c)
    sol_full, rhs_full, crs_full = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n), rng.uniform(-1, 1, nc)
    mk = lambda M: b200.CSR_lMatrix.from_csr(pf, *to_csr(M), n_cols=M.shape[1])
    offd = lambda M: mk(M) if ghost else None
    v = pf.vector
    # residual on the owned fine rows
    res = v(len(own_f))
    b200.gmg_residual(pf, mk(Ad), v(sol_full[own_f]), v(rhs_full[own_f]), res, offd(Ao),
                      v(sol_full[gA]) if ghost else None)
    ref = rhs_full[own_f] - A[own_f] @ sol_full
    check(b200, res.numpy(), ref, np.abs(A[own_f]) @ np.abs(sol_full) + np.abs(rhs_full[own_f]))
    # restriction of a fine vector to the owned coarse rows
    tmp_full = rng.uniform(-1, 1, n)
    rc = v(len(own_c))
    b200.gmg_restriction(pf, mk(Rd), v(tmp_full[own_f]), rc, offd(Ro), v(tmp_full[gR]) if ghost else None)
    check(b200, rc.numpy(), R[own_c] @ tmp_full, np.abs(R[own_c]) @ np.abs(tmp_full))
    # prolongation update of the owned fine rows
    sol = v(sol_full[own_f])
    b200.gmg_prolongation_add(pf, mk(Pd), v(crs_full[own_c]), sol, offd(Po), v(crs_full[gP]) if ghost else None)
    ref = sol_full[own_f] + P[own_f] @ crs_full
    check(b200, sol.numpy(), ref, np.abs(P[own_f]) @ np.abs(crs_full) + np.abs(sol_full[own_f]))


def test_gmg_rejects_bad_blocks(b200, pf):
    row, col, val = b200.q1_assemble(2, 4)
    n = len(row) - 1
    A = b200.CSR_lMatrix.from_csr(pf, row, col, val)
    O = b200.CSR_lMatrix.from_csr(pf, row[:6] - row[0], col[:row[5]], val[:row[5]], n_cols=n)   # 5 rows
    x, y, z = pf.vector(n), pf.vector(n), pf.vector(n)
    b200.gmg_residual(pf, A, x, y, y)                # res may overwrite rhs
    with pytest.raises(b200.B200Error):
        b200.gmg_residual(pf, A, x, y, x)            # res may not overwrite sol
    with pytest.raises(b200.B200Error):
        b200.gmg_restriction(pf, A, x, y, O, z)      # off-diagonal block with another row count


REF_GMG = __import__("os").path.join(__import__("os").path.dirname(__import__("os").path.dirname(
    __import__("os").path.abspath(__file__))), "baseline", "_ref", "libref_gpu_gmg.so")


@pytest.mark.parametrize("ghost", [False, True])
def test_gmg_level_steps_vs_reference_kernels(b200, pf, ghost):
    """The same level steps against HiFlow3's own GPU kernels (lmp/cuda/cuda_gmg.cu
    and cuda_gmg_kernel.h, compiled for sm_100a from the reference tree by
    baseline/Makefile into baseline/_ref): residual, restriction and updated
    solution, with and without the ghost block, within TOL per row."""
    import ctypes as C
    import os
    if not os.path.exists(REF_GMG):
        pytest.fail("baseline/_ref/libref_gpu_gmg.so is missing: build it with __graft_entry__.build() where the "
                    "HiFlow3 sources are present")
    L = C.CDLL(REF_GMG)
    _P, _I = C.c_void_p, C.c_int
    L.refgpu_gmg.argtypes = [_I, _I, _P, _P, _P, _I, _P, _P, _P, _I, _P, _P, _P, _P]
    L.refgpu_gmg.restype = _I
    rng = np.random.default_rng(11)
    Nc = 8
    row, col, val = b200.q1_assemble(2, 2 * Nc, 0, np.exp(rng.normal(0.0, 0.5, (2 * Nc) ** 2)))
    n = len(row) - 1
    A = dense(row, col, val, n)
    P = prolongation(Nc)
    R = P.T / 4.0
    nc = P.shape[1]
    own_f = np.arange(n // 2) if ghost else np.arange(n)
    own_c = np.arange(nc // 2) if ghost else np.arange(nc)
    v = pf.vector
    mk = lambda M: b200.CSR_lMatrix.from_csr(pf, *to_csr(M), n_cols=M.shape[1])

    def ref(mode, Md, Mo, in0, in1, io, ghost_vals):
        dr, dc, dv = to_csr(Md)
        args = [mode, Md.shape[0], dr.ctypes.data, dc.ctypes.data, dv.ctypes.data, Md.shape[1]]
        if Mo is not None:
            orr, oc, ov = to_csr(Mo)
            g = np.ascontiguousarray(ghost_vals, np.float64)
            args += [orr.ctypes.data, oc.ctypes.data, ov.ctypes.data, len(g), g.ctypes.data]
        else:
            args += [None, None, None, 0, None]
        a0 = np.ascontiguousarray(in0, np.float64)
        a1 = np.ascontiguousarray(in1 if in1 is not None else np.zeros(1), np.float64)
        out = np.ascontiguousarray(io, np.float64).copy()
        rc = L.refgpu_gmg(*args, a0.ctypes.data, a1.ctypes.data, out.ctypes.data)
        assert rc == 0, rc
        return out

    Ad, Ao, gA = split(A, own_f, own_f)
    Rd, Ro, gR = split(R, own_c, own_f)
    Pd, Po, gP = split(P, own_f, own_c)
    sol_f, rhs_f, crs = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n), rng.uniform(-1, 1, nc)
    tmp_f = rng.uniform(-1, 1, n)
    # residual
    res = v(len(own_f))
    b200.gmg_residual(pf, mk(Ad), v(sol_f[own_f]), v(rhs_f[own_f]), res, mk(Ao) if ghost else None,
                      v(sol_f[gA]) if ghost else None)
    want = ref(0, Ad, Ao if ghost else None, sol_f[own_f], rhs_f[own_f], np.zeros(len(own_f)), sol_f[gA])
    check(b200, res.numpy(), want, np.abs(A[own_f]) @ np.abs(sol_f) + np.abs(rhs_f[own_f]))
    # restriction
    rc = v(len(own_c))
    b200.gmg_restriction(pf, mk(Rd), v(tmp_f[own_f]), rc, mk(Ro) if ghost else None, v(tmp_f[gR]) if ghost else None)
    want = ref(1, Rd, Ro if ghost else None, tmp_f[own_f], None, np.zeros(len(own_c)), tmp_f[gR])
    check(b200, rc.numpy(), want, np.abs(R[own_c]) @ np.abs(tmp_f))
    # updated solution (prolongation update)
    sol = v(sol_f[own_f])
    b200.gmg_prolongation_add(pf, mk(Pd), v(crs[own_c]), sol, mk(Po) if ghost else None, v(crs[gP]) if ghost else None)
    want = ref(2, Pd, Po if ghost else None, crs[own_c], None, sol_f[own_f], crs[gP])
    check(b200, sol.numpy(), want, np.abs(P[own_f]) @ np.abs(crs) + np.abs(sol_f[own_f]))
