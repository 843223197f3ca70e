"""Asynchronous block-Jacobi iteration (b200la_async_jacobi) against the
solution of the system.  The iterates are not reproducible bit for bit by
design (rows read their neighbours' current values with no barrier, as in
src/linear_solver/gpu-based/async_iter_gpu.cc); the tests check the stop
decision and the solution it stops at."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pf(b200):
    return b200.Platform(0)


def dense(row, col, val, m=None):
    n = len(row) - 1
    A = np.zeros((n, m or n))
    for i in range(n):
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


@pytest.mark.parametrize("w", [1.0, 0.8])
def test_async_jacobi_converges(b200, pf, w):
    row, col, val = b200.q1_assemble(2, 16, 0, np.exp(np.random.default_rng(3).standard_normal(256)))
    n = len(row) - 1
    b = b200.q1_rhs(5, 2, 16)
    A = b200.CSR_lMatrix.from_csr(pf, row, col, val)
    x = pf.vector(n)
    out = b200.async_jacobi(pf, A, pf.vector(b), x, n_inner=4, n_block=8, w=w, reltol=1e-8, maxits=200000)
    assert out["status"] == b200.SUCCESS_REL
    assert out["iters"] % 4 == 0 and out["iters"] > 0
    D = dense(row, col, val)
    xs = x.numpy()
    assert np.linalg.norm(b - D @ xs) <= 1e-8 * out["res0"] * 1.0001
    xe = np.linalg.solve(D, b)
    assert np.linalg.norm(xs - xe) <= 1e-4 * np.linalg.norm(xe)


def test_async_jacobi_fp32(b200, pf):
    row, col, val = b200.q1_assemble(2, 12, 0)
    n = len(row) - 1
    b = b200.q1_rhs(9, 2, 12)
    A = b200.CSR_lMatrix.from_csr(pf, row, col, val, dtype=b200.F32)
    x = pf.vector(n, b200.F32)
    out = b200.async_jacobi(pf, A, pf.vector(b, b200.F32), x, n_inner=2, n_block=16, reltol=1e-4)
    assert out["status"] == b200.SUCCESS_REL
    xe = np.linalg.solve(dense(row, col, val), b)
    assert np.linalg.norm(x.numpy() - xe) <= 1e-2 * np.linalg.norm(xe)


def test_async_jacobi_with_ghost_block(b200, pf):
    # a "rank" owning the first half of the rows; the ghosts hold the other
    # half of the exact solution, so the local iteration converges to the
    # exact solution's own part
    row, col, val = b200.q1_assemble(2, 14, 0)
    n = len(row) - 1
    Dm = dense(row, col, val)
    b = b200.q1_rhs(2, 2, 14)
    xe = np.linalg.solve(Dm, b)
    own, rest = np.arange(n // 2), np.arange(n // 2, n)
    Ad = b200.CSR_lMatrix.from_csr(pf, *to_csr(Dm[np.ix_(own, own)]))
    Ao = b200.CSR_lMatrix.from_csr(pf, *to_csr(Dm[np.ix_(own, rest)]), n_cols=len(rest))
    x = pf.vector(len(own))
    out = b200.async_jacobi(pf, Ad, pf.vector(b[own]), x, n_inner=4, n_block=8, reltol=1e-10, maxits=400000,
                            A_offdiag=Ao, x_ghost=pf.vector(xe[rest]))
    assert out["status"] == b200.SUCCESS_REL
    assert np.linalg.norm(x.numpy() - xe[own]) <= 1e-6 * np.linalg.norm(xe[own])


def test_async_jacobi_rejects(b200, pf):
    row, col, val = b200.q1_assemble(2, 4, 0)
    n = len(row) - 1
    A = b200.CSR_lMatrix.from_csr(pf, row, col, val)
    with pytest.raises(b200.B200Error):
        b200.async_jacobi(pf, A, pf.vector(n), pf.vector(n), n_inner=0)
    with pytest.raises(b200.B200Error):
        b200.async_jacobi(pf, A, pf.vector(n), pf.vector(n), w=0.0)
