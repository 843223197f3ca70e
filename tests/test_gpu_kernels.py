"""GPU parity of the B200 platform's kernels against the oracle (C restatement
of the reference, pinned to the reference's own outputs).

Tolerances: FP64 SpMV 1e-13 relative to the row's magnitude sum_j |a_ij x_j|
(the stated SpMV bar), FP32 SpMV 1e-5 on the same scale; BLAS1 1e-13
relative in FP64; preconditioner applies 1e-12 relative (the sweeps sum each
row in a different order than the reference's serial loop).
"""
import os
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KAT_ROW = np.array([0, 3, 6, 9], np.int32)
KAT_COL = np.array([0, 1, 2] * 3, np.int32)
KAT_VAL = np.array([2, -1, 0, -1, 2, -1, 0, -1, 2.0])


@pytest.fixture(scope="module")
def pf(b200):
    return b200.Platform(0)


def row_scale(row, col, val, x):
    a = np.abs(val) * np.abs(x[col])
    return np.add.reduceat(a, row[:-1]) if len(a) else np.zeros(len(row) - 1)


def spmv_ok(y, y_ref, scale, tol):
    s = np.where(np.diff(np.r_[0, np.arange(len(scale))]) >= 0, scale, 0)
    return np.all(np.abs(y - y_ref) <= tol * np.maximum(s, np.finfo(float).tiny))


def random_csr(rng, n, m, long_rows=(), empty_rows=(), mean=7):
    rows = []
    for i in range(n):
        if i in empty_rows:
            k = 0
        elif i in long_rows:
            k = min(m, 5000)
        else:
            k = int(rng.integers(0, 2 * mean))
        rows.append(np.sort(rng.choice(m, size=k, replace=False)) if k else np.zeros(0, np.int64))
    row = np.zeros(n + 1, np.int32)
    row[1:] = np.cumsum([len(r) for r in rows])
    col = np.concatenate(rows).astype(np.int32) if row[-1] else np.zeros(0, np.int32)
    val = rng.standard_normal(row[-1])
    return row, col, val


def test_spmv_kat(pf, b200):
    # test-legacy/cuda_test.cc:27-100 and test-legacy/lmp_test.cc:38-89
    A = b200.CSR_lMatrix.from_csr(pf, KAT_ROW, KAT_COL, KAT_VAL)
    for xv, yv in [([1.2, -2.3, 0.7], [4.7, -6.5, 3.7]), ([1.0, -2.0, 0.0], [4.0, -5.0, 2.0])]:
        x, y = pf.vector(xv), pf.vector(3)
        A.VectorMult(x, y)
        np.testing.assert_allclose(y.numpy(), yv, atol=1e-12)


@pytest.mark.parametrize("dim,N,kind,coef", [(2, 8, 0, False), (2, 17, 1, False), (3, 7, 0, True),
                                             (2, 256, 0, False), (3, 32, 0, True), (2, 512, 1, False)])
def test_spmv_q1_vs_oracle(pf, b200, oracle, dim, N, kind, coef):
    rng = np.random.default_rng(dim * 1000 + N)
    kc = np.exp(rng.standard_normal(N ** dim)) if coef else None
    row, col, val = oracle.q1_assemble(dim, N, kind, kc, nu=1e-3, beta=(1.0, 0.5))
    n = len(row) - 1
    x = rng.uniform(-1, 1, n)
    y_ref = oracle.spmv(row, col, val, x)
    sc = row_scale(row, col, val, x)
    A = b200.CSR_lMatrix.from_csr(pf, row, col, val)
    xv, yv = pf.vector(x), pf.vector(n)
    A.VectorMult(xv, yv)
    assert spmv_ok(yv.numpy(), y_ref, sc, 1e-13)
    # y += A x
    y0 = rng.uniform(-1, 1, n)
    yv = pf.vector(y0)
    A.VectorMultAdd(xv, yv)
    assert np.all(np.abs(yv.numpy() - (y0 + y_ref)) <= 1e-13 * (sc + np.abs(y0)) + 1e-300)
    # fused y = A x, x.y
    d = A.VectorMultDot(xv, yv)
    assert abs(d - np.dot(x, y_ref)) <= 1e-12 * np.dot(np.abs(x), sc)
    # fused r = b - A x, ||r||^2
    b = rng.uniform(-1, 1, n)
    rv = pf.vector(n)
    nr = A.Residual(pf.vector(b), xv, rv)
    assert np.all(np.abs(rv.numpy() - (b - y_ref)) <= 1e-13 * (sc + np.abs(b)))
    np.testing.assert_allclose(nr, np.dot(b - y_ref, b - y_ref), rtol=1e-12)
    # FP32 copy (CastFrom) and FP32 SpMV
    A32 = A.CastFrom(b200.F32)
    x32 = x.astype(np.float32)
    y32_ref = oracle.spmv(row, col, val.astype(np.float32), x32)
    yv32 = pf.vector(n, b200.F32)
    A32.VectorMult(pf.vector(x32, b200.F32), yv32)
    sc32 = row_scale(row, col, val.astype(np.float32).astype(np.float64), x32.astype(np.float64))
    assert np.all(np.abs(yv32.numpy().astype(np.float64) - y32_ref) <= 2e-6 * sc32 + 1e-30)


def test_spmv_irregular_long_and_empty_rows(pf, b200, oracle):
    rng = np.random.default_rng(11)
    n, m = 3000, 7000
    row, col, val = random_csr(rng, n, m, long_rows={5, 1700, 2999}, empty_rows={0, 1, 2, 900, 2998})
    x = rng.uniform(-1, 1, m)
    # oracle works on square CSR; compute the reference product directly
    y_ref = np.zeros(n)
    for i in range(n):
        s = 0.0
        for j in range(row[i], row[i + 1]):
            s += val[j] * x[col[j]]
        y_ref[i] = s
    A = b200.CSR_lMatrix.from_csr(pf, row, col, val, n_cols=m)
    info = A.info()
    assert info["n_long_rows"] == 3
    yv = pf.vector(n)
    A.VectorMult(pf.vector(x), yv)
    assert spmv_ok(yv.numpy(), y_ref, row_scale(row, col, val, x), 1e-13)
    assert np.all(yv.numpy()[[0, 1, 2, 900, 2998]] == 0.0)


@pytest.mark.parametrize("lanes", ["auto", "1", "4", "32"])
def test_spmv_fp32_csr_irregular(pf, b200, lanes, monkeypatch):
    """FP32 CSR SpMV with 16-byte value/column loads: rows that start at any
    offset (not a multiple of four entries), long rows, empty rows (the last
    row among them), for the automatic and forced lanes-per-row choices.
    Tolerance: the FP32 rounding bound (row length + 16) * 2^-24 on the row's
    magnitude sum_j |a_ij x_j|, against the product in FP64 of the same FP32
    inputs."""
    if lanes != "auto":
        monkeypatch.setenv("B200LA_LANES", lanes)
    rng = np.random.default_rng(23)
    n, m = 2500, 4100
    row, col, val = random_csr(rng, n, m, long_rows={3, 1200}, empty_rows={0, 7, 2499}, mean=9)
    v32 = val.astype(np.float32)
    x32 = rng.uniform(-1, 1, m).astype(np.float32)
    vd, xd = v32.astype(np.float64), x32.astype(np.float64)
    y_ref = np.array([vd[row[i]:row[i + 1]] @ xd[col[row[i]:row[i + 1]]] for i in range(n)])
    scale = np.array([np.abs(vd[row[i]:row[i + 1]]) @ np.abs(xd[col[row[i]:row[i + 1]]]) for i in range(n)])
    A = b200.CSR_lMatrix.from_csr(pf, row, col, v32, n_cols=m, dtype=b200.F32)
    if lanes != "auto":
        assert A.info()["lanes_per_row"] == int(lanes)
    y = pf.vector(n, b200.F32)
    A.VectorMult(pf.vector(x32, b200.F32), y)
    yh = y.numpy().astype(np.float64)
    tol = (np.diff(row) + 16) * 2.0 ** -24 * np.maximum(scale, 1e-30)
    assert np.all(np.abs(yh - y_ref) <= tol)
    assert np.all(yh[[0, 7, 2499]] == 0.0)


@pytest.mark.parametrize("lanes", ["1", "2", "8", "32"])
def test_spmv_lane_layouts(pf, b200, oracle, lanes, monkeypatch):
    monkeypatch.setenv("B200LA_LANES", lanes)
    row, col, val = oracle.q1_assemble(3, 9, 0)
    x = np.random.default_rng(2).uniform(-1, 1, len(row) - 1)
    A = b200.CSR_lMatrix.from_csr(pf, row, col, val)
    assert A.info()["lanes_per_row"] == int(lanes)
    yv = pf.vector(len(row) - 1)
    A.VectorMult(pf.vector(x), yv)
    assert spmv_ok(yv.numpy(), oracle.spmv(row, col, val, x), row_scale(row, col, val, x), 1e-13)


@pytest.mark.parametrize("mode,stage,tma,stencil", [("0", "0", "0", "0"), ("2", "0", "0", "0"), ("2", "1", "0", "0"),
                                                   ("2", "0", "1", "0"), ("0", "0", "0", "2"), ("2", "0", "0", "2")])
@pytest.mark.parametrize("dim,N,kind", [(3, 10, 0), (2, 33, 1), (3, 21, 0), (2, 1, 0), (3, 40, 1)])
def test_spmv_pattern_dictionary(pf, b200, oracle, mode, stage, tma, stencil, dim, N, kind, monkeypatch):
    """SpMV through the row-pattern dictionary (mode 2, both precisions; sliced
    layout read directly or by bulk-copy tiles, or CSR value order with x
    staged in shared memory) and through the index-free stencil layout
    (stencil 2) equals SpMV through explicit column indices."""
    monkeypatch.setenv("B200LA_PATTERN", mode)
    monkeypatch.setenv("B200LA_STAGE_X", stage)
    monkeypatch.setenv("B200LA_SELL_TMA", tma)
    monkeypatch.setenv("B200LA_STENCIL", stencil)
    stencil_ok = N > 1     # N = 1: every row is a corner, the padding exceeds the limit
    # symmetric operators (Poisson, kind 0) take the half stencil layout
    want = (("half-stencil" if kind == 0 else "stencil") if (stencil == "2" and stencil_ok)
            else "dictionary" if mode == "2" else "csr")
    row, col, val = oracle.q1_assemble(dim, N, kind, None, nu=1e-3, beta=(1.0, 0.5))
    n = len(row) - 1
    x = np.random.default_rng(4).uniform(-1, 1, n)
    sc = row_scale(row, col, val, x)
    y_ref = oracle.spmv(row, col, val, x)
    A = b200.CSR_lMatrix.from_csr(pf, row, col, val)
    info = A.info()
    assert info["row_patterns"] == ((27 if dim == 3 else 9) if N > 1 else 2 ** dim)   # interior, faces, edges, corners
    assert info["storage"] == want
    yv = pf.vector(n)
    A.VectorMult(pf.vector(x), yv)
    assert spmv_ok(yv.numpy(), y_ref, sc, 1e-13)
    A32 = A.CastFrom(b200.F32)
    assert A32.info()["storage"] == ("stencil" if want == "half-stencil" else want)
    x32 = x.astype(np.float32)
    y32 = pf.vector(n, b200.F32)
    A32.VectorMult(pf.vector(x32, b200.F32), y32)
    y32_ref = oracle.spmv(row, col, val.astype(np.float32), x32)
    assert np.all(np.abs(y32.numpy().astype(np.float64) - y32_ref) <= 2e-6 * sc + 1e-30)


@pytest.mark.parametrize("dim,N,coef", [(2, 20, False), (2, 63, True), (3, 9, False), (3, 13, True), (3, 64, True)])
def test_spmv_half_stencil_bitwise(pf, b200, oracle, dim, N, coef, monkeypatch):
    """The half stencil layout (diagonal and upper half; the lower half read
    from the rows that own it) gives y bit for bit equal to the full stencil
    layout, in both precisions and in every fused epilogue (y = Ax, y += Ax,
    y = Ax with x.y, r = b - Ax with ||r||^2), and within the SpMV tolerance
    of the oracle."""
    rng = np.random.default_rng(100 * dim + N)
    kc = np.exp(rng.standard_normal(N ** dim)) if coef else None
    row, col, val = oracle.q1_assemble(dim, N, 0, kc)
    n = len(row) - 1
    x, y0, b = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)
    outs = {}
    for half in ("2", "0"):
        monkeypatch.setenv("B200LA_HALF_STENCIL", half)
        A = b200.CSR_lMatrix.from_csr(pf, row, col, val)
        A32 = A.CastFrom(b200.F32)
        assert A.info()["storage"] == A32.info()["storage"] == ("half-stencil" if half == "2" else "stencil")
        res = []
        for M, dt in ((A, b200.F64), (A32, b200.F32)):
            cast = (lambda v: v) if dt == b200.F64 else (lambda v: v.astype(np.float32))
            xv, yv = pf.vector(cast(x), dt), pf.vector(n, dt)
            M.VectorMult(xv, yv)
            res.append(yv.numpy())
            ya = pf.vector(cast(y0), dt)
            M.VectorMultAdd(xv, ya)
            res.append(ya.numpy())
            res.append(np.array([M.VectorMultDot(xv, yv)]))
            rv = pf.vector(n, dt)
            res.append(np.array([M.Residual(pf.vector(cast(b), dt), xv, rv)]))
            res.append(rv.numpy())
        outs[half] = res
    # vectors bit for bit; the fused reductions (x.y, ||r||^2) sum the same
    # products over a grid sized by each kernel's occupancy, so their order
    # of summation, and possibly their last bit, differ
    for k, (a, c) in enumerate(zip(outs["2"], outs["0"])):
        if k % 5 in (2, 3):
            np.testing.assert_allclose(a, c, rtol=1e-13)
        else:
            assert np.array_equal(a.view(np.uint8), c.view(np.uint8)), k
    assert spmv_ok(outs["2"][0], oracle.spmv(row, col, val, x), row_scale(row, col, val, x), 1e-13)
    # the default: FP64 operators take the half layout, FP32 ones the full one
    monkeypatch.delenv("B200LA_HALF_STENCIL")
    A = b200.CSR_lMatrix.from_csr(pf, row, col, val)
    assert A.info()["storage"] == "half-stencil" and A.CastFrom(b200.F32).info()["storage"] == "stencil"


def test_spmv_half_stencil_rejects_asymmetry(pf, b200, oracle):
    """One off-diagonal entry changed between two interior rows: the operator
    is no longer symmetric, the half layout is not used, and SpMV stays exact."""
    # 16^3 cells: small grids pad more than the stencil layout allows (30 %)
    row, col, val = oracle.q1_assemble(3, 16, 0, None)
    n = len(row) - 1
    r = (n // 2)
    j = next(k for k in range(row[r], row[r + 1]) if col[k] != r and val[k] != 0.0)
    val = val.copy()
    val[j] *= 1.0 + 2.0 ** -40
    A = b200.CSR_lMatrix.from_csr(pf, row, col, val)
    assert A.info()["storage"] == "stencil"
    x = np.random.default_rng(5).uniform(-1, 1, n)
    yv = pf.vector(n)
    A.VectorMult(pf.vector(x), yv)
    assert spmv_ok(yv.numpy(), oracle.spmv(row, col, val, x), row_scale(row, col, val, x), 1e-13)


def test_spmv_degenerate_shapes(pf, b200):
    A = b200.CSR_lMatrix.from_csr(pf, [0, 1], [0], [3.0])
    y = pf.vector(1)
    A.VectorMult(pf.vector([2.0]), y)
    assert y.numpy()[0] == 6.0
    Z = b200.CSR_lMatrix.from_csr(pf, np.zeros(6, np.int32), np.zeros(0, np.int32), np.zeros(0))
    y = pf.vector(np.ones(5))
    Z.VectorMult(pf.vector(np.ones(5)), y)
    assert np.all(y.numpy() == 0.0)


def test_malformed_csr_rejected(pf, b200):
    with pytest.raises(b200.B200Error) as e:
        b200.CSR_lMatrix.from_csr(pf, [0, 2, 1], [0, 1], [1.0, 2.0])
    assert e.value.code == 5
    with pytest.raises(b200.B200Error) as e:
        b200.CSR_lMatrix.from_csr(pf, [0, 1, 2], [0, 7], [1.0, 2.0])
    assert e.value.code == 5


@pytest.mark.parametrize("n", [1, 5, 1000, 1_000_003])
def test_blas1_vs_numpy(pf, b200, oracle, n):
    rng = np.random.default_rng(n)
    x, y = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)
    X, Y = pf.vector(x), pf.vector(y)
    np.testing.assert_allclose(X.Dot(Y), oracle.dot(x, y), rtol=1e-12, atol=1e-14 * n)
    np.testing.assert_allclose(X.Norm2(), np.sqrt(oracle.dot(x, x)), rtol=1e-13)
    Y.Axpy(X, 0.75)
    np.testing.assert_allclose(Y.numpy(), y + 0.75 * x, rtol=1e-15, atol=1e-15)
    Y = pf.vector(y)
    Y.ScaleAdd(-1.5, X)
    np.testing.assert_allclose(Y.numpy(), -1.5 * y + x, rtol=1e-15, atol=1e-15)
    Y.Scale(2.0)
    np.testing.assert_allclose(Y.numpy(), 2 * (-1.5 * y + x), rtol=1e-15, atol=1e-15)
    Y = pf.vector(y)
    Y.ElementWiseMult(X)
    np.testing.assert_array_equal(Y.numpy(), y * x)
    Z = pf.vector(n, b200.F32)
    Z.CastFrom(X)
    np.testing.assert_array_equal(Z.numpy(), x.astype(np.float32))
    W = pf.vector(n)
    W.CastFrom(Z)
    np.testing.assert_array_equal(W.numpy(), x.astype(np.float32).astype(np.float64))
    idx = rng.permutation(n)[: max(1, n // 3)]
    np.testing.assert_array_equal(X.GetIndexedValues(idx), x[idx])
    X.SetIndexedValues(idx, np.zeros(idx.size))
    xx = x.copy()
    xx[idx] = 0
    np.testing.assert_array_equal(X.numpy(), xx)
    perm = rng.permutation(n)
    X = pf.vector(x)
    X.Reorder(perm)
    np.testing.assert_array_equal(X.numpy(), x[perm])
    # float dot: FP32 products, FP64 global reduction
    xf, yf = x.astype(np.float32), y.astype(np.float32)
    d32 = pf.vector(xf, b200.F32).Dot(pf.vector(yf, b200.F32))
    np.testing.assert_allclose(d32, np.dot(xf.astype(np.float64), yf.astype(np.float64)), rtol=1e-5,
                               atol=1e-6 * np.sqrt(n))


def test_reference_gpu_kernel_baseline(oracle):
    """The reference's own GPU SpMV (kernel_spmv_csr_scalar, built for sm_100a
    into baseline/_ref and timed in bench.py beside the platform's kernels)
    computes y = A x: it is a correct baseline."""
    import ctypes as C
    so = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "baseline", "_ref",
                      "libref_gpu_spmv.so")
    if not os.path.exists(so):
        pytest.skip("the reference GPU baseline is built only where the HiFlow3 sources are present")
    L = C.CDLL(so)
    row, col, val = oracle.q1_assemble(3, 20, 0, np.exp(np.random.default_rng(2).standard_normal(20 ** 3)))
    n = len(row) - 1
    x = np.random.default_rng(3).uniform(-1, 1, n)
    for dtype, npd in ((0, np.float64), (1, np.float32)):
        v, xx = val.astype(npd), x.astype(npd)
        y = np.empty(n, npd)
        ms = C.c_double()
        assert L.refgpu_spmv(dtype, n, len(col), C.c_void_p(row.ctypes.data), C.c_void_p(col.ctypes.data),
                             C.c_void_p(v.ctypes.data), C.c_void_p(xx.ctypes.data), C.c_void_p(y.ctypes.data), 3,
                             C.byref(ms)) == 0
        y_ref = oracle.spmv(row, col, v.astype(np.float64), xx.astype(np.float64))
        sc = row_scale(row, col, v.astype(np.float64), xx.astype(np.float64))
        tol = 1e-13 if dtype == 0 else 2e-6
        assert np.all(np.abs(y.astype(np.float64) - y_ref) <= tol * sc + 1e-30)
        assert ms.value > 0
