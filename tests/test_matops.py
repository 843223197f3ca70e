"""CSR_lMatrix value and structure operations (Scale, ScaleOffdiag, Zeros,
extract_diagelements / extract_invdiagelements, extract_submatrix, Compress)
and the lVector BLAS1 members beyond the Krylov path (ArgMin, ArgMax, Norm1,
NormMax, Rot, Rotm, Rotg).

Fixtures (tests/golden/matops_golden.npz, made by gen_matops_golden.py) hold
the reference's own outputs (lmp/lmatrix_csr_cpu.cc:100-224, 1768-1843,
2395-2431, its CPU code compiled unmodified) on random CSRs with unsorted
rows, repeated columns and stored zeros, square and rectangular, and on a 2-D
Q1 convection-diffusion system, and of CPUsimple_lvector.cc:51-158, 448-600
on seeded vectors.  The oracle's restatement must equal them bit for bit
(CPU), and so must the device operations (GPU); Norm1 is summed in a
different order on the device and agrees within 1e-14 relative.  Rows without a
stored diagonal are left out of the diagonal comparisons: the reference
writes an uninitialised value there.
"""
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = ["rand", "rect", "q1"]
NBLOCKS = {"rand": 4, "rect": 3, "q1": 3}
BLOCKS = {"rand": [(0, 0, 60, 60), (5, 7, 40, 33), (10, 0, 11, 60), (59, 59, 60, 60)],
          "rect": [(0, 0, 50, 70), (3, 52, 47, 70), (20, 10, 30, 65)],
          "q1": [(0, 0, 121, 121), (11, 11, 110, 110), (40, 30, 80, 95)]}


@pytest.fixture(scope="module")
def gold():
    return np.load(os.path.join(HERE, "golden", "matops_golden.npz"))


def csr(gold, name):
    return gold[f"{name}_row"], gold[f"{name}_col"], gold[f"{name}_val"], int(gold[f"{name}_m"])


def bits(a):
    return np.ascontiguousarray(a, np.float64).view(np.uint64)


@pytest.mark.parametrize("name", CASES)
def test_oracle_matops_match_reference(oracle, gold, name):
    row, col, val, m = csr(gold, name)
    alpha = float(gold["alpha"])
    for mode in (0, 1, 2):
        assert np.array_equal(bits(oracle.csr_scale(row, col, val, alpha, mode)), bits(gold[f"{name}_scale{mode}"]))
    lo, hi = gold[f"{name}_diag_range"]
    has = gold[f"{name}_has_diag"]
    for inv in (0, 1):
        d = oracle.csr_diag(row, col, val, int(lo), int(hi), inv)
        assert np.array_equal(bits(d[has]), bits(gold[f"{name}_diag{inv}"][has]))
    for k, blk in enumerate(BLOCKS[name]):
        r, c, v = oracle.csr_extract(row, col, val, 0, *blk)
        assert np.array_equal(r, gold[f"{name}_sub{k}_row"]) and np.array_equal(c, gold[f"{name}_sub{k}_col"])
        assert np.array_equal(bits(v), bits(gold[f"{name}_sub{k}_val"]))
    r, c, v = oracle.csr_extract(row, col, val, 1)
    assert np.array_equal(r, gold[f"{name}_comp_row"]) and np.array_equal(c, gold[f"{name}_comp_col"])
    assert np.array_equal(bits(v), bits(gold[f"{name}_comp_val"]))


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_device_matops_match_reference(b200, gold, name):
    pf = b200.Platform(0)
    row, col, val, m = csr(gold, name)
    n = len(row) - 1
    alpha = float(gold["alpha"])
    for mode, op in enumerate(("Scale", "ScaleOffdiag", "Zeros")):
        A = b200.CSR_lMatrix.from_csr(pf, row, col, val, n_cols=m)
        getattr(A, op)(*(() if op == "Zeros" else (alpha,)))
        r, c, v = A.download()
        assert np.array_equal(r, row) and np.array_equal(c, col)
        assert np.array_equal(bits(v), bits(gold[f"{name}_scale{mode}"])), op
    A = b200.CSR_lMatrix.from_csr(pf, row, col, val, n_cols=m)
    lo, hi = (int(x) for x in gold[f"{name}_diag_range"])
    has = gold[f"{name}_has_diag"]
    for inv, op in enumerate(("extract_diagelements", "extract_invdiagelements")):
        vec = pf.vector(np.full(hi - lo, -7.0))
        getattr(A, op)(lo, hi, vec)
        d = vec.numpy()
        assert np.array_equal(bits(d[has]), bits(gold[f"{name}_diag{inv}"][has]))
        assert np.all(d[~has] == -7.0)        # rows without a diagonal: untouched
    for k, blk in enumerate(BLOCKS[name]):
        S = A.extract_submatrix(*blk)
        assert (S.n, S.m) == (blk[2] - blk[0], blk[3] - blk[1])
        r, c, v = S.download()
        assert np.array_equal(r, gold[f"{name}_sub{k}_row"]) and np.array_equal(c, gold[f"{name}_sub{k}_col"])
        assert np.array_equal(bits(v), bits(gold[f"{name}_sub{k}_val"]))
    A.Compress()
    r, c, v = A.download()
    assert np.array_equal(r, gold[f"{name}_comp_row"]) and np.array_equal(c, gold[f"{name}_comp_col"])
    assert np.array_equal(bits(v), bits(gold[f"{name}_comp_val"]))


@pytest.mark.gpu
def test_device_scale_feeds_the_spmv_layouts(b200, oracle, gold):
    """After ScaleOffdiag the SpMV (stencil layout for the Q1 operator, SELL
    or CSR otherwise) multiplies with the new values: 1e-13 of the row's
    magnitude sum against the oracle's SpMV of the reference's scaled values."""
    pf = b200.Platform(0)
    for name in ("q1", "rand"):
        row, col, val, m = csr(gold, name)
        if m != len(row) - 1:
            continue
        A = b200.CSR_lMatrix.from_csr(pf, row, col, val)
        A.ScaleOffdiag(float(gold["alpha"]))
        x = np.random.default_rng(3).uniform(-1, 1, m)
        y = pf.vector(len(row) - 1)
        A.VectorMult(pf.vector(x), y)
        vs = gold[f"{name}_scale1"]
        ref = oracle.spmv(row, col, vs, x)
        scale = np.array([np.abs(vs[row[i]:row[i + 1]]) @ np.abs(x[col[row[i]:row[i + 1]]])
                          for i in range(len(row) - 1)])
        assert np.all(np.abs(y.numpy() - ref) <= 1e-13 * np.maximum(scale, 1e-300))


@pytest.mark.gpu
def test_device_matops_fp32(b200, gold):
    """FP32 matrices: the same operations in float arithmetic (Scale and
    ScaleOffdiag products, 1 / a_ii in float) and the same submatrix
    structure; the Q1 operator has no repeated columns, so its block values
    are the float copies of the FP64 ones."""
    pf = b200.Platform(0)
    row, col, val, m = csr(gold, "q1")
    v32 = val.astype(np.float32)
    a32 = np.float32(gold["alpha"])
    A = b200.CSR_lMatrix.from_csr(pf, row, col, v32, dtype=b200.F32)
    A.ScaleOffdiag(float(gold["alpha"]))
    exp = v32.copy()
    off = col != np.repeat(np.arange(len(row) - 1), np.diff(row))
    exp[off] = exp[off] * a32
    assert np.array_equal(A.download()[2].view(np.uint32), exp.view(np.uint32))
    B = b200.CSR_lMatrix.from_csr(pf, row, col, v32, dtype=b200.F32)
    lo, hi = (int(x) for x in gold["q1_diag_range"])
    vec = pf.vector(hi - lo, b200.F32)
    B.extract_invdiagelements(lo, hi, vec)
    dg = np.array([v32[row[i]:row[i + 1]][col[row[i]:row[i + 1]] == i][-1] for i in range(lo, hi)])
    assert np.array_equal(vec.numpy().view(np.uint32), (np.float32(1) / dg).view(np.uint32))
    S = B.extract_submatrix(*BLOCKS["q1"][2])
    r, c, v = S.download()
    assert np.array_equal(r, gold["q1_sub2_row"]) and np.array_equal(c, gold["q1_sub2_col"])
    assert np.array_equal(v.view(np.uint32), gold["q1_sub2_val"].astype(np.float32).view(np.uint32))


@pytest.mark.gpu
def test_device_matops_reject_bad_ranges(b200, gold):
    pf = b200.Platform(0)
    row, col, val, m = csr(gold, "rect")
    A = b200.CSR_lMatrix.from_csr(pf, row, col, val, n_cols=m)
    for blk in [(5, 5, 5, 10), (0, 0, 51, 10), (0, 60, 10, 71), (-1, 0, 3, 3), (3, 9, 2, 12)]:
        with pytest.raises(b200.B200Error) as e:
            A.extract_submatrix(*blk)
        assert e.value.code == b200.ERR_ARG
    with pytest.raises(b200.B200Error):
        A.extract_diagelements(10, 51, pf.vector(41))


NVEC = 4


def test_oracle_vecops_match_reference(oracle, gold):
    for k in range(NVEC):
        x, y = gold[f"vec{k}_x"], gold[f"vec{k}_y"]
        ref = gold[f"vec{k}_reduce"]
        got = oracle.vec_reduce(x)
        assert (got[0], got[1]) == (int(ref[0]), int(ref[1]))
        assert bits(np.array(got[2:])).tolist() == bits(ref[2:]).tolist()
        for j, (c, s) in enumerate([(0.6, 0.8), (-0.3, 0.95)]):
            xo, yo = oracle.rot(x, y, c, s)
            assert np.array_equal(bits(xo), bits(gold[f"vec{k}_rot{j}_x"]))
            assert np.array_equal(bits(yo), bits(gold[f"vec{k}_rot{j}_y"]))
    for (a, b), ref in zip(gold["rotg_in"], gold["rotg_out"]):
        assert bits(np.array(oracle.rotg(a, b))).tolist() == bits(ref).tolist()


ROTM = [(-1, 0.3, -0.7, 1.2, 0.9), (0, 9, 0.25, -0.5, 9), (1, 1.5, 9, 9, -0.4), (-2, 1, 2, 3, 4)]


@pytest.mark.gpu
def test_device_vecops_match_reference(b200, gold):
    pf = b200.Platform(0)
    for k in range(NVEC):
        x, y = gold[f"vec{k}_x"], gold[f"vec{k}_y"]
        ref = gold[f"vec{k}_reduce"]
        xv = pf.vector(x)
        assert xv.ArgMin() == int(ref[0]) and xv.ArgMax() == int(ref[1])
        assert bits(np.array([xv.NormMax()])) == bits(ref[3:4])
        assert abs(xv.Norm1() - ref[2]) <= 1e-14 * ref[2]
        for j, (c, s) in enumerate([(0.6, 0.8), (-0.3, 0.95)]):
            a, b = pf.vector(x), pf.vector(y)
            a.Rot(b, c, s)
            assert np.array_equal(bits(a.numpy()), bits(gold[f"vec{k}_rot{j}_x"]))
            assert np.array_equal(bits(b.numpy()), bits(gold[f"vec{k}_rot{j}_y"]))
        for j, prm in enumerate(ROTM):
            a, b = pf.vector(x), pf.vector(y)
            a.Rotm(b, prm)
            assert np.array_equal(bits(a.numpy()), bits(gold[f"vec{k}_rotm{j}_x"])), prm
            assert np.array_equal(bits(b.numpy()), bits(gold[f"vec{k}_rotm{j}_y"])), prm
    for (a, b), ref in zip(gold["rotg_in"], gold["rotg_out"]):
        assert bits(np.array(pf.vector(1).Rotg(a, b))).tolist() == bits(ref).tolist()


@pytest.mark.gpu
def test_device_argmin_argmax_ties_and_nans(b200, oracle):
    """Large vectors (many CTAs): the first index of the extreme magnitude
    wins across CTAs; NaNs are skipped, except a NaN at index 0, which the
    reference's scan keeps."""
    pf = b200.Platform(0)
    rng = np.random.default_rng(12)
    n = 3_000_001
    x = rng.uniform(-1, 1, n)
    x[[5, 2_000_000, 2_999_999]] = -7.5          # the largest magnitude three times
    x[[17, 1_500_000]] = 1e-300                  # the smallest twice
    x[[100, 2_500_000]] = np.nan
    xv = pf.vector(x)
    assert (xv.ArgMin(), xv.ArgMax()) == (oracle.vec_reduce(x)[0], oracle.vec_reduce(x)[1]) == (17, 5)
    assert xv.NormMax() == 7.5
    x[0] = np.nan
    xv = pf.vector(x)
    assert (xv.ArgMin(), xv.ArgMax()) == (0, 0) == oracle.vec_reduce(x)[:2]
    x32 = rng.standard_normal(100_003).astype(np.float32)
    x32[[9, 99_999]] = np.float32(-40.0)
    v32 = pf.vector(x32, b200.F32)
    assert v32.ArgMax() == 9 and v32.NormMax() == 40.0
    assert v32.ArgMin() == int(np.argmin(np.abs(x32)))


@pytest.mark.gpu
def test_device_rot_fp32(b200):
    """FP32 Rot and Rotm: every product and sum rounded to float on its own."""
    pf = b200.Platform(0)
    rng = np.random.default_rng(4)
    x, y = rng.standard_normal(4099).astype(np.float32), rng.standard_normal(4099).astype(np.float32)
    c, s = np.float32(0.6), np.float32(0.8)
    a, b = pf.vector(x, b200.F32), pf.vector(y, b200.F32)
    a.Rot(b, 0.6, 0.8)
    assert np.array_equal(a.numpy(), c * x + s * y) and np.array_equal(b.numpy(), c * y - s * x)
    h = np.array([-1, 0.3, -0.7, 1.2, 0.9], np.float32)
    a, b = pf.vector(x, b200.F32), pf.vector(y, b200.F32)
    a.Rotm(b, h)
    assert np.array_equal(b.numpy(), y * h[1] + x * h[3]) and np.array_equal(a.numpy(), y * h[2] + x * h[4])


@pytest.mark.gpu
@pytest.mark.parametrize("dt", ["F64", "F32"])
def test_device_vector_index_and_range_access(b200, dt):
    """SetValues / GetValues / add_values with repeated indices, block and
    sub-vector copies, partial_add_subvector.  The expected values restate the
    reference's loops (lvector_cpu.cc:114-200, 419-545) one entry at a time,
    in the vector's own precision."""
    pf = b200.Platform(0)
    dtype = getattr(b200, dt)
    npt = np.float64 if dt == "F64" else np.float32
    rng = np.random.default_rng(8)
    n = 5000
    x0 = rng.standard_normal(n).astype(npt)
    idx = rng.integers(0, n, 3000).astype(np.int32)
    idx[:50] = 17                                  # one target fifty times
    vals = rng.standard_normal(3000).astype(npt)
    # add_values: buffer[indices[i]] += values[i], in order
    exp = x0.copy()
    for i, v in zip(idx, vals):
        exp[i] = npt(exp[i] + v)
    xv = pf.vector(x0, dtype)
    xv.add_values(idx, vals)
    assert np.array_equal(xv.numpy(), exp)
    xv.add_value(3, 2.5)
    exp[3] = npt(exp[3] + npt(2.5))
    assert np.array_equal(xv.numpy(), exp)
    # SetValues: buffer[index[i]] = values[i], the last write stays
    exp2 = x0.copy()
    for i, v in zip(idx, vals):
        exp2[i] = v
    xv = pf.vector(x0, dtype)
    xv.SetValues(idx, vals)
    assert np.array_equal(xv.numpy(), exp2)
    assert np.array_equal(xv.GetValues(idx[::7]), exp2[idx[::7]])
    # block and sub-vector copies
    xv.SetBlockValues(100, 140, np.arange(40))
    exp2[100:140] = np.arange(40)
    assert np.array_equal(xv.GetBlockValues(90, 150), exp2[90:150])
    sub = xv.extract_subvector(1000, 1300)
    assert np.array_equal(sub.numpy(), exp2[1000:1300])
    yv = pf.vector(n, dtype)
    yv.partial_replace_subvector(10, 5, 200, sub)
    expy = np.zeros(n, npt)
    expy[10:210] = exp2[1005:1205]
    assert np.array_equal(yv.numpy(), expy)
    yv.partial_add_subvector(0, 0, 300, 0.5, sub)
    expy[:300] += npt(0.5) * exp2[1000:1300]
    assert np.allclose(yv.numpy(), expy, rtol=0, atol=(1e-15 if dt == "F64" else 1e-6) * 4)
    with pytest.raises(b200.B200Error):
        xv.add_values([n], [1.0])
    with pytest.raises(b200.B200Error):
        xv.GetBlockValues(10, n + 1)


def test_rotg_host_abi_matches_reference(b200, gold):
    """b200la_rotg runs on the host: the library's own entry point (no GPU)
    against the reference's Rotg outputs, bit for bit, in FP64; FP32 against
    the same formulas evaluated in float."""
    import ctypes as C
    lib = b200.lib()
    for (a, b), ref in zip(gold["rotg_in"], gold["rotg_out"]):
        v = [C.c_double(a), C.c_double(b), C.c_double(), C.c_double()]
        assert lib.b200la_rotg(b200.F64, *[C.cast(C.byref(q), C.c_void_p) for q in v]) == 0
        assert bits(np.array([q.value for q in v])).tolist() == bits(ref).tolist()
    f = [C.c_float(3.0), C.c_float(4.0), C.c_float(), C.c_float()]
    assert lib.b200la_rotg(b200.F32, *[C.cast(C.byref(q), C.c_void_p) for q in f]) == 0
    assert [q.value for q in f] == [5.0, np.float32(1) / np.float32(0.6), np.float32(0.6), np.float32(0.8)]
    assert lib.b200la_rotg(7, None, None, None, None) == 1
