"""MatrixMarket and vector file I/O against HiFlow3's own reader and writer.

The fixtures (tests/golden/mm/, made by gen_mm_golden.py) hold this project's
own seeded input files together with what the reference's
CPU_CSR_lMatrix::ReadFile / WriteFile and CPU_lVector::ReadFile / WriteFile
(lmp/lmatrix_csr_cpu.cc:1733-1765, lmp/lmatrix_coo_cpu.cc:133-299,
lmp/lvector_cpu.cc:582-663) produced from them.  Reading must give the
reference's CSR entry for entry, writing its text byte for byte.
"""
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
MM = os.path.join(HERE, "golden", "mm")
MATRICES = ["general", "symmetric", "integer_rect", "skew", "random200"]


@pytest.fixture(scope="module")
def pf(b200):
    return b200.Platform(0)


@pytest.fixture(scope="module")
def gold():
    return np.load(os.path.join(MM, "mm_golden.npz"))


@pytest.mark.parametrize("name", MATRICES)
def test_mm_read_matches_reference(b200, gold, name):
    row, col, val, m = b200.read_matrix_market(os.path.join(MM, name + ".mtx"))
    n_ref, m_ref, nnz_ref = (int(v) for v in gold[f"{name}_shape"])
    assert (row.size - 1, m, col.size) == (n_ref, m_ref, nnz_ref)
    assert np.array_equal(row, gold[f"{name}_row"])
    assert np.array_equal(col, gold[f"{name}_col"])
    assert np.array_equal(val.view(np.uint64), gold[f"{name}_val"].view(np.uint64))


def test_mm_symmetric_expansion(b200, gold):
    # every off-diagonal entry of the lower triangle appears with its mirror
    row, col, val, _ = b200.read_matrix_market(os.path.join(MM, "symmetric.mtx"))
    n = row.size - 1
    A = np.zeros((n, n))
    for i in range(n):
        for j in range(row[i], row[i + 1]):
            A[i, col[j]] += val[j]
    assert np.array_equal(A, A.T)


@pytest.mark.parametrize("name", ["general", "integer_rect", "random200"])
def test_mm_write_matches_reference(b200, gold, name, tmp_path):
    n, m, _ = (int(v) for v in gold[f"{name}_shape"])
    p = tmp_path / "out.mtx"
    b200.write_matrix_market(p, gold[f"{name}_row"], gold[f"{name}_col"], gold[f"{name}_val"], n_cols=m)
    assert p.read_bytes() == bytes(gold[f"{name}_written"])


def test_mm_write_read_is_transpose(b200, gold, tmp_path):
    # the reference writes "column row value": reading a written file gives A^T
    row, col, val = gold["random200_row"], gold["random200_col"], gold["random200_val"]
    p = tmp_path / "t.mtx"
    b200.write_matrix_market(p, row, col, val)
    r2, c2, v2, _ = b200.read_matrix_market(p)
    n = row.size - 1
    A, B = np.zeros((n, n)), np.zeros((n, n))
    for i in range(n):
        for j in range(row[i], row[i + 1]):
            A[i, col[j]] += val[j]
        for j in range(r2[i], r2[i + 1]):
            B[i, c2[j]] += v2[j]
    assert np.allclose(B, A.T, rtol=1e-13, atol=0)


@pytest.mark.parametrize("name", ["vec_newline", "vec_no_newline", "vec_exp"])
def test_vec_read_matches_reference(b200, gold, name):
    x = b200.read_vector(os.path.join(MM, name + ".vec"))
    assert np.array_equal(x, gold[f"{name}_values"])


def test_vec_write_matches_reference(b200, gold, tmp_path):
    p = tmp_path / "v.txt"
    b200.write_vector(p, gold["vecwrite_input"])
    assert p.read_bytes() == bytes(gold["vecwrite_written"])


@pytest.mark.parametrize("text,code", [
    ("%%MatrixMarket matrix coordinate pattern general\n2 2 1\n1 1\n", "ERR_FORMAT"),
    ("%%MatrixMarket matrix coordinate complex general\n2 2 1\n1 1 1.0 0.0\n", "ERR_FORMAT"),
    ("%%MatrixMarket matrix array real general\n2 2\n1\n2\n3\n4\n", "ERR_FORMAT"),
    ("%%MatrixMarket matrix coordinate real hermitian\n2 2 1\n1 1 1.0\n", "ERR_FORMAT"),
    ("MatrixMarket matrix coordinate real general\n2 2 1\n1 1 1.0\n", "ERR_FORMAT"),
    ("%%MatrixMarket matrix coordinate real general\n2 2 3\n1 1 1.0\n2 2 2.0\n", "ERR_FORMAT"),
    ("%%MatrixMarket matrix coordinate real general\n2 2 1\n3 1 1.0\n", "ERR_CSR"),
    ("%%MatrixMarket matrix coordinate real general\n", "ERR_FORMAT"),
])
def test_mm_read_rejects(b200, tmp_path, text, code):
    # the reference exits the process on these; the platform returns a status
    p = tmp_path / "bad.mtx"
    p.write_text(text)
    with pytest.raises(b200.B200Error) as e:
        b200.read_matrix_market(p)
    assert e.value.code == getattr(b200, code)


def test_missing_files(b200, tmp_path):
    with pytest.raises(b200.B200Error) as e:
        b200.read_matrix_market(tmp_path / "nope.mtx")
    assert e.value.code == b200.ERR_IO
    with pytest.raises(b200.B200Error) as e:
        b200.read_vector(tmp_path / "nope.vec")
    assert e.value.code == b200.ERR_IO
    with pytest.raises(b200.B200Error) as e:
        b200.write_vector(tmp_path / "no_dir" / "v.txt", np.ones(3))
    assert e.value.code == b200.ERR_IO


@pytest.mark.gpu
def test_mm_file_to_device_spmv(b200, pf, gold, tmp_path):
    """A MatrixMarket file read onto the device and multiplied equals the
    reference's CSR times x; the device matrix written back gives the
    reference's text."""
    A = b200.CSR_lMatrix.ReadFile(pf, os.path.join(MM, "random200.mtx"))
    row, col, val = gold["random200_row"], gold["random200_col"], gold["random200_val"]
    x = np.random.default_rng(1).uniform(-1, 1, 200)
    y = pf.vector(200)
    A.VectorMult(pf.vector(x), y)
    ref = np.array([np.dot(val[row[i]:row[i + 1]], x[col[row[i]:row[i + 1]]]) for i in range(200)])
    scale = np.array([np.abs(val[row[i]:row[i + 1]]) @ np.abs(x[col[row[i]:row[i + 1]]]) for i in range(200)])
    assert np.all(np.abs(y.numpy() - ref) <= 1e-13 * np.maximum(scale, 1e-300))
    p = tmp_path / "dev.mtx"
    A.WriteFile(p)
    assert p.read_bytes() == bytes(gold["random200_written"])
    v = pf.vector_from_file(os.path.join(MM, "vec_newline.vec"))
    assert np.array_equal(v.numpy(), gold["vec_newline_values"])
