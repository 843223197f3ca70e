"""Pins the C restatement (oracle/oracle.c) to HiFlow3's own CPU lmp code.

The fixtures in tests/golden/lmp_golden.npz were produced by
tests/golden/gen_golden.py from the reference sources compiled unmodified
(oracle/_ref).  Integer and index results must match exactly; floating-point
results too, because the restatement keeps the reference's operation order.
"""
import numpy as np
import pytest

from pyoracle import control

CASES = [(2, 8), (2, 17), (3, 4), (3, 7)]
TAGS = [("p", 0), ("pk", 0), ("cd", 1)]


def test_kat_unordered_init_structure(oracle, golden):
    # test/LinearAlgebra/CPUsimple_CSR_lMatrix.cc:159-200
    r, c = oracle.coo_to_csr(3, [1, 2, 0, 0, 1], [2, 1, 0, 1, 1])
    assert r.tolist() == [0, 2, 4, 5] and c.tolist() == [0, 1, 1, 2, 1]
    assert np.array_equal(r, golden["kat_unordered_sq_row"]) and np.array_equal(c, golden["kat_unordered_sq_col"])
    r, c = oracle.coo_to_csr(3, [2, 0, 0, 1], [1, 0, 1, 1])
    assert r.tolist() == [0, 2, 3, 4] and c.tolist() == [0, 1, 1, 1]
    assert np.array_equal(r, golden["kat_unordered_rect_row"])


def test_kat_add_values(oracle, golden):
    # test/LinearAlgebra/CPUsimple_CSR_lMatrix.cc:79-99
    r, c = oracle.coo_to_csr(3, [0, 0, 1, 1, 1, 2, 2], [0, 1, 0, 1, 2, 1, 2])
    v = oracle.add_values(r, c, np.zeros(7), [0, 1, 2], [0, 1, 2], np.arange(1.0, 10.0))
    assert v.tolist() == [1, 2, 4, 5, 6, 8, 9]
    assert np.array_equal(v, golden["kat_addvalues_val"])


def test_kat_spmv(oracle, golden):
    # test-legacy/lmp_test.cc:38-89, test-legacy/cuda_test.cc:27-100
    row = np.array([0, 3, 6, 9], np.int32)
    col = np.array([0, 1, 2] * 3, np.int32)
    val = np.array([2, -1, 0, -1, 2, -1, 0, -1, 2.0])
    y = oracle.spmv(row, col, val, np.array([1.0, -2.0, 0.0]))
    np.testing.assert_allclose(y, [4.0, -5.0, 2.0], atol=1e-12)
    assert np.array_equal(y, golden["kat_spmv_lmp_y"])
    y = oracle.spmv(row, col, val, np.array([1.2, -2.3, 0.7]))
    np.testing.assert_allclose(y, [4.7, -6.5, 3.7], atol=1e-12)
    assert np.array_equal(y, golden["kat_spmv_cuda_y"])


def test_kat_cg(oracle, golden):
    # test/LinearAlgebra/cg.cc:35-91: x = (-0.25, -1.5, -0.75); an absolute
    # tolerance of 1e-300 stops on the exact zero residual the 3x3 system reaches
    row = np.array([0, 3, 6, 9], np.int32)
    col = np.array([0, 1, 2] * 3, np.int32)
    val = np.array([2, -1, 0, -1, 2, -1, 0, -1, 2.0])
    out = oracle.pcg(row, col, val, np.array([1.0, -2.0, 0.0]), ctl=control(100, 1e-300, 0.0, 1e6))
    np.testing.assert_allclose(out["x"], [-0.25, -1.5, -0.75], atol=1e-12)
    np.testing.assert_allclose(out["x"], golden["kat_cg_x"], atol=1e-12)
    out = oracle.gmres(row, col, val, np.array([1.0, -2.0, 0.0]), ctl=control(100, 1e-300, 0.0, 1e6))
    np.testing.assert_allclose(out["x"], [-0.25, -1.5, -0.75], atol=1e-12)


@pytest.mark.parametrize("dim,N", CASES)
@pytest.mark.parametrize("tag,kind", TAGS)
def test_assembly_and_kernels_bit_exact(oracle, golden, dim, N, tag, kind):
    key = f"{dim}d{N}_{tag}"
    kc = golden.get(key + "_kcell")
    row, col, val = oracle.q1_assemble(dim, N, kind, kc, nu=1e-3, beta=(1.0, 0.5, 0.25))
    assert np.array_equal(row, golden[key + "_row"])
    assert np.array_equal(col, golden[key + "_col"])
    assert np.array_equal(val, golden[key + "_val"])
    x = golden[key + "_x"]
    y = oracle.spmv(row, col, val, x)
    assert np.array_equal(y, golden[key + "_y"])
    assert oracle.dot(x, y) == golden[key + "_dot"][0]
    nc, sizes, perm = oracle.multicoloring(row, col)
    assert np.array_equal(sizes, golden[key + "_mc_sizes"]) and np.array_equal(perm, golden[key + "_mc_perm"])
    if dim == 3:
        assert nc == 8   # 27-point stencil: eight colours
    nl, lsz, lperm = oracle.levelscheduling(row, col)
    assert np.array_equal(lsz, golden[key + "_ls_sizes"]) and np.array_equal(lperm, golden[key + "_ls_perm"])
    ro = oracle.reorder(row, col, val, perm)
    for a, s in zip(ro, ("row", "col", "val")):
        assert np.array_equal(a, golden[f"{key}_re_{s}"])
    lu = oracle.ilu0(row, col, val)
    assert np.array_equal(lu, golden[key + "_ilu0"])
    assert np.array_equal(oracle.ilu_solve(row, col, lu, x), golden[key + "_ilusolve"])


@pytest.mark.parametrize("dim,N", CASES)
@pytest.mark.parametrize("tag,kind", TAGS)
@pytest.mark.parametrize("name", ["mcsgs", "iluls", "ilumc"])
def test_block_preconditioners_bit_exact(oracle, golden, dim, N, tag, kind, name):
    key = f"{dim}d{N}_{tag}"
    row, col, val = golden[key + "_row"], golden[key + "_col"], golden[key + "_val"]
    if name == "mcsgs":
        P, A = oracle.mcsgs_build(row, col, val)
    else:
        P, A = oracle.ilu0_build(row, col, val, 0 if name == "iluls" else 1)
    assert np.array_equal(P.perm, golden[f"{key}_{name}_perm"])
    assert np.array_equal(np.diff(P.block_off), golden[f"{key}_{name}_sizes"])
    for a, s in zip(A, ("Arow", "Acol", "Aval")):
        assert np.array_equal(a, golden[f"{key}_{name}_{s}"])
    z = P.apply(golden[key + "_x"])
    assert np.array_equal(z, golden[f"{key}_{name}_z"])


@pytest.mark.parametrize("dim,N", [(2, 32), (3, 12)])
def test_pcg_bit_exact(oracle, golden, dim, N):
    key = f"solve{dim}d{N}"
    row, col, val = oracle.q1_assemble(dim, N)
    b = oracle.q1_rhs(42, dim, N)
    assert np.array_equal(b, golden[key + "_b"])
    for name, pre, tol in [("none", None, 1e-10), ("jacobi", "jacobi", 1e-10), ("mcsgs", "mcsgs", 1e-8)]:
        if pre == "jacobi":
            out = oracle.pcg(row, col, val, b, precond=oracle.invdiag(row, col, val),
                             ctl=control(5000, 0, tol, 1e6), history=True)
        elif pre == "mcsgs":
            P, (Ar, Ac, Av) = oracle.mcsgs_build(row, col, val)
            out = oracle.pcg(Ar, Ac, Av, b[P.perm], precond=P, ctl=control(5000, 0, tol, 1e6), history=True)
        else:
            out = oracle.pcg(row, col, val, b, ctl=control(5000, 0, tol, 1e6), history=True)
        assert out["iters"] == golden[f"{key}_{name}_iters"][0]
        assert np.array_equal(out["x"], golden[f"{key}_{name}_x"])
        assert np.array_equal(out["history"], golden[f"{key}_{name}_hist"])


def test_gmres_ilu_bit_exact(oracle, golden):
    row, col, val = oracle.q1_assemble(2, 32, 1, None, nu=1e-3, beta=(1.0, 0.5))
    b = golden["gmres2d32_b"]
    P, (Ar, Ac, Av) = oracle.ilu0_build(row, col, val, 0)
    out = oracle.gmres(Ar, Ac, Av, b[P.perm], precond=P, m=30, ctl=control(1000, 0, 1e-9, 1e6))
    assert out["iters"] == golden["gmres2d32_iluls_iters"][0]
    assert np.array_equal(out["x"], golden["gmres2d32_iluls_x"])
    out = oracle.gmres(row, col, val, b, m=30, ctl=control(3000, 0, 1e-9, 1e6))
    assert out["iters"] == golden["gmres2d32_none_iters"][0]
    assert np.array_equal(out["x"], golden["gmres2d32_none_x"])


def test_q1_sizes_match_workloads(oracle):
    # 2-D 256^2 and 3-D 128^3 Q1 systems
    assert oracle.q1_sizes(2, 256) == (66049, 591361)
    assert oracle.q1_sizes(3, 128) == (2146689, 57066625)
    assert oracle.q1_sizes(2, 512) == (263169, 2362369)   # (3*512+1)^2
