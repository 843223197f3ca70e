"""Solver parity at the full sizes of the four device configurations.

The reference's own CPU lmp code solved each configuration at its full size
(tests/golden/gen_config_counts.py and gen_c3_counts.py, run from oracle/_ref);
its iteration counts, colour / level structure and solution checksums are in
tests/golden/config_counts.json and c3_counts.json.  Bars:

- the assembled CSR arrays, the colouring / level permutation, the colour or
  level sizes and the permuted operator: bit-exact (SHA-256 of the bytes);
- iterations within +-5% of the reference's count, with the same stop state;
- the solution: its true relative residual, recomputed on the host in FP64
  (scipy CSR product), below 1.5 times the solve's tolerance (the stop test
  reads the recursive residual), and its 2-norm and its dot
  product with the seeded weight vector within 1e-6 relative of the
  reference solution's (two solutions at relative residual tol differ by at
  most about cond(A) * tol; the checksums are size-independent).
"""
import hashlib
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def counts():
    with open(os.path.join(HERE, "golden", "config_counts.json")) as f:
        d = json.load(f)
    with open(os.path.join(HERE, "golden", "c3_counts.json")) as f:
        d["c3"] = json.load(f)
    return d


@pytest.fixture(scope="module")
def pf(b200):
    return b200.Platform(0)


def sha(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def within5(got, want):
    return abs(got - want) <= max(1, int(np.ceil(0.05 * want)))


def host_relres(row, col, val, b, x):
    import scipy.sparse as sp
    n = len(row) - 1
    r = b - sp.csr_matrix((val, col, row), shape=(n, n)) @ x
    return float(np.linalg.norm(r) / np.linalg.norm(b))


def check_solution(row, col, val, b, x, ref, tol, w_seed):
    rel = host_relres(row, col, val, b, x)
    # the stop test reads the recursive residual, which drifts from the true one by rounding
    assert rel <= 1.5 * tol, (rel, tol)
    w = np.random.default_rng(w_seed).uniform(-1.0, 1.0, len(x))
    xn, xw = float(np.linalg.norm(x)), float(np.dot(w, x))
    assert abs(xn - ref["x_norm2"]) <= 1e-6 * ref["x_norm2"], (xn, ref["x_norm2"])
    assert abs(xw - ref["x_dot_w"]) <= 1e-6 * np.linalg.norm(w) * ref["x_norm2"], (xw, ref["x_dot_w"])
    return rel


def test_c1_jacobi_pcg_256(pf, b200, counts):
    c = counts["c1"]
    row, col, val = b200.q1_assemble(2, 256)
    assert sha(row, col, val) == c["csr_sha256"]
    b = b200.q1_rhs(42, 2, 256)
    A = b200.CSR_lMatrix.from_csr(pf, row, col, val)
    cg = b200.CG(pf)
    cg.SetupOperator(A)
    cg.SetupPreconditioner(b200.Preconditioner.Jacobi(pf, A))
    cg.InitControl(100000, 0.0, 1e-10, 1e6)
    x = pf.vector(len(b))
    assert cg.Solve(pf.vector(b), x) == b200.SUCCESS_REL == c["status"]
    assert within5(cg.iter(), c["iters"]), (cg.iter(), c["iters"])
    check_solution(row, col, val, b, x.numpy(), c, 1e-10, counts["w_seed"])


def test_c2_mcsgs_pcg_128cubed(pf, b200, counts):
    c = counts["c2"]
    row, col, val = b200.q1_assemble(3, 128)
    assert sha(row, col, val) == c["csr_sha256"]
    b = b200.q1_rhs(42, 3, 128)
    P = b200.Preconditioner.MultiColoringSGS(pf, row, col, val)
    assert P.nblocks == c["precond_colours"] == 8
    assert [int(v) for v in P.block_sizes] == c["precond_sizes"]
    assert sha(np.asarray(P.perm, np.int32)) == c["precond_perm_sha256"]
    Ar, Ac, Av = P.A_perm.download()
    assert sha(Ar, Ac, Av) == c["permuted_csr_sha256"]
    bp = b[P.perm]
    cg = b200.CG(pf)
    cg.SetupOperator(P.A_perm)
    cg.SetupPreconditioner(P)
    cg.InitControl(100000, 0.0, 1e-8, 1e6)
    x = pf.vector(len(bp))
    assert cg.Solve(pf.vector(bp), x) == b200.SUCCESS_REL == c["status"]
    assert within5(cg.iter(), c["iters"]), (cg.iter(), c["iters"])
    check_solution(Ar, Ac, Av, bp, x.numpy(), c, 1e-8, counts["w_seed"])


def test_c3_mixed_and_fp64_128cubed(pf, b200, counts):
    import importlib
    c = counts["c3"]
    wl = importlib.import_module("hiflow3_b200.workloads")
    row, col, val, b, _ = wl.system(b200, "c3")
    A64 = b200.CSR_lMatrix.from_csr(pf, row, col, val)
    A32 = A64.CastFrom(b200.F32)
    mp = b200.MPIR(pf, max_outer=50)
    mp.SetupOperator(A64)
    mp.SetupLowPrecisionOperator(A32)
    mp.InitControl(50, 0.0, 1e-10, 1e6)
    mp.InitInnerControl(100000, 0.0, 1e-4, 1e6)
    bv, x = pf.vector(b), pf.vector(len(b))
    assert mp.Solve(bv, x) == b200.SUCCESS_REL
    r = mp.result
    assert abs(r.outer - c["mpir_outer"]) <= 1, (r.outer, c["mpir_outer"])
    assert within5(r.iters, c["mpir_inner_total"]), (r.iters, c["mpir_inner_total"])
    assert host_relres(row, col, val, b, x.numpy()) <= 1e-10
    cg = b200.CG(pf)
    cg.SetupOperator(A64)
    cg.SetupPreconditioner(b200.Preconditioner.Jacobi(pf, A64))
    cg.InitControl(200000, 0.0, 1e-10, 1e6)
    x64 = pf.vector(len(b))
    assert cg.Solve(bv, x64) == b200.SUCCESS_REL
    assert within5(cg.iter(), c["fp64_cg_iters"]), (cg.iter(), c["fp64_cg_iters"])
    assert host_relres(row, col, val, b, x64.numpy()) <= 1e-10


def test_c4_gmres_ilu0_ls_512(pf, b200, counts):
    c = counts["c4"]
    row, col, val = b200.q1_assemble(2, 512, 1, None, 1e-3, (1.0, 0.5, 0.0))
    assert sha(row, col, val) == c["csr_sha256"]
    b = b200.q1_rhs(42, 2, 512)
    P = b200.Preconditioner.ILU0(pf, row, col, val, b200.PRECOND_ILU0_LS)
    assert P.nblocks == c["levels"] == 1537
    assert sha(np.asarray(P.block_sizes, np.int32)) == c["level_sizes_sha256"]
    assert sha(np.asarray(P.perm, np.int32)) == c["levelscheduling_perm_sha256"]
    Ar, Ac, Av = P.A_perm.download()
    assert sha(Ar, Ac, Av) == c["permuted_csr_sha256"]
    bp = b[P.perm]
    gm = b200.GMRES(pf, 30)
    gm.SetupOperator(P.A_perm)
    gm.SetupPreconditioner(P)
    gm.InitControl(100000, 0.0, 1e-9, 1e6)
    x = pf.vector(len(bp))
    assert gm.Solve(pf.vector(bp), x) == b200.SUCCESS_REL == c["status"]
    assert within5(gm.iter(), c["iters"]), (gm.iter(), c["iters"])
    check_solution(Ar, Ac, Av, bp, x.numpy(), c, 1e-9, counts["w_seed"])
