"""ILU(p) with powered patterns (lPreconditioner_MultiColoring_ILUp with ilu_p > 0).

Fixtures (tests/golden/ilup_golden.npz, gen_ilup_golden.py) come from the
reference's own CPU code: MatrixSupSPower, ilup, the ILU(p) block
preconditioner build and apply, and GMRES(30) with ILU(1).  The platform's
host set-up and the oracle must reproduce the patterns and factors bit for
bit; the device preconditioner and solver are checked within the tolerances
of the other preconditioner tests.
"""
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = ["2d17_cd", "3d6_p", "2d12_pk"]
BUILDS = [(3, 1, 1), (3, 2, 1), (4, 1, 1), (4, 2, 1), (4, 1, 2), (4, 0, 2)]


@pytest.fixture(scope="module")
def gold():
    return np.load(os.path.join(HERE, "golden", "ilup_golden.npz"))


def same_bits(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return a.shape == b.shape and np.array_equal(a.view(np.uint8), b.view(np.uint8))


def A(gold, key):
    return gold[key + "_row"], gold[key + "_col"], gold[key + "_val"]


@pytest.mark.parametrize("key", CASES)
def test_power_pattern_and_factors_match_reference(b200, oracle, gold, key):
    row, col, val = A(gold, key)
    for p in (2, 3):
        ref = (gold[f"{key}_pow{p}_row"], gold[f"{key}_pow{p}_col"])
        for got in (b200.matrix_power_pattern(row, col, p), oracle.power_pattern(row, col, p)):
            assert same_bits(got[0], ref[0]) and same_bits(got[1], ref[1])
    for p in (1, 2):
        ref = (gold[f"{key}_ilu{p}_row"], gold[f"{key}_ilu{p}_col"], gold[f"{key}_ilu{p}_val"])
        for got in (b200.ilup(row, col, val, p), oracle.ilup(row, col, val, p)):
            assert all(same_bits(x, y) for x, y in zip(got, ref))


@pytest.mark.parametrize("key", CASES)
@pytest.mark.parametrize("mode,p,mp", BUILDS)
def test_oracle_ilup_build_matches_reference(oracle, gold, key, mode, p, mp):
    row, col, val = A(gold, key)
    P, (Ar, Ac, Av) = oracle.ilup_build(row, col, val, 0 if mode == 3 else 1, p, mp)
    b = f"{key}_b{mode}_{p}_{mp}"
    assert np.array_equal(P.perm, gold[b + "_perm"])
    assert np.array_equal(np.diff(P.block_off), gold[b + "_sizes"])
    assert same_bits(Av, gold[b + "_Aval"])
    assert same_bits(P.apply(gold[key + "_r"]), gold[b + "_z"])


def test_ilup_rejects(b200):
    row = np.array([0, 1, 2], np.int32)
    col = np.array([1, 0], np.int32)   # no diagonal
    with pytest.raises(b200.B200Error):
        b200.ilup(row, col, np.ones(2), 1)
    with pytest.raises(b200.B200Error):
        b200.matrix_power_pattern(row, col, 0)


@pytest.fixture(scope="module")
def pf(b200):
    return b200.Platform(0)


@pytest.mark.gpu
@pytest.mark.parametrize("key", CASES)
@pytest.mark.parametrize("mode,p,mp", BUILDS)
def test_ilup_precond_apply(pf, b200, gold, key, mode, p, mp):
    row, col, val = A(gold, key)
    P = b200.Preconditioner.ILUp(pf, row, col, val, p, mp, mode)
    b = f"{key}_b{mode}_{p}_{mp}"
    assert np.array_equal(P.perm, gold[b + "_perm"])
    assert np.array_equal(P.block_sizes, gold[b + "_sizes"])
    r = gold[key + "_r"]
    z = pf.vector(len(r))
    for _ in range(2):
        P.ApplyPreconditioner(pf.vector(r), z)
        zr = gold[b + "_z"]
        assert np.max(np.abs(z.numpy() - zr)) <= 1e-12 * np.max(np.abs(zr))


@pytest.mark.gpu
def test_gmres_ilu1_ls_vs_reference(pf, b200, gold):
    row, col, val = b200.q1_assemble(2, 32, 1, None, 1e-3, (1.0, 0.5))
    P = b200.Preconditioner.ILUp(pf, row, col, val, 1, 1, b200.PRECOND_ILU0_LS)
    b = gold["gmres2d32_b"][P.perm]
    gm = b200.GMRES(pf, 30)
    gm.SetupOperator(P.A_perm)
    gm.SetupPreconditioner(P)
    gm.InitControl(1000, 0.0, 1e-9, 1e6)
    x = pf.vector(len(b))
    assert gm.Solve(pf.vector(b), x) == b200.SUCCESS_REL
    ref_it = int(gold["gmres2d32_ilu1ls_iters"][0])
    assert abs(gm.iter() - ref_it) <= max(1, 0.05 * ref_it), (gm.iter(), ref_it)
    xr = gold["gmres2d32_ilu1ls_x"]
    assert np.linalg.norm(x.numpy() - xr) <= 1e-7 * np.linalg.norm(xr)
