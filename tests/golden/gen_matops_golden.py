"""Generate tests/golden/matops_golden.npz from HiFlow3's own CPU lmp code.

Matrices: the reference's CPU_CSR_lMatrix::Scale, ScaleOffdiag, Zeros,
extract_diagelements, extract_invdiagelements, extract_submatrix and Compress
(oracle/_ref/libhiflow_lmp_ref.so, the reference's unmodified sources) on
this project's seeded inputs: random CSRs with unsorted rows, repeated
columns and stored zeros (square and rectangular), and a 2-D Q1
convection-diffusion system whose Dirichlet rows hold stored zeros.
Vectors: CPUsimple_lVector::ArgMin, ArgMax, Norm1, NormMax, Rot, Rotm and
Rotg on seeded vectors with repeated magnitudes, signed zeros and lengths
around the reference's unroll-by-5.  The inputs and the reference's outputs
go into the fixture.

Usage:  make -C oracle REF=<HiFlow3 source tree> && python tests/golden/gen_matops_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
from pyoracle import Oracle, Ref  # noqa: E402

ALPHA = 1.7
BLOCKS = {"rand": [(0, 0, 60, 60), (5, 7, 40, 33), (10, 0, 11, 60), (59, 59, 60, 60)],
          "rect": [(0, 0, 50, 70), (3, 52, 47, 70), (20, 10, 30, 65)],
          "q1": [(0, 0, 121, 121), (11, 11, 110, 110), (40, 30, 80, 95)]}

VEC_SIZES = [1, 7, 10, 1003]
ROT_CS = [(0.6, 0.8), (-0.3, 0.95)]
ROTM_PARAMS = [(-1, 0.3, -0.7, 1.2, 0.9), (0, 9, 0.25, -0.5, 9), (1, 1.5, 9, 9, -0.4), (-2, 1, 2, 3, 4)]
ROTG_IN = [(3.0, 4.0), (-2.0, 1.0), (0.0, 0.0), (0.0, 5.0), (1e-300, -3e-300), (7.0, 0.0), (-1.5, -2.5)]


def rand_csr(rng, n, m):
    """Unsorted rows, a repeated column in some rows, stored zeros."""
    rows = []
    for i in range(n):
        k = int(rng.integers(0, 9))
        c = list(rng.choice(m, size=min(k, m), replace=False))
        if i < m and rng.random() < 0.8 and i not in c:
            c.append(i)
        if c and rng.random() < 0.2:
            c.append(c[0])
        rng.shuffle(c)
        rows.append(c)
    row = np.zeros(n + 1, np.int32)
    row[1:] = np.cumsum([len(r) for r in rows])
    col = np.array([x for r in rows for x in r], np.int32)
    val = rng.standard_normal(len(col))
    val[rng.random(len(col)) < 0.1] = 0.0
    return row, col, val


def main():
    R = Ref()
    rng = np.random.default_rng(20261204)
    cases = {"rand": rand_csr(rng, 60, 60) + (60,), "rect": rand_csr(rng, 50, 70) + (70,)}
    row, col, val = Oracle().q1_assemble(2, 10, 1, None, nu=1e-2, beta=(1.0, 0.5))
    cases["q1"] = (row, col, val, len(row) - 1)
    g = {}
    for name, (row, col, val, m) in cases.items():
        n = len(row) - 1
        g[f"{name}_row"], g[f"{name}_col"], g[f"{name}_val"], g[f"{name}_m"] = row, col, val, np.int64(m)
        for mode in (0, 1, 2):
            g[f"{name}_scale{mode}"] = R.csr_scale(row, col, val, ALPHA, mode, m=m)
        lo, hi = 3, min(n, m) - 2
        g[f"{name}_has_diag"] = np.array([i in col[row[i]:row[i + 1]] for i in range(lo, hi)])
        for inv in (0, 1):
            g[f"{name}_diag{inv}"] = R.csr_diag(row, col, val, lo, hi, inv, m=m)
        g[f"{name}_diag_range"] = np.array([lo, hi])
        for k, (sr, sc, er, ec) in enumerate(BLOCKS[name]):
            r, c, v = R.csr_extract(row, col, val, 0, sr, sc, er, ec, m=m)
            g[f"{name}_sub{k}_row"], g[f"{name}_sub{k}_col"], g[f"{name}_sub{k}_val"] = r, c, v
        r, c, v = R.csr_extract(row, col, val, 1, m=m)
        g[f"{name}_comp_row"], g[f"{name}_comp_col"], g[f"{name}_comp_val"] = r, c, v
    for k, n in enumerate(VEC_SIZES):
        x, y = rng.standard_normal(n), rng.standard_normal(n)
        if n > 6:
            x[n - 2] = -x[1]            # repeated magnitudes: the first index wins
            x[n // 2] = 0.0
            x[n // 3] = -0.0
        g[f"vec{k}_x"], g[f"vec{k}_y"] = x, y
        g[f"vec{k}_reduce"] = np.array(R.vec_reduce(x), dtype=np.float64)
        for j, (c, s) in enumerate(ROT_CS):
            g[f"vec{k}_rot{j}_x"], g[f"vec{k}_rot{j}_y"] = R.rot(x, y, c, s)
        for j, prm in enumerate(ROTM_PARAMS):
            g[f"vec{k}_rotm{j}_x"], g[f"vec{k}_rotm{j}_y"] = R.rot(x, y, param=np.array(prm, np.float64))
    g["rotg_in"] = np.array(ROTG_IN, np.float64)
    g["rotg_out"] = np.array([R.rotg(a, b) for a, b in ROTG_IN], np.float64)
    g["alpha"] = np.float64(ALPHA)
    out = os.path.join(HERE, "matops_golden.npz")
    np.savez_compressed(out, **g)
    print("wrote", out, len(g), "arrays")


if __name__ == "__main__":
    main()
