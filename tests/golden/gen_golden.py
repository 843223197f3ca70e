"""Generate the golden fixtures in tests/golden/ from HiFlow3's own CPU lmp code.

Runs oracle/_ref/libhiflow_lmp_ref.so (the reference's unmodified CPU lmp
sources compiled by oracle/Makefile) on small seeded inputs and writes
``lmp_golden.npz``.  The known-answer tests of the reference's own test suite
are written out beside them:

* test/LinearAlgebra/CPUsimple_CSR_lMatrix.cc:79-200 (add_values, unordered
  init_structure),
* test-legacy/lmp_test.cc:38-89 and test-legacy/cuda_test.cc:27-100 (SpMV),
* test/LinearAlgebra/cg.cc:35-91 and gmres.cc:35-91 (3x3 solve).

Usage:  make -C oracle REF=<HiFlow3 source tree> && python tests/golden/gen_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
from pyoracle import Oracle, Ref  # noqa: E402

CASES = [(2, 8), (2, 17), (3, 4), (3, 7)]
SOLVE_CASES = [(2, 32), (3, 12)]


def main():
    ref, orc = Ref(), Oracle()
    g = {}
    # --- KATs of the reference test suite ---
    r, c = ref.coo_to_csr(3, [1, 2, 0, 0, 1], [2, 1, 0, 1, 1])
    g["kat_unordered_sq_row"], g["kat_unordered_sq_col"] = r, c
    r, c = ref.coo_to_csr(3, [2, 0, 0, 1], [1, 0, 1, 1])
    g["kat_unordered_rect_row"], g["kat_unordered_rect_col"] = r, c
    r, c = ref.coo_to_csr(3, [0, 0, 1, 1, 1, 2, 2], [0, 1, 0, 1, 2, 1, 2])
    g["kat_addvalues_val"] = ref.add_values(r, c, np.zeros(7), [0, 1, 2], [0, 1, 2],
                                            np.arange(1.0, 10.0))
    r3 = np.array([0, 3, 6, 9], np.int32)
    c3 = np.array([0, 1, 2] * 3, np.int32)
    v3 = np.array([2, -1, 0, -1, 2, -1, 0, -1, 2.0])
    g["kat_spmv_lmp_y"] = ref.spmv(r3, c3, v3, np.array([1.0, -2.0, 0.0]))
    g["kat_spmv_cuda_y"] = ref.spmv(r3, c3, v3, np.array([1.2, -2.3, 0.7]))
    rc, x = ref.lmp_cg(r3, c3, v3, np.array([1.0, -2.0, 0.0]), 0.0, 0.0, 100)
    g["kat_cg_x"] = x
    # --- structured cases ---
    rng = np.random.default_rng(20261203)
    for dim, N in CASES:
        n, nnz = orc.q1_sizes(dim, N)
        kcell = np.exp(rng.standard_normal(N ** dim))
        x = rng.uniform(-1.0, 1.0, n)
        for kind, kc, tag in [(0, None, "p"), (0, kcell, "pk"), (1, None, "cd")]:
            key = f"{dim}d{N}_{tag}"
            row, col, val = ref.q1_assemble(dim, N, kind, kc, nu=1e-3, beta=(1.0, 0.5, 0.25))
            g[key + "_row"], g[key + "_col"], g[key + "_val"] = row, col, val
            if kc is not None:
                g[key + "_kcell"] = kc
            g[key + "_x"] = x
            g[key + "_y"] = ref.spmv(row, col, val, x)
            g[key + "_dot"] = np.array([ref.dot(x, g[key + "_y"])])
            nc, sizes, perm = ref.multicoloring(row, col, val)
            g[key + "_mc_sizes"], g[key + "_mc_perm"] = sizes, perm
            nl, lsz, lperm = ref.levelscheduling(row, col, val)
            g[key + "_ls_sizes"], g[key + "_ls_perm"] = lsz, lperm
            ro = ref.reorder(row, col, val, perm)
            g[key + "_re_row"], g[key + "_re_col"], g[key + "_re_val"] = ro
            lu = ref.ilu0(row, col, val)
            g[key + "_ilu0"] = lu
            g[key + "_ilusolve"] = ref.ilu_solve(row, col, lu, x)
            for kindp, name in [(2, "mcsgs"), (3, "iluls"), (4, "ilumc")]:
                # r in the permuted numbering: the same x, permuted by the block order
                res = ref.block_precond(kindp, row, col, val, x)
                g[f"{key}_{name}_perm"] = res["perm"]
                g[f"{key}_{name}_sizes"] = res["sizes"]
                g[f"{key}_{name}_z"] = res["z"]
                g[f"{key}_{name}_Arow"], g[f"{key}_{name}_Acol"], g[f"{key}_{name}_Aval"] = res["A"]
    # --- solves ---
    for dim, N in SOLVE_CASES:
        key = f"solve{dim}d{N}"
        row, col, val = ref.q1_assemble(dim, N)
        b = orc.q1_rhs(42, dim, N)
        g[key + "_b"] = b
        for p, name, tol in [(0, "none", 1e-10), (1, "jacobi", 1e-10), (2, "mcsgs", 1e-8)]:
            if p == 2:
                perm = ref.block_precond(2, row, col, val, b)["perm"]
                rhs = b[perm]
            else:
                rhs = b
            out = ref.pcg(row, col, val, rhs, precond=p, maxits=5000, reltol=tol, history=True)
            g[f"{key}_{name}_iters"] = np.array([out["iters"]])
            g[f"{key}_{name}_x"] = out["x"]
            g[f"{key}_{name}_hist"] = out["history"]
    row, col, val = ref.q1_assemble(2, 32, 1, None, nu=1e-3, beta=(1.0, 0.5))
    b = orc.q1_rhs(7, 2, 32)
    g["gmres2d32_b"] = b
    perm = ref.block_precond(3, row, col, val, b)["perm"]
    out = ref.gmres(row, col, val, b[perm], precond=3, m=30, maxits=1000, reltol=1e-9)
    g["gmres2d32_iluls_iters"] = np.array([out["iters"]])
    g["gmres2d32_iluls_x"] = out["x"]
    out = ref.gmres(row, col, val, b, precond=0, m=30, maxits=3000, reltol=1e-9)
    g["gmres2d32_none_iters"] = np.array([out["iters"]])
    g["gmres2d32_none_x"] = out["x"]
    np.savez_compressed(os.path.join(HERE, "lmp_golden.npz"), **g)
    print("wrote", len(g), "arrays")


if __name__ == "__main__":
    main()
