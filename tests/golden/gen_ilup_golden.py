"""Generate the ILU(p) fixtures (tests/golden/ilup_golden.npz) from HiFlow3's own CPU lmp code.

Runs oracle/_ref/libhiflow_lmp_ref.so (the reference's unmodified CPU lmp
sources) on small Q1 operators assembled by the reference's own code path:
  - CPU_CSR_lMatrix::MatrixSupSPower (lmatrix_csr_cpu.cc:1641-1664): powered patterns;
  - CPU_CSR_lMatrix::ilup (lmatrix_csr_cpu.cc:1933-2104): ILU(p) factors;
  - lPreconditioner_MultiColoring_ILUp (lpreconditioner_mc_ilup.cc:84-262) with
    ILU(p) and the colouring on the pattern of A^mat_power: permutation, block
    sizes, permuted operator and one apply;
  - right-preconditioned GMRES(30) with ILU(1) level-scheduled: iterations and x.

Usage:  make -C oracle REF=<HiFlow3 source tree> && python tests/golden/gen_ilup_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
from pyoracle import Oracle, Ref  # noqa: E402

CASES = [(2, 17, 1, "cd"), (3, 6, 0, "p"), (2, 12, 0, "pk")]
BUILDS = [(3, 1, 1), (3, 2, 1), (4, 1, 1), (4, 2, 1), (4, 1, 2), (4, 0, 2)]   # (mode, ilu_p, mat_power)


def main():
    ref, orc = Ref(), Oracle()
    g = {}
    for dim, N, kind, tag in CASES:
        key = f"{dim}d{N}_{tag}"
        kc = np.exp(np.random.default_rng(N).standard_normal(N ** dim)) if tag == "pk" else None
        row, col, val = ref.q1_assemble(dim, N, kind, kc, nu=1e-2, beta=(1.0, 0.5, 0.25))
        n = len(row) - 1
        g[key + "_row"], g[key + "_col"], g[key + "_val"] = row, col, val
        for p in (2, 3):
            r, c = ref.power_pattern(row, col, p)
            g[f"{key}_pow{p}_row"], g[f"{key}_pow{p}_col"] = r, c
        for p in (1, 2):
            r, c, v = ref.ilup(row, col, val, p)
            g[f"{key}_ilu{p}_row"], g[f"{key}_ilu{p}_col"], g[f"{key}_ilu{p}_val"] = r, c, v
        rv = orc.q1_rhs(11, dim, N)
        g[key + "_r"] = rv
        for mode, p, mp in BUILDS:
            out = ref.block_precond_ilup(mode, p, mp, row, col, val, rv)
            b = f"{key}_b{mode}_{p}_{mp}"
            g[b + "_perm"], g[b + "_sizes"], g[b + "_z"] = out["perm"], out["sizes"], out["z"]
            g[b + "_Aval"] = out["A"][2]
    row, col, val = ref.q1_assemble(2, 32, 1, None, nu=1e-3, beta=(1.0, 0.5))
    b = orc.q1_rhs(7, 2, 32)
    perm = ref.block_precond_ilup(3, 1, 1, row, col, val, b)["perm"]
    out = ref.gmres(row, col, val, b[perm], precond=3, m=30, maxits=1000, reltol=1e-9, ilu_p=1)
    g["gmres2d32_b"] = b
    g["gmres2d32_ilu1ls_iters"] = np.array([out["iters"]])
    g["gmres2d32_ilu1ls_x"] = out["x"]
    np.savez_compressed(os.path.join(HERE, "ilup_golden.npz"), **g)
    print("wrote", len(g), "arrays; GMRES ILU(1)-LS iterations", out["iters"])


if __name__ == "__main__":
    main()
