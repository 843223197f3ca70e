"""Full-size reference results of the four device configurations, from the
reference's own CPU lmp code (oracle/_ref), written to config_counts.json.

For every configuration the reference assembles the system itself
(init_structure + add_values + ZeroRows of its CPU_CSR_lMatrix) and solves
it with its own lmp objects driving the CG / GMRES loops of
src/linear_solver/cg.cc:164-248 and gmres.cc:285-510:

  c1  2-D Q1 Poisson 256^2, Jacobi-PCG to 1e-10
  c2  3-D Q1 Poisson 128^3, 8-colour MC-SGS PCG to 1e-8
      (lPreconditioner_MultiColoring_SymmetricGaussSeidel: colours, colour
      sizes and the permutation from CPU_CSR_lMatrix::Multicoloring,
      lmatrix_csr_cpu.cc:2175-2290)
  c3  3-D Q1 128^3 with k = exp(GRF): see c3_counts.json (gen_c3_counts.py)
  c4  2-D Q1 convection-diffusion 512^2, GMRES(30) + ILU(0) level-scheduled
      to 1e-9 (levels and permutation from Levelscheduling,
      lmatrix_csr_cpu.cc:2295-2392)

Recorded: SHA-256 of the assembled CSR arrays (row, col, val bytes), the
colour / level counts, sizes and a SHA-256 of the permutation, the iteration
count, stop state and final residual, and two size-independent checksums of
the solution (its 2-norm and its dot product with a seeded weight vector
w = numpy default_rng(7).uniform(-1, 1, n)), plus its true relative residual.
The solution vectors themselves (17 MB at 128^3) are not stored.

Usage:  make -C oracle REF=<HiFlow3 source tree> && python tests/golden/gen_config_counts.py [c1 c2 c4]
"""
import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.join(HERE, "..", "..")
sys.path.insert(0, os.path.join(ROOT, "oracle"))
from pyoracle import Oracle, Ref  # noqa: E402

OUT = os.path.join(HERE, "config_counts.json")
W_SEED = 7


def sha(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def spmv(row, col, val, x):
    import scipy.sparse as sp
    n = len(row) - 1
    return sp.csr_matrix((val, col, row), shape=(n, n)) @ x


def solution_summary(row, col, val, b, x):
    w = np.random.default_rng(W_SEED).uniform(-1.0, 1.0, len(x))
    r = b - spmv(row, col, val, x)
    return dict(x_norm2=float(np.linalg.norm(x)), x_dot_w=float(np.dot(w, x)),
                relres_true=float(np.linalg.norm(r) / np.linalg.norm(b)))


def c1(orc, ref, nt):
    row, col, val = ref.q1_assemble(2, 256)
    b = orc.q1_rhs(42, 2, 256)
    t = time.time()
    s = ref.pcg(row, col, val, b, precond=1, impl=1, nthreads=nt, maxits=100000, reltol=1e-10)
    out = dict(dim=2, N=256, seed=42, n=len(b), nnz=len(col), csr_sha256=sha(row, col, val),
               method="Jacobi-PCG", reltol=1e-10, iters=s["iters"], status=s["status"], res=s["res"],
               seconds=time.time() - t)
    out.update(solution_summary(row, col, val, b, s["x"]))
    return out


def c2(orc, ref, nt):
    row, col, val = ref.q1_assemble(3, 128)
    b = orc.q1_rhs(42, 3, 128)
    t = time.time()
    nc, sizes, perm_mc = ref.multicoloring(row, col, val)
    t_col = time.time() - t
    # the block preconditioner's permutation and permuted operator (the numbering CG runs in)
    blk = ref.block_precond(2, row, col, val, np.zeros(len(b)))
    Ar, Ac, Av = blk["A"]
    bp = b[blk["perm"]]
    t = time.time()
    s = ref.pcg(row, col, val, bp, precond=2, impl=1, nthreads=nt, maxits=100000, reltol=1e-8)
    out = dict(dim=3, N=128, seed=42, n=len(b), nnz=len(col), csr_sha256=sha(row, col, val),
               colours=int(nc), colour_sizes=[int(v) for v in sizes],
               multicoloring_perm_sha256=sha(perm_mc.astype(np.int32)),
               precond_perm_sha256=sha(blk["perm"].astype(np.int32)),
               precond_colours=int(blk["nblocks"]), precond_sizes=[int(v) for v in blk["sizes"]],
               permuted_csr_sha256=sha(Ar, Ac, Av),
               method="MC-SGS PCG (permuted numbering, b[perm])", reltol=1e-8,
               iters=s["iters"], status=s["status"], res=s["res"],
               seconds_colouring=t_col, seconds=time.time() - t)
    out.update(solution_summary(Ar, Ac, Av, bp, s["x"]))
    return out


def c4(orc, ref, nt):
    row, col, val = ref.q1_assemble(2, 512, 1, None, 1e-3, (1.0, 0.5, 0.0))
    b = orc.q1_rhs(42, 2, 512)
    t = time.time()
    nl, lsizes, lperm = ref.levelscheduling(row, col, val)
    t_ls = time.time() - t
    # lPreconditioner_MultiColoring_ILUp with level scheduling permutes the
    # operator by the levels of its ILU(0) factors, whose pattern is the
    # operator's (lpreconditioner_mc.cc:157-199, 264-356); its block build
    # extracts every level pair and costs O(levels^2 nnz), so the solve below
    # applies the same reordered factors with the reference's ilu_solve
    # (precond kind 5 of ref_gmres; identical iteration counts and solutions
    # to 3e-16 against the block preconditioner on the 32^2 and 64^2 cases).
    Ar, Ac, Av = ref.reorder(row, col, val, lperm)
    bp = b[lperm]
    t = time.time()
    s = ref.gmres(row, col, val, bp, precond=5, m=30, impl=1, nthreads=nt, maxits=100000, reltol=1e-9)
    out = dict(dim=2, N=512, seed=42, nu=1e-3, beta=[1.0, 0.5], n=len(b), nnz=len(col),
               csr_sha256=sha(row, col, val), levels=int(nl), level_sizes_sha256=sha(lsizes.astype(np.int32)),
               levelscheduling_perm_sha256=sha(lperm.astype(np.int32)), permuted_csr_sha256=sha(Ar, Ac, Av),
               method="GMRES(30) + ILU(0) level-scheduled, right-preconditioned (permuted numbering, b[perm])",
               reltol=1e-9, iters=s["iters"], status=s["status"], res=s["res"], seconds_levels=t_ls,
               seconds=time.time() - t)
    out.update(solution_summary(Ar, Ac, Av, bp, s["x"]))
    return out


def main():
    which = sys.argv[1:] or ["c1", "c2", "c4"]
    orc, ref = Oracle(), Ref()
    nt = ref.max_threads()
    data = {}
    if os.path.exists(OUT):
        with open(OUT) as f:
            data = json.load(f)
    data["w_seed"] = W_SEED
    data["threads"] = nt
    for name in which:
        t = time.time()
        data[name] = globals()[name](orc, ref, nt)
        print(name, json.dumps(data[name]), f"({time.time() - t:.1f} s)", flush=True)
        with open(OUT, "w") as f:
            json.dump(data, f, indent=1)


if __name__ == "__main__":
    main()
