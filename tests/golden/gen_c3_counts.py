"""Iteration counts of the 3-D 128^3 variable-coefficient system, from the
reference's own CPU lmp code (oracle/_ref), written to c3_counts.json.

The CPU baseline times a bounded sample of the reference's mixed-precision
solve (MPIR, FP32 Jacobi-CG inside FP64 defect correction) and of its FP64
Jacobi-CG, and scales the per-iteration cost by these full-solve counts.

Usage:  make -C oracle REF=<HiFlow3 source tree> && python tests/golden/gen_c3_counts.py [N]
"""
import importlib.util
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.join(HERE, "..", "..")
sys.path.insert(0, os.path.join(ROOT, "oracle"))
from pyoracle import Oracle, Ref, ref_mpir, ref_pcg_timed  # noqa: E402

spec = importlib.util.spec_from_file_location("b200_workloads", os.path.join(ROOT, "hiflow3_2.0_b200", "workloads.py"))
wl = importlib.util.module_from_spec(spec)
spec.loader.exec_module(wl)


def main():
    N = int(sys.argv[1]) if len(sys.argv) > 1 else 128
    orc, ref = Oracle(), Ref()
    kc = np.exp(wl.grf_cells(N, 3))
    row, col, val = orc.q1_assemble(3, N, 0, kc)
    b = orc.q1_rhs(42, 3, N)
    nt = ref.max_threads()
    t = time.time()
    m = ref_mpir(ref, row, col, val, b, nt, max_outer=50, reltol=1e-10, inner_reltol=1e-4)
    t_m = time.time() - t
    t = time.time()
    p = ref_pcg_timed(ref, row, col, val, b, nt, reltol=1e-10)
    t_p = time.time() - t
    r = b - orc.spmv(row, col, val, m["x"])
    out = dict(N=N, seed=42, grf=dict(sigma=1.0, ell=0.1, seed=2024, covariance="squared-exponential"),
               mpir_outer=m["outer"], mpir_inner_total=m["inner_total"],
               mpir_relres=float(np.linalg.norm(r) / np.linalg.norm(b)),
               fp64_cg_iters=p["iters"], threads=nt, seconds_mpir=t_m, seconds_fp64=t_p,
               kcell_contrast=float(kc.max() / kc.min()))
    name = "c3_counts.json" if N == 128 else f"c3_counts_{N}.json"
    with open(os.path.join(HERE, name), "w") as f:
        json.dump(out, f, indent=1)
    print(json.dumps(out))


if __name__ == "__main__":
    main()
