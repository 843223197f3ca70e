"""Generate the file-I/O fixtures in tests/golden/mm/ from HiFlow3's own CPU lmp code.

Writes seeded MatrixMarket and vector files (this project's own test inputs),
reads each with the reference's CPU_CSR_lMatrix::ReadFile /
CPU_lVector::ReadFile (oracle/_ref/libhiflow_lmp_ref.so, the reference's
unmodified CPU lmp sources), writes CSR matrices and vectors with the
reference's WriteFile, and stores the reference's CSR arrays, values and
written texts in ``mm/mm_golden.npz``.

Usage:  make -C oracle REF=<HiFlow3 source tree> && python tests/golden/gen_mm_golden.py
"""
import ctypes as C
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "mm")
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
from pyoracle import Ref  # noqa: E402

_i32p = np.ctypeslib.ndpointer(np.int32, flags="C")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C")


def _lib():
    L = Ref().lib
    L.ref_mm_read.argtypes = [C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int), _i32p, _i32p, _f64p, C.c_int,
                              C.c_int]
    L.ref_mm_read.restype = C.c_int
    L.ref_mm_write.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int, _i32p, _i32p, _f64p]
    L.ref_vec_read.argtypes = [C.c_char_p, _f64p, C.c_int]
    L.ref_vec_read.restype = C.c_int
    L.ref_vec_write.argtypes = [C.c_char_p, C.c_int, _f64p]
    return L


def entries_text(rows, cols, vals, fmt):
    return "".join(f"{r} {c} {fmt(v)}\n" for r, c, v in zip(rows, cols, vals))


def matrix_files(rng):
    """name -> file text.  Each file exercises one rule of the reader."""
    f = {}
    # general real, unsorted entries, a duplicate pair, comments, mixed-case
    # banner words, blank line before the size line
    rows = [3, 1, 7, 2, 5, 1, 4, 6, 7, 3, 1, 2]
    cols = [2, 5, 7, 2, 1, 1, 4, 3, 1, 2, 3, 6]
    vals = rng.uniform(-4, 4, len(rows))
    f["general.mtx"] = ("%%MatrixMarket Matrix Coordinate Real General\n% a comment line\n%\n\n7 7 12\n" +
                        entries_text(rows, cols, vals, lambda v: f"{v:.17g}"))
    # symmetric: lower triangle with the diagonal
    ent = [(i, j) for i in range(1, 7) for j in range(1, i + 1) if (i + j) % 3 != 1 or i == j]
    vals = rng.uniform(-1, 1, len(ent))
    f["symmetric.mtx"] = (f"%%MatrixMarket matrix coordinate real symmetric\n6 6 {len(ent)}\n" +
                          entries_text([e[0] for e in ent], [e[1] for e in ent], vals, lambda v: f"{v:.17g}"))
    # integer, rectangular
    rows = [1, 2, 2, 3, 5, 4, 1]
    cols = [4, 1, 3, 2, 4, 1, 1]
    f["integer_rect.mtx"] = ("%%MatrixMarket matrix coordinate integer general\n5 4 7\n" +
                             entries_text(rows, cols, rng.integers(-9, 10, len(rows)), str))
    # skew-symmetric: read as general by the reference
    f["skew.mtx"] = ("%%MatrixMarket matrix coordinate real skew-symmetric\n4 4 3\n" +
                     entries_text([2, 3, 4], [1, 1, 3], [0.5, -1.25, 2.0], lambda v: f"{v:.17g}"))
    # random 200 x 200, values in exponent notation and integers mixed
    n, m = 200, 2000
    rows, cols = rng.integers(1, n + 1, m), rng.integers(1, n + 1, m)
    vals = rng.standard_normal(m) * 10.0 ** rng.integers(-6, 7, m)
    f["random200.mtx"] = (f"%%MatrixMarket matrix coordinate real general\n{n} {n} {m}\n" +
                          entries_text(rows, cols, vals, lambda v: f"{v:.12e}"))
    return f


def vector_files(rng):
    x = rng.standard_normal(9)
    body = "".join(f"{v:.17g}\n" for v in x)
    return {"vec_newline.vec": body,                      # last value followed by a line break
            "vec_no_newline.vec": body.rstrip("\n"),       # the reference drops the last value
            "vec_exp.vec": "1e-3\n  -2.5E+02\n3\n\n7.125\n"}


def main():
    L = _lib()
    rng = np.random.default_rng(20261203)
    os.makedirs(OUT, exist_ok=True)
    g = {}
    for name, text in matrix_files(rng).items():
        path = os.path.join(OUT, name)
        with open(path, "w") as fh:
            fh.write(text)
        nr, nc = C.c_int(), C.c_int()
        cap = 8192
        row, col, val = np.zeros(cap, np.int32), np.zeros(cap, np.int32), np.zeros(cap)
        nnz = L.ref_mm_read(path.encode(), C.byref(nr), C.byref(nc), row, col, val, cap, cap)
        assert nnz >= 0
        key = name.split(".")[0]
        g[f"{key}_shape"] = np.array([nr.value, nc.value, nnz], np.int64)
        g[f"{key}_row"], g[f"{key}_col"], g[f"{key}_val"] = row[:nr.value + 1].copy(), col[:nnz].copy(), val[:nnz].copy()
    with tempfile.TemporaryDirectory() as td:
        # WriteFile of two CSR matrices: the general one read above, and a
        # rectangular one with values of many magnitudes
        for key in ("general", "integer_rect", "random200"):
            nr, nc, nnz = (int(v) for v in g[f"{key}_shape"])
            p = os.path.join(td, key + ".out")
            L.ref_mm_write(p.encode(), nr, nc, nnz, g[f"{key}_row"], g[f"{key}_col"], g[f"{key}_val"])
            g[f"{key}_written"] = np.frombuffer(open(p, "rb").read(), np.uint8).copy()
        for name, text in vector_files(rng).items():
            path = os.path.join(OUT, name)
            with open(path, "w") as fh:
                fh.write(text)
            x = np.zeros(64)
            n = L.ref_vec_read(path.encode(), x, x.size)
            assert n >= 0
            key = name.split(".")[0]
            g[f"{key}_values"] = x[:n].copy()
        xw = np.concatenate([rng.standard_normal(6), [0.0, -0.0, 1e-300, 6.02e23, 123456789.0]])
        p = os.path.join(td, "vec.out")
        L.ref_vec_write(p.encode(), xw.size, xw)
        g["vecwrite_input"] = xw
        g["vecwrite_written"] = np.frombuffer(open(p, "rb").read(), np.uint8).copy()
    np.savez_compressed(os.path.join(OUT, "mm_golden.npz"), **g)
    print("wrote", os.path.join(OUT, "mm_golden.npz"), len(g), "arrays")


if __name__ == "__main__":
    main()
