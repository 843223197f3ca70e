"""ctypes bindings of the CPU checker libraries (test infrastructure only).

``Oracle`` wraps ``oracle/liboracle.so`` (the C restatement of HiFlow3's lmp
hot path) and ``Ref`` wraps ``oracle/_ref/libhiflow_lmp_ref.so`` (HiFlow3's own
CPU lmp sources compiled unmodified, plus ``ref_driver.cc``).  Only tests,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` import this
module; the product library never does.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libhiflow_lmp_ref.so")

_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class _Control(C.Structure):
    _fields_ = [("maxits", C.c_int), ("abstol", C.c_double), ("reltol", C.c_double),
                ("divtol", C.c_double)]


class _Result(C.Structure):
    _fields_ = [("iters", C.c_int), ("status", C.c_int), ("res0", C.c_double), ("res", C.c_double)]


class _Block(C.Structure):
    _fields_ = [("n", C.c_int), ("nblocks", C.c_int), ("block_off", C.POINTER(C.c_int)),
                ("perm", C.POINTER(C.c_int)), ("row", C.POINTER(C.c_int)),
                ("col", C.POINTER(C.c_int)), ("val", C.POINTER(C.c_double)),
                ("Dv", C.POINTER(C.c_double)), ("iDv", C.POINTER(C.c_double)),
                ("kind", C.c_int), ("omega", C.c_double)]


class _Jacobi(C.Structure):
    _fields_ = [("n", C.c_int), ("invdiag", C.POINTER(C.c_double))]


_PRECOND_FN = C.CFUNCTYPE(None, C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double))

# IterateControl states (src/common/iterate_control.h)
ITERATE, SUCCESS_ABS, SUCCESS_REL, FAIL_DIV, FAIL_MAXITS = range(5)


def control(maxits=1000, abstol=0.0, reltol=1e-10, divtol=1e6):
    return _Control(maxits, abstol, reltol, divtol)


class BlockPrecond:
    """A built colour/level block preconditioner (owned C struct)."""

    def __init__(self, lib, st):
        self._lib, self.st = lib, st
        n, nb = st.n, st.nblocks
        self.n, self.nblocks = n, nb
        self.block_off = np.ctypeslib.as_array(st.block_off, (nb + 1,)).copy()
        self.perm = np.ctypeslib.as_array(st.perm, (n,)).copy()
        nnz = st.row[n]
        self.row = np.ctypeslib.as_array(st.row, (n + 1,)).copy()
        self.col = np.ctypeslib.as_array(st.col, (nnz,)).copy() if nnz else np.zeros(0, np.int32)
        self.val = np.ctypeslib.as_array(st.val, (nnz,)).copy() if nnz else np.zeros(0)
        self.Dv = np.ctypeslib.as_array(st.Dv, (n,)).copy()
        self.iDv = np.ctypeslib.as_array(st.iDv, (n,)).copy()

    def apply(self, r):
        r = _f64(r)
        z = np.zeros_like(r)
        self._lib.orc_block_apply(C.byref(self.st), r, z)
        return z

    def __del__(self):
        try:
            self._lib.orc_block_free(C.byref(self.st))
        except Exception:
            pass


class Oracle:
    def __init__(self, path=ORACLE_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle`")
        L = self.lib = C.CDLL(path)
        L.orc_q1_sizes.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int64)]
        L.orc_q1_structure.argtypes = [C.c_int, C.c_int, _i32p, _i32p]
        L.orc_q1_element.argtypes = [C.c_int, C.c_double, C.c_int, C.c_double, _f64p, _f64p]
        L.orc_q1_element.restype = None
        L.orc_q1_dirichlet.argtypes = [C.c_int, C.c_int, _i32p]
        L.orc_q1_assemble.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_double, _f64p,
                                      _i32p, _i32p, _f64p]
        L.orc_q1_rhs.argtypes = [C.c_uint64, C.c_int, C.c_int, _f64p]
        L.orc_q1_rhs.restype = None
        L.orc_coo_to_csr.argtypes = [C.c_int, C.c_int, _i32p, _i32p, C.c_void_p, _i32p, _i32p, C.c_void_p]
        L.orc_coo_to_csr.restype = None
        L.orc_add_values.argtypes = [_i32p, _i32p, _f64p, _i32p, C.c_int, _i32p, C.c_int, _f64p]
        L.orc_add_values.restype = None
        L.orc_zero_rows.argtypes = [_i32p, _i32p, _f64p, _i32p, C.c_int, C.c_double]
        L.orc_zero_rows.restype = None
        L.orc_spmv_d.argtypes = [C.c_int, _i32p, _i32p, _f64p, _f64p, _f64p]
        L.orc_spmv_d.restype = None
        L.orc_spmv_f.argtypes = [C.c_int, _i32p, _i32p, _f32p, _f32p, _f32p]
        L.orc_spmv_f.restype = None
        L.orc_spmv_add_d.argtypes = [C.c_int, _i32p, _i32p, _f64p, _f64p, _f64p]
        L.orc_spmv_add_d.restype = None
        L.orc_dot_d.argtypes = [C.c_int, _f64p, _f64p]
        L.orc_dot_d.restype = C.c_double
        L.orc_dot_f_acc_d.argtypes = [C.c_int, _f32p, _f32p]
        L.orc_dot_f_acc_d.restype = C.c_double
        L.orc_multicoloring.argtypes = [C.c_int, _i32p, _i32p, C.POINTER(C.c_int), _i32p, _i32p]
        L.orc_levelscheduling.argtypes = [C.c_int, _i32p, _i32p, C.POINTER(C.c_int), _i32p, _i32p]
        L.orc_reorder_csr.argtypes = [C.c_int, _i32p, _i32p, _f64p, _i32p, _i32p, _i32p, _f64p]
        L.orc_reorder_csr.restype = None
        L.orc_ilu0.argtypes = [C.c_int, _i32p, _i32p, _f64p]
        L.orc_ilu0.restype = None
        L.orc_ilu_solve.argtypes = [C.c_int, _i32p, _i32p, _f64p, _f64p, _f64p]
        L.orc_ilu_solve.restype = None
        L.orc_mcsgs_build.argtypes = [C.c_int, _i32p, _i32p, _f64p, C.c_double, C.POINTER(_Block),
                                      _i32p, _i32p, _f64p]
        L.orc_ilu0_build.argtypes = [C.c_int, _i32p, _i32p, _f64p, C.c_int, C.POINTER(_Block),
                                     _i32p, _i32p, _f64p]
        L.orc_ilup_build.argtypes = [C.c_int, _i32p, _i32p, _f64p, C.c_int, C.c_int, C.c_int, C.POINTER(_Block),
                                     _i32p, _i32p, _f64p]
        _pp, _dp = C.POINTER(C.POINTER(C.c_int)), C.POINTER(C.POINTER(C.c_double))
        L.orc_power_pattern.argtypes = [C.c_int, _i32p, _i32p, C.c_int, _pp, _pp]
        L.orc_ilup.argtypes = [C.c_int, _i32p, _i32p, _f64p, C.c_int, _pp, _pp, _dp]
        L.orc_free.argtypes = [C.c_void_p]
        L.orc_csr_scale.argtypes = [C.c_int, _i32p, _i32p, _f64p, C.c_double, C.c_int]
        L.orc_iamin.argtypes = L.orc_iamax.argtypes = [C.c_int, _f64p]
        L.orc_asum.argtypes = [C.c_int, _f64p]
        L.orc_asum.restype = C.c_double
        L.orc_rot.argtypes = [C.c_int, _f64p, _f64p, C.c_double, C.c_double]
        L.orc_rot.restype = None
        L.orc_rotm.argtypes = [C.c_int, _f64p, _f64p, _f64p]
        L.orc_rotm.restype = None
        L.orc_rotg.argtypes = [C.POINTER(C.c_double)] * 4
        L.orc_rotg.restype = None
        L.orc_csr_scale.restype = None
        L.orc_csr_diag.argtypes = [_i32p, _i32p, _f64p, C.c_int, C.c_int, C.c_int, _f64p]
        L.orc_csr_diag.restype = None
        L.orc_csr_extract.argtypes = [C.c_int, _i32p, _i32p, _f64p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                      _pp, _pp, _dp]
        L.orc_free.restype = None
        L.orc_block_apply.argtypes = [C.POINTER(_Block), _f64p, _f64p]
        L.orc_block_apply.restype = None
        L.orc_block_free.argtypes = [C.POINTER(_Block)]
        L.orc_block_free.restype = None
        L.orc_invdiag.argtypes = [C.c_int, _i32p, _i32p, _f64p, _f64p]
        L.orc_invdiag.restype = None
        L.orc_pcg.argtypes = [C.c_int, _i32p, _i32p, _f64p, C.c_void_p, C.c_void_p, _f64p, _f64p,
                              C.POINTER(_Control), C.POINTER(_Result), C.c_void_p]
        L.orc_gmres.argtypes = [C.c_int, _i32p, _i32p, _f64p, C.c_void_p, C.c_void_p, C.c_int, _f64p,
                                _f64p, C.POINTER(_Control), C.POINTER(_Result)]
        L.orc_pcg_f32.argtypes = [C.c_int, _i32p, _i32p, _f32p, _f32p, _f32p, _f32p,
                                  C.POINTER(_Control), C.POINTER(_Result)]
        L.orc_mpir.argtypes = [C.c_int, _i32p, _i32p, _f64p, _f64p, _f64p, C.POINTER(_Control),
                               C.POINTER(_Control), C.c_int, C.c_int, C.POINTER(_Result),
                               C.POINTER(C.c_int)]
        self._jacobi_fn = C.cast(L.orc_jacobi_apply, C.c_void_p)
        self._block_fn = C.cast(L.orc_block_apply_cb, C.c_void_p)

    # ---- systems ----
    def q1_sizes(self, dim, N):
        n, nnz = C.c_int(), C.c_int64()
        if self.lib.orc_q1_sizes(dim, N, C.byref(n), C.byref(nnz)):
            raise ValueError("bad Q1 size")
        return n.value, nnz.value

    def q1_structure(self, dim, N):
        n, nnz = self.q1_sizes(dim, N)
        r, c = np.empty(nnz, np.int32), np.empty(nnz, np.int32)
        self.lib.orc_q1_structure(dim, N, r, c)
        return r, c

    def q1_element(self, dim, h, kind=0, coef=1.0, beta=(0.0, 0.0, 0.0)):
        Ke = np.empty((1 << dim) ** 2)
        self.lib.orc_q1_element(dim, h, kind, coef, _f64(list(beta) + [0.0] * (3 - len(beta))), Ke)
        return Ke.reshape(1 << dim, 1 << dim)

    def q1_dirichlet(self, dim, N):
        n, _ = self.q1_sizes(dim, N)
        idx = np.empty(n, np.int32)
        c = self.lib.orc_q1_dirichlet(dim, N, idx)
        return idx[:c].copy()

    def q1_assemble(self, dim, N, kind=0, kcell=None, nu=1.0, beta=(0.0, 0.0, 0.0)):
        n, nnz = self.q1_sizes(dim, N)
        row, col, val = np.empty(n + 1, np.int32), np.empty(nnz, np.int32), np.empty(nnz)
        kc = None
        if kcell is not None:
            kc = _f64(kcell)
            assert kc.size == N ** dim
        b3 = _f64(list(beta) + [0.0] * (3 - len(beta)))
        rc = self.lib.orc_q1_assemble(dim, N, kind, kc.ctypes.data if kc is not None else None,
                                      nu, b3, row, col, val)
        if rc:
            raise RuntimeError(f"orc_q1_assemble: {rc}")
        return row, col, val

    def q1_rhs(self, seed, dim, N):
        n, _ = self.q1_sizes(dim, N)
        b = np.empty(n)
        self.lib.orc_q1_rhs(seed, dim, N, b)
        return b

    # ---- CSR primitives ----
    def coo_to_csr(self, n, coo_row, coo_col, coo_val=None):
        coo_row, coo_col = _i32(coo_row), _i32(coo_col)
        nnz = coo_row.size
        row, col = np.empty(n + 1, np.int32), np.empty(nnz, np.int32)
        if coo_val is not None:
            cv = _f64(coo_val)
            val = np.empty(nnz)
            self.lib.orc_coo_to_csr(n, nnz, coo_row, coo_col, cv.ctypes.data, row, col, val.ctypes.data)
            return row, col, val
        self.lib.orc_coo_to_csr(n, nnz, coo_row, coo_col, None, row, col, None)
        return row, col

    def add_values(self, row, col, val, rows, cols, values):
        val = _f64(val).copy()
        rows, cols = _i32(rows), _i32(cols)
        self.lib.orc_add_values(_i32(row), _i32(col), val, rows, rows.size, cols, cols.size, _f64(values))
        return val

    def zero_rows(self, row, col, val, idx, alpha=1.0):
        val = _f64(val).copy()
        idx = _i32(idx)
        self.lib.orc_zero_rows(_i32(row), _i32(col), val, idx, idx.size, alpha)
        return val

    def spmv(self, row, col, val, x):
        n = len(row) - 1
        if np.asarray(val).dtype == np.float32:
            y = np.empty(n, np.float32)
            self.lib.orc_spmv_f(n, _i32(row), _i32(col), np.ascontiguousarray(val),
                                np.ascontiguousarray(x, dtype=np.float32), y)
            return y
        y = np.empty(n)
        self.lib.orc_spmv_d(n, _i32(row), _i32(col), _f64(val), _f64(x), y)
        return y

    def spmv_add(self, row, col, val, x, y):
        y = _f64(y).copy()
        self.lib.orc_spmv_add_d(len(row) - 1, _i32(row), _i32(col), _f64(val), _f64(x), y)
        return y

    def dot(self, x, y):
        x = np.asarray(x)
        if x.dtype == np.float32:
            return self.lib.orc_dot_f_acc_d(x.size, np.ascontiguousarray(x), np.ascontiguousarray(y, dtype=np.float32))
        return self.lib.orc_dot_d(x.size, _f64(x), _f64(y))

    # ---- analysis ----
    def multicoloring(self, row, col):
        n = len(row) - 1
        nc, sizes, perm = C.c_int(), np.empty(n, np.int32), np.empty(n, np.int32)
        if self.lib.orc_multicoloring(n, _i32(row), _i32(col), C.byref(nc), sizes, perm):
            raise RuntimeError("multicoloring failed")
        return nc.value, sizes[:nc.value].copy(), perm

    def levelscheduling(self, row, col):
        n = len(row) - 1
        nl, sizes, perm = C.c_int(), np.empty(n, np.int32), np.empty(n, np.int32)
        if self.lib.orc_levelscheduling(n, _i32(row), _i32(col), C.byref(nl), sizes, perm):
            raise RuntimeError("levelscheduling did not finish")
        return nl.value, sizes[:nl.value].copy(), perm

    def reorder(self, row, col, val, perm):
        n = len(row) - 1
        r2, c2, v2 = np.empty(n + 1, np.int32), np.empty(len(col), np.int32), np.empty(len(col))
        self.lib.orc_reorder_csr(n, _i32(row), _i32(col), _f64(val), _i32(perm), r2, c2, v2)
        return r2, c2, v2

    def ilu0(self, row, col, val):
        v = _f64(val).copy()
        self.lib.orc_ilu0(len(row) - 1, _i32(row), _i32(col), v)
        return v

    def ilu_solve(self, row, col, val, r):
        z = np.empty(len(row) - 1)
        self.lib.orc_ilu_solve(len(row) - 1, _i32(row), _i32(col), _f64(val), _f64(r), z)
        return z

    def invdiag(self, row, col, val):
        d = np.empty(len(row) - 1)
        self.lib.orc_invdiag(len(row) - 1, _i32(row), _i32(col), _f64(val), d)
        return d

    # ---- preconditioners ----
    def mcsgs_build(self, row, col, val, omega=1.0):
        n = len(row) - 1
        st = _Block()
        Ar, Ac, Av = np.empty(n + 1, np.int32), np.empty(len(col), np.int32), np.empty(len(col))
        if self.lib.orc_mcsgs_build(n, _i32(row), _i32(col), _f64(val), omega, C.byref(st), Ar, Ac, Av):
            raise RuntimeError("mcsgs build failed")
        return BlockPrecond(self.lib, st), (Ar, Ac, Av)

    def ilu0_build(self, row, col, val, mode=0):
        n = len(row) - 1
        st = _Block()
        Ar, Ac, Av = np.empty(n + 1, np.int32), np.empty(len(col), np.int32), np.empty(len(col))
        if self.lib.orc_ilu0_build(n, _i32(row), _i32(col), _f64(val), mode, C.byref(st), Ar, Ac, Av):
            raise RuntimeError("ilu0 build failed")
        return BlockPrecond(self.lib, st), (Ar, Ac, Av)

    def power_pattern(self, row, col, p):
        n = len(row) - 1
        r, c = C.POINTER(C.c_int)(), C.POINTER(C.c_int)()
        m = self.lib.orc_power_pattern(n, _i32(row), _i32(col), p, C.byref(r), C.byref(c))
        out = (np.ctypeslib.as_array(r, (n + 1,)).copy(), np.ctypeslib.as_array(c, (max(m, 1),))[:m].copy())
        self.lib.orc_free(C.cast(r, C.c_void_p))
        self.lib.orc_free(C.cast(c, C.c_void_p))
        return out

    def ilup(self, row, col, val, p):
        n = len(row) - 1
        r, c, v = C.POINTER(C.c_int)(), C.POINTER(C.c_int)(), C.POINTER(C.c_double)()
        m = self.lib.orc_ilup(n, _i32(row), _i32(col), _f64(val), p, C.byref(r), C.byref(c), C.byref(v))
        out = (np.ctypeslib.as_array(r, (n + 1,)).copy(), np.ctypeslib.as_array(c, (max(m, 1),))[:m].copy(),
               np.ctypeslib.as_array(v, (max(m, 1),))[:m].copy())
        for q in (r, c, v):
            self.lib.orc_free(C.cast(q, C.c_void_p))
        return out

    def vec_reduce(self, x):
        """ArgMin, ArgMax, Norm1, NormMax of x."""
        x = _f64(x)
        n = x.size
        k = self.lib.orc_iamax(n, x)
        return self.lib.orc_iamin(n, x), k, self.lib.orc_asum(n, x), abs(x[k])

    def rot(self, x, y, c=None, s=None, param=None):
        """Rot (c, s) or Rotm (param); returns the new (x, y)."""
        x, y = _f64(x).copy(), _f64(y).copy()
        if param is None:
            self.lib.orc_rot(x.size, x, y, c, s)
        else:
            self.lib.orc_rotm(x.size, x, y, _f64(param))
        return x, y

    def rotg(self, a, b):
        v = [C.c_double(a), C.c_double(b), C.c_double(), C.c_double()]
        self.lib.orc_rotg(*[C.byref(q) for q in v])
        return tuple(q.value for q in v)

    def csr_scale(self, row, col, val, alpha, mode):
        """Scale (mode 0), ScaleOffdiag (1), Zeros (2): the new values."""
        v = _f64(val).copy()
        self.lib.orc_csr_scale(len(row) - 1, _i32(row), _i32(col), v, alpha, mode)
        return v

    def csr_diag(self, row, col, val, start, end, inverse=False, fill=0.0):
        """extract_diagelements / extract_invdiagelements of rows [start, end);
        rows without a diagonal entry keep `fill`."""
        out = np.full(end - start, fill)
        self.lib.orc_csr_diag(_i32(row), _i32(col), _f64(val), start, end, int(inverse), out)
        return out

    def csr_extract(self, row, col, val, mode, sr=0, sc=0, er=0, ec=0):
        """extract_submatrix (mode 0, block [sr, er) x [sc, ec)) or Compress (mode 1)."""
        n = len(row) - 1
        r, c, v = C.POINTER(C.c_int)(), C.POINTER(C.c_int)(), C.POINTER(C.c_double)()
        m = self.lib.orc_csr_extract(n, _i32(row), _i32(col), _f64(val), mode, sr, sc, er, ec, C.byref(r),
                                     C.byref(c), C.byref(v))
        rows = (er - sr if mode == 0 else n) + 1
        out = (np.ctypeslib.as_array(r, (rows,)).copy(), np.ctypeslib.as_array(c, (max(m, 1),))[:m].copy(),
               np.ctypeslib.as_array(v, (max(m, 1),))[:m].copy())
        for q in (r, c, v):
            self.lib.orc_free(C.cast(q, C.c_void_p))
        return out

    def ilup_build(self, row, col, val, mode, ilu_p, mat_power=1):
        n = len(row) - 1
        st = _Block()
        Ar, Ac, Av = np.empty(n + 1, np.int32), np.empty(len(col), np.int32), np.empty(len(col))
        if self.lib.orc_ilup_build(n, _i32(row), _i32(col), _f64(val), mode, ilu_p, mat_power, C.byref(st),
                                   Ar, Ac, Av):
            raise RuntimeError("ilup build failed")
        return BlockPrecond(self.lib, st), (Ar, Ac, Av)

    # ---- solvers ----
    def _precond_args(self, precond):
        if precond is None:
            return None, None, None
        if isinstance(precond, BlockPrecond):
            return self._block_fn, C.cast(C.byref(precond.st), C.c_void_p), None
        d = _f64(precond)  # a Jacobi inverse diagonal
        j = _Jacobi(d.size, d.ctypes.data_as(C.POINTER(C.c_double)))
        return self._jacobi_fn, C.cast(C.byref(j), C.c_void_p), (d, j)

    def pcg(self, row, col, val, b, x0=None, precond=None, ctl=None, history=False):
        n = len(row) - 1
        x = np.zeros(n) if x0 is None else _f64(x0).copy()
        ctl = ctl or control()
        fn, ctx, keep = self._precond_args(precond)
        res = _Result()
        hist = np.zeros(ctl.maxits + 1) if history else None
        self.lib.orc_pcg(n, _i32(row), _i32(col), _f64(val), fn, ctx, _f64(b), x, C.byref(ctl),
                         C.byref(res), hist.ctypes.data if history else None)
        out = dict(x=x, iters=res.iters, status=res.status, res0=res.res0, res=res.res)
        if history:
            out["history"] = hist[:res.iters + 1]
        return out

    def gmres(self, row, col, val, b, x0=None, precond=None, m=30, ctl=None):
        n = len(row) - 1
        x = np.zeros(n) if x0 is None else _f64(x0).copy()
        ctl = ctl or control()
        fn, ctx, keep = self._precond_args(precond)
        res = _Result()
        self.lib.orc_gmres(n, _i32(row), _i32(col), _f64(val), fn, ctx, m, _f64(b), x, C.byref(ctl),
                           C.byref(res))
        return dict(x=x, iters=res.iters, status=res.status, res0=res.res0, res=res.res)

    def pcg_f32(self, row, col, val32, invdiag32, b32, ctl=None):
        n = len(row) - 1
        x = np.zeros(n, np.float32)
        ctl = ctl or control()
        res = _Result()
        self.lib.orc_pcg_f32(n, _i32(row), _i32(col), np.ascontiguousarray(val32, np.float32),
                             np.ascontiguousarray(invdiag32, np.float32),
                             np.ascontiguousarray(b32, np.float32), x, C.byref(ctl), C.byref(res))
        return dict(x=x, iters=res.iters, status=res.status, res0=res.res0, res=res.res)

    def mpir(self, row, col, val, b, outer=None, inner=None, max_outer=50, res0_mode=0):
        n = len(row) - 1
        x = np.zeros(n)
        outer = outer or control(reltol=1e-10)
        inner = inner or control(reltol=1e-4)
        res, tot = _Result(), C.c_int()
        self.lib.orc_mpir(n, _i32(row), _i32(col), _f64(val), _f64(b), x, C.byref(outer), C.byref(inner),
                          max_outer, res0_mode, C.byref(res), C.byref(tot))
        return dict(x=x, outer=res.iters, inner_total=tot.value, res0=res.res0, res=res.res,
                    status=res.status)


class Ref:
    """HiFlow3's own CPU lmp code (compiled from the reference sources)."""

    def __init__(self, path=REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: build it with `make -C oracle REF=<HiFlow3 source tree>` where the "
                                    "reference sources are present")
        L = self.lib = C.CDLL(path)
        L.ref_coo_to_csr.argtypes = [C.c_int, C.c_int, _i32p, _i32p, C.c_void_p, _i32p, _i32p, C.c_void_p]
        L.ref_q1_assemble.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_double, _f64p, _i32p,
                                      _i32p, _f64p]
        L.ref_add_values.argtypes = [C.c_int, C.c_int, _i32p, _i32p, _f64p, _i32p, C.c_int, _i32p,
                                     C.c_int, _f64p]
        L.ref_spmv.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, _i32p, _i32p, _f64p, _f64p, _f64p]
        L.ref_dot.argtypes = [C.c_int, C.c_int, _f64p, _f64p]
        L.ref_dot.restype = C.c_double
        L.ref_multicoloring.argtypes = [C.c_int, C.c_int, _i32p, _i32p, _f64p, C.POINTER(C.c_int), _i32p, _i32p]
        L.ref_levelscheduling.argtypes = [C.c_int, C.c_int, _i32p, _i32p, _f64p, C.POINTER(C.c_int), _i32p,
                                          _i32p]
        L.ref_reorder.argtypes = [C.c_int, C.c_int, _i32p, _i32p, _f64p, _i32p, _i32p, _i32p, _f64p]
        L.ref_ilu0.argtypes = [C.c_int, C.c_int, _i32p, _i32p, _f64p]
        L.ref_ilu_solve.argtypes = [C.c_int, C.c_int, _i32p, _i32p, _f64p, _f64p, _f64p]
        L.ref_block_precond.argtypes = [C.c_int, C.c_double, C.c_int, C.c_int, _i32p, _i32p, _f64p, _f64p,
                                        _f64p, _i32p, C.POINTER(C.c_int), _i32p, _i32p, _i32p, _f64p]
        L.ref_block_precond_ilup.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _i32p, _i32p, _f64p,
                                             _f64p, _f64p, _i32p, C.POINTER(C.c_int), _i32p, _i32p, _i32p, _f64p]
        L.ref_ilup.argtypes = [C.c_int, C.c_int, _i32p, _i32p, _f64p, C.c_int, C.c_int, _i32p, _i32p, _f64p]
        L.ref_set_ilup.argtypes = [C.c_int, C.c_int]
        L.ref_set_ilup.restype = None
        L.ref_power_pattern.argtypes = [C.c_int, C.c_int, _i32p, _i32p, C.c_int, C.c_int, _i32p, _i32p]
        L.ref_pcg.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _i32p, _i32p, _f64p, _f64p,
                              _f64p, C.c_int, C.c_double, C.c_double, C.c_double, C.POINTER(C.c_int),
                              C.POINTER(C.c_double), C.c_void_p]
        L.ref_gmres.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _i32p, _i32p, _f64p,
                                _f64p, _f64p, C.c_int, C.c_double, C.c_double, C.c_double,
                                C.POINTER(C.c_int), C.POINTER(C.c_double)]
        L.ref_lmp_cg.argtypes = [C.c_int, C.c_int, _i32p, _i32p, _f64p, _f64p, _f64p, C.c_double,
                                 C.c_double, C.c_int]
        L.ref_time_spmv.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, _i32p, _i32p, _f64p, _f64p, _f64p]
        L.ref_time_spmv.restype = C.c_double
        L.ref_max_threads.restype = C.c_int
        L.ref_csr_scale.argtypes = [C.c_int, C.c_int, C.c_int, _i32p, _i32p, _f64p, C.c_double, C.c_int]
        L.ref_vec_reduce.argtypes = [C.c_int, _f64p, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                     C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.ref_vec_reduce.restype = None
        L.ref_vec_rot.argtypes = [C.c_int, _f64p, _f64p, C.c_double, C.c_double, C.c_void_p]
        L.ref_vec_rot.restype = None
        L.ref_rotg.argtypes = [C.POINTER(C.c_double)] * 4
        L.ref_rotg.restype = None
        L.ref_csr_scale.restype = None
        L.ref_csr_diag.argtypes = [C.c_int, C.c_int, C.c_int, _i32p, _i32p, _f64p, C.c_int, C.c_int, C.c_int, _f64p]
        L.ref_csr_diag.restype = None
        L.ref_csr_extract.argtypes = [C.c_int, C.c_int, C.c_int, _i32p, _i32p, _f64p, C.c_int, C.c_int, C.c_int,
                                      C.c_int, C.c_int, C.c_int, _i32p, _i32p, _f64p]

    def coo_to_csr(self, n, coo_row, coo_col, coo_val=None):
        coo_row, coo_col = _i32(coo_row), _i32(coo_col)
        nnz = coo_row.size
        row, col = np.empty(n + 1, np.int32), np.empty(nnz, np.int32)
        if coo_val is not None:
            cv, val = _f64(coo_val), np.empty(nnz)
            self.lib.ref_coo_to_csr(n, nnz, coo_row, coo_col, cv.ctypes.data, row, col, val.ctypes.data)
            return row, col, val
        self.lib.ref_coo_to_csr(n, nnz, coo_row, coo_col, None, row, col, None)
        return row, col

    def q1_assemble(self, dim, N, kind=0, kcell=None, nu=1.0, beta=(0.0, 0.0, 0.0)):
        n = (N + 1) ** dim
        nnz = (3 * N + 1) ** dim
        row, col, val = np.empty(n + 1, np.int32), np.empty(nnz, np.int32), np.empty(nnz)
        kc = _f64(kcell) if kcell is not None else None
        b3 = _f64(list(beta) + [0.0] * (3 - len(beta)))
        self.lib.ref_q1_assemble(dim, N, kind, kc.ctypes.data if kc is not None else None, nu, b3,
                                 row, col, val)
        return row, col, val

    def add_values(self, row, col, val, rows, cols, values):
        row, col, val = _i32(row).copy(), _i32(col).copy(), _f64(val).copy()
        rows, cols = _i32(rows), _i32(cols)
        self.lib.ref_add_values(len(row) - 1, len(col), row, col, val, rows, rows.size, cols, cols.size,
                                _f64(values))
        return val

    def spmv(self, row, col, val, x, impl=0, nthreads=1):
        n = len(row) - 1
        y = np.empty(n)
        self.lib.ref_spmv(impl, nthreads, n, len(col), _i32(row), _i32(col), _f64(val), _f64(x), y)
        return y

    def dot(self, x, y, impl=0):
        x = _f64(x)
        return self.lib.ref_dot(impl, x.size, x, _f64(y))

    def multicoloring(self, row, col, val):
        n = len(row) - 1
        nc, sizes, perm = C.c_int(), np.empty(n, np.int32), np.empty(n, np.int32)
        self.lib.ref_multicoloring(n, len(col), _i32(row), _i32(col), _f64(val), C.byref(nc), sizes, perm)
        return nc.value, sizes[:nc.value].copy(), perm

    def levelscheduling(self, row, col, val):
        n = len(row) - 1
        nl, sizes, perm = C.c_int(), np.empty(n, np.int32), np.empty(n, np.int32)
        self.lib.ref_levelscheduling(n, len(col), _i32(row), _i32(col), _f64(val), C.byref(nl), sizes, perm)
        return nl.value, sizes[:nl.value].copy(), perm

    def reorder(self, row, col, val, perm):
        n = len(row) - 1
        r2, c2, v2 = np.empty(n + 1, np.int32), np.empty(len(col), np.int32), np.empty(len(col))
        self.lib.ref_reorder(n, len(col), _i32(row), _i32(col), _f64(val), _i32(perm), r2, c2, v2)
        return r2, c2, v2

    def ilu0(self, row, col, val):
        v = _f64(val).copy()
        self.lib.ref_ilu0(len(row) - 1, len(col), _i32(row), _i32(col), v)
        return v

    def ilu_solve(self, row, col, val, r):
        z = np.empty(len(row) - 1)
        self.lib.ref_ilu_solve(len(row) - 1, len(col), _i32(row), _i32(col), _f64(val), _f64(r), z)
        return z

    def block_precond(self, kind, row, col, val, r_perm, omega=1.0):
        """kind 2 MC-SGS, 3 ILU(0)+level scheduling, 4 ILU(0) multicoloured."""
        n, nnz = len(row) - 1, len(col)
        z, perm, sizes = np.empty(n), np.empty(n, np.int32), np.empty(n, np.int32)
        nb = C.c_int()
        Ar, Ac, Av = np.empty(n + 1, np.int32), np.empty(nnz, np.int32), np.empty(nnz)
        self.lib.ref_block_precond(kind, omega, n, nnz, _i32(row), _i32(col), _f64(val), _f64(r_perm), z,
                                   perm, C.byref(nb), sizes, Ar, Ac, Av)
        return dict(z=z, perm=perm, nblocks=nb.value, sizes=sizes[:nb.value].copy(), A=(Ar, Ac, Av))

    def block_precond_ilup(self, mode, ilu_p, mat_power, row, col, val, r_perm):
        """lPreconditioner_MultiColoring_ILUp with ILU(ilu_p); mode 3 levels, 4 colours."""
        n, nnz = len(row) - 1, len(col)
        z, perm, sizes = np.empty(n), np.empty(n, np.int32), np.empty(n, np.int32)
        nb = C.c_int()
        Ar, Ac, Av = np.empty(n + 1, np.int32), np.empty(nnz, np.int32), np.empty(nnz)
        self.lib.ref_block_precond_ilup(mode, ilu_p, mat_power, n, nnz, _i32(row), _i32(col), _f64(val),
                                        _f64(r_perm), z, perm, C.byref(nb), sizes, Ar, Ac, Av)
        return dict(z=z, perm=perm, nblocks=nb.value, sizes=sizes[:nb.value].copy(), A=(Ar, Ac, Av))

    def ilup(self, row, col, val, p, cap=None):
        n, nnz = len(row) - 1, len(col)
        cap = cap or 40 * nnz + 16
        r, c, v = np.empty(n + 1, np.int32), np.empty(cap, np.int32), np.empty(cap)
        m = self.lib.ref_ilup(n, nnz, _i32(row), _i32(col), _f64(val), p, cap, r, c, v)
        assert m >= 0
        return r, c[:m].copy(), v[:m].copy()

    def vec_reduce(self, x):
        a, b, c, d = C.c_int(), C.c_int(), C.c_double(), C.c_double()
        self.lib.ref_vec_reduce(len(x), _f64(x), C.byref(a), C.byref(b), C.byref(c), C.byref(d))
        return a.value, b.value, c.value, d.value

    def rot(self, x, y, c=0.0, s=0.0, param=None):
        x, y = _f64(x).copy(), _f64(y).copy()
        p = None if param is None else _f64(param)
        self.lib.ref_vec_rot(x.size, x, y, c, s, None if p is None else p.ctypes.data)
        return x, y

    def rotg(self, a, b):
        v = [C.c_double(a), C.c_double(b), C.c_double(), C.c_double()]
        self.lib.ref_rotg(*[C.byref(q) for q in v])
        return tuple(q.value for q in v)

    def csr_scale(self, row, col, val, alpha, mode, m=None):
        n = len(row) - 1
        v = _f64(val).copy()
        self.lib.ref_csr_scale(n, m or n, len(col), _i32(row), _i32(col), v, alpha, mode)
        return v

    def csr_diag(self, row, col, val, start, end, inverse=False, m=None):
        n = len(row) - 1
        out = np.empty(end - start)
        self.lib.ref_csr_diag(n, m or n, len(col), _i32(row), _i32(col), _f64(val), start, end, int(inverse), out)
        return out

    def csr_extract(self, row, col, val, mode, sr=0, sc=0, er=0, ec=0, m=None):
        n, nnz = len(row) - 1, len(col)
        rows = (er - sr if mode == 0 else n) + 1
        r, c, v = np.empty(rows, np.int32), np.empty(max(nnz, 1), np.int32), np.empty(max(nnz, 1))
        k = self.lib.ref_csr_extract(n, m or n, nnz, _i32(row), _i32(col), _f64(val), mode, sr, sc, er, ec,
                                     max(nnz, 1), r, c, v)
        assert k >= 0
        return r, c[:k].copy(), v[:k].copy()

    def power_pattern(self, row, col, p, cap=None):
        n, nnz = len(row) - 1, len(col)
        cap = cap or 60 * nnz + 16
        r, c = np.empty(n + 1, np.int32), np.empty(cap, np.int32)
        m = self.lib.ref_power_pattern(n, nnz, _i32(row), _i32(col), p, cap, r, c)
        assert m >= 0
        return r, c[:m].copy()

    def pcg(self, row, col, val, b, precond=0, impl=0, nthreads=1, maxits=1000, abstol=0.0,
            reltol=1e-10, divtol=1e6, history=False):
        n = len(row) - 1
        x = np.zeros(n)
        it, res = C.c_int(), C.c_double()
        hist = np.zeros(maxits + 1) if history else None
        conv = self.lib.ref_pcg(precond, impl, nthreads, n, len(col), _i32(row), _i32(col), _f64(val),
                                _f64(b), x, maxits, abstol, reltol, divtol, C.byref(it), C.byref(res),
                                hist.ctypes.data if history else None)
        out = dict(x=x, iters=it.value, res=res.value, status=conv)
        if history:
            out["history"] = hist[:it.value + 1]
        return out

    def gmres(self, row, col, val, b, precond=0, m=30, impl=0, nthreads=1, maxits=1000, abstol=0.0,
              reltol=1e-9, divtol=1e6, ilu_p=0, mat_power=1):
        n = len(row) - 1
        x = np.zeros(n)
        it, res = C.c_int(), C.c_double()
        self.lib.ref_set_ilup(ilu_p, mat_power)
        conv = self.lib.ref_gmres(precond, impl, nthreads, m, n, len(col), _i32(row), _i32(col), _f64(val),
                                  _f64(b), x, maxits, abstol, reltol, divtol, C.byref(it), C.byref(res))
        self.lib.ref_set_ilup(0, 1)
        return dict(x=x, iters=it.value, res=res.value, status=conv)

    def lmp_cg(self, row, col, val, b, rel_eps=0.0, abs_eps=0.0, max_iter=100):
        x = np.zeros(len(row) - 1)
        rc = self.lib.ref_lmp_cg(len(row) - 1, len(col), _i32(row), _i32(col), _f64(val), _f64(b), x,
                                 rel_eps, abs_eps, max_iter)
        return rc, x

    def lmp_cg_iters(self, row, col, val, b, rel_eps=0.0, abs_eps=0.0, max_iter=100, jacobi=False):
        """CGFunctor<double, true> on CPUsimple objects, optionally with
        lPreconditioner_Jacobi: (code, x, iterations)."""
        L = self.lib
        L.ref_lmp_cg_iters.argtypes = [C.c_int, C.c_int, _i32p, _i32p, _f64p, _f64p, _f64p, C.c_double, C.c_double,
                                       C.c_int, C.c_int, C.POINTER(C.c_int)]
        x = np.zeros(len(row) - 1)
        it = C.c_int()
        rc = L.ref_lmp_cg_iters(len(row) - 1, len(col), _i32(row), _i32(col), _f64(val), _f64(b), x, rel_eps,
                                abs_eps, max_iter, int(jacobi), C.byref(it))
        return rc, x, it.value

    def time_spmv(self, row, col, val, x, nthreads, reps):
        y = np.empty(len(row) - 1)
        t = self.lib.ref_time_spmv(nthreads, reps, len(row) - 1, len(col), _i32(row), _i32(col),
                                   _f64(val), _f64(x), y)
        return t, y

    def max_threads(self):
        return self.lib.ref_max_threads()

    def q1_rhs(self, seed, dim, N):
        """The seeded right-hand side (the C restatement linked into this library)."""
        b = np.empty((N + 1) ** dim)
        self.lib.orc_q1_rhs.argtypes = [C.c_uint64, C.c_int, C.c_int, _f64p]
        self.lib.orc_q1_rhs.restype = None
        self.lib.orc_q1_rhs(seed, dim, N, b)
        return b


def _ref_timing_sigs(L):
    L.ref_mpir.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, _i32p, _i32p, _f64p, _f64p, _f64p, C.c_int,
                           C.c_double, C.c_double, C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int),
                           C.POINTER(C.c_double)]
    L.ref_mpir.restype = C.c_double
    L.ref_pcg_timed.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, _i32p, _i32p, _f64p, _f64p, _f64p,
                                C.c_double, C.c_int, C.POINTER(C.c_int)]
    L.ref_pcg_timed.restype = C.c_double


def ref_mpir(ref, row, col, val, b, nthreads, max_outer=50, reltol=1e-10, inner_reltol=1e-4,
             inner_maxits=100000, sample_inner=0, impl=1):
    """The reference's lmp objects driving MPIR (FP64 outer, FP32 Jacobi-CG inner)."""
    _ref_timing_sigs(ref.lib)
    n = len(row) - 1
    x = np.zeros(n)
    o, i, r = C.c_int(), C.c_int(), C.c_double()
    dt = ref.lib.ref_mpir(impl, nthreads, n, len(col), _i32(row), _i32(col), _f64(val), _f64(b), x, max_outer,
                          reltol, inner_reltol, inner_maxits, sample_inner, C.byref(o), C.byref(i), C.byref(r))
    return dict(seconds=dt, outer=o.value, inner_total=i.value, res=r.value, x=x)


def ref_pcg_timed(ref, row, col, val, b, nthreads, reltol=1e-10, maxits=100000, impl=1):
    _ref_timing_sigs(ref.lib)
    n = len(row) - 1
    x = np.zeros(n)
    it = C.c_int()
    dt = ref.lib.ref_pcg_timed(impl, nthreads, n, len(col), _i32(row), _i32(col), _f64(val), _f64(b), x, reltol,
                               maxits, C.byref(it))
    return dict(seconds=dt, iters=it.value, x=x)


class RefMpirSession:
    """The reference's MPIR over CPUopenmp objects that persist between
    solves (ref_mpir_create / ref_mpir_run / ref_mpir_threads), so that each
    timed solve excludes the matrix copies and the preconditioner build."""

    def __init__(self, ref, row, col, val, nthreads):
        L = self.lib = ref.lib
        L.ref_mpir_create.argtypes = [C.c_int, C.c_int, C.c_int, _i32p, _i32p, _f64p]
        L.ref_mpir_create.restype = C.c_void_p
        L.ref_mpir_threads.argtypes = [C.c_void_p, C.c_int]
        L.ref_mpir_threads.restype = None
        L.ref_mpir_run.argtypes = [C.c_void_p, _f64p, _f64p, C.c_int, C.c_double, C.c_double, C.c_int, C.c_int,
                                   C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_double)]
        L.ref_mpir_run.restype = C.c_double
        L.ref_mpir_destroy.argtypes = [C.c_void_p]
        L.ref_mpir_destroy.restype = None
        self.n = len(row) - 1
        self.h = L.ref_mpir_create(nthreads, self.n, len(col), _i32(row), _i32(col), _f64(val))

    def threads(self, nthreads):
        self.lib.ref_mpir_threads(self.h, nthreads)

    def run(self, b, max_outer=50, reltol=1e-10, inner_reltol=1e-4, inner_maxits=100000, sample_inner=0):
        x = np.zeros(self.n)
        o, i, r = C.c_int(), C.c_int(), C.c_double()
        dt = self.lib.ref_mpir_run(self.h, _f64(b), x, max_outer, reltol, inner_reltol, inner_maxits, sample_inner,
                                   C.byref(o), C.byref(i), C.byref(r))
        return dict(seconds=dt, outer=o.value, inner_total=i.value, res=r.value, x=x)

    def close(self):
        if self.h:
            self.lib.ref_mpir_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()
