"""B200 lmp platform for HiFlow3 -- Python mirror of the reference's operator API.

The product is ``libb200la.so`` (this directory), a C-ABI library of
hand-written sm_100a kernels and their host orchestration; this module binds it
with ctypes so tests and benchmarks read like the reference's own
(``test/LinearAlgebra/cg.cc``, ``gmres.cc``): ``CSR_lMatrix.VectorMult``,
``lVector.Dot / Axpy / ScaleAdd``, ``CG.SetupOperator / InitControl / Solve``.
Device memory is owned by PyTorch CUDA tensors (plumbing only); every
arithmetic operation runs in the library's kernels.  There is no CPU fallback:
constructing a ``Platform`` without a B200 raises.

The directory name is not a Python identifier; load it with
``importlib.util.spec_from_file_location``.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libb200la.so")

F64, F32 = 0, 1
NOALLOC_MAX_N = 67108864      # B200LA_NOALLOC_MAX_N of include/b200la.h
PRECOND_JACOBI, PRECOND_MCSGS, PRECOND_ILU0_LS, PRECOND_ILU0_MC = 1, 2, 3, 4
ITERATE, SUCCESS_ABS, SUCCESS_REL, FAIL_DIV, FAIL_MAXITS = range(5)

STATUS = {0: "ok", 1: "invalid argument", 2: "CUDA error", 3: "allocation failed",
          4: "no usable sm_100 device", 5: "malformed CSR", 6: "refused by memory budget",
          7: "bounded device wait gave up", 8: "preconditioner setup failed", 9: "unknown request",
          10: "request pending", 11: "file I/O failed", 12: "unsupported or malformed file"}
PENDING = 10
ERR_ARG, ERR_CSR, ERR_IO, ERR_FORMAT = 1, 5, 11, 12
SERVE_CG, SERVE_GMRES = 0, 1
SERVE_F64, SERVE_MIXED = 0, 1


class B200Error(RuntimeError):
    def __init__(self, code, msg=""):
        self.code = code
        super().__init__(f"b200la error {code} ({STATUS.get(code, '?')}){': ' + msg if msg else ''}")


class Control(C.Structure):
    """IterateControl (src/common/iterate_control.h)."""
    _fields_ = [("maxits", C.c_int), ("abstol", C.c_double), ("reltol", C.c_double), ("divtol", C.c_double)]


class Result(C.Structure):
    _fields_ = [("iters", C.c_int), ("status", C.c_int), ("res0", C.c_double), ("res", C.c_double),
                ("outer", C.c_int), ("launches", C.c_int), ("solve_ms", C.c_double)]


class ServeConfig(C.Structure):
    """b200la_serve_config."""
    _fields_ = [("device", C.c_int), ("budget_bytes", C.c_double), ("max_slots", C.c_int),
                ("active_bytes", C.c_double), ("max_active", C.c_int), ("iters_per_round", C.c_int),
                ("autotune", C.c_int), ("warps", C.c_int), ("ctas_per_sm", C.c_int), ("chunks_per_warp", C.c_int)]


class Request(C.Structure):
    """b200la_request."""
    _fields_ = [("method", C.c_int), ("precision", C.c_int), ("n", C.c_int), ("nnz", C.c_int),
                ("row", C.c_void_p), ("col", C.c_void_p), ("val", C.c_void_p),
                ("q1_dim", C.c_int), ("q1_N", C.c_int), ("q1_kind", C.c_int), ("q1_kcell", C.c_void_p),
                ("q1_nu", C.c_double), ("q1_beta", C.c_double * 3), ("b", C.c_void_p), ("rhs_seed", C.c_uint64),
                ("x", C.c_void_p), ("ctl", Control), ("inner", Control), ("max_outer", C.c_int),
                ("gmres_m", C.c_int), ("gmres_precond", C.c_int)]


class ServeResult(C.Structure):
    """b200la_serve_result."""
    _fields_ = [("status", C.c_int), ("iters", C.c_int), ("outer", C.c_int), ("res0", C.c_double),
                ("res", C.c_double), ("t_submit", C.c_double), ("t_admit", C.c_double), ("t_ready", C.c_double),
                ("t_done", C.c_double), ("bytes", C.c_double)]


class ServeInfo(C.Structure):
    """b200la_serve_info."""
    _fields_ = [("submitted", C.c_longlong), ("completed", C.c_longlong), ("failed", C.c_longlong),
                ("rounds", C.c_longlong), ("batch_iters", C.c_longlong), ("busy_ms", C.c_double),
                ("resident_bytes", C.c_double), ("peak_resident_bytes", C.c_double), ("peak_active", C.c_int),
                ("warps", C.c_int), ("ctas_per_sm", C.c_int), ("chunks_per_warp", C.c_int),
                ("iters_per_round", C.c_int), ("active_bytes", C.c_double)]


def build(force=False):
    """Compile libb200la.so in place (nvcc, sm_100a)."""
    if force or not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-C", HERE, "-j8"], check=True)
    return LIB_PATH


_lib = None

_P = C.c_void_p
_I = C.c_int
_D = C.c_double


def lib():
    """Load libb200la.so, declaring every entry point of include/b200la.h."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C {HERE}` (no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    sig = {
        "b200la_create": ([_I, C.POINTER(_P)], _I),
        "b200la_destroy": ([_P], _I),
        "b200la_set_stream": ([_P, _P], _I),
        "b200la_get_stream": ([_P], _P),
        "b200la_sync": ([_P], _I),
        "b200la_last_error": ([_P], C.c_char_p),
        "b200la_status_string": ([_I], C.c_char_p),
        "b200la_num_sms": ([_P], _I),
        "b200la_malloc": ([_P, C.c_size_t, C.POINTER(_P)], _I),
        "b200la_free": ([_P, _P], _I),
        "b200la_memcpy_h2d": ([_P, _P, _P, C.c_size_t], _I),
        "b200la_memcpy_d2h": ([_P, _P, _P, C.c_size_t], _I),
        "b200la_memcpy_d2d": ([_P, _P, _P, C.c_size_t], _I),
        "b200la_memset_zero": ([_P, _P, C.c_size_t], _I),
        "b200la_host_alloc": ([_P, C.c_size_t, C.POINTER(_P)], _I),
        "b200la_host_free": ([_P, _P], _I),
        "b200la_timer_start": ([_P], _I),
        "b200la_timer_stop": ([_P, C.POINTER(_D)], _I),
        "b200la_csr_create": ([_P, _I, _I, _I, _P, _P, _P, _I, C.POINTER(_P)], _I),
        "b200la_csr_create_segmented": ([_P, _I, _I, _I, _P, _P, _P, _I, _I, _P, C.POINTER(_P)], _I),
        "b200la_csr_destroy": ([_P], _I),
        "b200la_csr_cast": ([_P, _P, _I, C.POINTER(_P)], _I),
        "b200la_csr_info": ([_P] + [C.POINTER(_I)] * 7, _I),
        "b200la_csr_download": ([_P, _P, _P, _P, _P], _I),
        "b200la_csr_format": ([_P, C.POINTER(_I), C.POINTER(_I)], _I),
        "b200la_csr_set_values": ([_P, _P, _P], _I),
        "b200la_csr_invdiag": ([_P, _P, _P], _I),
        "b200la_csr_scale": ([_P, _P, _D, _I], _I),
        "b200la_iamin": ([_P, _I, _I, _P, C.POINTER(_I)], _I),
        "b200la_iamax": ([_P, _I, _I, _P, C.POINTER(_I)], _I),
        "b200la_normmax": ([_P, _I, _I, _P, C.POINTER(_D)], _I),
        "b200la_asum": ([_P, _I, _I, _P, C.POINTER(_D)], _I),
        "b200la_rot": ([_P, _I, _I, _P, _P, _D, _D], _I),
        "b200la_rotm": ([_P, _I, _I, _P, _P, C.POINTER(_D)], _I),
        "b200la_rotg": ([_I, _P, _P, _P, _P], _I),
        "b200la_vec_add_values": ([_P, _I, _I, _P, _I, _P, _P], _I),
        "b200la_spmv_add_remote": ([_P, _P, _P, _P, _P, _P], _I),
        "b200la_enable_peer_access": ([_I, _I], _I),
        "b200la_comm_unique_id": ([_P], _I),
        "b200la_comm_create_nccl": ([_P, _P, _I, _I, _P], _I),
        "b200la_comm_create_local": ([_I, _P], _I),
        "b200la_comm_info": ([_P, C.POINTER(_I), C.POINTER(_I)], _I),
        "b200la_comm_destroy": ([_P], _I),
        "b200la_coupled_create": ([_P, _P, _P, _P, _P, _P, _P, _P], _I),
        "b200la_coupled_destroy": ([_P], _I),
        "b200la_coupled_update_ghost": ([_P, _P, _P, _P], _I),
        "b200la_coupled_spmv": ([_P, _P, _P, _P], _I),
        "b200la_coupled_dot": ([_P, _P, _P, _P, C.POINTER(_D)], _I),
        "b200la_coupled_cg": ([_P, _P, _P, _P, _P, C.POINTER(Control), C.POINTER(Result)], _I),
        "b200la_vec_set_values": ([_P, _I, _I, _P, _I, _P, _P], _I),
        "b200la_csr_diag": ([_P, _P, _I, _I, _I, _P], _I),
        "b200la_csr_extract_submatrix": ([_P, _P, _I, _I, _I, _I, C.POINTER(_P)], _I),
        "b200la_csr_compress": ([_P, _P, C.POINTER(_P)], _I),
        "b200la_spmv": ([_P, _P, _P, _P], _I),
        "b200la_spmv_add": ([_P, _P, _P, _P], _I),
        "b200la_spmv_dot": ([_P, _P, _P, _P, _P], _I),
        "b200la_residual": ([_P, _P, _P, _P, _P, _P], _I),
        "b200la_dot": ([_P, _I, _I, _P, _P, C.POINTER(_D)], _I),
        "b200la_nrm2": ([_P, _I, _I, _P, C.POINTER(_D)], _I),
        "b200la_dot_dev": ([_P, _I, _I, _P, _P, _P], _I),
        "b200la_dot_noalloc": ([_I, _I, _P, _P, _P, _P], _I),
        "b200la_axpy": ([_P, _I, _I, _D, _P, _P], _I),
        "b200la_scaleadd": ([_P, _I, _I, _D, _P, _P], _I),
        "b200la_scale": ([_P, _I, _I, _D, _P], _I),
        "b200la_ewmul": ([_P, _I, _I, _P, _P], _I),
        "b200la_cast": ([_P, _I, _P, _I, _P, _I], _I),
        "b200la_gather": ([_P, _I, _I, _P, _P, _P], _I),
        "b200la_scatter": ([_P, _I, _I, _P, _P, _P], _I),
        "b200la_permute": ([_P, _I, _I, _P, _P, _P], _I),
        "b200la_coo_to_csr": ([_I, _I, _P, _P, _P, _P, _P, _P], _I),
        "b200la_async_jacobi": ([_P, _P, _P, _P, _P, _P, _I, _I, C.c_double, C.POINTER(Control), C.POINTER(Result)],
                                _I),
        "b200la_gmg_residual": ([_P, _P, _P, _P, _P, _P, _P], _I),
        "b200la_gmg_restriction": ([_P, _P, _P, _P, _P, _P], _I),
        "b200la_gmg_prolongation_add": ([_P, _P, _P, _P, _P, _P], _I),
        "b200la_rowblock_split": ([_I, _I, _P, _P, _P, _I, _I, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P], _I),
        "b200la_mm_read_info": ([C.c_char_p, _P, _P, _P], _I),
        "b200la_mm_read_csr": ([C.c_char_p, _I, _I, _P, _P, _P], _I),
        "b200la_mm_write_csr": ([C.c_char_p, _I, _I, _I, _P, _P, _P], _I),
        "b200la_vec_read_info": ([C.c_char_p, _P], _I),
        "b200la_vec_read": ([C.c_char_p, _I, _P], _I),
        "b200la_vec_write": ([C.c_char_p, _I, _P], _I),
        "b200la_add_values": ([_P, _P, _P, _P, _I, _P, _I, _P], _I),
        "b200la_zero_rows": ([_P, _P, _P, _P, _I, _D], _I),
        "b200la_multicoloring": ([_I, _P, _P, C.POINTER(_I), _P, _P], _I),
        "b200la_levelscheduling": ([_I, _P, _P, C.POINTER(_I), _P, _P], _I),
        "b200la_reorder_csr": ([_I, _P, _P, _P, _P, _P, _P, _P], _I),
        "b200la_ilu0": ([_I, _P, _P, _P], _I),
        "b200la_matrix_power_pattern": ([_I, _P, _P, _I, _P, _P, _P], _I),
        "b200la_ilup": ([_I, _P, _P, _P, _I, _P, _P, _P, _P], _I),
        "b200la_q1_sizes": ([_I, _I, C.POINTER(_I), C.POINTER(C.c_int64)], _I),
        "b200la_q1_assemble": ([_I, _I, _I, _P, _D, _P, _P, _P, _P], _I),
        "b200la_q1_rhs": ([C.c_uint64, _I, _I, _P], _I),
        "b200la_precond_jacobi": ([_P, _P, C.POINTER(_P)], _I),
        "b200la_precond_mcsgs": ([_P, _I, _P, _P, _P, _D, _I, C.POINTER(_P), C.POINTER(_P)], _I),
        "b200la_precond_ilu0": ([_P, _I, _P, _P, _P, _I, _I, C.POINTER(_P), C.POINTER(_P)], _I),
        "b200la_precond_ilup": ([_P, _I, _P, _P, _P, _I, _I, _I, _I, C.POINTER(_P), C.POINTER(_P)], _I),
        "b200la_precond_info": ([_P, C.POINTER(_I), C.POINTER(_I), C.POINTER(_I), _P, _P], _I),
        "b200la_precond_apply": ([_P, _P, _P, _P], _I),
        "b200la_precond_destroy": ([_P], _I),
        "b200la_cg": ([_P, _P, _P, _P, _P, C.POINTER(Control), C.POINTER(Result)], _I),
        "b200la_cg_hist": ([_P, _P, _P, _P, _P, C.POINTER(Control), C.POINTER(Result), _P, _I], _I),
        "b200la_gmres": ([_P, _P, _P, _I, _P, _P, C.POINTER(Control), C.POINTER(Result)], _I),
        "b200la_mpir": ([_P, _P, _P, _P, _P, C.POINTER(Control), C.POINTER(Control), _I, C.POINTER(Result)], _I),
        "b200la_mpir_gmres": ([_P, _P, _P, _P, _I, _P, _P, C.POINTER(Control), C.POINTER(Control), _I,
                               C.POINTER(Result)], _I),
        "b200la_q1_assemble_device": ([_P, _I, _I, _I, _P, _D, _P, _P, _P, _P], _I),
        "b200la_q1_rhs_device": ([_P, C.c_uint64, _I, _I, _P], _I),
        "b200la_serve_start": ([C.POINTER(ServeConfig), C.POINTER(_P)], _I),
        "b200la_serve_submit": ([_P, C.POINTER(Request), C.POINTER(C.c_longlong)], _I),
        "b200la_serve_poll": ([_P, C.c_longlong, C.POINTER(ServeResult)], _I),
        "b200la_serve_wait": ([_P, C.c_longlong, _D, C.POINTER(ServeResult)], _I),
        "b200la_serve_stats": ([_P, C.POINTER(ServeInfo)], _I),
        "b200la_serve_stop": ([_P], _I),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


def exported_symbols():
    """Names of the entry points declared in include/b200la.h."""
    import re
    hdr = open(os.path.join(HERE, "..", "include", "b200la.h")).read()
    decl = r"^\s*(?:int|void|const char)\s*\*?\s*(b200la_[a-z0-9_]+)\s*\("
    return sorted(set(re.findall(decl, hdr, flags=re.M)))


def _np_ptr(a):
    return a.ctypes.data_as(C.c_void_p)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


# ----------------------------------------------------------------- host setup
# The one-time host algorithms of the platform (results identical to the
# reference's: CSR assembly, colouring, level scheduling, ILU(0)).

def _check(rc, what=""):
    if rc != 0:
        raise B200Error(rc, what)


def q1_sizes(dim, N):
    n, nnz = C.c_int(), C.c_int64()
    _check(lib().b200la_q1_sizes(dim, N, C.byref(n), C.byref(nnz)), "q1_sizes")
    return n.value, nnz.value


def q1_assemble(dim, N, kind=0, kcell=None, nu=1.0, beta=(0.0, 0.0, 0.0)):
    n, nnz = q1_sizes(dim, N)
    row, col, val = np.empty(n + 1, np.int32), np.empty(nnz, np.int32), np.empty(nnz)
    kc = _f64(kcell) if kcell is not None else None
    b3 = _f64(list(beta) + [0.0] * (3 - len(beta)))
    _check(lib().b200la_q1_assemble(dim, N, kind, _np_ptr(kc) if kc is not None else None, nu, _np_ptr(b3),
                                    _np_ptr(row), _np_ptr(col), _np_ptr(val)), "q1_assemble")
    return row, col, val


def q1_rhs(seed, dim, N):
    n, _ = q1_sizes(dim, N)
    b = np.empty(n)
    _check(lib().b200la_q1_rhs(seed, dim, N, _np_ptr(b)), "q1_rhs")
    return b


def coo_to_csr(n, coo_row, coo_col, coo_val=None):
    coo_row, coo_col = _i32(coo_row), _i32(coo_col)
    nnz = coo_row.size
    row, col = np.empty(n + 1, np.int32), np.empty(nnz, np.int32)
    if coo_val is None:
        _check(lib().b200la_coo_to_csr(n, nnz, _np_ptr(coo_row), _np_ptr(coo_col), None, _np_ptr(row),
                                       _np_ptr(col), None), "coo_to_csr")
        return row, col
    cv, val = _f64(coo_val), np.empty(nnz)
    _check(lib().b200la_coo_to_csr(n, nnz, _np_ptr(coo_row), _np_ptr(coo_col), _np_ptr(cv), _np_ptr(row),
                                   _np_ptr(col), _np_ptr(val)), "coo_to_csr")
    return row, col, val


# ----------------------------------------------------------------- file I/O
# MatrixMarket matrices and plain-text vectors with the reference's reading
# and writing rules (CPU_CSR_lMatrix::ReadFile / WriteFile,
# lmp/lmatrix_csr_cpu.cc:1733-1765; CPU_lVector::ReadFile / WriteFile,
# lmp/lvector_cpu.cc:582-663).  B200Error with B200LA_ERR_IO / _FORMAT / _CSR
# where the reference would exit.

def _path(path):
    return os.fsencode(os.fspath(path))


def read_matrix_market(path):
    """(row, col, val, n_cols) of a MatrixMarket file, as the reference's CSR."""
    n, m, nnz = C.c_int(), C.c_int(), C.c_int()
    _check(lib().b200la_mm_read_info(_path(path), C.byref(n), C.byref(m), C.byref(nnz)), f"read {path}")
    row, col, val = np.empty(n.value + 1, np.int32), np.empty(nnz.value, np.int32), np.empty(nnz.value)
    _check(lib().b200la_mm_read_csr(_path(path), n.value, nnz.value, _np_ptr(row), _np_ptr(col), _np_ptr(val)),
           f"read {path}")
    return row, col, val, m.value


def write_matrix_market(path, row, col, val, n_cols=None):
    """Write a host CSR as the reference does (entries as "column row value")."""
    row, col, val = _i32(row), _i32(col), _f64(val)
    n = row.size - 1
    _check(lib().b200la_mm_write_csr(_path(path), n, n if n_cols is None else int(n_cols), col.size, _np_ptr(row),
                                     _np_ptr(col), _np_ptr(val)), f"write {path}")


def read_vector(path):
    """The values of a one-value-per-line text file, counted as the reference counts them."""
    n = C.c_int()
    _check(lib().b200la_vec_read_info(_path(path), C.byref(n)), f"read {path}")
    x = np.empty(max(n.value, 0))
    _check(lib().b200la_vec_read(_path(path), x.size, _np_ptr(x)), f"read {path}")
    return x


def write_vector(path, x):
    x = _f64(x)
    _check(lib().b200la_vec_write(_path(path), x.size, _np_ptr(x)), f"write {path}")


def add_values(row, col, val, rows, cols, values):
    row, col, val = _i32(row), _i32(col), _f64(val).copy()
    rows, cols, values = _i32(rows), _i32(cols), _f64(values)
    _check(lib().b200la_add_values(_np_ptr(row), _np_ptr(col), _np_ptr(val), _np_ptr(rows), rows.size,
                                   _np_ptr(cols), cols.size, _np_ptr(values)), "add_values")
    return val


def zero_rows(row, col, val, idx, alpha=1.0):
    row, col, val, idx = _i32(row), _i32(col), _f64(val).copy(), _i32(idx)
    _check(lib().b200la_zero_rows(_np_ptr(row), _np_ptr(col), _np_ptr(val), _np_ptr(idx), idx.size, alpha))
    return val


def multicoloring(row, col):
    row, col = _i32(row), _i32(col)
    n = row.size - 1
    nc, sizes, perm = C.c_int(), np.empty(n, np.int32), np.empty(n, np.int32)
    _check(lib().b200la_multicoloring(n, _np_ptr(row), _np_ptr(col), C.byref(nc), _np_ptr(sizes), _np_ptr(perm)),
           "multicoloring")
    return nc.value, sizes[:nc.value].copy(), perm


def levelscheduling(row, col):
    row, col = _i32(row), _i32(col)
    n = row.size - 1
    nl, sizes, perm = C.c_int(), np.empty(n, np.int32), np.empty(n, np.int32)
    _check(lib().b200la_levelscheduling(n, _np_ptr(row), _np_ptr(col), C.byref(nl), _np_ptr(sizes),
                                        _np_ptr(perm)), "levelscheduling")
    return nl.value, sizes[:nl.value].copy(), perm


def reorder_csr(row, col, val, perm):
    row, col, val, perm = _i32(row), _i32(col), _f64(val), _i32(perm)
    n = row.size - 1
    r2, c2, v2 = np.empty(n + 1, np.int32), np.empty(col.size, np.int32), np.empty(col.size)
    _check(lib().b200la_reorder_csr(n, _np_ptr(row), _np_ptr(col), _np_ptr(val), _np_ptr(perm), _np_ptr(r2),
                                    _np_ptr(c2), _np_ptr(v2)), "reorder_csr")
    return r2, c2, v2


def ilu0(row, col, val):
    row, col, v = _i32(row), _i32(col), _f64(val).copy()
    _check(lib().b200la_ilu0(row.size - 1, _np_ptr(row), _np_ptr(col), _np_ptr(v)), "ilu0")
    return v


def rowblock_split(row, col, val, n_global, col_begin, col_end):
    """The rows of one rank split into (diag CSR, offdiag CSR, ghost global
    numbers): CoupledMatrix::InitStructure with LaCouplings' ghost numbering."""
    row, col, val = _i32(row), _i32(col), _f64(val)
    n = row.size - 1
    nd, no, ng = C.c_int(), C.c_int(), C.c_int()
    args = (n, n_global, _np_ptr(row), _np_ptr(col), _np_ptr(val), col_begin, col_end)
    _check(lib().b200la_rowblock_split(*args, C.byref(nd), C.byref(no), C.byref(ng), *([None] * 7)), "rowblock_split")
    rd, cd, vd = np.empty(n + 1, np.int32), np.empty(nd.value, np.int32), np.empty(nd.value)
    ro, co, vo = np.empty(n + 1, np.int32), np.empty(no.value, np.int32), np.empty(no.value)
    g = np.empty(ng.value, np.int32)
    _check(lib().b200la_rowblock_split(*args, C.byref(nd), C.byref(no), C.byref(ng), _np_ptr(rd), _np_ptr(cd),
                                       _np_ptr(vd), _np_ptr(ro), _np_ptr(co), _np_ptr(vo), _np_ptr(g)),
           "rowblock_split")
    return (rd, cd, vd), (ro, co, vo), g


def matrix_power_pattern(row, col, p):
    """(row, col) of the pattern of A^p (MatrixSupSPower)."""
    row, col = _i32(row), _i32(col)
    n, nnz = row.size - 1, C.c_int()
    _check(lib().b200la_matrix_power_pattern(n, _np_ptr(row), _np_ptr(col), p, C.byref(nnz), None, None),
           "matrix_power_pattern")
    ro, co = np.empty(n + 1, np.int32), np.empty(nnz.value, np.int32)
    _check(lib().b200la_matrix_power_pattern(n, _np_ptr(row), _np_ptr(col), p, C.byref(nnz), _np_ptr(ro),
                                             _np_ptr(co)), "matrix_power_pattern")
    return ro, co


def ilup(row, col, val, p):
    """ILU(p) factors (row, col, val) on the level-of-fill pattern (ilup)."""
    row, col, val = _i32(row), _i32(col), _f64(val)
    n, nnz = row.size - 1, C.c_int()
    _check(lib().b200la_ilup(n, _np_ptr(row), _np_ptr(col), _np_ptr(val), p, C.byref(nnz), None, None, None), "ilup")
    ro, co, vo = np.empty(n + 1, np.int32), np.empty(nnz.value, np.int32), np.empty(nnz.value)
    _check(lib().b200la_ilup(n, _np_ptr(row), _np_ptr(col), _np_ptr(val), p, C.byref(nnz), _np_ptr(ro), _np_ptr(co),
                             _np_ptr(vo)), "ilup")
    return ro, co, vo


# ----------------------------------------------------------------- device side

def _torch():
    import torch
    return torch


class Platform:
    """init_platform for the B200 (src/linear_algebra/lmp/platform_management.cc:135-185)."""

    def __init__(self, device=0):
        torch = _torch()
        if not torch.cuda.is_available():
            raise B200Error(4, "no CUDA device visible (the B200 platform has no CPU fallback)")
        torch.cuda.set_device(device)
        torch.cuda.init()
        self.device = device
        h = C.c_void_p()
        _check(lib().b200la_create(device, C.byref(h)), "b200la_create")
        self.h = h

    def check(self, rc, what=""):
        if rc != 0:
            msg = lib().b200la_last_error(self.h).decode()
            raise B200Error(rc, f"{what}: {msg}" if what else msg)

    def sync(self):
        self.check(lib().b200la_sync(self.h), "sync")

    def stream(self):
        """The platform's CUDA stream (every kernel of this platform runs on it)
        as a torch stream, for ordering other work against it with events."""
        torch = _torch()
        if getattr(self, "_ts", None) is None:
            self._ts = torch.cuda.ExternalStream(lib().b200la_get_stream(self.h) or 0, device=f"cuda:{self.device}")
        return self._ts

    def on_stream(self):
        """Context in which torch allocates, fills and copies on the
        platform's stream.  Every device tensor the platform hands to the
        library is made inside it: the caching allocator then reuses a freed
        block only in that stream's order, after the library's kernels that
        still read it (a temporary input freed as soon as the call returns)."""
        return _torch().cuda.stream(self.stream())

    def num_sms(self):
        return lib().b200la_num_sms(self.h)

    def timer_start(self):
        self.check(lib().b200la_timer_start(self.h), "timer_start")

    def timer_stop(self):
        ms = C.c_double()
        self.check(lib().b200la_timer_stop(self.h, C.byref(ms)), "timer_stop")
        return ms.value

    def host_alloc(self, nbytes):
        """A page-locked host buffer (returned as a ctypes pointer; free with host_free)."""
        p = C.c_void_p()
        self.check(lib().b200la_host_alloc(self.h, nbytes, C.byref(p)), "host_alloc")
        return p

    def host_free(self, p):
        self.check(lib().b200la_host_free(self.h, p), "host_free")

    def close(self):
        if getattr(self, "h", None):
            lib().b200la_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def vector_from_file(self, path, dtype=F64):
        """A vector read from a one-value-per-line file (CPU_lVector::ReadFile)."""
        return self.vector(read_vector(path), dtype)

    # vectors are torch CUDA tensors
    def vector(self, data_or_n, dtype=F64):
        torch = _torch()
        td = torch.float64 if dtype == F64 else torch.float32
        with self.on_stream():
            if isinstance(data_or_n, int):
                return lVector(self, torch.zeros(data_or_n, dtype=td, device=f"cuda:{self.device}"))
            a = np.ascontiguousarray(data_or_n, dtype=np.float64 if dtype == F64 else np.float32)
            return lVector(self, torch.from_numpy(a).to(f"cuda:{self.device}"))


def _dt(t):
    torch = _torch()
    if t.dtype == torch.float64:
        return F64
    if t.dtype == torch.float32:
        return F32
    raise TypeError("vectors are float64 or float32")


class lVector:
    """lVector<T> on the B200 (src/linear_algebra/lmp/lvector.h:39-335)."""

    def __init__(self, platform, tensor):
        self.pf, self.t = platform, tensor
        self.dtype = _dt(tensor)

    @property
    def ptr(self):
        return C.c_void_p(self.t.data_ptr())

    def get_size(self):
        return self.t.numel()

    def numpy(self):
        self.pf.sync()
        return self.t.cpu().numpy()

    def WriteFile(self, path):
        """One value per line (CPU_lVector::WriteFile)."""
        write_vector(path, self.numpy())

    def Zeros(self):
        self.pf.check(lib().b200la_memset_zero(self.pf.h, self.ptr, self.t.numel() * self.t.element_size()))

    def CopyFrom(self, other):
        self.pf.check(lib().b200la_memcpy_d2d(self.pf.h, self.ptr, other.ptr, self.t.numel() * self.t.element_size()))

    def CloneWithoutContent(self):
        with self.pf.on_stream():
            return lVector(self.pf, _torch().zeros_like(self.t))

    def Dot(self, other):
        out = C.c_double()
        self.pf.check(lib().b200la_dot(self.pf.h, self.dtype, self.get_size(), self.ptr, other.ptr, C.byref(out)),
                      "Dot")
        return out.value

    def Norm2(self):
        out = C.c_double()
        self.pf.check(lib().b200la_nrm2(self.pf.h, self.dtype, self.get_size(), self.ptr, C.byref(out)), "Norm2")
        return out.value

    def ArgMin(self):
        """First index of the smallest |x_i| (CPUsimple_lvector.cc:51-70)."""
        out = C.c_int()
        self.pf.check(lib().b200la_iamin(self.pf.h, self.dtype, self.get_size(), self.ptr, C.byref(out)), "ArgMin")
        return out.value

    def ArgMax(self):
        """First index of the largest |x_i| (CPUsimple_lvector.cc:73-92)."""
        out = C.c_int()
        self.pf.check(lib().b200la_iamax(self.pf.h, self.dtype, self.get_size(), self.ptr, C.byref(out)), "ArgMax")
        return out.value

    def NormMax(self):
        out = C.c_double()
        self.pf.check(lib().b200la_normmax(self.pf.h, self.dtype, self.get_size(), self.ptr, C.byref(out)),
                      "NormMax")
        return out.value

    def Norm1(self):
        out = C.c_double()
        self.pf.check(lib().b200la_asum(self.pf.h, self.dtype, self.get_size(), self.ptr, C.byref(out)), "Norm1")
        return out.value

    def Rot(self, vec, sc, ss):
        """self, vec <- sc self + ss vec, sc vec - ss self (CPUsimple_lvector.cc:448-466)."""
        self.pf.check(lib().b200la_rot(self.pf.h, self.dtype, self.get_size(), self.ptr, vec.ptr, sc, ss), "Rot")

    def Rotm(self, vec, sparam):
        """The modified Givens rotation sparam = (flag, h11, h21, h12, h22) (CPUsimple_lvector.cc:540-600)."""
        p = (C.c_double * 5)(*[float(v) for v in sparam])
        self.pf.check(lib().b200la_rotm(self.pf.h, self.dtype, self.get_size(), self.ptr, vec.ptr, p), "Rotm")

    def Rotg(self, sa, sb):
        """Givens rotation of (sa, sb) (CPUsimple_lvector.cc:492-535): returns (r, z, c, s)."""
        T = C.c_double if self.dtype == F64 else C.c_float
        v = [T(sa), T(sb), T(), T()]
        _check(lib().b200la_rotg(self.dtype, *[C.cast(C.byref(q), C.c_void_p) for q in v]), "Rotg")
        return tuple(q.value for q in v)

    def Axpy(self, vec, scalar):
        self.pf.check(lib().b200la_axpy(self.pf.h, self.dtype, self.get_size(), scalar, vec.ptr, self.ptr), "Axpy")

    def ScaleAdd(self, scalar, vec):
        self.pf.check(lib().b200la_scaleadd(self.pf.h, self.dtype, self.get_size(), scalar, vec.ptr, self.ptr),
                      "ScaleAdd")

    def Scale(self, scalar):
        self.pf.check(lib().b200la_scale(self.pf.h, self.dtype, self.get_size(), scalar, self.ptr), "Scale")

    def ElementWiseMult(self, vec):
        self.pf.check(lib().b200la_ewmul(self.pf.h, self.dtype, self.get_size(), vec.ptr, self.ptr),
                      "ElementWiseMult")

    def CastFrom(self, vec):
        self.pf.check(lib().b200la_cast(self.pf.h, vec.dtype, vec.ptr, self.dtype, self.ptr, self.get_size()),
                      "CastFrom")

    def GetIndexedValues(self, idx):
        torch = _torch()
        with self.pf.on_stream():
            idx_t = torch.as_tensor(_i32(idx), device=self.t.device)
            out = torch.empty(idx_t.numel(), dtype=self.t.dtype, device=self.t.device)
        self.pf.check(lib().b200la_gather(self.pf.h, self.dtype, idx_t.numel(), C.c_void_p(idx_t.data_ptr()),
                                          self.ptr, C.c_void_p(out.data_ptr())), "GetIndexedValues")
        self.pf.sync()
        return out.cpu().numpy()

    def SetIndexedValues(self, idx, values):
        torch = _torch()
        with self.pf.on_stream():
            idx_t = torch.as_tensor(_i32(idx), device=self.t.device)
            v = torch.as_tensor(np.asarray(values), dtype=self.t.dtype, device=self.t.device)
        self.pf.check(lib().b200la_scatter(self.pf.h, self.dtype, idx_t.numel(), C.c_void_p(idx_t.data_ptr()),
                                           C.c_void_p(v.data_ptr()), self.ptr), "SetIndexedValues")
        self.pf.sync()

    # index and range access (src/linear_algebra/lmp/lvector_cpu.cc:114-200, 419-550)
    def _at(self, i):
        return C.c_void_p(self.t.data_ptr() + i * self.t.element_size())

    def _host(self, values, n):
        a = np.ascontiguousarray(values, dtype=np.float64 if self.dtype == F64 else np.float32).reshape(-1)
        if a.size != n:
            raise ValueError("values has the wrong length")
        return a

    def _range(self, start, end):
        if not 0 <= start <= end <= self.get_size():
            raise B200Error(1, "range outside the vector")

    def SetValues(self, index, values):
        """x[index[k]] = values[k] (a repeated index keeps its last value)."""
        idx = _i32(index)
        v = self._host(values, idx.size)
        self.pf.check(lib().b200la_vec_set_values(self.pf.h, self.dtype, self.get_size(), self.ptr, idx.size,
                                                  _np_ptr(idx), _np_ptr(v)), "SetValues")

    def GetValues(self, index):
        """x[index[k]] for every k."""
        return self.GetIndexedValues(index)

    def add_values(self, indices, values):
        """x[indices[k]] += values[k] in order (lvector_cpu.cc:123-135)."""
        idx = _i32(indices)
        v = self._host(values, idx.size)
        self.pf.check(lib().b200la_vec_add_values(self.pf.h, self.dtype, self.get_size(), self.ptr, idx.size,
                                                  _np_ptr(idx), _np_ptr(v)), "add_values")

    def add_value(self, i, val):
        self.add_values([i], [val])

    def SetBlockValues(self, start, end, values):
        """x[start:end] = values."""
        self._range(start, end)
        v = self._host(values, end - start)
        if end > start:
            self.pf.check(lib().b200la_memcpy_h2d(self.pf.h, self._at(start), _np_ptr(v), v.nbytes), "SetBlockValues")
            self.pf.sync()

    def GetBlockValues(self, start, end):
        self._range(start, end)
        out = np.empty(end - start, np.float64 if self.dtype == F64 else np.float32)
        if end > start:
            self.pf.check(lib().b200la_memcpy_d2h(self.pf.h, _np_ptr(out), self._at(start), out.nbytes),
                          "GetBlockValues")
        return out

    def extract_subvector(self, start, end):
        """A new vector holding x[start:end] (lvector_cpu.cc:419-457)."""
        self._range(start, end)
        with self.pf.on_stream():
            sub = lVector(self.pf, _torch().empty(end - start, dtype=self.t.dtype, device=self.t.device))
        if end > start:
            self.pf.check(lib().b200la_memcpy_d2d(self.pf.h, sub.ptr, self._at(start), (end - start) *
                                                  self.t.element_size()), "extract_subvector")
        return sub

    def partial_replace_subvector(self, start_i, start_sub, size, sub):
        """x[start_i + k] = sub[start_sub + k], k < size (lvector_cpu.cc:460-500)."""
        self._range(start_i, start_i + size)
        sub._range(start_sub, start_sub + size)
        if size:
            self.pf.check(lib().b200la_memcpy_d2d(self.pf.h, self._at(start_i), sub._at(start_sub),
                                                  size * self.t.element_size()), "partial_replace_subvector")

    def partial_add_subvector(self, start_i, start_sub, size, weight, sub):
        """x[start_i + k] += weight sub[start_sub + k], k < size (lvector_cpu.cc:504-545)."""
        self._range(start_i, start_i + size)
        sub._range(start_sub, start_sub + size)
        if size:
            self.pf.check(lib().b200la_axpy(self.pf.h, self.dtype, size, weight, sub._at(start_sub),
                                            self._at(start_i)), "partial_add_subvector")

    def CopyTo(self, other):
        other.CopyFrom(self)

    def CastTo(self, other):
        other.CastFrom(self)

    def Reorder(self, perm):
        """out[i] = in[perm[i]] (CPU_lVector::Reorder, lvector_cpu.cc:75-94)."""
        torch = _torch()
        with self.pf.on_stream():
            p = torch.as_tensor(_i32(perm), device=self.t.device)
            out = torch.empty_like(self.t)
        self.pf.check(lib().b200la_permute(self.pf.h, self.dtype, self.get_size(), C.c_void_p(p.data_ptr()),
                                           self.ptr, C.c_void_p(out.data_ptr())), "Reorder")
        self.pf.sync()
        self.t = out


class CSR_lMatrix:
    """CSR_lMatrix<T> on the B200 (src/linear_algebra/lmp/lmatrix_csr.h)."""

    def __init__(self, platform, handle, n, m, nnz, dtype):
        self.pf, self.h, self.n, self.m, self.nnz, self.dtype = platform, handle, n, m, nnz, dtype

    @classmethod
    def from_csr(cls, platform, row, col, val, n_cols=None, dtype=F64, segments=None):
        row, col = _i32(row), _i32(col)
        n = row.size - 1
        m = n if n_cols is None else n_cols
        v = np.ascontiguousarray(val, dtype=np.float64 if dtype == F64 else np.float32)
        h = C.c_void_p()
        if segments is None:
            rc = lib().b200la_csr_create(platform.h, n, m, col.size, _np_ptr(row), _np_ptr(col), _np_ptr(v),
                                         dtype, C.byref(h))
        else:
            so = _i32(segments)
            rc = lib().b200la_csr_create_segmented(platform.h, n, m, col.size, _np_ptr(row), _np_ptr(col),
                                                   _np_ptr(v), dtype, so.size - 1, _np_ptr(so), C.byref(h))
        platform.check(rc, "csr_create")
        return cls(platform, h, n, m, col.size, dtype)

    def info(self):
        vals = [C.c_int() for _ in range(7)]
        self.pf.check(lib().b200la_csr_info(self.h, *[C.byref(v) for v in vals]))
        keys = ["n_rows", "n_cols", "nnz", "dtype", "lanes_per_row", "n_tiles", "n_long_rows"]
        out = dict(zip(keys, [v.value for v in vals]))
        npat, uses = C.c_int(), C.c_int()
        self.pf.check(lib().b200la_csr_format(self.h, C.byref(npat), C.byref(uses)))
        out["row_patterns"], out["uses_pattern_dictionary"] = npat.value, bool(uses.value)
        out["storage"] = {0: "csr", 1: "dictionary", 2: "stencil", 3: "half-stencil", 4: "lattice"}[uses.value]
        return out

    def CastFrom(self, dtype):
        """A copy of this matrix in another precision (lMatrix::CastFrom)."""
        h = C.c_void_p()
        self.pf.check(lib().b200la_csr_cast(self.pf.h, self.h, dtype, C.byref(h)), "CastFrom")
        return CSR_lMatrix(self.pf, h, self.n, self.m, self.nnz, dtype)

    @classmethod
    def ReadFile(cls, platform, path, dtype=F64):
        """A MatrixMarket file on the device (CPU_CSR_lMatrix::ReadFile)."""
        row, col, val, m = read_matrix_market(path)
        return cls.from_csr(platform, row, col, val, n_cols=m, dtype=dtype)

    def WriteFile(self, path):
        """This matrix as a MatrixMarket file (CPU_CSR_lMatrix::WriteFile)."""
        row, col, val = self.download()
        write_matrix_market(path, row, col, val, n_cols=self.m)

    def download(self):
        row = np.empty(self.n + 1, np.int32)
        col = np.empty(self.nnz, np.int32)
        val = np.empty(self.nnz, np.float64 if self.dtype == F64 else np.float32)
        self.pf.check(lib().b200la_csr_download(self.pf.h, self.h, _np_ptr(row), _np_ptr(col), _np_ptr(val)))
        return row, col, val

    def VectorMult(self, x, y):
        self.pf.check(lib().b200la_spmv(self.pf.h, self.h, x.ptr, y.ptr), "VectorMult")

    def VectorMultAdd(self, x, y):
        self.pf.check(lib().b200la_spmv_add(self.pf.h, self.h, x.ptr, y.ptr), "VectorMultAdd")

    def VectorMultDot(self, x, y):
        torch = _torch()
        with self.pf.on_stream():
            d = torch.zeros(1, dtype=torch.float64, device=x.t.device)
        self.pf.check(lib().b200la_spmv_dot(self.pf.h, self.h, x.ptr, y.ptr, C.c_void_p(d.data_ptr())),
                      "VectorMultDot")
        self.pf.sync()
        return float(d.item())

    def Residual(self, b, x, r):
        torch = _torch()
        with self.pf.on_stream():
            d = torch.zeros(1, dtype=torch.float64, device=x.t.device)
        self.pf.check(lib().b200la_residual(self.pf.h, self.h, b.ptr, x.ptr, r.ptr, C.c_void_p(d.data_ptr())),
                      "Residual")
        self.pf.sync()
        return float(d.item())

    def extract_diagelements(self, start, end, vec):
        """vec[0 .. end - start) = a_ii of rows [start, end) (lmatrix_csr_cpu.cc:2395-2412);
        a row without a stored diagonal leaves its entry of vec unchanged."""
        self.pf.check(lib().b200la_csr_diag(self.pf.h, self.h, start, end, 0, vec.ptr), "extract_diagelements")

    def extract_invdiagelements(self, start, end, vec):
        """vec[0 .. end - start) = 1 / a_ii of rows [start, end) (lmatrix_csr_cpu.cc:2414-2431)."""
        self.pf.check(lib().b200la_csr_diag(self.pf.h, self.h, start, end, 1, vec.ptr), "extract_invdiagelements")

    def Scale(self, alpha):
        """Every value times alpha (lmatrix_csr_cpu.cc:205-212)."""
        self.pf.check(lib().b200la_csr_scale(self.pf.h, self.h, alpha, 0), "Scale")

    def ScaleOffdiag(self, alpha):
        """The values off the diagonal times alpha (lmatrix_csr_cpu.cc:215-224)."""
        self.pf.check(lib().b200la_csr_scale(self.pf.h, self.h, alpha, 1), "ScaleOffdiag")

    def Zeros(self):
        """Every value zero, the structure kept (lmatrix_csr_cpu.cc:100-103)."""
        self.pf.check(lib().b200la_csr_scale(self.pf.h, self.h, 0.0, 2), "Zeros")

    def extract_submatrix(self, start_row, start_col, end_row, end_col):
        """A new matrix of the block [start_row, end_row) x [start_col, end_col)
        (lmatrix_csr_cpu.cc:1768-1843)."""
        h = C.c_void_p()
        self.pf.check(lib().b200la_csr_extract_submatrix(self.pf.h, self.h, start_row, start_col, end_row, end_col,
                                                         C.byref(h)), "extract_submatrix")
        return CSR_lMatrix._wrap(self.pf, h, self.dtype)

    def Compress(self):
        """Drop the entries whose value is zero (lmatrix_csr_cpu.cc:142-202), in place."""
        h = C.c_void_p()
        self.pf.check(lib().b200la_csr_compress(self.pf.h, self.h, C.byref(h)), "Compress")
        lib().b200la_csr_destroy(self.h)
        self.h = h
        self.nnz = self.info()["nnz"]

    @classmethod
    def _wrap(cls, platform, h, dtype):
        vals = [C.c_int() for _ in range(7)]
        platform.check(lib().b200la_csr_info(h, *[C.byref(v) for v in vals]))
        return cls(platform, h, vals[0].value, vals[1].value, vals[2].value, dtype)

    def close(self):
        if getattr(self, "h", None):
            lib().b200la_csr_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _h(m):
    return m.h if m is not None else None


def _vp(v):
    return v.ptr if v is not None else None


def gmg_residual(pf, A_diag, sol, rhs, res, A_offdiag=None, sol_ghost=None):
    """res = rhs - A_diag sol - A_offdiag sol_ghost (lmp/cuda/cuda_gmg.h)."""
    pf.check(lib().b200la_gmg_residual(pf.h, A_diag.h, _h(A_offdiag), sol.ptr, rhs.ptr, _vp(sol_ghost), res.ptr),
             "gmg_residual")


def gmg_restriction(pf, R_diag, tmp, res, R_offdiag=None, res_ghost=None):
    """res = R_diag tmp + R_offdiag res_ghost."""
    pf.check(lib().b200la_gmg_restriction(pf.h, R_diag.h, _h(R_offdiag), tmp.ptr, _vp(res_ghost), res.ptr),
             "gmg_restriction")


def gmg_prolongation_add(pf, P_diag, res, sol, P_offdiag=None, res_ghost=None):
    """sol += P_diag res + P_offdiag res_ghost."""
    pf.check(lib().b200la_gmg_prolongation_add(pf.h, P_diag.h, _h(P_offdiag), res.ptr, _vp(res_ghost), sol.ptr),
             "gmg_prolongation_add")


def async_jacobi(pf, A, b, x, n_inner=10, n_block=10, w=1.0, maxits=100000, abstol=0.0, reltol=1e-8, divtol=1e6,
                 A_offdiag=None, x_ghost=None):
    """Asynchronous block-Jacobi solve (AsynchronousIterationGPU); returns a dict
    with iters (sweeps), status, res0, res."""
    ctl, res = Control(maxits, abstol, reltol, divtol), Result()
    pf.check(lib().b200la_async_jacobi(pf.h, A.h, _h(A_offdiag), b.ptr, x.ptr, _vp(x_ghost), n_inner, n_block, w,
                                       C.byref(ctl), C.byref(res)), "async_jacobi")
    return dict(iters=res.iters, status=res.status, res0=res.res0, res=res.res, launches=res.launches)


class Preconditioner:
    """lPreconditioner on the B200: Jacobi, MC-SGS or ILU(0) (level-scheduled / coloured)."""

    def __init__(self, platform, handle, kind, n, A_perm=None):
        self.pf, self.h, self.kind, self.n, self.A_perm = platform, handle, kind, n, A_perm
        kind_c, n_c, nb = C.c_int(), C.c_int(), C.c_int()
        sizes = np.zeros(n, np.int32)
        perm = np.arange(n, dtype=np.int32)
        lib().b200la_precond_info(handle, C.byref(kind_c), C.byref(n_c), C.byref(nb), _np_ptr(sizes),
                                  _np_ptr(perm))
        self.nblocks = nb.value
        self.block_sizes = sizes[:nb.value].copy()
        self.perm = perm if nb.value else None

    @classmethod
    def Jacobi(cls, platform, A):
        h = C.c_void_p()
        platform.check(lib().b200la_precond_jacobi(platform.h, A.h, C.byref(h)), "precond_jacobi")
        return cls(platform, h, PRECOND_JACOBI, A.n)

    @classmethod
    def MultiColoringSGS(cls, platform, row, col, val, omega=1.0, dtype=F64):
        row, col, val = _i32(row), _i32(col), _f64(val)
        n = row.size - 1
        h, Ap = C.c_void_p(), C.c_void_p()
        platform.check(lib().b200la_precond_mcsgs(platform.h, n, _np_ptr(row), _np_ptr(col), _np_ptr(val), omega,
                                                  dtype, C.byref(h), C.byref(Ap)), "precond_mcsgs")
        A = CSR_lMatrix(platform, Ap, n, n, col.size, dtype)
        return cls(platform, h, PRECOND_MCSGS, n, A)

    @classmethod
    def ILU0(cls, platform, row, col, val, mode=PRECOND_ILU0_LS, dtype=F64):
        row, col, val = _i32(row), _i32(col), _f64(val)
        n = row.size - 1
        h, Ap = C.c_void_p(), C.c_void_p()
        platform.check(lib().b200la_precond_ilu0(platform.h, n, _np_ptr(row), _np_ptr(col), _np_ptr(val), mode,
                                                 dtype, C.byref(h), C.byref(Ap)), "precond_ilu0")
        A = CSR_lMatrix(platform, Ap, n, n, col.size, dtype)
        return cls(platform, h, mode, n, A)

    @classmethod
    def ILUp(cls, platform, row, col, val, ilu_p, mat_power=1, mode=PRECOND_ILU0_MC, dtype=F64):
        """lPreconditioner_MultiColoring_ILUp with ILU(ilu_p) factors and the
        colouring on the pattern of A^mat_power (level scheduling: mat_power 1)."""
        row, col, val = _i32(row), _i32(col), _f64(val)
        n = row.size - 1
        h, Ap = C.c_void_p(), C.c_void_p()
        platform.check(lib().b200la_precond_ilup(platform.h, n, _np_ptr(row), _np_ptr(col), _np_ptr(val), mode,
                                                 ilu_p, mat_power, dtype, C.byref(h), C.byref(Ap)), "precond_ilup")
        A = CSR_lMatrix(platform, Ap, n, n, col.size, dtype)
        return cls(platform, h, mode, n, A)

    def ApplyPreconditioner(self, r, z):
        self.pf.check(lib().b200la_precond_apply(self.pf.h, self.h, r.ptr, z.ptr), "ApplyPreconditioner")

    def close(self):
        if getattr(self, "h", None):
            lib().b200la_precond_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class _Solver:
    def __init__(self, platform):
        self.pf = platform
        self.op = None
        self.precond = None
        self.ctl = Control(1000, 0.0, 1e-10, 1e6)
        self.result = Result()

    def SetupOperator(self, A):
        self.op = A

    def SetupPreconditioner(self, P):
        self.precond = P

    def InitControl(self, maxits, abstol, reltol, divtol):
        self.ctl = Control(maxits, abstol, reltol, divtol)

    def iter(self):
        return self.result.iters

    def res(self):
        return self.result.res


class CG(_Solver):
    """CG<LAD> (src/linear_solver/cg.cc) on the device."""

    def Solve(self, b, x, history=0):
        P = self.precond.h if self.precond is not None else None
        if history:
            hist = np.zeros(history)
            rc = lib().b200la_cg_hist(self.pf.h, self.op.h, P, b.ptr, x.ptr, C.byref(self.ctl),
                                      C.byref(self.result), _np_ptr(hist), history)
            self.history = hist[:self.result.iters + 1]
        else:
            rc = lib().b200la_cg(self.pf.h, self.op.h, P, b.ptr, x.ptr, C.byref(self.ctl), C.byref(self.result))
        self.pf.check(rc, "CG::Solve")
        return self.result.status


class GMRES(_Solver):
    """GMRES<LAD>::SolveRight (src/linear_solver/gmres.cc) on the device."""

    def __init__(self, platform, size_basis=30):
        super().__init__(platform)
        self.size_basis = size_basis

    def Solve(self, b, x):
        P = self.precond.h if self.precond is not None else None
        rc = lib().b200la_gmres(self.pf.h, self.op.h, P, self.size_basis, b.ptr, x.ptr, C.byref(self.ctl),
                                C.byref(self.result))
        self.pf.check(rc, "GMRES::Solve")
        return self.result.status


class MPIR(_Solver):
    """MPIR<LAD_high, LAD_low> (src/linear_solver/mpir.cc): FP64 defect correction
    around an FP32 Jacobi-CG, or around an FP32 GMRES(m) with an FP32
    preconditioner (SetupInnerGMRES)."""

    def __init__(self, platform, max_outer=50):
        super().__init__(platform)
        self.inner = Control(10000, 0.0, 1e-4, 1e6)
        self.max_outer = max_outer
        self.op32 = None
        self.gmres_m = 0
        self.prec32 = None

    def SetupLowPrecisionOperator(self, A32):
        self.op32 = A32

    def SetupInnerGMRES(self, m, precond32=None):
        self.gmres_m = m
        self.prec32 = precond32

    def InitInnerControl(self, maxits, abstol, reltol, divtol):
        self.inner = Control(maxits, abstol, reltol, divtol)

    def Solve(self, b, x):
        A32 = self.op32.h if self.op32 is not None else None
        if self.gmres_m > 0:
            P32 = self.prec32.h if self.prec32 is not None else None
            rc = lib().b200la_mpir_gmres(self.pf.h, self.op.h, A32, P32, self.gmres_m, b.ptr, x.ptr,
                                         C.byref(self.ctl), C.byref(self.inner), self.max_outer,
                                         C.byref(self.result))
        else:
            rc = lib().b200la_mpir(self.pf.h, self.op.h, A32, b.ptr, x.ptr, C.byref(self.ctl), C.byref(self.inner),
                                   self.max_outer, C.byref(self.result))
        self.pf.check(rc, "MPIR::Solve")
        return self.result.status
