"""Continuous-batching solve server: Python mirror of the b200la_serve_* C ABI,
plus the seeded request stream of the serving benchmark.

A ``Server`` owns a device, admits requests against a device-memory budget,
and iterates every admitted SPD request inside one batched launch sequence
(CUDA-graph replays of the three batched Krylov kernels); nonsymmetric
requests run one at a time on a second stream.  ``submit`` returns an id at
once; ``wait`` / ``poll`` give the result (status, iterations, residuals,
timestamps) and the solution array.

The request stream stands in for a production arrival process: 80 % 2-D Q1
Poisson systems with N x N cells, N uniform in [32, 512] and a log-normal
coefficient k = exp(g) (g a Gaussian random field, sigma = 0.5, correlation
length 0.1); 20 % 3-D Q1 Poisson systems with M^3 cells, M uniform in
[16, 64]; FP64 and mixed-precision requests, all to a 1e-10 relative residual;
Poisson arrivals at a given rate.  The coefficient fields come from a bank of
eight realisations on 512 x 512 cells, each request reading one realisation at
its own cell centres (a restriction of a Gaussian field keeps its covariance).
"""
import ctypes as C

import numpy as np

from . import (Control, PRECOND_JACOBI, Request, ServeConfig, ServeInfo, ServeResult, B200Error, PENDING,
               SERVE_CG, SERVE_F64, SERVE_MIXED, lib, q1_sizes, _f64, _i32)
from .workloads import grf_cells


def _ctl(c):
    if isinstance(c, Control):
        return c
    maxits, abstol, reltol, divtol = c
    return Control(int(maxits), float(abstol), float(reltol), float(divtol))


class Server:
    """b200la_serve_start ... b200la_serve_stop."""

    def __init__(self, device=0, budget_bytes=60e9, max_slots=4096, active_bytes=0.0, max_active=0,
                 iters_per_round=0, autotune=False, warps=0, ctas_per_sm=0, chunks_per_warp=0):
        cfg = ServeConfig(device, float(budget_bytes), int(max_slots), float(active_bytes), int(max_active),
                          int(iters_per_round), int(bool(autotune)), int(warps), int(ctas_per_sm),
                          int(chunks_per_warp))
        h = C.c_void_p()
        rc = lib().b200la_serve_start(C.byref(cfg), C.byref(h))
        if rc:
            raise B200Error(rc, "serve_start")
        self.h = h
        self._keep = {}

    def submit(self, q1=None, csr=None, b=None, rhs_seed=0, precision=SERVE_F64, method=SERVE_CG,
               ctl=(100000, 0.0, 1e-10, 1e6), inner=(100000, 0.0, 1e-4, 1e6), max_outer=50, gmres_m=30,
               gmres_precond=PRECOND_JACOBI):
        """Queue one solve.  q1 = dict(dim, N, kind=0, kcell=None, nu=1.0, beta=(0, 0, 0)) for a
        structured Q1 system assembled on the device, or csr = (row, col, val) host arrays; b the
        right-hand side (default: the Q1 stream of rhs_seed).  Returns the request id."""
        r = Request()
        r.method, r.precision = method, precision
        keep = []
        if csr is not None:
            row, col, val = _i32(csr[0]), _i32(csr[1]), _f64(csr[2])
            keep += [row, col, val]
            n = row.size - 1
            r.n, r.nnz = n, col.size
            r.row, r.col, r.val = row.ctypes.data, col.ctypes.data, val.ctypes.data
        else:
            n, _ = q1_sizes(q1["dim"], q1["N"])
            r.q1_dim, r.q1_N, r.q1_kind = q1["dim"], q1["N"], q1.get("kind", 0)
            kc = q1.get("kcell")
            if kc is not None:
                kc = _f64(kc)
                keep.append(kc)
                r.q1_kcell = kc.ctypes.data
            r.q1_nu = q1.get("nu", 1.0)
            beta = list(q1.get("beta", (0.0, 0.0, 0.0))) + [0.0] * 3
            for d in range(3):
                r.q1_beta[d] = beta[d]
        if b is not None:
            bb = _f64(b)
            keep.append(bb)
            r.b = bb.ctypes.data
        r.rhs_seed = int(rhs_seed)
        x = np.zeros(n)
        keep.append(x)
        r.x = x.ctypes.data
        r.ctl, r.inner = _ctl(ctl), _ctl(inner)
        r.max_outer, r.gmres_m, r.gmres_precond = int(max_outer), int(gmres_m), int(gmres_precond)
        rid = C.c_longlong()
        rc = lib().b200la_serve_submit(self.h, C.byref(r), C.byref(rid))
        if rc:
            raise B200Error(rc, "serve_submit")
        self._keep[rid.value] = (x, keep)
        return rid.value

    def _out(self, rid, res):
        x = self._keep.pop(rid)[0]
        d = {f: getattr(res, f) for f, _ in ServeResult._fields_}
        d["x"] = x
        d["latency"] = res.t_done - res.t_submit
        return d

    def poll(self, rid):
        res = ServeResult()
        rc = lib().b200la_serve_poll(self.h, rid, C.byref(res))
        if rc == PENDING:
            return None
        if rc:
            raise B200Error(rc, "serve_poll")
        return self._out(rid, res)

    def wait(self, rid, timeout=600.0):
        res = ServeResult()
        rc = lib().b200la_serve_wait(self.h, rid, float(timeout), C.byref(res))
        if rc == PENDING:
            raise TimeoutError(f"request {rid} still running after {timeout} s")
        if rc:
            raise B200Error(rc, "serve_wait")
        return self._out(rid, res)

    def stats(self):
        s = ServeInfo()
        rc = lib().b200la_serve_stats(self.h, C.byref(s))
        if rc:
            raise B200Error(rc, "serve_stats")
        return {f: getattr(s, f) for f, _ in ServeInfo._fields_}

    def stop(self):
        if self.h:
            rc = lib().b200la_serve_stop(self.h)
            self.h = None
            if rc:
                raise B200Error(rc, "serve_stop")

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.stop()

    def __del__(self):
        try:
            self.stop()
        except Exception:
            pass


# ------------------------------------------------------------------ workload

class FieldBank:
    """Log-normal coefficient fields k = exp(g), g a Gaussian random field
    (squared exponential, sigma, correlation length ell) on res x res cells;
    ``kcell(N, j)`` reads realisation j at the centres of N x N cells."""

    def __init__(self, count=8, res=512, sigma=0.5, ell=0.1, seed=9000):
        self.res = res
        self.fields = [np.exp(grf_cells(res, 2, sigma=sigma, ell=ell, seed=seed + j)).reshape(res, res)
                       for j in range(count)]

    def kcell(self, N, j):
        idx = ((2 * np.arange(N) + 1) * self.res) // (2 * N)
        f = self.fields[j % len(self.fields)]
        return np.ascontiguousarray(f[np.ix_(idx, idx)]).reshape(-1)


def c5_stream(count=4096, seed=2025, mixed_fraction=0.5, frac2d=0.8, n2d=(32, 512), m3d=(16, 64)):
    """The seeded request mix: list of dicts (dim, N, precision, rhs_seed, field)."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        if rng.random() < frac2d:
            dim, N = 2, int(rng.integers(n2d[0], n2d[1] + 1))
        else:
            dim, N = 3, int(rng.integers(m3d[0], m3d[1] + 1))
        prec = SERVE_MIXED if rng.random() < mixed_fraction else SERVE_F64
        out.append(dict(dim=dim, N=N, precision=prec, rhs_seed=seed * 100003 + k, field=k % 8))
    return out


def poisson_arrivals(count, rate, seed=77):
    """Arrival times (seconds) of a Poisson process of the given rate."""
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate, size=count))


def percentiles(lat, qs=(50, 99)):
    a = np.sort(np.asarray(lat, dtype=float))
    return {f"p{q}": float(np.percentile(a, q)) if a.size else float("nan") for q in qs}
