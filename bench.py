#!/usr/bin/env python
"""Benchmark of the B200 lmp platform on the 3-D Q1 128^3 variable-coefficient system.

One step = one complete mixed-precision solve to a 1e-10 relative residual:
FP64 outer defect correction (MPIR) around an FP32 Jacobi-CG with tolerance
1e-4, on the 128^3-cell trilinear Q1 operator with k = exp(GRF), sigma = 1,
correlation length 0.1 (2,146,689 DoFs, 57,066,625 stored nonzeros).
`value` is whole-job solves/s with the system resident in HBM; the line also
carries the plain FP64 Jacobi-CG time to the same tolerance, the speed-up of
the mixed form over it, the SpMV bandwidth against the measured HBM peak,
the end-to-end rate through the C ABI with host buffers, and the reference's
CPU code timed on this host.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference] [--N 128]

For N > 1 (torchrun, one rank per GPU) every rank solves its own replica of
the system: the path has no data-parallel exchange (replicas only), and the
time is the maximum over ranks.
"""
import argparse
import datetime
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
METRIC = "3D Q1 128³ CG time-to-1e-10: mixed vs FP64; SpMV HBM GB/s; serving p50/p99"
UNIT = "solves/s"


def load_platform():
    name = "hiflow3_b200"
    if name in sys.modules:
        return sys.modules[name]
    path = os.path.join(ROOT, "hiflow3_2.0_b200", "__init__.py")
    spec = importlib.util.spec_from_file_location(name, path, submodule_search_locations=[os.path.dirname(path)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def load_workloads():
    load_platform()
    import importlib
    return importlib.import_module("hiflow3_b200.workloads")


def profiled_traffic(name="spmv_stencil_f32_128cubed.md"):
    """DRAM bytes per launch of the dominant kernel from the committed ncu
    summary (dram__bytes_read.sum + dram__bytes_write.sum of one capture)."""
    import re
    p = os.path.join(ROOT, "profiles", name)
    if os.path.exists(p):
        m = re.search(r"^traffic_bytes_per_launch:\s*(\d+)", open(p).read(), flags=re.M)
        if m:
            return int(m.group(1))
    return None


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi samples of SM clock and throttle reasons during a region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu, self.rows, self.proc = gpu, [], None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        time.sleep(0.3)
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
                for k, nm in enumerate(names):
                    if r[5 + k].lower().startswith("active"):
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def spmv_bytes(n, nnz, vbytes):
    """Algorithmic bytes of one CSR SpMV: values + column indices + row
    pointer, x read once, y written once."""
    return vbytes * nnz + 4 * nnz + 4 * (n + 1) + 2 * vbytes * n


def dict_spmv_bytes(n, nnz, vbytes):
    """Algorithmic bytes of one SpMV on the row-pattern dictionary in the
    sliced layout: values, a 2-byte pattern id per row, one offset per
    32-row chunk, x read once, y written once (padding of short rows and the
    few-KB pattern table excluded)."""
    return vbytes * nnz + 2 * n + 4 * ((n + 31) // 32 + 1) + 2 * vbytes * n


def stencil_spmv_bytes(n, nb, vbytes):
    """Algorithmic bytes of one SpMV on the stencil layout: the values of
    3 nb positions per row (zero-padded chunks of 32 rows; FP32 positions in
    groups of four), x read once, y written once; no indices."""
    w = 4 if vbytes == 4 else 1
    slots = (3 * nb + w - 1) // w * w
    return vbytes * slots * 32 * ((n + 31) // 32) + 2 * vbytes * n


def half_spmv_bytes(n, nb, vbytes):
    """Algorithmic bytes of one SpMV on the half stencil layout of a symmetric
    stencil operator: the diagonal and upper-half values (FP64: 2 + 3 U
    positions per row; FP32: max(U, 2) groups of four, U = (nb - 1) / 2) in
    zero-padded chunks of 32 rows, one identity-row mask word per chunk, x
    read once, y written once.  The lower half is the same values read a
    second time, from L2, by the neighbouring rows."""
    u = (nb - 1) // 2
    slots = 4 * max(u, 2) if vbytes == 4 else 2 + 3 * u
    nch = (n + 31) // 32
    return vbytes * slots * 32 * nch + 4 * nch + 2 * vbytes * n


def reference_gpu_spmv(row, col, val, x, reps=20):
    """The reference's own GPU SpMV (kernel_spmv_csr_scalar of
    lmp/cuda/cuda_spmv_kernel_csr_scalar.h, one thread per row, 256 per block,
    as GPUscalar_CSR_lMatrix::VectorMult launches it), built for sm_100a into
    baseline/_ref and timed on the same FP64 CSR matrix: mean kernel time of
    back-to-back launches, and y for a check.  None when the library is absent."""
    import ctypes as C
    so = os.path.join(ROOT, "baseline", "_ref", "libref_gpu_spmv.so")
    if not os.path.exists(so):
        return None
    L = C.CDLL(so)
    n = len(row) - 1
    y = np.empty(n)
    ms = C.c_double()
    rc = L.refgpu_spmv(0, n, len(col), C.c_void_p(row.ctypes.data), C.c_void_p(col.ctypes.data),
                       C.c_void_p(val.ctypes.data), C.c_void_p(x.ctypes.data), C.c_void_p(y.ctypes.data), reps,
                       C.byref(ms))
    return (ms.value, y) if rc == 0 else None


# --------------------------------------------------------------- ranks

def reduce_max(x, dist, device):
    """Max of a float over all ranks (x itself on a single process)."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def shard(items, rank, world):
    """Rank's share of a request stream: every world-th item from rank."""
    return items[rank::world]


# --------------------------------------------------------------- CPU baseline

def load_workloads_file():
    """workloads.py loaded by path: numpy only, so the reference arm loads no
    library of this platform."""
    name = "b200_workloads_file"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, os.path.join(ROOT, "hiflow3_2.0_b200", "workloads.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def host_cpu():
    """The host's CPU model, physical cores (distinct physical id / core id
    pairs of /proc/cpuinfo), the logical CPUs this process may run on, and
    OMP_NUM_THREADS."""
    model, cores = None, set()
    try:
        phys = None
        with open("/proc/cpuinfo") as f:
            for line in f:
                k, _, v = line.partition(":")
                k, v = k.strip(), v.strip()
                if k == "model name" and model is None:
                    model = v
                elif k == "physical id":
                    phys = v
                elif k == "core id":
                    cores.add((phys, v))
    except OSError:
        pass
    return {"model": model, "physical_cores": len(cores) or None,
            "logical_cpus_available": len(os.sched_getaffinity(0)),
            "omp_num_threads": os.environ.get("OMP_NUM_THREADS")}


def repo_libraries():
    """Shared libraries of this repository mapped into this process."""
    libs = set()
    try:
        with open("/proc/self/maps") as f:
            for line in f:
                path = line.split()[-1]
                if path.endswith(".so") and os.path.realpath(path).startswith(os.path.realpath(ROOT)):
                    libs.add(os.path.relpath(os.path.realpath(path), os.path.realpath(ROOT)))
    except OSError:
        pass
    return sorted(libs)


def pyoracle_module():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    return pyoracle


def reference_system(N):
    """The 3-D Q1 N^3 GRF system assembled by the reference's own code
    (oracle/_ref: CPU_CSR_lMatrix init_structure + add_values + ZeroRows),
    bit-identical to the platform's assembler."""
    pyoracle = pyoracle_module()
    ref = pyoracle.Ref()
    wl = load_workloads_file()
    kc = np.exp(wl.grf_cells(N, 3))
    row, col, val = ref.q1_assemble(3, N, 0, kc)
    b = ref.q1_rhs(42, 3, N)
    return ref, row, col, val, b


def cpu_baseline(row, col, val, b, single_thread=False, ref=None):
    """The reference's own CPU code (oracle/_ref: HiFlow3's CPUopenmp lmp
    objects driving the restated MPIR loop of mpir.cc:69-326), one full
    mixed-precision solve to 1e-10 timed with every host thread, and (with
    single_thread) one more with one thread."""
    pyoracle = pyoracle_module()
    if not os.path.exists(pyoracle.REF_SO):
        return None
    ref = ref or pyoracle.Ref()
    threads = len(os.sched_getaffinity(0))
    sess = pyoracle.RefMpirSession(ref, row, col, val, threads)
    sess.run(b, sample_inner=16)                      # warm-up: threads started, pages touched
    m = sess.run(b)
    out = dict(value=1.0 / m["seconds"], unit=UNIT, cores=threads, kind="reference",
               sample=(f"one full solve to 1e-10 of the same system by the reference's CPUopenmp lmp objects "
                       f"(MPIR: {m['outer']} corrections, {m['inner_total']} FP32 inner iterations), "
                       f"{threads} OpenMP threads"),
               solve_s=m["seconds"], outer=m["outer"], inner_total=m["inner_total"], cpu=host_cpu())
    if single_thread:
        sess.threads(1)
        sess.run(b, sample_inner=4)
        m1 = sess.run(b)
        out["one_thread"] = dict(value=1.0 / m1["seconds"], unit=UNIT, cores=1, solve_s=m1["seconds"],
                                 outer=m1["outer"], inner_total=m1["inner_total"])
    sess.close()
    return out


def run_reference(args):
    """The reference's own CPU implementation of the path (oracle/_ref, built
    from the reference's lmp sources), on the same system, timed per step as
    one full solve to 1e-10; warm-up steps are untimed solves cut after 16
    inner iterations.  Nothing of this platform is loaded."""
    pyoracle = pyoracle_module()
    if not os.path.exists(pyoracle.REF_SO):
        return {"impl": "reference", "unavailable": "oracle/_ref (the reference's CPU lmp build) is missing"}
    t0 = time.time()
    ref, row, col, val, b = reference_system(args.N)
    t_asm = time.time() - t0
    threads = len(os.sched_getaffinity(0))
    sess = pyoracle.RefMpirSession(ref, row, col, val, threads)
    for _ in range(args.warmup):
        sess.run(b, sample_inner=16)
    secs = []
    for _ in range(args.steps):
        m = sess.run(b)
        secs.append(m["seconds"])
    sess.close()
    r = b - ref.spmv(row, col, val, m["x"], impl=1, nthreads=threads)
    relres = float(np.linalg.norm(r) / np.linalg.norm(b))
    total = sum(secs)
    v = args.steps / total
    wl = load_workloads_file()
    cb = {"value": v, "unit": UNIT, "cores": threads, "kind": "reference",
          "sample": (f"{args.steps} full solves to 1e-10 by the reference's CPUopenmp lmp objects (MPIR: "
                     f"{m['outer']} corrections, {m['inner_total']} FP32 inner iterations), {threads} OpenMP threads"),
          "cpu": host_cpu()}
    return {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32-inner/f64-outer", "data": "synthetic (seeded)",
            "impl": "reference",
            "config": {"workload": wl.CONFIGS["c3"]["desc"], "cells": args.N ** 3, "dofs": len(b), "nnz": len(col)},
            "solve": {"outer": m["outer"], "inner_total": m["inner_total"], "relres_true": relres,
                      "seconds_min": min(secs), "seconds_max": max(secs)},
            "setup_s": {"grf_and_assembly": t_asm}, "libraries_loaded": repo_libraries(),
            "cpu_baseline": cb, "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


# --------------------------------------------------------------- B200 arm

def run_b200(args, rank, world, local_rank, dist):
    import torch
    b200 = load_platform()
    wl = load_workloads()
    torch.cuda.set_device(local_rank)
    pf = b200.Platform(local_rank)
    t0 = time.time()
    row, col, val, b, _ = wl.system(b200, "c3", N=args.N)
    t_asm = time.time() - t0
    n, nnz = len(row) - 1, len(col)
    t0 = time.time()
    A64 = b200.CSR_lMatrix.from_csr(pf, row, col, val)
    A32 = A64.CastFrom(b200.F32)
    pf.sync()
    t_up = time.time() - t0
    bv, x = pf.vector(b), pf.vector(n)

    mp = b200.MPIR(pf, max_outer=50)
    mp.SetupOperator(A64)
    mp.SetupLowPrecisionOperator(A32)
    mp.InitControl(50, 0.0, 1e-10, 1e6)
    mp.InitInnerControl(100000, 0.0, 1e-4, 1e6)

    def step():
        x.Zeros()
        mp.Solve(bv, x)
        return mp.result

    for _ in range(args.warmup):
        step()
    if world > 1:
        dist.barrier()
    pf.sync()
    launches = 0
    with Clocks(local_rank) as clk:
        pf.timer_start()
        for _ in range(args.steps):
            r = step()
            launches += r.launches
        ms = pf.timer_stop()
    res_mixed = dict(outer=r.outer, inner_total=r.iters, res0=r.res0, res=r.res, status=r.status)
    ms = reduce_max(ms, dist if world > 1 else None, "cuda")
    ms_step = ms / args.steps
    value = world * args.steps / (ms / 1e3)
    x_mixed = x.numpy()

    # true residual of the mixed solution, in FP64 on the device
    rv = pf.vector(n)
    relres = float(np.sqrt(A64.Residual(bv, x, rv)) / np.linalg.norm(b))

    # plain FP64 Jacobi-CG to the same tolerance (the comparison)
    cg = b200.CG(pf)
    cg.SetupOperator(A64)
    J64 = b200.Preconditioner.Jacobi(pf, A64)
    cg.SetupPreconditioner(J64)
    cg.InitControl(200000, 0.0, 1e-10, 1e6)
    x64 = pf.vector(n)
    cg.Solve(bv, x64)          # warm-up
    k64 = max(1, min(3, args.steps))
    pf.sync()
    pf.timer_start()
    for _ in range(k64):
        x64.Zeros()
        cg.Solve(bv, x64)
    fp64_ms = pf.timer_stop() / k64
    fp64_iters = cg.iter()
    # FP64 reference solution at 1e-12 for the error of the mixed result
    cg.InitControl(400000, 0.0, 1e-12, 1e6)
    xr = pf.vector(n)
    cg.Solve(bv, xr)
    xr_h = xr.numpy()
    err = float(np.linalg.norm(x_mixed - xr_h) / np.linalg.norm(xr_h))
    err64 = float(np.linalg.norm(x64.numpy() - xr_h) / np.linalg.norm(xr_h))

    # SpMV bandwidth: the fused SpMV+dot kernel of the CG iteration, FP64 and
    # FP32, events on the library's stream around back-to-back launches
    # (matrix 0.5-0.7 GB, well above L2)
    def spmv_rate(A, vbytes):
        dt = b200.F64 if vbytes == 8 else b200.F32
        xx, yy = pf.vector(np.random.default_rng(1).uniform(-1, 1, n), dt), pf.vector(n, dt)
        import ctypes
        with pf.on_stream():
            d = torch.zeros(1, dtype=torch.float64, device="cuda")
        L = b200.lib()
        for _ in range(3):
            L.b200la_spmv_dot(pf.h, A.h, xx.ptr, yy.ptr, ctypes.c_void_p(d.data_ptr()))
        reps = 40
        pf.sync()
        pf.timer_start()
        for _ in range(reps):
            L.b200la_spmv_dot(pf.h, A.h, xx.ptr, yy.ptr, ctypes.c_void_p(d.data_ptr()))
        t_ms = pf.timer_stop() / reps
        storage = A.info()["storage"]
        by = {"csr": spmv_bytes(n, nnz, vbytes), "dictionary": dict_spmv_bytes(n, nnz, vbytes),
              "stencil": stencil_spmv_bytes(n, 9, vbytes), "half-stencil": half_spmv_bytes(n, 9, vbytes)}[storage]
        return by, t_ms, by / (t_ms * 1e-3) / 1e9, storage

    by64, t64, gbs64, st64 = spmv_rate(A64, 8)
    by32, t32, gbs32, st32 = spmv_rate(A32, 4)
    # the FP64 operator with explicit column indices (CSR) as well: the
    # reference's storage; FP64 CG on it for comparison
    os.environ["B200LA_STENCIL"] = "0"
    A64c = b200.CSR_lMatrix.from_csr(pf, row, col, val)
    del os.environ["B200LA_STENCIL"]
    by64c, t64c, gbs64c, st64c = spmv_rate(A64c, 8)
    cgc = b200.CG(pf)
    cgc.SetupOperator(A64c)
    cgc.SetupPreconditioner(b200.Preconditioner.Jacobi(pf, A64c))
    cgc.InitControl(200000, 0.0, 1e-10, 1e6)
    xc = pf.vector(n)
    cgc.Solve(bv, xc)
    pf.sync()
    pf.timer_start()
    for _ in range(k64):
        xc.Zeros()
        cgc.Solve(bv, xc)
    fp64c_ms = pf.timer_stop() / k64
    fp64c_iters = cgc.iter()
    del A64c, cgc, xc
    peak, peak_kind = measured_peaks()
    # the reference's own GPU kernel on the same FP64 CSR matrix
    xr = np.random.default_rng(1).uniform(-1, 1, n)
    rg = reference_gpu_spmv(row, col, val, xr)
    ref_gpu = None
    if rg is not None:
        import scipy.sparse as sp
        y_host = sp.csr_matrix((val, col, row), shape=(n, n)) @ xr
        scale = sp.csr_matrix((np.abs(val), col, row), shape=(n, n)) @ np.abs(xr)
        by_ref = spmv_bytes(n, nnz, 8)
        ref_gpu = {"kernel": "kernel_spmv_csr_scalar<double> (the reference's GPUscalar CSR SpMV, sm_100a build)",
                   "us": rg[0] * 1e3, "gbs": by_ref / (rg[0] * 1e-3) / 1e9, "bytes": by_ref,
                   "frac_of_peak": by_ref / (rg[0] * 1e-3) / 1e9 / peak,
                   "max_rel_err": float(np.max(np.abs(rg[1] - y_host) / np.maximum(scale, 1e-300)))}
    # SURVEY units: one FP64 / FP32 SpMV of this operator (CSR algorithmic bytes)
    unit64, unit32 = spmv_bytes(n, nnz, 8), spmv_bytes(n, nnz, 4)

    # end to end through the C ABI: host b in, host x out, per step
    import ctypes
    L = b200.lib()
    hb = pf.host_alloc(8 * n)
    hx = pf.host_alloc(8 * n)
    ctypes.memmove(hb, b.ctypes.data, 8 * n)
    ctl = b200.Control(50, 0.0, 1e-10, 1e6)
    ictl = b200.Control(100000, 0.0, 1e-4, 1e6)
    db, dx = ctypes.c_void_p(), ctypes.c_void_p()
    pf.check(L.b200la_malloc(pf.h, 8 * n, ctypes.byref(db)))
    pf.check(L.b200la_malloc(pf.h, 8 * n, ctypes.byref(dx)))
    res = b200.Result()

    def e2e_step():
        pf.check(L.b200la_memcpy_h2d(pf.h, db, hb, 8 * n))
        pf.check(L.b200la_memset_zero(pf.h, dx, 8 * n))
        pf.check(L.b200la_mpir(pf.h, A64.h, A32.h, db, dx, ctypes.byref(ctl), ctypes.byref(ictl), 50,
                               ctypes.byref(res)))
        pf.check(L.b200la_memcpy_d2h(pf.h, hx, dx, 8 * n))

    for _ in range(min(args.warmup, 2)):
        e2e_step()
    if world > 1:
        dist.barrier()
    pf.sync()
    pf.timer_start()
    for _ in range(args.steps):
        e2e_step()
    e2e_ms = pf.timer_stop()
    e2e_ms = reduce_max(e2e_ms, dist if world > 1 else None, "cuda")
    xh = np.ctypeslib.as_array(ctypes.cast(hx, ctypes.POINTER(ctypes.c_double)), (n,)).copy()
    e2e_ok = bool(np.array_equal(xh, x_mixed))
    L.b200la_free(pf.h, db)
    L.b200la_free(pf.h, dx)
    pf.host_free(hb)
    pf.host_free(hx)

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32-inner/f64-outer", "data": "synthetic (seeded GRF coefficient and RHS)",
        "config": {"workload": wl.CONFIGS["c3"]["desc"], "cells": args.N ** 3, "dofs": n, "nnz": nnz,
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                   "l2": "inputs larger than L2 (matrix 0.46-0.69 GB)"},
        "mixed": {"ms": ms_step, "outer": res_mixed["outer"], "inner_iters": res_mixed["inner_total"],
                  "relres_true": relres, "err_vs_fp64_solution": err},
        "fp64_cg": {"ms": fp64_ms, "iters": fp64_iters, "err_vs_fp64_solution": err64},
        "mixed_speedup_vs_fp64": fp64_ms / ms_step,
        "fp64_cg_csr": {"ms": fp64c_ms, "iters": fp64c_iters,
                        "note": "FP64 Jacobi-CG with the operator in CSR (explicit column indices)"},
        "mixed_speedup_vs_fp64_csr": fp64c_ms / ms_step,
        "spmv": {"fp64": {"storage": st64, "us": t64 * 1e3, "gbs": gbs64, "bytes": by64, "frac_of_peak": gbs64 / peak,
                          "csr_unit_gbs": unit64 / (t64 * 1e-3) / 1e9},
                 "fp64_csr": {"us": t64c * 1e3, "gbs": gbs64c, "bytes": by64c, "frac_of_peak": gbs64c / peak},
                 "fp32_inner": {"storage": st32, "us": t32 * 1e3, "gbs": gbs32, "bytes": by32,
                                "frac_of_peak": gbs32 / peak, "csr_unit_gbs": unit32 / (t32 * 1e-3) / 1e9},
                 "csr_unit_bytes": {"fp64": unit64, "fp32": unit32},
                 "reference_gpu_fp64_csr": ref_gpu},
        "roofline": {"bound": "hbm",
                     "kernel": f"FP32 SpMV + p.Ap of the inner CG ({st32} layout)",
                     "achieved": gbs32, "peak": peak, "unit": "GB/s", "frac": gbs32 / peak,
                     "peak_source": peak_kind, "bytes_per_launch": by32,
                     "bytes_basis": "the layout's own bytes: values, x once, y once (no indices)",
                     "csr_unit_bytes_per_launch": unit32, "achieved_csr_unit": unit32 / (t32 * 1e-3) / 1e9,
                     "traffic": profiled_traffic() if args.N == 128 else None,
                     "traffic_source": "profiles/spmv_stencil_f32_128cubed.md (ncu, one launch)"},
        "gpu_launches": launches,
        "e2e": {"value": world * args.steps / (e2e_ms / 1e3), "unit": UNIT, "h2d_bytes_per_step": 8 * n,
                "d2h_bytes_per_step": 8 * n, "matches_device_run": e2e_ok},
        "setup_s": {"assembly": t_asm, "upload_and_cast": t_up},
        "clocks": clk.summary(),
    }
    if not args.no_configs:
        line["configs"] = other_configs(b200, pf, wl)
    if args.serve_requests > 0:
        line["serving"] = serving_bench(b200, pf, args.serve_requests, rank=rank, world=world,
                                        dist=dist if world > 1 else None)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb = cpu_baseline(row, col, val, b, single_thread=True)
        line["cpu_baseline"] = cb if cb else {"value": None, "unit": UNIT, "cores": 0, "kind": "reference",
                                              "sample": "oracle/_ref missing"}
    pf.close()
    return line


def other_configs(b200, pf, wl):
    """Time to solution of the other configurations: C1 (2-D Poisson 256^2,
    Jacobi-CG to 1e-10, FP64; the reference's own CPU case), C2 (3-D
    Poisson 128^3, 8-colour MC-SGS PCG to 1e-8, FP64) and C4 (2-D
    convection-diffusion 512^2, GMRES(30) + level-scheduled ILU(0) to 1e-9,
    FP64 and mixed: FP32 factors and Arnoldi inside FP64 defect correction)."""
    out = {}
    # C1
    row, col, val, b, _ = wl.system(b200, "c1")
    A1 = b200.CSR_lMatrix.from_csr(pf, row, col, val)
    cg = b200.CG(pf)
    cg.SetupOperator(A1)
    cg.SetupPreconditioner(b200.Preconditioner.Jacobi(pf, A1))
    cg.InitControl(100000, 0.0, 1e-10, 1e6)
    bv, x = pf.vector(b), pf.vector(len(b))
    cg.Solve(bv, x)
    times = []
    for _ in range(5):
        x.Zeros()
        pf.sync()
        pf.timer_start()
        cg.Solve(bv, x)
        times.append(pf.timer_stop())
    out["c1_jacobi_cg_fp64"] = {"ms": float(np.median(times)), "iters": cg.iter(), "status": cg.result.status,
                                "storage": A1.info()["storage"], "n": len(b), "nnz": len(col),
                                "note": "median of 5 timed solves (the system fits in L2)"}
    # C2
    row, col, val, b, _ = wl.system(b200, "c2")
    t0 = time.perf_counter()
    P = b200.Preconditioner.MultiColoringSGS(pf, row, col, val)
    pf.sync()
    t_setup = time.perf_counter() - t0
    bp = b[P.perm]
    cg = b200.CG(pf)
    cg.SetupOperator(P.A_perm)
    cg.SetupPreconditioner(P)
    cg.InitControl(100000, 0.0, 1e-8, 1e6)
    bv, x = pf.vector(bp), pf.vector(len(bp))
    cg.Solve(bv, x)
    x.Zeros()
    pf.sync()
    pf.timer_start()
    cg.Solve(bv, x)
    ms = pf.timer_stop()
    out["c2_mcsgs_cg_fp64"] = {"ms": ms, "iters": cg.iter(), "status": cg.result.status,
                               "colours": P.nblocks, "setup_s": t_setup,
                               "storage": P.A_perm.info()["storage"]}
    # one MC-SGS apply (2 x colours sweep launches) and one SpMV of the
    # coloured operator, events around back-to-back calls (operands > L2)
    n = len(bp)
    rv, zv, yv = pf.vector(np.random.default_rng(3).uniform(-1, 1, n)), pf.vector(n), pf.vector(n)
    for _ in range(3):
        P.ApplyPreconditioner(rv, zv)
    pf.sync()
    pf.timer_start()
    for _ in range(20):
        P.ApplyPreconditioner(rv, zv)
    t_apply = pf.timer_stop() / 20
    for _ in range(3):
        P.A_perm.VectorMult(rv, yv)
    pf.sync()
    pf.timer_start()
    for _ in range(20):
        P.A_perm.VectorMult(rv, yv)
    t_spmv = pf.timer_stop() / 20
    nnz = len(col)
    lattice = P.A_perm.info()["storage"] == "lattice"
    # algorithmic bytes: lattice -- values by slot (26 or 27 per row, padded
    # chunks counted as stored) and the vector passes; CSR -- SURVEY's units
    nch = (n + 31) // 32 + 8
    apply_bytes = (8 * 26 * 32 * nch + 48 * n) if lattice else (12 * (nnz - n) + 8 * (n + 1) + 48 * n)
    spmv_b = (8 * 27 * 32 * nch + 16 * n) if lattice else spmv_bytes(n, nnz, 8)
    peak, _ = measured_peaks()
    out["c2_mcsgs_cg_fp64"]["mcsgs_apply"] = {"us": t_apply * 1e3, "bytes": apply_bytes,
                                              "gbs": apply_bytes / (t_apply * 1e-3) / 1e9,
                                              "frac_of_peak": apply_bytes / (t_apply * 1e-3) / 1e9 / peak}
    out["c2_mcsgs_cg_fp64"]["coloured_spmv"] = {"us": t_spmv * 1e3, "bytes": spmv_b,
                                                "gbs": spmv_b / (t_spmv * 1e-3) / 1e9,
                                                "frac_of_peak": spmv_b / (t_spmv * 1e-3) / 1e9 / peak}
    del P, cg, bv, x, rv, zv, yv
    # C4
    row, col, val, b, _ = wl.system(b200, "c4")
    t0 = time.perf_counter()
    P64 = b200.Preconditioner.ILU0(pf, row, col, val, b200.PRECOND_ILU0_LS)
    P32 = b200.Preconditioner.ILU0(pf, row, col, val, b200.PRECOND_ILU0_LS, dtype=b200.F32)
    pf.sync()
    t_setup = time.perf_counter() - t0
    bp = b[P64.perm]
    bv = pf.vector(bp)
    gm = b200.GMRES(pf, 30)
    gm.SetupOperator(P64.A_perm)
    gm.SetupPreconditioner(P64)
    gm.InitControl(100000, 0.0, 1e-9, 1e6)
    x = pf.vector(len(bp))
    gm.Solve(bv, x)
    x.Zeros()
    pf.sync()
    pf.timer_start()
    gm.Solve(bv, x)
    ms64 = pf.timer_stop()
    x64 = x.numpy()
    it64 = gm.iter()
    m = b200.MPIR(pf, max_outer=50)
    m.SetupOperator(P64.A_perm)
    m.SetupLowPrecisionOperator(P32.A_perm)
    m.SetupInnerGMRES(30, P32)
    m.InitControl(50, 0.0, 1e-9, 1e6)
    m.InitInnerControl(100000, 0.0, 1e-4, 1e6)
    xm = pf.vector(len(bp))
    m.Solve(bv, xm)
    xm.Zeros()
    pf.sync()
    pf.timer_start()
    m.Solve(bv, xm)
    msm = pf.timer_stop()
    rv = pf.vector(len(bp))
    true = float(np.sqrt(P64.A_perm.Residual(bv, xm, rv)) / np.linalg.norm(bp))
    out["c4_gmres_ilu_fp64"] = {"ms": ms64, "iters": it64, "levels": P64.nblocks, "setup_s": t_setup}
    out["c4_gmres_ilu_mixed"] = {"ms": msm, "outer": m.result.outer, "inner_iters": m.result.iters,
                                 "relres_true": true,
                                 "rel_diff_vs_fp64": float(np.linalg.norm(xm.numpy() - x64) / np.linalg.norm(x64)),
                                 "speedup_vs_fp64": ms64 / msm}
    return out


def serving_bench(b200, pf, nreq, sample=128, seed=2025, rank=0, world=1, dist=None):
    """The serving loop on the seeded request stream: saturation throughput
    (every request offered at t = 0), p50/p99 latency at Poisson arrival rates
    below saturation, and the drop-in FP64 Jacobi-CG solving a sample of the
    same requests one at a time.  With several ranks every rank serves its
    shard of the stream on its own GPU (replicas); the job's rate is all
    requests over the slowest rank's time."""
    import importlib
    srv = importlib.import_module("hiflow3_b200.serving")
    fb = srv.FieldBank()
    stream = shard(srv.c5_stream(nreq, seed=seed), rank, world)
    nreq = len(stream)
    kcache = {}

    def kcell(r):
        key = (r["N"], r["field"])
        if key not in kcache:
            kcache[key] = fb.kcell(r["N"], r["field"])
        return kcache[key]

    def req(r):
        kc = kcell(r) if r["dim"] == 2 else None
        return dict(q1=dict(dim=r["dim"], N=r["N"], kcell=kc), rhs_seed=r["rhs_seed"], precision=r["precision"],
                    ctl=(100000, 0.0, 1e-10, 1e6), inner=(100000, 0.0, 1e-4, 1e6), max_outer=50)

    reqs = [req(r) for r in stream]

    def ok(r):
        return r["status"] in (b200.SUCCESS_ABS, b200.SUCCESS_REL) and r["res"] <= 1e-10 * r["res0"]

    s = srv.Server(autotune=True)
    t0 = time.perf_counter()
    ids = [s.submit(**a) for a in reqs]
    res = [s.wait(i) for i in ids]
    t_sat = time.perf_counter() - t0
    st = s.stats()
    s.stop()
    sat = len(res) / t_sat
    t_job = reduce_max(t_sat, dist if world > 1 else None, "cuda")
    shape = dict(warps=st["warps"], ctas_per_sm=st["ctas_per_sm"], chunks_per_warp=st["chunks_per_warp"])
    lat = [r["latency"] for r in res]
    out = {"requests": len(res) * world, "solves_per_s": len(res) * world / t_job, "wall_s": t_job,
           "met_1e-10": sum(map(ok, res)),
           "latency_ms": {k: v * 1e3 for k, v in srv.percentiles(lat).items()},
           "iterations": int(sum(r["iters"] for r in res)), "rounds": st["rounds"],
           "batch_iterations": st["batch_iters"], "gpu_busy_s": st["busy_ms"] / 1e3,
           "peak_active": st["peak_active"], "peak_resident_gb": st["peak_resident_bytes"] / 1e9,
           "kernel_shape": shape, "active_bytes": st["active_bytes"],
           "mix": {"2d": sum(r["dim"] == 2 for r in stream), "3d": sum(r["dim"] == 3 for r in stream),
                   "mixed_precision": sum(r["precision"] == b200.SERVE_MIXED for r in stream)}}
    sweeps = []
    m = min(nreq, 1024)
    for frac in (0.5, 0.8):
        rate = frac * sat
        arr = srv.poisson_arrivals(m, rate, seed=int(frac * 100))
        s = srv.Server(**shape)
        t0 = time.perf_counter()
        ids = []
        for k in range(m):
            dt = t0 + arr[k] - time.perf_counter()
            if dt > 0:
                time.sleep(dt)
            ids.append(s.submit(**reqs[k]))
        rs = [s.wait(i) for i in ids]
        t_all = time.perf_counter() - t0
        s.stop()
        pc = srv.percentiles([r["latency"] for r in rs])
        sweeps.append({"offered_per_s": rate, "served_per_s": m / t_all, "requests": m,
                       "p50_ms": pc["p50"] * 1e3, "p99_ms": pc["p99"] * 1e3, "met_1e-10": sum(map(ok, rs))})
    out["rate_sweep"] = sweeps
    # one at a time: the drop-in FP64 Jacobi-CG (lMatrix upload, solve, download)
    solve_s = full_s = 0.0
    err = 0.0
    for k in range(min(sample, nreq)):
        r = stream[k]
        kc = kcell(r) if r["dim"] == 2 else None
        row, col, val = b200.q1_assemble(r["dim"], r["N"], 0, kc)
        bh = b200.q1_rhs(r["rhs_seed"], r["dim"], r["N"])
        pf.sync()
        ta = time.perf_counter()
        A = b200.CSR_lMatrix.from_csr(pf, row, col, val)
        P = b200.Preconditioner.Jacobi(pf, A)
        cg = b200.CG(pf)
        cg.SetupOperator(A)
        cg.SetupPreconditioner(P)
        cg.InitControl(100000, 0.0, 1e-10, 1e6)
        xv, bv = pf.vector(len(bh)), pf.vector(bh)
        pf.sync()
        tb = time.perf_counter()
        cg.Solve(bv, xv)
        pf.sync()
        tc = time.perf_counter()
        xh = xv.numpy()
        td = time.perf_counter()
        solve_s += tc - tb
        full_s += td - ta
        err = max(err, float(np.linalg.norm(res[k]["x"] - xh) / np.linalg.norm(xh)))
    ns = min(sample, nreq)
    out["one_at_a_time_fp64"] = {"sample": ns, "solves_per_s": ns / solve_s,
                                 "solves_per_s_with_upload": ns / full_s}
    out["speedup_vs_one_at_a_time"] = sat / (ns / solve_s)
    out["max_rel_diff_vs_fp64_one_at_a_time"] = err
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--N", type=int, default=128)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-configs", action="store_true", help="skip the C2 / C4 time-to-solution runs")
    ap.add_argument("--serve-requests", type=int, default=4096,
                    help="requests of the serving stream (0: skip the serving measurement)")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if args.impl == "reference":
        # rank 0 alone times the reference's CPU code; other ranks exit at once
        if rank == 0:
            print(json.dumps(run_reference(args)), flush=True)
        return
    if world > 1:
        import torch.distributed as dist
        import torch
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        line = run_b200(args, rank, world, local_rank, dist)
        if rank == 0:
            print(json.dumps(line), flush=True)
    finally:
        if dist is not None:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
