"""CPU tests of the serving layer's host side: the ctypes mirror of the
serving structs against the C header (compiled here with gcc), and the seeded
request stream of the serving benchmark."""
import ctypes as C
import importlib
import os
import subprocess
import tempfile

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def srv(b200):
    return importlib.import_module("hiflow3_b200.serving")


def test_struct_layout_matches_header(b200):
    """sizeof and field offsets of the serving structs agree between the C
    header and the ctypes mirror."""
    structs = {"b200la_serve_config": b200.ServeConfig, "b200la_request": b200.Request,
               "b200la_serve_result": b200.ServeResult, "b200la_serve_info": b200.ServeInfo,
               "b200la_control": b200.Control, "b200la_result": b200.Result}
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "b200la.h"', "int main(void) {"]
    for cname, py in structs.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for f, _ in py._fields_:
            lines.append(f'printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    lines.append("return 0; }")
    with tempfile.TemporaryDirectory() as d:
        src, exe = os.path.join(d, "abi.c"), os.path.join(d, "abi")
        open(src, "w").write("\n".join(lines))
        subprocess.run(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), src, "-o", exe], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {}
    for ln in out:
        if ln:
            a, b, c = ln.split()
            got[(a, b)] = int(c)
    for cname, py in structs.items():
        assert got[(cname, "size")] == C.sizeof(py), cname
        for f, _ in py._fields_:
            assert got[(cname, f)] == getattr(py, f).offset, (cname, f)


def test_c5_stream_is_seeded_and_shaped(srv, b200):
    a = srv.c5_stream(4096, seed=5)
    b = srv.c5_stream(4096, seed=5)
    assert a == b
    dims = np.array([r["dim"] for r in a])
    assert abs((dims == 2).mean() - 0.8) < 0.03
    n2 = np.array([r["N"] for r in a if r["dim"] == 2])
    n3 = np.array([r["N"] for r in a if r["dim"] == 3])
    assert n2.min() >= 32 and n2.max() <= 512 and abs(n2.mean() - 272) < 12
    assert n3.min() >= 16 and n3.max() <= 64 and abs(n3.mean() - 40) < 3
    mixed = np.array([r["precision"] == b200.SERVE_MIXED for r in a])
    assert abs(mixed.mean() - 0.5) < 0.03
    assert len({r["rhs_seed"] for r in a}) == 4096


def test_poisson_arrivals_and_percentiles(srv):
    t = srv.poisson_arrivals(20000, rate=250.0, seed=3)
    assert np.all(np.diff(t) > 0)
    assert abs(20000 / t[-1] - 250.0) < 10.0
    p = srv.percentiles(np.arange(1, 101))
    assert p["p50"] == pytest.approx(50.5) and p["p99"] == pytest.approx(99.01)


def test_field_bank_restriction(srv):
    fb = srv.FieldBank(count=2, res=64, sigma=0.5, ell=0.1, seed=1)
    k = fb.kcell(16, 1)
    assert k.shape == (256,) and np.all(k > 0)
    # each coarse cell reads the fine cell containing its centre
    f = fb.fields[1]
    assert k[0] == f[2, 2] and k[17] == f[6, 6]
    assert np.array_equal(fb.kcell(64, 0), fb.fields[0].reshape(-1))
