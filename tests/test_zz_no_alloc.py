"""The allocation-free dot product, b200la_dot_noalloc, against b200la_dot.

b200la_dot_noalloc exists for callers that cannot allocate device memory: an
application that owns all device memory through its own pool, or a
stream-ordered pipeline in which cudaMalloc (which may synchronise the device)
is not allowed after set-up.  It keeps its scratch in a fixed array inside the
library.  This file is collected last so that a run stopping at the first
failure has run every other test before it.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def test_dot_noalloc_matches_dot_twice_in_a_row(b200):
    import torch
    pf = b200.Platform(0)
    L = b200.lib()
    for dtype, td, npd in [(b200.F64, torch.float64, np.float64), (b200.F32, torch.float32, np.float32)]:
        for n in (1_000_003, 4096 * 37 + 5, 1):
            rng = np.random.default_rng(n + dtype)
            x = torch.from_numpy(rng.uniform(-1, 1, n).astype(npd)).cuda()
            y = torch.from_numpy(rng.uniform(-1, 1, n).astype(npd)).cuda()
            ref = C.c_double()
            pf.check(L.b200la_dot(pf.h, dtype, n, _ptr(x), _ptr(y), C.byref(ref)))
            out = torch.full((2,), float("nan"), dtype=torch.float64, device="cuda")
            for call in range(2):
                rc = L.b200la_dot_noalloc(dtype, n, _ptr(x), _ptr(y), C.c_void_p(out.data_ptr() + 8 * call), None)
                assert rc == 0
            torch.cuda.synchronize()
            got = out.cpu().numpy()
            # the BLAS1 tolerances of the other GPU tests
            if dtype == b200.F64:
                np.testing.assert_allclose(got, ref.value, rtol=1e-12, atol=1e-14 * n)
            else:
                np.testing.assert_allclose(got, ref.value, rtol=1e-5, atol=1e-6 * np.sqrt(n))
            assert got[0] == got[1]   # same order of summation on every call


def test_dot_noalloc_full_scratch_and_explicit_stream(b200):
    """n at the limit fills every partial slot (the last one included); the
    call is also made on a caller's stream and checked against b200la_dot."""
    import torch
    pf = b200.Platform(0)
    L = b200.lib()
    n = b200.NOALLOC_MAX_N
    x = torch.ones(n, dtype=torch.float32, device="cuda")
    out = torch.full((2,), float("nan"), dtype=torch.float64, device="cuda")
    assert L.b200la_dot_noalloc(b200.F32, n, _ptr(x), _ptr(x), _ptr(out), None) == 0
    torch.cuda.synchronize()
    assert out[0].item() == float(n)          # exact: every product is 1
    del x
    m = 3_000_017
    rng = np.random.default_rng(11)
    a = torch.from_numpy(rng.uniform(-1, 1, m)).cuda()
    c = torch.from_numpy(rng.uniform(-1, 1, m)).cuda()
    ref = C.c_double()
    pf.check(L.b200la_dot(pf.h, b200.F64, m, _ptr(a), _ptr(c), C.byref(ref)))
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        assert L.b200la_dot_noalloc(b200.F64, m, _ptr(a), _ptr(c), C.c_void_p(out.data_ptr() + 8),
                                    C.c_void_p(s.cuda_stream)) == 0
    s.synchronize()
    np.testing.assert_allclose(out[1].item(), ref.value, rtol=1e-12, atol=1e-14 * m)


def test_dot_noalloc_rejects_sizes_beyond_its_scratch(b200):
    import torch
    L = b200.lib()
    x = torch.zeros(16, dtype=torch.float64, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    assert L.b200la_dot_noalloc(b200.F64, b200.NOALLOC_MAX_N + 1, _ptr(x), _ptr(x), _ptr(out), None) == 1
    assert L.b200la_dot_noalloc(b200.F64, 16, _ptr(x), _ptr(x), None, None) == 1
