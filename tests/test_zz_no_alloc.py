"""The allocation-free merge entry point, scphd_merge_components_static.

It exists for callers that must not allocate device memory (a host running inside
another framework's memory pool, or a latency-bounded loop where cudaMalloc and
cudaFree could stall).  Its result must equal the allocating entry point's on the
same inputs, on consecutive calls that share its static device scratch.  This file
is collected last so that a run stopping at the first failure has run every other
test first.
"""
import ctypes

import numpy as np
import pytest

from conftest import gpu_available

pytestmark = pytest.mark.gpu

MAX = 512   # SCPHD_STATIC_MERGE_MAX in include/scphd.h


def _static_fn(pkg):
    lib = pkg.load_library()
    fn = lib.scphd_merge_components_static
    P = ctypes.POINTER
    fn.restype = ctypes.c_int32
    fn.argtypes = [P(ctypes.c_double), P(ctypes.c_uint8), ctypes.c_int32, ctypes.c_double, ctypes.c_int32,
                   P(ctypes.c_double), P(ctypes.c_int32), P(ctypes.c_int32)]
    return lib, fn


def _call_static(fn, comps, flags, min_sep, prec):
    n = comps.shape[0]
    comps = np.ascontiguousarray(comps, np.float64)
    flags = np.ascontiguousarray(flags, np.uint8)
    out = np.zeros((max(n, 1), 28))
    mem = np.zeros(max(n, 1), np.int32)
    n_out = ctypes.c_int32(-1)
    st = fn(comps.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
            flags.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), n, float(min_sep), int(prec),
            out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), ctypes.byref(n_out),
            mem.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)))
    return st, out[: n_out.value], mem[:n]


def _components(rng, n):
    comps = np.zeros((n, 28))
    centers = rng.uniform(0, 100, (max(1, n // 4), 6))
    for i in range(n):
        c = centers[rng.integers(len(centers))]
        A = rng.normal(0, 1, (6, 6)) * 0.5
        C = A @ A.T + np.diag(rng.uniform(0.5, 3, 6))
        comps[i, 0] = rng.choice([rng.uniform(1e-3, 1), 0.25])
        comps[i, 1:7] = c + rng.normal(0, 1.0, 6)
        comps[i, 7:] = [C[a, b] for a in range(6) for b in range(a + 1)]
    flags = (rng.uniform(size=n) < 0.1).astype(np.uint8)
    return comps, flags


@pytest.mark.parametrize("prec", [1, 0])
def test_static_merge_equals_allocating_merge(pkg, orc, prec):
    """Both entry points, and the FP64 oracle's greedy merge, on the largest list the
    static entry point accepts and then a small one."""
    if not gpu_available():
        pytest.skip("no CUDA device")
    _, fn = _static_fn(pkg)
    rng = np.random.default_rng(17 + prec)
    # two calls in a row with different sizes: the second must not see the first's data
    for n in (MAX, 37):
        comps, flags = _components(rng, n)
        if prec == 0:
            comps = comps.astype(np.float32).astype(np.float64)
        st, out_s, mem_s = _call_static(fn, comps, flags, 6.0, prec)
        assert st == 0, pkg.load_library().scphd_last_error()
        out_a, mem_a = pkg.merge_components(comps, flags, 6.0, prec)
        assert out_s.shape == out_a.shape
        assert np.array_equal(mem_s, mem_a)
        tol = dict(rtol=1e-10, atol=1e-10) if prec == 1 else dict(rtol=2e-4, atol=2e-4)
        np.testing.assert_allclose(out_s, out_a, **tol)
        out_o, mem_o = orc.merge(comps, flags, 6.0)
        assert out_s.shape == out_o.shape, f"n={n}: {out_s.shape} vs oracle {out_o.shape}"
        assert np.array_equal(mem_s, mem_o), f"n={n}: membership differs from the oracle"
        np.testing.assert_allclose(out_s, out_o, **tol)


def test_static_merge_rejects_oversize(pkg):
    if not gpu_available():
        pytest.skip("no CUDA device")
    lib, fn = _static_fn(pkg)
    comps, flags = _components(np.random.default_rng(3), MAX + 1)
    st, _, _ = _call_static(fn, comps, flags, 6.0, 1)
    assert st == 3   # SCPHD_ERR_CAPACITY
    assert b"at most 512" in lib.scphd_last_error()
