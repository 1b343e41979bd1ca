"""jsi_eval_grid_noalloc: the grid-evaluation entry point for callers that
cannot allocate device memory (a host application whose memory pool owns the
whole device, or a loop that cannot take cudaMalloc's implicit
synchronisation).  It must give the same records as the context-based
jsi_eval_grid, call after call, although every call reuses one fixed device
array that still holds the previous call's data.

This file is collected last so that a run stopping at the first failure has
already run every other test; it passes alone or after the others.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import load_npz, surface_from

pytestmark = pytest.mark.gpu


def _call_noalloc(lib, s, us, vs, u0, v0, nuv):
    out = np.full(nuv * nuv * 18, np.nan, dtype=np.float32)
    iv = np.ascontiguousarray(s.ivec, np.int32)
    da = np.ascontiguousarray(s.data, np.float32)
    st = lib.jsi_eval_grid_noalloc(iv.ctypes.data_as(ctypes.c_void_p), da.ctypes.data_as(ctypes.c_void_p),
                                   int(da.shape[0]), float(us), float(vs), float(u0), float(v0), nuv,
                                   out.ctypes.data_as(ctypes.c_void_p))
    return st, out


def test_noalloc_grid_equals_context_grid_on_consecutive_calls():
    import jsi_cad_next_versions_b200 as J
    from jsi_cad_next_versions_b200 import _capi
    lib = _capi.load()
    g = load_npz("ref_eval_grids.npz")
    # A larger rational grid first, then a smaller non-rational one: the second
    # call runs on an array that still holds the first call's data.
    cases = [("deg5x4_rat", 40), ("sine_a", 33)]
    with J.Context(0) as ctx:
        for name, nuv in cases:
            s = surface_from(g[f"{name}/ivec"], g[f"{name}/data"])
            r = s.rect()
            us = np.float32((r[2] - r[0]) / np.float32(nuv))
            vs = np.float32((r[3] - r[1]) / np.float32(nuv))
            st, got = _call_noalloc(lib, s, us, vs, r[0], r[1], nuv)
            assert st == 0, _capi.STATUS_NAMES.get(st, st)
            exp = ctx.eval_grid(s.ivec, s.data, us, vs, r[0], r[1], nuv)
            # this kernel is bit-exact against the reference, so the tolerance is zero
            assert np.array_equal(got.view(np.uint32), exp.view(np.uint32)), name


def test_noalloc_rejects_grids_beyond_its_array():
    from jsi_cad_next_versions_b200 import _capi
    lib = _capi.load()
    g = load_npz("ref_eval_grids.npz")
    s = surface_from(g["sine_a/ivec"], g["sine_a/data"])
    nuv = 1024  # 1024^2 * 18 floats = 72 MiB > 32 MiB
    st, out = _call_noalloc(lib, s, 0.001, 0.001, 0.0, 0.0, nuv)
    assert st == -4  # JSI_ERR_CAPACITY
    assert np.isnan(out).all()
