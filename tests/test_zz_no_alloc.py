"""jsi_eval_grid_noalloc: the grid-evaluation entry point for callers that
cannot allocate device memory (a host application whose memory pool owns the
whole device, or a loop that cannot take cudaMalloc's implicit
synchronisation).  It must give the same records as the context-based
jsi_eval_grid, call after call, although every call reuses one fixed device
array that still holds the previous call's data, and it must not take device
memory.

This file is collected last so that a run stopping at the first failure has
already run every other test; it passes alone or after the others.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import load_npz, surface_from


def _call_noalloc(lib, s, us, vs, u0, v0, nuv, ndata=None):
    out = np.full(nuv * nuv * 18, np.nan, dtype=np.float32)
    iv = np.ascontiguousarray(s.ivec, np.int32)
    da = np.ascontiguousarray(s.data, np.float32)
    nd = int(da.shape[0]) if ndata is None else ndata
    st = lib.jsi_eval_grid_noalloc(iv.ctypes.data_as(ctypes.c_void_p), da.ctypes.data_as(ctypes.c_void_p),
                                   nd, float(us), float(vs), float(u0), float(v0), nuv,
                                   out.ctypes.data_as(ctypes.c_void_p))
    return st, out


def _steps(s, nuv):
    r = s.rect()
    return np.float32((r[2] - r[0]) / np.float32(nuv)), np.float32((r[3] - r[1]) / np.float32(nuv)), r[0], r[1]


@pytest.mark.gpu
def test_noalloc_grid_equals_context_grid_on_consecutive_calls():
    import jsi_cad_next_versions_b200 as J
    from jsi_cad_next_versions_b200 import _capi
    lib = _capi.load()
    g = load_npz("ref_eval_grids.npz")
    # Rational, non-rational, rational: each call runs on an array that still
    # holds the previous call's data, and the last rational call copies its
    # weights into the lane the non-rational call left stale.
    cases = [("deg5x4_rat", 40), ("sine_a", 33), ("saddle_rat", 37)]
    with J.Context(0) as ctx:
        for name, nuv in cases:
            s = surface_from(g[f"{name}/ivec"], g[f"{name}/data"])
            us, vs, u0, v0 = _steps(s, nuv)
            st, got = _call_noalloc(lib, s, us, vs, u0, v0, nuv)
            assert st == 0, _capi.STATUS_NAMES.get(st, st)
            exp = ctx.eval_grid(s.ivec, s.data, us, vs, u0, v0, nuv)
            # this kernel is bit-exact against the reference, so the tolerance is zero
            assert np.array_equal(got.view(np.uint32), exp.view(np.uint32)), name


@pytest.mark.gpu
def test_noalloc_takes_no_device_memory():
    import torch
    from jsi_cad_next_versions_b200 import _capi
    lib = _capi.load()
    g = load_npz("ref_eval_grids.npz")
    s = surface_from(g["saddle_rat/ivec"], g["saddle_rat/data"])
    us, vs, u0, v0 = _steps(s, 64)
    assert _call_noalloc(lib, s, us, vs, u0, v0, 64)[0] == 0  # warm-up: kernel code loaded
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(0)
    for nuv in (64, 128, 200):
        us, vs, u0, v0 = _steps(s, nuv)
        assert _call_noalloc(lib, s, us, vs, u0, v0, nuv)[0] == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(0)
    assert free1 >= free0, (free0, free1)


@pytest.mark.gpu
def test_noalloc_rejects_grids_beyond_its_array():
    from jsi_cad_next_versions_b200 import _capi
    lib = _capi.load()
    g = load_npz("ref_eval_grids.npz")
    s = surface_from(g["sine_a/ivec"], g["sine_a/data"])
    nuv = 1024  # 1024^2 * 18 floats = 72 MiB > 32 MiB
    st, out = _call_noalloc(lib, s, 0.001, 0.001, 0.0, 0.0, nuv)
    assert st == -4  # JSI_ERR_CAPACITY
    assert np.isnan(out).all()


def test_noalloc_rejects_bad_lengths_before_device_work():
    """Header and length errors return before any CUDA call, so this runs
    without a GPU: a negative data length with a control net whose 16-byte
    points would wrap a 64-bit size, and a data array one float short."""
    from jsi_cad_next_versions_b200 import _capi
    lib = _capi.load()
    g = load_npz("ref_eval_grids.npz")
    s = surface_from(g["sine_a/ivec"], g["sine_a/data"])
    huge = surface_from(np.array([1, 3, 1 << 30, (1 << 30) + 4, 3, 1 << 30, (1 << 30) + 4], np.int32),
                        s.data)
    st, out = _call_noalloc(lib, huge, 0.1, 0.1, 0.0, 0.0, 4, ndata=-1)
    assert st == -5  # JSI_ERR_SURFACE
    st, _ = _call_noalloc(lib, s, 0.1, 0.1, 0.0, 0.0, 4, ndata=-1)
    assert st == -5
    st, _ = _call_noalloc(lib, s, 0.1, 0.1, 0.0, 0.0, 4, ndata=int(s.data.shape[0]) - 1)
    assert st == -5
    assert np.isnan(out).all()
