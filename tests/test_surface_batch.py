"""Packed host surface sets (SurfaceBatch): the arrays handed to
jsi_surface_upload_many point at exact copies of every surface's data, with
the surface's own header and length, and slices are views of the same set."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from jsi_cad_next_versions_b200 import SurfaceBatch, synth


def _surfaces():
    rng = synth.SplitMix64(21)
    out = [synth.random_surface(rng) for _ in range(7)]
    out += list(synth.distance_pair_hard_wave(seed_a=5, seed_b=6)[:2])
    return out


def test_pointers_headers_and_lengths():
    surfs = _surfaces()
    hs = SurfaceBatch(surfs)
    assert len(hs) == len(surfs)
    assert hs.ivec.flags["C_CONTIGUOUS"] and hs.ivec.shape == (len(surfs), 7) and hs.ivec.dtype == np.int32
    assert hs.ptrs.dtype == np.uintp and hs.ndata.dtype == np.int32
    for q, s in enumerate(surfs):
        assert np.array_equal(hs.ivec[q], np.asarray(s.ivec, np.int32))
        assert hs.ndata[q] == s.ndata
        assert int(hs.ptrs[q]) % 64 == 0
        raw = (ctypes.c_float * s.ndata).from_address(int(hs.ptrs[q]))
        assert np.array_equal(np.frombuffer(raw, np.float32).view(np.uint32), s.data.view(np.uint32))
        iv, data = hs.surface(q)
        assert np.array_equal(iv, hs.ivec[q]) and data.ctypes.data == int(hs.ptrs[q])
    # records do not overlap
    order = np.argsort(hs.ptrs)
    ends = hs.ptrs[order].astype(np.int64) + 4 * hs.ndata[order].astype(np.int64)
    assert np.all(ends[:-1] <= hs.ptrs[order][1:].astype(np.int64))


def test_slices_are_views():
    surfs = _surfaces()
    hs = SurfaceBatch(surfs)
    sub = hs[2:6]
    assert len(sub) == 4 and sub.data is hs.data
    assert np.array_equal(sub.ptrs, hs.ptrs[2:6]) and np.array_equal(sub.ivec, hs.ivec[2:6])
    assert sub.ivec.flags["C_CONTIGUOUS"] and sub.ptrs.flags["C_CONTIGUOUS"] and sub.ndata.flags["C_CONTIGUOUS"]
    assert len(hs[5:5]) == 0
    with pytest.raises(TypeError):
        hs[::2]
    with pytest.raises(TypeError):
        hs[3]


def test_empty_set_and_bad_header():
    assert len(SurfaceBatch([])) == 0
    s = _surfaces()[0]
    bad = synth.Surface(ivec=np.asarray(s.ivec)[:6], data=s.data)
    with pytest.raises(ValueError):
        SurfaceBatch([bad])
