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


class _FakeLib:
    """Stands in for the C library: records what jsi_surface_upload_many
    receives (read back through the pointers it is given) and hands out ids."""

    def __init__(self):
        self.calls = []
        self.next_id = 1

    def jsi_surface_upload_many(self, handle, n, ivecs, datas, ndatas, out):
        iv = np.ctypeslib.as_array((ctypes.c_int * (7 * n)).from_address(ivecs)).reshape(n, 7).copy()
        ptrs = np.ctypeslib.as_array((ctypes.c_size_t * n).from_address(datas)).copy()
        nd = np.ctypeslib.as_array((ctypes.c_int * n).from_address(ndatas)).copy()
        data = [np.frombuffer((ctypes.c_float * int(nd[q])).from_address(int(ptrs[q])), np.float32).copy()
                for q in range(n)]
        self.calls.append((iv, data))
        ids = (ctypes.c_int * n).from_address(out)
        for q in range(n):
            ids[q] = self.next_id
            self.next_id += 1
        return 0

    def jsi_last_error(self, handle):
        return b""


def _fake_context():
    from jsi_cad_next_versions_b200 import Context
    ctx = object.__new__(Context)
    ctx.lib = _FakeLib()
    ctx.handle = None
    return ctx


def test_upload_many_passes_each_slice_to_the_c_call():
    """Chunked uploads of a packed set hand the C call exactly the surfaces
    of each slice (headers, lengths and data), the same as a list upload."""
    surfs = _surfaces()
    hs = SurfaceBatch(surfs)
    ctx = _fake_context()
    ids = ctx.upload_many(hs[0:4]) + ctx.upload_many(hs[4:len(surfs)])
    assert ids == list(range(1, len(surfs) + 1))
    ref = _fake_context()
    ref.upload_many(surfs)
    got_iv = np.concatenate([c[0] for c in ctx.lib.calls])
    got_data = [d for c in ctx.lib.calls for d in c[1]]
    assert np.array_equal(got_iv, ref.lib.calls[0][0])
    for a, b in zip(got_data, ref.lib.calls[0][1]):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert ctx.upload_many(hs[2:2]) == []
    assert len(ctx.lib.calls) == 2
