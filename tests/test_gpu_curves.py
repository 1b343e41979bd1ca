"""Intersection curves: Newton points linked into polylines.

No counterpart in the reference (it stops at per-round overlap counts); the
checks are geometric: every vertex lies on both surfaces, consecutive vertices
are within the link tolerance, a straight intersection gives one open
monotone polyline, and a cap cut by a plane gives a closed loop."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rect32
from jsi_cad_next_versions_b200 import synth

pytestmark = pytest.mark.gpu


def _tasks(ctx, A, B, nuv):
    return (ctx.task(ctx.upload(A), rect32(A), nuv, 1), ctx.task(ctx.upload(B), rect32(B), nuv, 2))


def _check_polylines(res):
    assert res.points_found > 0 and len(res.curves) >= 1
    for cv in res.curves:
        assert cv.shape[0] >= 2
        steps = np.linalg.norm(np.diff(cv[:, :3], axis=0), axis=1)
        assert np.all(steps <= res.link_tol * (1 + 1e-12))
    assert sum(cv.shape[0] for cv in res.curves) <= res.points_found


def test_curves_crossing_planes(gpu_ctx):
    """z = 0 against z = 0.3 x - 0.1: the line x = 1/3, z = 0."""
    X, Y = np.meshgrid(np.linspace(0, 1, 6), np.linspace(0, 1, 5))
    P0 = synth.make_surface(np.stack([X, Y, 0 * X], -1), 3, 3)
    X2, Y2 = np.meshgrid(np.linspace(0, 1, 7), np.linspace(0, 1, 6))
    Pt = synth.make_surface(np.stack([X2, Y2, 0.3 * X2 - 0.1], -1), 2, 3)
    ta, tb = _tasks(gpu_ctx, P0, Pt, 16)
    res = gpu_ctx.intersection_curves(ta, tb, rounds=3)
    _check_polylines(res)
    assert len(res.curves) == 1 and not res.closed[0]
    cv = res.curves[0]
    assert np.allclose(cv[:, 0], 1.0 / 3.0, atol=1e-9) and np.allclose(cv[:, 2], 0.0, atol=1e-9)
    dy = np.diff(cv[:, 1])
    assert np.all(dy > 0) or np.all(dy < 0)  # ordered along the line
    # spans the sampled part of the overlap (the reference's grid leaves the
    # last strip of every refined cell unsampled)
    assert cv[:, 1].max() - cv[:, 1].min() > 0.8


def test_curves_closed_loop(gpu_ctx):
    """A cap (z = 0.5 - (x - 0.5)^2 - (y - 0.5)^2 sampled on a 12 x 12 net)
    cut by the plane z = 0.45: one closed loop around the cap's top."""
    X, Y = np.meshgrid(np.linspace(0, 1, 12), np.linspace(0, 1, 12))
    cap = synth.make_surface(np.stack([X, Y, 0.5 - (X - 0.5) ** 2 - (Y - 0.5) ** 2], -1), 3, 3)
    Xp, Yp = np.meshgrid(np.linspace(-0.1, 1.1, 5), np.linspace(-0.1, 1.1, 5))
    plane = synth.make_surface(np.stack([Xp, Yp, 0 * Xp + 0.45], -1), 3, 3)
    ta, tb = _tasks(gpu_ctx, cap, plane, 32)
    res = gpu_ctx.intersection_curves(ta, tb, rounds=3)
    _check_polylines(res)
    main = max(range(len(res.curves)), key=lambda k: res.curves[k].shape[0])
    cv = res.curves[main]
    assert res.closed[main]
    assert np.allclose(cv[:, 2], 0.45, atol=1e-9)
    r = np.hypot(cv[:, 0] - 0.5, cv[:, 1] - 0.5)
    assert r.min() > 0.1 and r.max() < 0.35  # a loop around the top, radius ~0.22


def test_curves_saddle_plane(gpu_ctx, orc):
    """The rational saddle / wavy plane pair of the intersection config: two
    branches; sampled vertices evaluated on both surfaces by the oracle
    coincide with each other and with the vertex."""
    C, D, _ = synth.intersection_pair_saddle_plane()
    ta, tb = _tasks(gpu_ctx, C, D, 64)
    for rounds in (3, 4):
        res = gpu_ctx.intersection_curves(ta, tb, rounds=rounds)
        _check_polylines(res)
        assert len(res.curves) <= 4 and not any(res.closed)
        allv = np.concatenate(res.curves)
        for v in allv[:: max(1, allv.shape[0] // 40)]:
            p1 = orc.eval_grid(C, 0.0, 0.0, v[3], v[4], 1, dtype=np.float64)[:3]
            p2 = orc.eval_grid(D, 0.0, 0.0, v[5], v[6], 1, dtype=np.float64)[:3]
            assert np.linalg.norm(p1 - p2) <= 1e-8
            assert np.linalg.norm(p1 - v[:3]) <= 1e-8
