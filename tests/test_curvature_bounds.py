"""jsi_surface_curvature_bounds: per-coordinate bounds on |S_uu| and |S_vv|
over a whole surface (the pads of the bounds mode), host only.

Checked against the oracle's FP64 second derivatives (records P, Pu, Pv,
Puu, Puv, Pvv; evaluation.cu:221-290 restated) on a dense grid that covers
the domain's ends: every sampled |S_uu[c]| / |S_vv[c]| must be at or below
the bound.  Non-rational and rational surfaces of degree 1 to 5, the
rational saddle of the intersection configuration among them."""
from __future__ import annotations

import numpy as np
import pytest

import jsi_cad_next_versions_b200 as J
from jsi_cad_next_versions_b200 import synth


def _sampled_maxima(orc, s, n=81):
    r = np.array(s.rect(), np.float64)
    us = (r[2] - r[0]) / (n - 1)
    vs = (r[3] - r[1]) / (n - 1)
    g = orc.eval_grid(s, us, vs, r[0], r[1], n, dtype=np.float64).reshape(n * n, 18)
    return np.abs(g[:, 9:12]).max(0), np.abs(g[:, 15:18]).max(0)


def _surfaces():
    rng = synth.SplitMix64(707)
    out = [synth.random_surface(rng) for _ in range(16)]
    C, D, _ = synth.intersection_pair_saddle_plane()
    A, B, _ = synth.distance_pair_sine()
    return out + [C, D, A, B]


@pytest.mark.parametrize("idx", range(20))
def test_curvature_bounds_dominate_sampled_second_derivatives(orc, idx):
    s = _surfaces()[idx]
    mu, mv = J.curvature_bounds(s)
    su, sv = _sampled_maxima(orc, s)
    assert np.all(np.isfinite(mu)) and np.all(np.isfinite(mv))
    # degree-1 directions have no second derivative
    if int(s.ivec[1]) < 2:
        assert np.all(mu == 0)
    if int(s.ivec[4]) < 2:
        assert np.all(mv == 0)
    assert np.all(su <= mu), (su, mu)
    assert np.all(sv <= mv), (sv, mv)


def _sub_rects(s, rng, n):
    """Random parameter rectangles: inside one knot span, across several,
    and exactly one span (ends on knots)."""
    r = np.array(s.rect(), np.float64)
    iv = [int(x) for x in s.ivec]
    U = s.data[:iv[3]].astype(np.float64)
    V = s.data[iv[3]:iv[3] + iv[6]].astype(np.float64)
    ku = np.unique(U[(U >= r[0]) & (U <= r[2])])
    kv = np.unique(V[(V >= r[1]) & (V <= r[3])])
    out = []
    for k in range(n):
        a = np.sort(rng.uniform(2, r[0], r[2]))
        b = np.sort(rng.uniform(2, r[1], r[3]))
        if k % 3 == 1 and ku.size > 1 and kv.size > 1:
            i = int(rng.uniform(1, 0, ku.size - 1)[0])
            j = int(rng.uniform(1, 0, kv.size - 1)[0])
            a = np.array([ku[i], ku[i + 1]])
            b = np.array([kv[j], kv[j + 1]])
        elif k % 3 == 2:
            a = a[0] + (a - a[0]) * 0.05
            b = b[0] + (b - b[0]) * 0.05
        out.append((a[0], b[0], a[1], b[1]))
    return out


@pytest.mark.parametrize("idx", range(20))
def test_curvature_bounds_per_rectangle(orc, idx):
    """The bounds mode's per-region rule (largest per-span bound over the
    spans a rectangle touches) against the oracle's second derivatives on a
    17 x 17 grid of each rectangle.  The grid stops 1e-7 of the width inside
    the upper ends: S_uu jumps at a knot, and an evaluation exactly on a knot
    takes the next span's polynomial, which the rule leaves out (the
    rectangle's interpolation error needs S_uu only almost everywhere)."""
    s = _surfaces()[idx]
    rng = synth.SplitMix64(4000 + idx)
    for rect in _sub_rects(s, rng, 6):
        mu, mv = J.curvature_bounds(s, rect=rect)
        n = 17
        wu, wv = (rect[2] - rect[0]) * (1 - 1e-7), (rect[3] - rect[1]) * (1 - 1e-7)
        g = orc.eval_grid(s, wu / (n - 1), wv / (n - 1), rect[0], rect[1], n, dtype=np.float64).reshape(n * n, 18)
        su, sv = np.abs(g[:, 9:12]).max(0), np.abs(g[:, 15:18]).max(0)
        assert np.all(su <= mu), (rect, su, mu)
        assert np.all(sv <= mv), (rect, sv, mv)


def test_curvature_bounds_per_span_tighter_for_rational():
    """Random weights in [0.5, 2] make the whole-surface quotient bound tens
    of times the sampled maximum; the per-span bounds are far tighter."""
    A0, _, _ = synth.distance_pair_sine()
    cp, _ = A0.control_net()
    w = synth.SplitMix64(900).uniform(cp.shape[0] * cp.shape[1], 0.5, 2.0)
    R = synth.make_surface(cp.astype(np.float64), int(A0.ivec[1]), int(A0.ivec[4]),
                           weights=w.reshape(cp.shape[0], cp.shape[1]))
    glob, _ = J.curvature_bounds(R)
    U = np.unique(R.data[:int(R.ivec[3])].astype(np.float64))
    loc = [J.curvature_bounds(R, rect=(U[i], U[i], U[i + 1], U[i + 1]))[0] for i in range(U.size - 1)]
    assert np.median(np.array(loc), 0).max() < 0.2 * glob.max()


def test_curvature_bounds_rational_cases_present():
    rats = [s for s in _surfaces() if int(s.ivec[0]) & 2]
    assert len(rats) >= 4


def test_curvature_bounds_nonrational_equals_rational_with_unit_weights():
    """A rational record whose weights are all 1 is the same surface: the
    bound may differ only by the rounding slack (relative 1e-9 here)."""
    rng = synth.SplitMix64(99)
    s = synth.random_surface(rng)
    while int(s.ivec[0]) & 2:
        s = synth.random_surface(rng)
    cp, _ = s.control_net()
    r = synth.make_surface(cp.astype(np.float64), int(s.ivec[1]), int(s.ivec[4]),
                           weights=np.ones(cp.shape[:2]))
    mu0, mv0 = J.curvature_bounds(s)
    mu1, mv1 = J.curvature_bounds(r)
    np.testing.assert_allclose(mu1, mu0, rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(mv1, mv0, rtol=1e-9, atol=1e-12)


def test_curvature_bounds_rejects_bad_records():
    s = synth.random_surface(synth.SplitMix64(5))
    with pytest.raises(J.JsiError):
        J.curvature_bounds(ivec=s.ivec, data=s.data[:-1])
    cp, _ = s.control_net()
    w = np.ones(cp.shape[:2])
    w[0, 0] = -1.0
    bad = synth.make_surface(cp.astype(np.float64), int(s.ivec[1]), int(s.ivec[4]), weights=w)
    with pytest.raises(J.JsiError) as e:
        J.curvature_bounds(bad)
    assert e.value.status == -7  # JSI_ERR_UNSUPPORTED
