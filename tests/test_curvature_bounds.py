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
