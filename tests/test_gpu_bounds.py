"""Bounds mode: a rigorous interval lb <= (minimum distance) <= ub.

There is no counterpart in the reference, so the checks are the interval's
own properties: an analytic case (parallel planes), the ordering against the
minimum over a dense FP64 sample of both surfaces taken by the oracle (every
sample pair is a pair of surface points, so that minimum is >= the true one
and must be >= lb), the Newton pair as ub, and refinement tightening lb."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rect32
from jsi_cad_next_versions_b200 import synth

pytestmark = pytest.mark.gpu


def _dense_min(orc, A, B, n=96):
    """min |S1 - S2| over n x n FP64 samples per surface (a sample grid that
    includes the rectangle ends)."""
    pts = []
    for s in (A, B):
        r = rect32(s).astype(np.float64)
        us = (r[2] - r[0]) / (n - 1)
        vs = (r[3] - r[1]) / (n - 1)
        g = orc.eval_grid(s, us, vs, r[0], r[1], n, dtype=np.float64).reshape(n * n, 18)[:, :3]
        pts.append(g)
    P, Q = pts
    best = np.inf
    for i in range(0, P.shape[0], 512):
        d = P[i:i + 512, None, :] - Q[None, :, :]
        best = min(best, float(np.sqrt((d * d).sum(-1)).min()))
    return best


def _tasks(ctx, A, B, nuv):
    return (ctx.task(ctx.upload(A), rect32(A), nuv, 1), ctx.task(ctx.upload(B), rect32(B), nuv, 2))


def test_bounds_parallel_planes(gpu_ctx):
    """z = 0 and z = 0.5 over overlapping squares: the distance is 0.5."""
    X, Y = np.meshgrid(np.linspace(0, 1, 6), np.linspace(0, 1, 5))
    P0 = synth.make_surface(np.stack([X, Y, 0 * X], -1), 3, 3)
    X2, Y2 = np.meshgrid(np.linspace(0, 1, 7), np.linspace(0, 1, 6))
    P1 = synth.make_surface(np.stack([0.9 * X2 + 0.05, 0.8 * Y2 + 0.1, 0 * X2 + 0.5], -1), 3, 2)
    ta, tb = _tasks(gpu_ctx, P0, P1, 20)
    r = gpu_ctx.distance_bounds(ta, tb)
    assert r.lb <= 0.5 <= r.ub
    assert r.certified and r.ub - r.lb <= 1e-6 * r.ub * (1 + 1e-9)
    assert abs(r.ub - 0.5) < 1e-9


@pytest.mark.parametrize("seeds", [(1, 2), (21, 22)])
def test_bounds_sine_pair(gpu_ctx, orc, seeds):
    A, B, _ = synth.distance_pair_sine(seed_a=seeds[0], seed_b=seeds[1])
    ta, tb = _tasks(gpu_ctx, A, B, 64)
    r = gpu_ctx.distance_bounds(ta, tb, rel_tol=1e-6)
    dense = _dense_min(orc, A, B)
    assert 0.0 <= r.lb <= r.ub
    assert r.lb <= dense
    assert r.ub <= dense * (1 + 1e-9) + 1e-12  # Newton's pair is at least as close as any sample pair
    assert np.all(np.diff(r.lb_round) >= 0)
    assert r.certified, (r.lb, r.ub, r.kept)
    fp64 = gpu_ctx.min_distance(ta, tb, precision="fp64", newton=True)
    assert abs(fp64.newton_distance - r.ub) <= 1e-9 * r.ub


@pytest.mark.parametrize("want_rational", [False, True])
def test_bounds_random_surfaces(gpu_ctx, orc, want_rational):
    """Random pairs of degree 1-5; the rational case takes pairs with at
    least one rational surface (the quotient-rule curvature bound and the
    weight-scaled evaluation allowance)."""
    rng = synth.SplitMix64(515 if not want_rational else 616)
    done = 0
    while done < 3:
        A, B = synth.random_surface(rng), synth.random_surface(rng)
        rat = bool(int(A.ivec[0]) & 2 or int(B.ivec[0]) & 2)
        if rat != want_rational:
            continue
        ta, tb = _tasks(gpu_ctx, A, B, 32)
        r = gpu_ctx.distance_bounds(ta, tb, max_rounds=8)
        assert 0.0 <= r.lb <= r.ub
        assert r.lb <= _dense_min(orc, A, B, n=64)
        assert np.all(np.diff(r.lb_round) >= 0)
        done += 1


def test_bounds_hard_wave_full_size(gpu_ctx):
    """The headline pair at nuv0 = 512: the interval closes in a few rounds."""
    A, B, _ = synth.distance_pair_hard_wave()
    ta, tb = _tasks(gpu_ctx, A, B, 512)
    r = gpu_ctx.distance_bounds(ta, tb, rel_tol=1e-6)
    assert 0.0 < r.lb <= r.ub
    assert r.ub - r.lb <= 1e-3 * r.ub
    assert np.all(np.diff(r.lb_round) >= 0)


def test_bounds_rational_saddle_plane(gpu_ctx, orc):
    """The rational intersection pair: the surfaces cross, so the minimum
    distance is 0 and the interval must close onto it from above."""
    C, D, _ = synth.intersection_pair_saddle_plane()
    ta, tb = _tasks(gpu_ctx, C, D, 32)
    r = gpu_ctx.distance_bounds(ta, tb, max_rounds=4)
    assert 0.0 <= r.lb <= r.ub
    assert r.lb <= _dense_min(orc, C, D, n=64)
    assert r.ub < 1e-3


def test_bounds_rational_separated_pair(gpu_ctx, orc):
    """A rational sine pair (seeded weights in [0.5, 2] on both nets) held
    apart: the interval certifies and brackets the dense sample minimum."""
    A0, B0, _ = synth.distance_pair_sine()
    out = []
    for k, s in enumerate((A0, B0)):
        cp, _ = s.control_net()
        w = synth.SplitMix64(900 + k).uniform(cp.shape[0] * cp.shape[1], 0.5, 2.0)
        out.append(synth.make_surface(cp.astype(np.float64), int(s.ivec[1]), int(s.ivec[4]),
                                      weights=w.reshape(cp.shape[0], cp.shape[1])))
    A, B = out
    ta, tb = _tasks(gpu_ctx, A, B, 64)
    r = gpu_ctx.distance_bounds(ta, tb, rel_tol=1e-6)
    dense = _dense_min(orc, A, B)
    assert 0.0 < r.lb <= r.ub
    assert r.lb <= dense
    assert r.ub <= dense * (1 + 1e-9) + 1e-12
    assert r.certified, (r.lb, r.ub, r.kept)


def test_bounds_rejects_nonpositive_weight(gpu_ctx):
    import jsi_cad_next_versions_b200 as J
    A0, _, _ = synth.distance_pair_sine()
    cp, _ = A0.control_net()
    w = np.ones(cp.shape[:2])
    w[1, 1] = 0.0
    A = synth.make_surface(cp.astype(np.float64), int(A0.ivec[1]), int(A0.ivec[4]), weights=w)
    ta, tb = _tasks(gpu_ctx, A, A0, 16)
    with pytest.raises(J.JsiError):
        gpu_ctx.distance_bounds(ta, tb)
