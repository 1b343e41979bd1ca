"""FP64 Newton refinement: closest points of the distance query and
intersection points of the intersection query.  The reference stops at cell
centres and has no such outputs, so these are pinned against the oracle's
restatement (same start points, tolerance 1e-10 relative) and against
analytic cases (parallel planes, crossing planes)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rect32
from jsi_cad_next_versions_b200 import synth

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _planes():
    X, Y = np.meshgrid(np.linspace(0, 1, 6), np.linspace(0, 1, 5))
    P0 = synth.make_surface(np.stack([X, Y, 0 * X], -1), 3, 3, name="plane z=0")
    X2, Y2 = np.meshgrid(np.linspace(0, 1, 7), np.linspace(0, 1, 6))
    P1 = synth.make_surface(np.stack([0.9 * X2 + 0.05, 0.8 * Y2 + 0.1, 0 * X2 + 0.5], -1), 3, 2, name="z=0.5")
    Pt = synth.make_surface(np.stack([X2, Y2, 0.3 * X2 - 0.1], -1), 2, 3, name="z=0.3x-0.1")
    return P0, P1, Pt


def _dom(a, b):
    ra, rb = rect32(a).astype(np.float64), rect32(b).astype(np.float64)
    return np.array([ra[0], ra[2], ra[1], ra[3], rb[0], rb[2], rb[1], rb[3]])


@pytest.mark.parametrize("precision", ["v5_fp32", "fp64", "fp32_screen"])
def test_newton_parallel_planes(gpu_ctx, precision):
    P0, P1, _ = _planes()
    sa, sb = gpu_ctx.upload(P0), gpu_ctx.upload(P1)
    r = gpu_ctx.min_distance(gpu_ctx.task(sa, rect32(P0), 20, 1), gpu_ctx.task(sb, rect32(P1), 20, 2),
                             precision=precision, newton=True)
    gpu_ctx.release(sa)
    gpu_ctx.release(sb)
    assert abs(r.newton_distance - 0.5) <= 1e-12
    assert abs(r.point1[2]) <= 1e-12 and abs(r.point2[2] - 0.5) <= 1e-12
    assert abs(r.point1[0] - r.point2[0]) <= 1e-9 and abs(r.point1[1] - r.point2[1]) <= 1e-9


@pytest.mark.parametrize("case", ["sine", "hardwave", "random"])
def test_newton_distance_matches_oracle(gpu_ctx, orc, case):
    if case == "sine":
        A, B, _ = synth.distance_pair_sine()
        nuv0, k = 64, 8
    elif case == "hardwave":
        A, B, _ = synth.distance_pair_hard_wave()
        nuv0, k = 64, 8
    else:
        rng = synth.SplitMix64(404)
        A, B = synth.random_surface(rng), synth.random_surface(rng)
        nuv0, k = 40, 5
    sa, sb = gpu_ctx.upload(A), gpu_ctx.upload(B)
    r = gpu_ctx.min_distance(gpu_ctx.task(sa, rect32(A), nuv0, 1), gpu_ctx.task(sb, rect32(B), nuv0, 2), k=k,
                             precision="fp64", newton=True)
    gpu_ctx.release(sa)
    gpu_ctx.release(sb)
    o = orc.dist_query(A, B, rect32(A).astype(np.float64), rect32(B).astype(np.float64), nuv0, 16, k, 4,
                       dtype=np.float64)
    dom = _dom(A, B)
    sols = [orc.newton_distance(A, B, dom, x0) for x0 in o["starts"]]
    best = min(range(len(sols)), key=lambda q: (sols[q][0], q))
    exp = sols[best]
    assert abs(r.newton_distance - exp[0]) <= TOL * max(exp[0], 1e-300)
    assert np.allclose([*r.uv1, *r.uv2], exp[1:5], rtol=0, atol=1e-8)
    # the refined distance never exceeds the best centre distance by more than a cell
    assert r.newton_distance <= r.distance + 0.01


def test_newton_intersection_points_crossing_planes(gpu_ctx):
    P0, _, Pt = _planes()
    sa, sb = gpu_ctx.upload(P0), gpu_ctx.upload(Pt)
    r = gpu_ctx.intersect(gpu_ctx.task(sa, rect32(P0), 16, 1), gpu_ctx.task(sb, rect32(Pt), 16, 2), use_k=True,
                          rounds=3, points=True)
    gpu_ctx.release(sa)
    gpu_ctx.release(sb)
    pts = r.points
    assert pts.shape[0] == r.counts[-1] > 0
    conv = pts[pts[:, 7] <= 1e-9]
    assert conv.shape[0] == r.points_converged > 0
    # every converged point lies on the line z = 0 = 0.3 x - 0.1
    assert np.allclose(conv[:, 0], 1.0 / 3.0, atol=1e-9)
    assert np.allclose(conv[:, 2], 0.0, atol=1e-9)


@pytest.mark.parametrize("precision", ["v5_fp32", "fp64"])
def test_newton_intersection_points_match_oracle(gpu_ctx, orc, precision):
    C, D, _ = synth.intersection_pair_saddle_plane()
    nuv0 = 24
    sa, sb = gpu_ctx.upload(C), gpu_ctx.upload(D)
    r = gpu_ctx.intersect(gpu_ctx.task(sa, rect32(C), nuv0, 1), gpu_ctx.task(sb, rect32(D), nuv0, 2), use_k=False,
                          rounds=3, precision=precision, points=True)
    gpu_ctx.release(sa)
    gpu_ctx.release(sb)
    dt = np.float32 if precision == "v5_fp32" else np.float64
    o = orc.inter_query(C, D, rect32(C).astype(dt), rect32(D).astype(dt), nuv0, 16, 0, rounds=3, dtype=dt,
                        starts_cap=1 << 16)
    assert r.points.shape[0] == o["starts"].shape[0]
    dom = _dom(C, D)
    for q in range(0, r.points.shape[0], max(1, r.points.shape[0] // 64)):
        exp = orc.newton_point(C, D, dom, o["starts"][q])
        got = r.points[q]
        assert np.allclose(got[:7], exp[:7], rtol=TOL, atol=1e-12), q
    assert r.points_converged > 0.5 * r.points.shape[0]
