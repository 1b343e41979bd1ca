"""The FP32-screen form's candidate sets, checked as sets.

* Intersection: the first round's FP32 screen (FP32 samples, curvature
  terms, boxes and overlap tests, widened by a rigorous rounding-error bound)
  must return a superset of the FP64 form's first-round overlap pairs, and
  after the FP64 re-check every round's pair list must equal the FP64 form's
  and the oracle's (intersection.cu:259-309 over boxes from :106-148 padded
  by compute_K, common.cu:149-172).  Full size: the rational saddle / plane
  pair at nuv0 = 256 (4.2e9 first-round box tests), curvature padding on and
  off, against the reference's own counts and the oracle's per-round list
  digests (tests/golden/make_oracle_digests.py).
* Distance: the FP32 screen's candidates must contain every pair whose FP64
  squared centre distance is at most the FP64 k-th value
  (distance_analysis.cu:202-207, 246-338).

Tolerance: zero.  The lists are integer index triples and must match
exactly; intersection points and distances of the two forms are compared
bit for bit, because the FP64 re-check makes every later step identical.
"""
from __future__ import annotations

import hashlib
import json

import numpy as np
import pytest

from conftest import GOLDEN, load_npz, rect32, surface_from
from jsi_cad_next_versions_b200 import synth

pytestmark = pytest.mark.gpu


def _keys(p: np.ndarray) -> np.ndarray:
    """(slot, i, j) triples as one sortable int64 each."""
    p = np.asarray(p, np.int64).reshape(-1, 3)
    return (p[:, 0] << 42) | (p[:, 1] << 21) | p[:, 2]


def _contains(sup: np.ndarray, sub: np.ndarray) -> bool:
    return bool(np.isin(_keys(sub), _keys(sup), assume_unique=False).all())


def _digest(p) -> str:
    return hashlib.sha256(np.ascontiguousarray(p, dtype=np.int32).tobytes()).hexdigest()


def _inter(ctx, A, B, nuv0, use_k, **kw):
    sa, sb = ctx.upload(A), ctx.upload(B)
    try:
        return ctx.intersect(ctx.task(sa, rect32(A), nuv0, 1), ctx.task(sb, rect32(B), nuv0, 2), use_k=bool(use_k),
                             **kw)
    finally:
        ctx.release(sa)
        ctx.release(sb)


@pytest.mark.parametrize("use_k", [1, 0])
def test_saddle_plane_full_size_screen_superset_and_exact(gpu_ctx, use_k):
    C, D, _ = synth.intersection_pair_saddle_plane()
    ref = load_npz("ref_inter_synth.npz")
    dig = json.loads((GOLDEN / "oracle_inter_n256.json").read_text())
    v5 = _inter(gpu_ctx, C, D, 256, use_k, precision="v5_fp32", trace=True)
    assert np.array_equal(v5.counts, ref[f"n256/k{use_k}/counts"])
    assert [_digest(p) for p in v5.pairs] == dig[f"f32/k{use_k}"]["sha256"]
    f64 = _inter(gpu_ctx, C, D, 256, use_k, precision="fp64", trace=True, points=True)
    scr = _inter(gpu_ctx, C, D, 256, use_k, precision="fp32_screen", trace=True, points=True, screen_trace=True)
    assert f64.counts.tolist() == dig[f"f64/k{use_k}"]["counts"]
    assert [_digest(p) for p in f64.pairs] == dig[f"f64/k{use_k}"]["sha256"]
    # the FP32 screen's first-round candidates hold every FP64 pair ...
    assert scr.screen_written >= f64.counts[0]
    # ... are the same on every run (the widening is a fixed bound per region
    # pair) and only slightly more
    again = _inter(gpu_ctx, C, D, 256, use_k, precision="fp32_screen")
    assert again.screen_written == scr.screen_written
    assert scr.screen_written <= 1.02 * f64.counts[0] + 256
    assert scr.screen_pairs.shape[0] == scr.screen_written
    assert _contains(scr.screen_pairs, f64.pairs[0])
    # ... and after the FP64 re-check every round equals the FP64 form's
    assert np.array_equal(scr.counts, f64.counts)
    for r in range(f64.rounds):
        assert np.array_equal(scr.pairs[r], f64.pairs[r]), f"round {r + 1}"
    assert scr.pad == f64.pad
    if use_k:
        assert np.float64(scr.pad[0]) == np.float64(dig["f64/k1"]["pads"][0])
        assert 0 < scr.kmax_rechecked < 2 * 256 * 256
    # same final pairs and regions: the FP64 Newton points are identical
    assert np.array_equal(scr.points.view(np.uint64), f64.points.view(np.uint64))
    assert scr.points_converged == f64.points_converged > 0


@pytest.mark.parametrize("case", [3, 4])
@pytest.mark.parametrize("use_k", [1, 0])
def test_reference_cases_screen_equals_oracle_fp64(gpu_ctx, orc, case, use_k):
    g = load_npz("ref_intersection.npz")
    A = surface_from(g[f"case{case}/ivec1"], g[f"case{case}/data1"])
    B = surface_from(g[f"case{case}/ivec2"], g[f"case{case}/data2"])
    scr = _inter(gpu_ctx, A, B, 16, use_k, precision="fp32_screen", trace=True, screen_trace=True)
    o = orc.inter_query(A, B, rect32(A).astype(np.float64), rect32(B).astype(np.float64), 16, 16, use_k,
                        dtype=np.float64)
    assert np.array_equal(scr.counts, o["counts"])
    for r in range(scr.rounds):
        assert np.array_equal(scr.pairs[r], o["pairs"][r]), f"round {r + 1}"
    assert _contains(scr.screen_pairs, o["pairs"][0])


@pytest.mark.parametrize("seed", [41, 42, 43, 44, 45, 46])
def test_random_pairs_screen_equals_oracle_fp64(gpu_ctx, orc, seed):
    """Mixed degrees 1-5, about 30% rational surfaces, uneven nuv0."""
    rng = synth.SplitMix64(seed)
    A = synth.random_surface(rng)
    B = synth.random_surface(rng)
    nuv0 = 14 + 5 * (seed % 9)
    use_k = seed % 2
    scr = _inter(gpu_ctx, A, B, nuv0, use_k, precision="fp32_screen", rounds=4, trace=True, screen_trace=True)
    o = orc.inter_query(A, B, rect32(A).astype(np.float64), rect32(B).astype(np.float64), nuv0, 16, use_k,
                        rounds=4, dtype=np.float64)
    assert np.array_equal(scr.counts, o["counts"])
    for r in range(scr.rounds):
        if o["pairs"][r] is not None:
            assert np.array_equal(scr.pairs[r], o["pairs"][r]), f"round {r + 1}"
    if scr.rounds:
        assert _contains(scr.screen_pairs, o["pairs"][0])


# ---------------------------------------------------------------------------
# distance: the screen's candidates hold every pair at or below the k-th d2
# ---------------------------------------------------------------------------

def _dist(ctx, A, B, nuv0, k, precision):
    sa, sb = ctx.upload(A), ctx.upload(B)
    try:
        return ctx.min_distance(ctx.task(sa, rect32(A), nuv0, 1), ctx.task(sb, rect32(B), nuv0, 2), k=k,
                                precision=precision, trace=True, cand_trace=True)
    finally:
        ctx.release(sa)
        ctx.release(sb)


def _check_distance_superset(ctx, A, B, nuv0, k):
    f64 = _dist(ctx, A, B, nuv0, k, "fp64")
    scr = _dist(ctx, A, B, nuv0, k, "fp32_screen")
    kth = f64.kth_d2[0]
    # every FP64 pair with d2 <= the k-th value (the FP64 form's exact culling
    # keeps them all among its own candidates)
    exact = f64.cand_pairs[f64.cand_d2 <= kth]
    assert exact.shape[0] >= f64.npairs[0]
    assert _contains(exact, f64.pairs[0])
    assert _contains(scr.cand_pairs, exact)
    # the FP64 d2 the screen path re-checked agree with the FP64 form's
    common = np.isin(_keys(scr.cand_pairs), _keys(exact))
    sk = np.argsort(_keys(scr.cand_pairs)[common])
    ek = np.argsort(_keys(exact))
    assert np.array_equal(scr.cand_d2[common][sk].view(np.uint64), f64.cand_d2[f64.cand_d2 <= kth][ek].view(np.uint64))
    assert np.array_equal(scr.kth_d2, f64.kth_d2)
    return exact.shape[0], scr.cand_pairs.shape[0]


def test_distance_hardwave_full_size_screen_superset(gpu_ctx):
    A, B, _ = synth.distance_pair_hard_wave()
    _check_distance_superset(gpu_ctx, A, B, 512, 8)


@pytest.mark.parametrize("seed", [51, 52, 53, 54])
def test_distance_random_rational_screen_superset(gpu_ctx, seed):
    rng = synth.SplitMix64(seed)
    A = synth.random_surface(rng)
    B = synth.random_surface(rng)
    if not (A.rational or B.rational):
        # make one side rational: same net, seeded weights in [0.5, 2]
        cp, _ = A.control_net()
        w = synth.SplitMix64(seed + 1000).uniform(cp.shape[0] * cp.shape[1], 0.5, 2.0)
        A = synth.make_surface(cp.astype(np.float64), int(A.ivec[1]), int(A.ivec[4]),
                               weights=w.reshape(cp.shape[0], cp.shape[1]))
    _check_distance_superset(gpu_ctx, A, B, 48 + 8 * (seed % 4), [1, 5, 8, 33][seed % 4])


def test_distance_sine_screen_superset_matches_brute_force(gpu_ctx, orc):
    """At nuv0 = 64 the exact set {d2 <= k-th} is enumerated on the CPU from
    the oracle's FP64 cell centres and must equal the GPU FP64 form's."""
    A, B, _ = synth.distance_pair_sine()
    f64 = _dist(gpu_ctx, A, B, 64, 8, "fp64")
    ca = orc.region_cells(A, rect32(A).astype(np.float64), 64, radii=False, dtype=np.float64)[0].reshape(-1, 3)
    cb = orc.region_cells(B, rect32(B).astype(np.float64), 64, radii=False, dtype=np.float64)[0].reshape(-1, 3)
    d2 = ((ca[:, None, 0] - cb[None, :, 0]) ** 2 + (ca[:, None, 1] - cb[None, :, 1]) ** 2
          + (ca[:, None, 2] - cb[None, :, 2]) ** 2)
    ii, jj = np.nonzero(d2 <= f64.kth_d2[0])
    brute = np.stack([np.zeros_like(ii), ii, jj], 1)
    exact = f64.cand_pairs[f64.cand_d2 <= f64.kth_d2[0]]
    assert np.array_equal(np.sort(_keys(brute)), np.sort(_keys(exact)))
    n_exact, n_scr = _check_distance_superset(gpu_ctx, A, B, 64, 8)
    assert n_scr >= n_exact
