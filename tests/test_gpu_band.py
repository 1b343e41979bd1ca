"""First-round cells on large grids (the band kernel) against the oracle.

Grids of at least 16 tiles per side (nuv0 >= 129) with degrees <= 3 build
their first-round cells band by band. These cases cover each variant of that
kernel: full bicubic units (fast path) with and without weights, bands that
need one more control-net row (clustered knots), bands that need too many
rows for the factored form, lower degrees (general loop), and ragged last
tiles and bands (nuv0 - 1 not a multiple of 8). The V5_FP32 and FP64 forms
must match the oracle bit for bit (k-th squared distances and every round's
candidate list in order); the FP32 screen must match the FP64 form."""
from __future__ import annotations

import math

import numpy as np
import pytest

from conftest import rect32
from jsi_cad_next_versions_b200 import synth

pytestmark = pytest.mark.gpu


def _net(n_u, n_v, seed, lift=0.0, amp=0.05, f=3.0):
    rng = synth.SplitMix64(seed)
    x = np.arange(n_u, dtype=np.float64) / (n_u - 1)
    y = np.arange(n_v, dtype=np.float64) / (n_v - 1)
    X, Y = np.meshgrid(x, y)
    Z = amp * np.sin(2 * math.pi * f * X) * np.cos(2 * math.pi * f * Y) + lift
    Z = Z + rng.uniform(n_u * n_v, -1e-3, 1e-3).reshape(n_v, n_u)
    return np.stack([X, Y, Z], axis=-1)


def _clustered_knots(ncp, deg):
    """Clamped knots whose interior has two tiny spans at 0.5 and an uneven
    split near 0.3."""
    n_int = ncp - deg - 1
    base = list(np.linspace(0.04, 0.96, n_int - 3))
    inner = sorted(base + [0.5003, 0.5006, 0.3001])
    return np.array([0.0] * (deg + 1) + inner + [1.0] * (deg + 1))


def _weights(n_u, n_v, seed):
    return synth.SplitMix64(seed).uniform(n_u * n_v, 0.5, 2.0).reshape(n_v, n_u)


def _case(name):
    other = synth.make_surface(_net(16, 16, 91, lift=0.2, f=2.0), 3, 3)
    if name == "rational_bicubic":
        A = synth.make_surface(_net(20, 18, 11), 3, 3, weights=_weights(20, 18, 12))
        return A, other, 136
    if name == "clustered_knots":
        A = synth.make_surface(_net(24, 24, 13), 3, 3, uknots=_clustered_knots(24, 3),
                               vknots=_clustered_knots(24, 3))
        return A, other, 160
    if name == "biquadratic":
        A = synth.make_surface(_net(18, 18, 14), 2, 2)
        return A, synth.make_surface(_net(14, 14, 92, lift=0.2), 2, 2), 129
    if name == "mixed_3x2_rational":
        A = synth.make_surface(_net(19, 17, 15), 3, 2, weights=_weights(19, 17, 16))
        return A, other, 144
    raise KeyError(name)


CASES = ["rational_bicubic", "clustered_knots", "biquadratic", "mixed_3x2_rational"]


def _query(ctx, A, B, nuv0, precision, k=8, rounds=4):
    sa, sb = ctx.upload(A), ctx.upload(B)
    try:
        return ctx.min_distance(ctx.task(sa, rect32(A), nuv0, 1), ctx.task(sb, rect32(B), nuv0, 2), k=k,
                                rounds=rounds, precision=precision, trace=True)
    finally:
        ctx.release(sa)
        ctx.release(sb)


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("precision", ["v5_fp32", "fp64"])
def test_band_cells_match_oracle(gpu_ctx, orc, name, precision):
    A, B, nuv0 = _case(name)
    res = _query(gpu_ctx, A, B, nuv0, precision)
    dt = np.float32 if precision == "v5_fp32" else np.float64
    o = orc.dist_query(A, B, rect32(A).astype(dt), rect32(B).astype(dt), nuv0, 16, 8, 4, dtype=dt)
    assert np.array_equal(res.kth_d2.astype(dt).view(np.uint32 if dt == np.float32 else np.uint64),
                          o["kth_d2"].view(np.uint32 if dt == np.float32 else np.uint64))
    for r in range(len(o["pairs"])):
        assert np.array_equal(res.pairs[r], o["pairs"][r]), f"round {r + 1} candidate list"


@pytest.mark.parametrize("name", CASES)
def test_band_screen_equals_fp64(gpu_ctx, name):
    A, B, nuv0 = _case(name)
    scr = _query(gpu_ctx, A, B, nuv0, "fp32_screen")
    ref = _query(gpu_ctx, A, B, nuv0, "fp64")
    assert np.array_equal(scr.kth_d2.view(np.uint64), ref.kth_d2.view(np.uint64))
    for r in range(4):
        assert np.array_equal(scr.pairs[r], ref.pairs[r]), f"round {r + 1}"


def test_band_clustered_knots_take_all_band_forms():
    """The clustered-knot case has bands over D + 2, D + 3 and more net rows
    (checked on the host from the knots and the sample positions)."""
    A, _, nuv0 = _case("clustered_knots")
    ku = A.data[:A.ivec[3]].astype(np.float64)
    deg = int(A.ivec[1])
    u = ku[deg] + (ku[-deg - 1] - ku[deg]) * np.arange(nuv0) / (nuv0 - 1)
    span = np.searchsorted(ku, u, side="right") - 1
    span = np.minimum(span, len(ku) - deg - 2)
    rows = set()
    for b0 in range(0, nuv0 - 1, 8):
        s = span[b0:min(b0 + 9, nuv0)]
        rows.add(int(s.max() - s.min() + 1 + deg))
    assert {deg + 1, deg + 2}.issubset(rows) or {deg + 2, deg + 3}.issubset(rows)
    assert max(rows) > deg + 3
