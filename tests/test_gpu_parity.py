"""Parity of the CUDA path (through the C ABI) with the reference and the oracle.

* V5_FP32 form: bit-for-bit against the reference's golden vectors and, per
  round, against the oracle's float instantiation (candidate sets in order).
* FP64 form: bit-for-bit against the oracle's double instantiation (the
  plain-FP64 restatement of the same algorithm): same candidate sets, same
  k-th squared distances.
"""
from __future__ import annotations

import json

import numpy as np
import pytest

from conftest import GOLDEN, load_npz, rect32, surface_from
from jsi_cad_next_versions_b200 import synth

pytestmark = pytest.mark.gpu


def _task(ctx, sid, rect, nuv, side):
    return ctx.task(sid, rect, nuv, side)


def _grid_names():
    g = load_npz("ref_eval_grids.npz")
    return sorted({k.split("/")[0] for k in g})


# ---------------------------------------------------------------------------
# grid evaluation
# ---------------------------------------------------------------------------

@pytest.mark.parametrize("name", _grid_names())
@pytest.mark.parametrize("nuv", [5, 16])
def test_eval_grid_matches_reference_bits(gpu_ctx, name, nuv):
    g = load_npz("ref_eval_grids.npz")
    us, vs, u0, v0 = g[f"{name}/n{nuv}/params"]
    got = gpu_ctx.eval_grid(g[f"{name}/ivec"], g[f"{name}/data"], us, vs, u0, v0, nuv)
    exp = g[f"{name}/n{nuv}/records"]
    assert np.array_equal(got.view(np.uint32), exp.view(np.uint32))


@pytest.mark.parametrize("name", _grid_names())
def test_eval_grid_f64_matches_oracle_bits(gpu_ctx, orc, name):
    g = load_npz("ref_eval_grids.npz")
    s = surface_from(g[f"{name}/ivec"], g[f"{name}/data"])
    r = [float(x) for x in s.rect()]
    nuv = 13
    us, vs = (r[2] - r[0]) / nuv, (r[3] - r[1]) / nuv
    got = gpu_ctx.eval_grid(s.ivec, s.data, us, vs, r[0], r[1], nuv, dtype=np.float64)
    exp = orc.eval_grid(s, us, vs, r[0], r[1], nuv, dtype=np.float64)
    assert np.array_equal(got.view(np.uint64), exp.view(np.uint64))


def test_eval_with_cuda_name(gpu_ctx):
    """The reference's evalWithCuda entry point name, over the default context."""
    import jsi_cad_next_versions_b200 as J
    g = load_npz("ref_eval_grids.npz")
    s = surface_from(g["sine_a/ivec"], g["sine_a/data"])
    r = s.rect()
    us = np.float32((r[2] - r[0]) / np.float32(33))
    J.init_cad()
    try:
        out = np.zeros(33 * 33 * J.ONE_UV_SIZE, np.float32)
        J.evalWithCuda(s.ivec, s.data, s.ndata, us, us, r[0], r[1], 33, out)
    finally:
        J.deinit_cad()
    assert np.array_equal(out.view(np.uint32), g["sine_a/evalWithCuda33"].view(np.uint32))


# ---------------------------------------------------------------------------
# minimum distance
# ---------------------------------------------------------------------------

def _dist_both(ctx, orc, A, B, nuv0, k, rounds=4, nuv_b=None, precision="v5_fp32"):
    ra, rb = rect32(A), rect32(B)
    sa, sb = ctx.upload(A), ctx.upload(B)
    try:
        res = ctx.min_distance(_task(ctx, sa, ra, nuv0, 1), _task(ctx, sb, rb, nuv_b or nuv0, 2), k=k,
                               rounds=rounds, precision=precision, trace=True)
    finally:
        ctx.release(sa)
        ctx.release(sb)
    return res


@pytest.mark.parametrize("key", ["sine/n64/k8", "sine/n64/k64", "sine/n32/k8", "hardwave/n64/k8",
                                 "hardwave/n128/k8"])
def test_distance_v5_matches_reference_and_oracle(gpu_ctx, orc, key):
    g = load_npz("ref_distance.npz")
    name, n, k = key.split("/")
    nuv0, k = int(n[1:]), int(k[1:])
    A, B, _ = synth.distance_pair_sine() if name == "sine" else synth.distance_pair_hard_wave()
    res = _dist_both(gpu_ctx, orc, A, B, nuv0, k)
    per_round = np.sqrt(res.kth_d2.astype(np.float32))
    assert np.array_equal(per_round.view(np.uint32), g[key + "/per_round"].view(np.uint32))
    assert np.float32(res.v5_value) == g[key + "/per_round"][-1]
    o = orc.dist_query(A, B, rect32(A), rect32(B), nuv0, 16, k, 4)
    for r in range(4):
        assert np.array_equal(res.pairs[r], o["pairs"][r]), f"round {r + 1} candidate list"


@pytest.mark.parametrize("key", ["sine/n64/k8", "sine/n64/k64", "hardwave/n64/k8"])
def test_distance_fp64_matches_oracle(gpu_ctx, orc, key):
    name, n, k = key.split("/")
    nuv0, k = int(n[1:]), int(k[1:])
    A, B, _ = synth.distance_pair_sine() if name == "sine" else synth.distance_pair_hard_wave()
    res = _dist_both(gpu_ctx, orc, A, B, nuv0, k, precision="fp64")
    o = orc.dist_query(A, B, rect32(A).astype(np.float64), rect32(B).astype(np.float64), nuv0, 16, k, 4,
                       dtype=np.float64)
    assert np.array_equal(res.kth_d2.view(np.uint64), o["kth_d2"].view(np.uint64))
    for r in range(4):
        assert np.array_equal(res.pairs[r], o["pairs"][r])
    assert res.distance == np.sqrt(o["kth_d2"][-1])


def test_distance_full_size_hardwave(gpu_ctx):
    """Hard-wave pair at full size, nuv0 = 512: the reference's own value."""
    path = GOLDEN / "ref_full.json"
    if not path.exists():
        pytest.skip("full-size fixture not generated")
    full = json.loads(path.read_text())["hardwave_n512_k8"]
    A, B, _ = synth.distance_pair_hard_wave()
    sa, sb = gpu_ctx.upload(A), gpu_ctx.upload(B)
    res = gpu_ctx.min_distance(_task(gpu_ctx, sa, rect32(A), 512, 1), _task(gpu_ctx, sb, rect32(B), 512, 2))
    gpu_ctx.release(sa)
    gpu_ctx.release(sb)
    assert np.float32(res.v5_value).view(np.uint32) == full["value_bits"]


@pytest.mark.parametrize("seed", [11, 12, 13, 14])
@pytest.mark.parametrize("precision", ["v5_fp32", "fp64"])
def test_distance_random_pairs(gpu_ctx, orc, seed, precision):
    """Mixed degrees 2..5, rational and non-rational, uneven nuv per side."""
    rng = synth.SplitMix64(seed)
    A = synth.random_surface(rng)
    B = synth.random_surface(rng)
    nuv_a, nuv_b = 17 + seed, 23 + 2 * seed
    k = [1, 5, 8, 33][seed % 4]
    res = _dist_both(gpu_ctx, orc, A, B, nuv_a, k, nuv_b=nuv_b, precision=precision)
    dt = np.float32 if precision == "v5_fp32" else np.float64
    # The oracle's dist_query uses one nuv for both sides: compare round by round
    # through the oracle's per-side interface only when nuv_a == nuv_b.
    res2 = _dist_both(gpu_ctx, orc, A, B, nuv_a, k, precision=precision)
    o = orc.dist_query(A, B, rect32(A).astype(dt), rect32(B).astype(dt), nuv_a, 16, k, 4, dtype=dt)
    assert np.array_equal(res2.kth_d2.astype(dt), o["kth_d2"])
    for r in range(len(o["pairs"])):
        assert np.array_equal(res2.pairs[r], o["pairs"][r])
    assert res.rounds >= 1


def test_distance_k_larger_than_pairs(gpu_ctx, orc):
    """k beyond the number of cell pairs keeps every pair (min(k, num),
    distance_analysis.cu:142, :236-240)."""
    A, B, _ = synth.distance_pair_sine()
    res = _dist_both(gpu_ctx, orc, A, B, 3, 64, rounds=2)
    o = orc.dist_query(A, B, rect32(A), rect32(B), 3, 16, 64, 2)
    assert res.npairs[0] == 16
    for r in range(2):
        assert np.array_equal(res.pairs[r], o["pairs"][r])
    assert np.array_equal(res.kth_d2.astype(np.float32), o["kth_d2"])


# ---------------------------------------------------------------------------
# intersection
# ---------------------------------------------------------------------------

def _inter(ctx, A, B, nuv0, use_k, precision="v5_fp32", rounds=6):
    sa, sb = ctx.upload(A), ctx.upload(B)
    try:
        return ctx.intersect(_task(ctx, sa, rect32(A), nuv0, 1), _task(ctx, sb, rect32(B), nuv0, 2),
                             use_k=bool(use_k), precision=precision, rounds=rounds, trace=True)
    finally:
        ctx.release(sa)
        ctx.release(sb)


@pytest.mark.parametrize("case", [3, 4])
@pytest.mark.parametrize("use_k", [1, 0])
def test_intersection_reference_cases(gpu_ctx, orc, case, use_k):
    g = load_npz("ref_intersection.npz")
    A = surface_from(g[f"case{case}/ivec1"], g[f"case{case}/data1"])
    B = surface_from(g[f"case{case}/ivec2"], g[f"case{case}/data2"])
    res = _inter(gpu_ctx, A, B, 16, use_k)
    assert np.array_equal(res.counts, g[f"case{case}/k{use_k}/counts"])
    o = orc.inter_query(A, B, rect32(A), rect32(B), 16, 16, use_k)
    for r in range(res.rounds):
        assert np.array_equal(res.pairs[r], o["pairs"][r]), f"round {r + 1}"
    assert np.float32(res.pad[0]) == o["pads"][0] and np.float32(res.pad[1]) == o["pads"][1]


@pytest.mark.parametrize("case", [3, 4])
@pytest.mark.parametrize("use_k", [1, 0])
def test_intersection_fp64_matches_oracle(gpu_ctx, orc, case, use_k):
    g = load_npz("ref_intersection.npz")
    A = surface_from(g[f"case{case}/ivec1"], g[f"case{case}/data1"])
    B = surface_from(g[f"case{case}/ivec2"], g[f"case{case}/data2"])
    res = _inter(gpu_ctx, A, B, 16, use_k, precision="fp64")
    o = orc.inter_query(A, B, rect32(A).astype(np.float64), rect32(B).astype(np.float64), 16, 16, use_k,
                        dtype=np.float64)
    assert np.array_equal(res.counts, o["counts"])
    for r in range(res.rounds):
        assert np.array_equal(res.pairs[r], o["pairs"][r]), f"round {r + 1}"


@pytest.mark.parametrize("nuv0", [16, 32])
@pytest.mark.parametrize("use_k", [1, 0])
def test_intersection_saddle_plane_counts(gpu_ctx, nuv0, use_k):
    g = load_npz("ref_inter_synth.npz")
    C, D, _ = synth.intersection_pair_saddle_plane()
    res = _inter(gpu_ctx, C, D, nuv0, use_k)
    assert np.array_equal(res.counts, g[f"n{nuv0}/k{use_k}/counts"])


@pytest.mark.parametrize("seed", [21, 22, 23])
@pytest.mark.parametrize("precision", ["v5_fp32", "fp64"])
def test_intersection_random_pairs(gpu_ctx, orc, seed, precision):
    rng = synth.SplitMix64(seed)
    A = synth.random_surface(rng)
    B = synth.random_surface(rng)
    dt = np.float32 if precision == "v5_fp32" else np.float64
    nuv0 = 12 + seed % 7
    res = _inter(gpu_ctx, A, B, nuv0, 1, precision=precision, rounds=4)
    o = orc.inter_query(A, B, rect32(A).astype(dt), rect32(B).astype(dt), nuv0, 16, 1, rounds=4, dtype=dt)
    assert np.array_equal(res.counts, o["counts"])
    for r in range(res.rounds):
        if o["pairs"][r] is not None:
            assert np.array_equal(res.pairs[r], o["pairs"][r])


@pytest.mark.parametrize("case", [1, 2])
def test_intersection_degree11_reference_inputs(gpu_ctx, ref, orc, case):
    """The reference's own degree-11 inputs (345x356 control points), read
    from the compiled reference data when oracle/_ref is present."""
    ia, da = ref.face(f"inter_case{case}_obj1")
    ib, db = ref.face(f"inter_case{case}_obj2")
    A, B = surface_from(ia, da), surface_from(ib, db)
    res = _inter(gpu_ctx, A, B, 16, 1)
    o = orc.inter_query(A, B, rect32(A), rect32(B), 16, 16, 1, pair_cap=1 << 20)
    assert np.array_equal(res.counts, o["counts"])
    for r in range(res.rounds):
        if o["pairs"][r] is not None:
            assert np.array_equal(res.pairs[r], o["pairs"][r])


# ---------------------------------------------------------------------------
# FP32-screen form: FP32 evaluation and screening with rigorous bounds, FP64
# re-check; its candidate lists and k-th distances must equal the FP64 form's.
# ---------------------------------------------------------------------------

@pytest.mark.parametrize("key", ["sine/n64/k8", "sine/n64/k64", "sine/n32/k8", "hardwave/n64/k8",
                                 "hardwave/n128/k8"])
def test_distance_screen_equals_fp64(gpu_ctx, orc, key):
    name, n, k = key.split("/")
    nuv0, k = int(n[1:]), int(k[1:])
    A, B, _ = synth.distance_pair_sine() if name == "sine" else synth.distance_pair_hard_wave()
    scr = _dist_both(gpu_ctx, orc, A, B, nuv0, k, precision="fp32_screen")
    ref = _dist_both(gpu_ctx, orc, A, B, nuv0, k, precision="fp64")
    assert np.array_equal(scr.kth_d2.view(np.uint64), ref.kth_d2.view(np.uint64))
    for r in range(4):
        assert np.array_equal(scr.pairs[r], ref.pairs[r]), f"round {r + 1}"
        # the FP32 screen passed a superset of the kept pairs
        assert scr.candidates[r] >= scr.npairs[r]
    assert scr.distance == ref.distance


@pytest.mark.parametrize("seed", [31, 32, 33, 34, 35, 36])
def test_distance_screen_random_pairs(gpu_ctx, orc, seed):
    """Mixed degrees, 30% rational, nuv0 per side, k in {1, 5, 8, 33}."""
    rng = synth.SplitMix64(seed)
    A = synth.random_surface(rng)
    B = synth.random_surface(rng)
    nuv0 = 20 + 3 * seed % 40
    k = [1, 5, 8, 33][seed % 4]
    scr = _dist_both(gpu_ctx, orc, A, B, nuv0, k, precision="fp32_screen")
    o = orc.dist_query(A, B, rect32(A).astype(np.float64), rect32(B).astype(np.float64), nuv0, 16, k, 4,
                       dtype=np.float64)
    assert np.array_equal(scr.kth_d2, o["kth_d2"])
    for r in range(len(o["pairs"])):
        assert np.array_equal(scr.pairs[r], o["pairs"][r])


def test_distance_screen_full_size(gpu_ctx):
    """Full-size hard-wave pair (nuv0 = 512): screen form == FP64 form."""
    A, B, _ = synth.distance_pair_hard_wave()
    sa, sb = gpu_ctx.upload(A), gpu_ctx.upload(B)
    ta, tb = _task(gpu_ctx, sa, rect32(A), 512, 1), _task(gpu_ctx, sb, rect32(B), 512, 2)
    scr = gpu_ctx.min_distance(ta, tb, precision="fp32_screen", trace=True)
    ref = gpu_ctx.min_distance(ta, tb, precision="fp64", trace=True)
    gpu_ctx.release(sa)
    gpu_ctx.release(sb)
    assert np.array_equal(scr.kth_d2, ref.kth_d2)
    for r in range(4):
        assert np.array_equal(scr.pairs[r], ref.pairs[r])


def test_distance_4x_scaled_nuv2048(gpu_ctx):
    """The 4x geometrically scaled hard-wave pair at nuv0 = 2048 (4.19M cells
    per side, 1.76e13 cell pairs brute force): the FP32-screen form equals the
    FP64 form round by round, and the V5-FP32 value agrees with FP64 to FP32
    precision.  (The CPU paths would need hours at this size.)"""
    A, B, _ = synth.distance_pair_hard_wave(scale=4.0)
    sa, sb = gpu_ctx.upload(A), gpu_ctx.upload(B)
    ta, tb = _task(gpu_ctx, sa, rect32(A), 2048, 1), _task(gpu_ctx, sb, rect32(B), 2048, 2)
    r64 = gpu_ctx.min_distance(ta, tb, precision="fp64", trace=True)
    scr = gpu_ctx.min_distance(ta, tb, precision="fp32_screen", trace=True)
    v5 = gpu_ctx.min_distance(ta, tb, precision="v5_fp32", trace=True)
    gpu_ctx.release(sa)
    gpu_ctx.release(sb)
    assert np.array_equal(scr.kth_d2, r64.kth_d2)
    for r in range(4):
        assert np.array_equal(scr.pairs[r], r64.pairs[r])
    assert abs(v5.distance - r64.distance) <= 1e-5 * r64.distance
    # round 1 examined a tiny fraction of the (2047^2)^2 pairs
    assert r64.pair_tests[0] < 1e9


@pytest.mark.parametrize("precision", ["v5_fp32", "fp64", "fp32_screen"])
@pytest.mark.parametrize("k", [1, 8, 300])
def test_distance_heavy_exact_ties(gpu_ctx, orc, precision, k):
    """Parallel planes on regular grids: thousands of cell pairs share the
    k-th squared distance exactly; the kept pairs are the first k under the
    reference's (d2, slot, i, j) order."""
    X, Y = np.meshgrid(np.linspace(0, 1, 6), np.linspace(0, 1, 5))
    P0 = synth.make_surface(np.stack([X, Y, 0 * X], -1), 3, 3)
    X2, Y2 = np.meshgrid(np.linspace(0, 1, 7), np.linspace(0, 1, 6))
    P1 = synth.make_surface(np.stack([0.9 * X2 + 0.05, 0.8 * Y2 + 0.1, 0 * X2 + 0.5], -1), 3, 2)
    res = _dist_both(gpu_ctx, orc, P0, P1, 20, k, rounds=2, precision=precision)
    dt = np.float32 if precision == "v5_fp32" else np.float64
    o = orc.dist_query(P0, P1, rect32(P0).astype(dt), rect32(P1).astype(dt), 20, 16, k, 2, dtype=dt)
    for r in range(2):
        assert np.array_equal(res.pairs[r], o["pairs"][r])
    assert np.array_equal(res.kth_d2.astype(dt), o["kth_d2"])


def _run_example(binary, case, use_k):
    import os
    import re
    import subprocess
    env = dict(os.environ, CAD_INTERSECT_USE_K=str(use_k), OMP_NUM_THREADS="4")
    out = subprocess.run([str(binary), str(case)], env=env, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stdout[-2000:] + out.stderr[-2000:]
    return [int(m.group(2)) for m in re.finditer(r"Round (\d+): overlap pairs = (\d+)", out.stdout)]


@pytest.mark.parametrize("case", [3, 4])
@pytest.mark.parametrize("use_k", [1, 0])
def test_reference_example_linked_to_b200_library(case, use_k):
    """The reference's own examples/intersection_example.cu, compiled
    unchanged and linked against libjsi_v5_shim.so (the reference's C++ API
    over this library's C ABI), prints the reference's per-round counts."""
    from conftest import ROOT
    binary = ROOT / "oracle" / "_ref" / "test_intersect_b200"
    if not binary.exists():
        pytest.skip("reference example not built (needs the reference checkout at build time)")
    g = load_npz("ref_intersection.npz")
    assert _run_example(binary, case, use_k) == g[f"case{case}/k{use_k}/counts"].tolist()


@pytest.mark.parametrize("case", [1, 2])
def test_reference_example_degree11_linked_to_b200_library(case):
    from conftest import ROOT
    b200 = ROOT / "oracle" / "_ref" / "test_intersect_b200"
    ref = ROOT / "oracle" / "_ref" / "test_intersect_ref"
    if not (b200.exists() and ref.exists()):
        pytest.skip("reference example not built")
    assert _run_example(b200, case, 1) == _run_example(ref, case, 1)
