"""Generates the committed golden fixtures of tests/golden/ from the reference.

Run in a container where the reference checkout is present:

    make -C oracle ref && python tests/golden/make_golden.py [--full]

Every number here comes from the reference VERSION5 itself, compiled from its
own sources into oracle/_ref/libjsi_v5_ref.so (oracle/Makefile):

* ref_eval_grids.npz    EG_spline2dDeriv_irrational records (evaluation.cu:358-374)
                        and compute_K (common.cu:149-172) on synthetic surfaces
* ref_intersection.npz  the reference's built-in inputs inter_case3/4 (ivec, data),
                        per-round "overlap pairs" counts of intersection()
                        (intersection.cu:338-475), K on and off, the printed initial
                        paddings, and the round-1 overlap lists
* ref_distance.npz      per-round k-th distances of minimum_distance()
                        (distance_analysis.cu:356-506) obtained by running it with
                        max_layers = 1..rounds, and the round-1 top-k lists
* ref_inter_synth.npz   per-round counts (and round-1 paddings) on the saddle/plane pair at
                        nuv0 = 16, 32 and the full-size 256
* ref_full.json         (--full) the full-size hard-wave distance (nuv0 = 512)

Synthetic surfaces are regenerated by jsi_cad_next_versions_b200.synth; each
fixture stores a digest of the float32 data it was made from.
"""
from __future__ import annotations

import hashlib
import json
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402
from jsi_cad_next_versions_b200 import synth  # noqa: E402

OUT = Path(__file__).resolve().parent


def digest(s) -> str:
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(s.ivec, np.int32).tobytes())
    h.update(np.ascontiguousarray(s.data, np.float32).tobytes())
    return h.hexdigest()[:16]


def eval_surfaces():
    """Surfaces for the evaluation fixtures: a spread of degrees, rational and
    non-rational, clamped knots, plus the reference's own case-3/4 inputs."""
    out = {}
    A, B, _ = synth.distance_pair_sine()
    out["sine_a"] = A
    out["sine_b"] = B
    C, D, _ = synth.intersection_pair_saddle_plane()
    out["saddle_rat"] = C
    out["plane_rat"] = D
    rng = synth.SplitMix64(99)
    for q in range(6):
        out[f"rand{q}"] = synth.random_surface(rng, name=f"rand{q}")
    # forced low / high degrees and a degree-1 direction
    X, Y = np.meshgrid(np.linspace(0, 1, 6), np.linspace(0, 1, 5))
    Z = 0.3 * np.sin(3 * X) * np.cos(2 * Y)
    out["deg1x2"] = synth.make_surface(np.stack([X, Y, Z], -1), 1, 2, name="deg1x2")
    X, Y = np.meshgrid(np.linspace(0, 1, 9), np.linspace(0, 1, 8))
    Z = 0.2 * np.sin(5 * X + 1) * np.cos(4 * Y)
    W = 0.5 + 1.5 * (np.sin(7 * X * Y) ** 2)
    out["deg5x4_rat"] = synth.make_surface(np.stack([X, Y, Z], -1), 5, 4, weights=W, name="deg5x4_rat")
    return out


def main(full: bool = False):
    R = oracle.Reference()
    t0 = time.time()

    # --- evaluation grids -------------------------------------------------
    grids = {}
    meta = {}
    for name, s in eval_surfaces().items():
        r = s.rect()
        for nuv in (5, 16):
            us = np.float32((r[2] - r[0]) / np.float32(nuv))
            vs = np.float32((r[3] - r[1]) / np.float32(nuv))
            g = R.eval_grid(s, us, vs, r[0], r[1], nuv)
            grids[f"{name}/n{nuv}/records"] = g
            grids[f"{name}/n{nuv}/K"] = np.array([R.compute_k(g, nuv)], np.float32)
            grids[f"{name}/n{nuv}/params"] = np.array([us, vs, r[0], r[1]], np.float32)
        grids[f"{name}/ivec"] = s.ivec
        grids[f"{name}/data"] = s.data
        meta[name] = digest(s)
    # evalWithCuda (strip driver) on one surface
    s = eval_surfaces()["sine_a"]
    r = s.rect()
    us = np.float32((r[2] - r[0]) / np.float32(33))
    grids["sine_a/evalWithCuda33"] = R.eval_with_cuda(s, us, us, r[0], r[1], 33)
    np.savez_compressed(OUT / "ref_eval_grids.npz", **grids)
    (OUT / "ref_eval_grids.json").write_text(json.dumps(meta, indent=1))
    print(f"eval grids done {time.time() - t0:.1f}s")

    # --- reference intersection cases 3 and 4 -----------------------------
    inter = {}
    for case in (3, 4):
        ia, da = R.face(f"inter_case{case}_obj1")
        ib, db = R.face(f"inter_case{case}_obj2")
        inter[f"case{case}/ivec1"], inter[f"case{case}/data1"] = ia, da
        inter[f"case{case}/ivec2"], inter[f"case{case}/data2"] = ib, db
        SA, SB = synth.Surface(ia, da), synth.Surface(ib, db)
        ra, rb = np.array(SA.rect(), np.float32), np.array(SB.rect(), np.float32)
        for use_k in (1, 0):
            res = R.intersection(SA, SB, ra, rb, 16, 16, use_k)
            inter[f"case{case}/k{use_k}/counts"] = res["counts"]
            r1 = R.inter_round1(SA, SB, ra, rb, 16, use_k)
            inter[f"case{case}/k{use_k}/round1_i"] = r1["i"]
            inter[f"case{case}/k{use_k}/round1_j"] = r1["j"]
            if use_k:
                inter[f"case{case}/k1/pads_printed"] = np.array(res["pads"], np.float64)
    np.savez_compressed(OUT / "ref_intersection.npz", **inter)
    print(f"intersection cases done {time.time() - t0:.1f}s")

    # --- distance ----------------------------------------------------------
    dist = {}
    dmeta = {}
    cases = []
    A, B, q = synth.distance_pair_sine()
    cases += [("sine", A, B, 64, 8), ("sine", A, B, 64, 64), ("sine", A, B, 32, 8)]
    HA, HB, _ = synth.distance_pair_hard_wave()
    cases += [("hardwave", HA, HB, 64, 8), ("hardwave", HA, HB, 128, 8)]
    for name, a, b, nuv0, k in cases:
        ra, rb = np.array(a.rect(), np.float32), np.array(b.rect(), np.float32)
        key = f"{name}/n{nuv0}/k{k}"
        dist[key + "/per_round"] = np.array(
            [R.minimum_distance(a, b, ra, rb, nuv0, 16, k, r) for r in (1, 2, 3, 4)], np.float32)
        r1 = R.dist_round1(a, b, ra, rb, nuv0, k)
        dist[key + "/round1_d2"] = r1["d2"]
        dist[key + "/round1_i"] = r1["i"]
        dist[key + "/round1_j"] = r1["j"]
        dmeta[name] = [digest(a), digest(b)]
    np.savez_compressed(OUT / "ref_distance.npz", **dist)
    (OUT / "ref_distance.json").write_text(json.dumps(dmeta, indent=1))
    print(f"distance done {time.time() - t0:.1f}s")

    # --- synthetic intersection (saddle / plane, rational) ----------------
    syn = {}
    C, D, _ = synth.intersection_pair_saddle_plane()
    rc, rd = np.array(C.rect(), np.float32), np.array(D.rect(), np.float32)
    # nuv0 = 256 is the configuration's full size (4.2e9 first-round box tests).
    for nuv0 in (16, 32, 256):
        for use_k in (1, 0):
            res = R.intersection(C, D, rc, rd, nuv0, 16, use_k)
            syn[f"n{nuv0}/k{use_k}/counts"] = res["counts"]
            if res["pads"]:
                syn[f"n{nuv0}/k{use_k}/pads"] = np.array(res["pads"], np.float32)
    np.savez_compressed(OUT / "ref_inter_synth.npz", **syn)
    (OUT / "ref_inter_synth.json").write_text(json.dumps({"saddle_plane": [digest(C), digest(D)]}, indent=1))
    print(f"synthetic intersection done {time.time() - t0:.1f}s")

    if full:
        t1 = time.time()
        ra, rb = np.array(HA.rect(), np.float32), np.array(HB.rect(), np.float32)
        v = R.minimum_distance(HA, HB, ra, rb, 512, 16, 8, 4)
        el = time.time() - t1
        (OUT / "ref_full.json").write_text(json.dumps({
            "hardwave_n512_k8": {"value": float(v), "value_bits": int(np.float32(v).view(np.uint32)),
                                 "seconds": el, "digests": [digest(HA), digest(HB)]}}, indent=1))
        print(f"full-size hard-wave distance {v!r} in {el:.1f}s")


if __name__ == "__main__":
    main(full="--full" in sys.argv)
