"""The oracle against the reference itself (oracle/_ref, compiled from the
reference sources), on inputs too large for committed fixtures: the
reference's own degree-11 intersection inputs inter_case1/2."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rect32, surface_from


@pytest.mark.parametrize("case", [1, 2])
@pytest.mark.parametrize("use_k", [1, 0])
def test_reference_degree11_intersection_counts(ref, orc, case, use_k):
    ia, da = ref.face(f"inter_case{case}_obj1")
    ib, db = ref.face(f"inter_case{case}_obj2")
    A, B = surface_from(ia, da), surface_from(ib, db)
    exp = ref.intersection(A, B, rect32(A), rect32(B), 16, 16, use_k)["counts"]
    got = orc.inter_query(A, B, rect32(A), rect32(B), 16, 16, use_k, pair_cap=1 << 10)["counts"]
    assert np.array_equal(got, exp)


def test_reference_round1_distance_pairs_random(ref, orc):
    from jsi_cad_next_versions_b200 import synth
    rng = synth.SplitMix64(5)
    for _ in range(3):
        A, B = synth.random_surface(rng), synth.random_surface(rng)
        r = ref.dist_round1(A, B, rect32(A), rect32(B), 24, 16)
        o = orc.dist_query(A, B, rect32(A), rect32(B), 24, 16, 16, 1)
        assert np.array_equal(o["pairs"][0][:, 1], r["i"]) and np.array_equal(o["pairs"][0][:, 2], r["j"])
        assert np.array_equal(o["kth_d2"][:1], r["d2"][-1:])
