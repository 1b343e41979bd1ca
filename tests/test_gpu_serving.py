"""Worker lanes, batches and queued queries: each result is bit-identical to
the same query run alone, whatever runs beside it on the device."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import load_npz, rect32, surface_from
from jsi_cad_next_versions_b200 import synth

pytestmark = pytest.mark.gpu


def _mixed_distance_queries(ctx):
    out = []
    A, B, _ = synth.distance_pair_sine()
    out.append((A, B, 64))
    HA, HB, _ = synth.distance_pair_hard_wave()
    out.append((HA, HB, 128))
    rng = synth.SplitMix64(77)
    for q in range(6):
        out.append((synth.random_surface(rng), synth.random_surface(rng), 20 + 7 * q))
    tasks = []
    for a, b, nuv in out:
        sa, sb = ctx.upload(a), ctx.upload(b)
        tasks.append((ctx.task(sa, rect32(a), nuv, 1), ctx.task(sb, rect32(b), nuv, 2), sa, sb))
    return tasks


@pytest.mark.parametrize("precision", ["v5_fp32", "fp64", "fp32_screen"])
def test_batch_results_equal_single_results(precision):
    import jsi_cad_next_versions_b200 as J
    with J.Context(0) as ctx:
        tasks = _mixed_distance_queries(ctx)
        alone = [ctx.min_distance(ta, tb, k=8, precision=precision, trace=True) for ta, tb, _, _ in tasks]
        ctx.workers(4)
        batch, ms = ctx.min_distance_batch([(ta, tb) for ta, tb, _, _ in tasks] * 2, k=8, precision=precision,
                                           trace=True)
        assert ms > 0
        for q, r in enumerate(batch):
            a = alone[q % len(alone)]
            assert np.array_equal(r.kth_d2, a.kth_d2)
            for rr in range(a.rounds):
                assert np.array_equal(r.pairs[rr], a.pairs[rr])
        ctx.workers(0)


def test_queued_mix_of_distance_and_intersection():
    """Continuous submission: distance and intersection queries interleaved on
    3 lanes; every result equals the one computed alone."""
    import jsi_cad_next_versions_b200 as J
    g = load_npz("ref_intersection.npz")
    with J.Context(0) as ctx:
        dtasks = _mixed_distance_queries(ctx)
        C3 = surface_from(g["case3/ivec1"], g["case3/data1"])
        D3 = surface_from(g["case3/ivec2"], g["case3/data2"])
        sc, sd = ctx.upload(C3), ctx.upload(D3)
        itask = (ctx.task(sc, rect32(C3), 16, 1), ctx.task(sd, rect32(D3), 16, 2))
        alone_d = [ctx.min_distance(ta, tb, precision="fp64", trace=True) for ta, tb, _, _ in dtasks]
        alone_i = ctx.intersect(*itask, trace=True)
        ctx.workers(3)
        tickets = []
        for q, (ta, tb, _, _) in enumerate(dtasks):
            tickets.append(("d", q, ctx.submit_distance(ta, tb, precision="fp64", trace=True)))
            if q % 3 == 0:
                tickets.append(("i", q, ctx.submit_intersect(*itask, trace=True)))
        for kind, q, t in tickets:
            r = ctx.wait(t)
            if kind == "d":
                assert np.array_equal(r.kth_d2, alone_d[q].kth_d2)
                for rr in range(r.rounds):
                    assert np.array_equal(r.pairs[rr], alone_d[q].pairs[rr])
            else:
                assert np.array_equal(r.counts, alone_i.counts)
                for rr in range(r.rounds):
                    assert np.array_equal(r.pairs[rr], alone_i.pairs[rr])
        assert ctx.queue_depth() == (0, 0)
        ctx.workers(0)
