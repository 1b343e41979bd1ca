"""Mixed batches: queries of different degrees, rational flags and kinds in
one call must give, query by query, exactly what the same query gives alone
(jsi_min_distance / jsi_intersect).  Tolerance: zero (the batched kernels
run the same arithmetic on the same inputs)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rect32
from jsi_cad_next_versions_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lanes_ctx():
    import jsi_cad_next_versions_b200 as J
    ctx = J.Context(0)
    ctx.workers(3)
    ctx.batch_chunk(16)
    yield ctx
    ctx.close()


def _random_pairs(seed, n):
    rng = synth.SplitMix64(seed)
    return [(synth.random_surface(rng), synth.random_surface(rng)) for _ in range(n)]


@pytest.mark.parametrize("precision", ["v5_fp32", "fp64", "fp32_screen"])
def test_mixed_shape_lockstep_batch_equals_alone(lanes_ctx, precision):
    """Degrees 2-5 and rational flags differ inside each lockstep batch (one
    first-round nuv): the batch runs the mixed cell build."""
    ctx = lanes_ctx
    pairs = _random_pairs(61, 40)
    ids = [(ctx.upload(A), ctx.upload(B)) for A, B in pairs]
    tasks = [(ctx.task(a, rect32(A), 72, 1), ctx.task(b, rect32(B), 72, 2)) for (a, b), (A, B) in zip(ids, pairs)]
    try:
        res, _ = ctx.min_distance_batch(tasks, k=8, rounds=4, precision=precision, trace=True, newton=True)
        assert len({(int(A.ivec[1]), int(A.ivec[4]), A.rational) for A, _ in pairs}) > 4  # really mixed
        for q, (ta, tb) in enumerate(tasks):
            alone = ctx.min_distance(ta, tb, k=8, rounds=4, precision=precision, trace=True, newton=True)
            got = res[q]
            assert np.array_equal(got.kth_d2.view(np.uint64), alone.kth_d2.view(np.uint64)), q
            for r in range(alone.rounds):
                assert np.array_equal(got.pairs[r], alone.pairs[r]), (q, r)
            assert got.newton_distance == alone.newton_distance, q
    finally:
        for a, b in ids:
            ctx.release(a)
            ctx.release(b)


@pytest.mark.parametrize("precision", ["fp64", "fp32_screen"])
def test_query_batch_equals_alone(lanes_ctx, precision):
    """The mixed configuration's generator (degrees 2-5, nets 4-64, 30%
    rational, half distance and half intersection), first-round nuv scaled to
    16-63 so that the alone runs stay short."""
    ctx = lanes_ctx
    batch = synth.mixed_batch(48, seed=11)
    ids = [(ctx.upload(a), ctx.upload(b)) for a, b, _ in batch]
    queries = []
    for (sa, sb), (a, b, m) in zip(ids, batch):
        nuv0 = 16 + m["nuv0"] % 48
        queries.append((m["kind"], ctx.task(sa, rect32(a), nuv0, 1), ctx.task(sb, rect32(b), nuv0, 2)))
    try:
        cap = 1 << 16
        res, status, ms = ctx.query_batch(queries, precision=precision, newton=True, points=True, trace=True,
                                          points_cap=cap, trace_cap=1 << 22)
        assert all(s == 0 for s in status)
        assert ms > 0
        for q, (kind, ta, tb) in enumerate(queries):
            if kind == "distance":
                alone = ctx.min_distance(ta, tb, k=8, rounds=4, precision=precision, newton=True)
                assert np.array_equal(res[q].kth_d2.view(np.uint64), alone.kth_d2.view(np.uint64)), q
                assert res[q].newton_distance == alone.newton_distance, q
            else:
                alone = ctx.intersect(ta, tb, precision=precision, points=True, trace=True)
                assert np.array_equal(res[q].counts, alone.counts), q
                for r in range(alone.rounds):
                    # a round beyond a trace buffer's capacity is not traced
                    # (the batch's buffers are smaller than the alone run's)
                    if res[q].pairs[r] is not None:
                        assert np.array_equal(res[q].pairs[r], alone.pairs[r]), (q, r)
                m = min(cap, alone.points.shape[0])
                assert res[q].points.shape[0] == m, q
                assert np.array_equal(res[q].points.view(np.uint64), alone.points[:m].view(np.uint64)), q
    finally:
        for a, b in ids:
            ctx.release(a)
            ctx.release(b)
