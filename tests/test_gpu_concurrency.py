"""Host-side concurrency of the worker lanes.

* The caller's thread turns per-kernel timing on and off and reads its
  totals while the lanes run queries (the lanes write the same timing state;
  it is guarded by a per-lane mutex).
* Lockstep batches replayed as CUDA graphs: a graph is keyed by everything
  its launches depend on, including the degrees and rational flags of the
  batch, so a batch of another shape with the same sizes never replays it.

Every result must equal the same query run alone (tolerance zero)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rect32
from jsi_cad_next_versions_b200 import synth

pytestmark = pytest.mark.gpu


def _bicubic(seed, rational):
    rng = synth.SplitMix64(seed)
    n = 12
    X, Y = np.meshgrid(np.linspace(0, 1, n), np.linspace(0, 1, n))
    Z = 0.1 * np.sin(2 * np.pi * (X + rng.uniform())) * np.cos(2 * np.pi * (Y + rng.uniform()))
    W = rng.uniform(n * n, 0.5, 2.0).reshape(n, n) if rational else None
    return synth.make_surface(np.stack([X, Y, Z], -1), 3, 3, weights=W)


def test_timing_toggled_while_lanes_run():
    import jsi_cad_next_versions_b200 as J
    with J.Context(0) as ctx:
        ctx.workers(3)
        rng = synth.SplitMix64(71)
        pairs = [(synth.random_surface(rng), synth.random_surface(rng)) for _ in range(24)]
        ids = [(ctx.upload(A), ctx.upload(B)) for A, B in pairs]
        tasks = [(ctx.task(a, rect32(A), 36, 1), ctx.task(b, rect32(B), 36, 2)) for (a, b), (A, B) in zip(ids, pairs)]
        tickets = []
        for q, (ta, tb) in enumerate(tasks):
            if q % 3 == 2:
                tickets.append(("i", ctx.submit_intersect(ta, tb, precision="fp64")))
            else:
                tickets.append(("d", ctx.submit_distance(ta, tb, precision="fp64")))
        for it in range(60):
            ctx.kernel_timing(it % 2 == 0)
            ctx.kernel_times()
        ctx.kernel_timing(False)
        got = [ctx.wait(t) for _, t in tickets]
        for (kind, _), (ta, tb), r in zip(tickets, tasks, got):
            if kind == "d":
                alone = ctx.min_distance(ta, tb, precision="fp64")
                assert np.array_equal(r.kth_d2.view(np.uint64), alone.kth_d2.view(np.uint64))
            else:
                alone = ctx.intersect(ta, tb, precision="fp64")
                assert np.array_equal(r.counts, alone.counts)


def test_graph_replay_keyed_by_shape():
    import jsi_cad_next_versions_b200 as J
    with J.Context(0) as ctx:
        ctx.workers(1)
        ctx.batch_chunk(8)
        ctx.batch_graphs(True)
        groups = []
        for rational in (False, True):
            pairs = [(_bicubic(100 + 2 * q + 10 * rational, rational), _bicubic(101 + 2 * q + 10 * rational, rational))
                     for q in range(8)]
            ids = [(ctx.upload(A), ctx.upload(B)) for A, B in pairs]
            groups.append([(ctx.task(a, rect32(A), 40, 1), ctx.task(b, rect32(B), 40, 2))
                           for (a, b), (A, B) in zip(ids, pairs)])
        for tasks in groups:
            # first run eager, second captured, third replayed
            for _ in range(3):
                res, _ = ctx.min_distance_batch(tasks, precision="fp64", trace=True)
            for q, (ta, tb) in enumerate(tasks):
                alone = ctx.min_distance(ta, tb, precision="fp64", trace=True)
                assert np.array_equal(res[q].kth_d2.view(np.uint64), alone.kth_d2.view(np.uint64))
        assert ctx.batch_graphs() >= 2
