"""Lockstep batches of distance queries (one launch per stage for a whole
batch of same-shape queries): every result equals the same query run alone
on the per-query path, bit for bit, including the per-round kept pairs, the
Newton refinement and queries that overflow a batch list and are re-run."""
from __future__ import annotations

import os

import numpy as np
import pytest

from conftest import rect32
from jsi_cad_next_versions_b200 import synth

pytestmark = pytest.mark.gpu

PRECISIONS = ["v5_fp32", "fp64", "fp32_screen"]


def _upload_pairs(ctx, pairs, nuv):
    tasks = []
    for a, b in pairs:
        sa, sb = ctx.upload(a), ctx.upload(b)
        tasks.append((ctx.task(sa, rect32(a), nuv, 1), ctx.task(sb, rect32(b), nuv, 2)))
    return tasks


def _hard_wave_pairs(n, seed0=100):
    return [synth.distance_pair_hard_wave(seed_a=seed0 + 2 * q, seed_b=seed0 + 2 * q + 1)[:2] for q in range(n)]


def _sine_pairs(n, seed0=200):
    return [synth.distance_pair_sine(seed_a=seed0 + 2 * q, seed_b=seed0 + 2 * q + 1)[:2] for q in range(n)]


def _same(r, a, newton=False):
    """Equal results (pair-test and candidate counts may differ: they depend
    on the order the screen visits tile pairs in)."""
    assert r.rounds == a.rounds
    assert np.array_equal(r.npairs, a.npairs)
    assert np.array_equal(r.kth_d2, a.kth_d2)
    for rr in range(a.rounds):
        assert np.array_equal(r.pairs[rr], a.pairs[rr])
    assert r.v5_value == a.v5_value
    assert r.distance == a.distance
    if newton:
        assert r.newton_distance == a.newton_distance
        assert r.uv1 == a.uv1 and r.uv2 == a.uv2


def _check_batch(ctx, tasks, *, k=8, rounds=4, precision="fp64", newton=False, lanes=2):
    alone = [ctx.min_distance(ta, tb, k=k, rounds=rounds, precision=precision, newton=newton, trace=True)
             for ta, tb in tasks]
    ctx.workers(lanes)
    try:
        batch, ms = ctx.min_distance_batch(tasks, k=k, rounds=rounds, precision=precision, newton=newton,
                                           trace=True)
    finally:
        ctx.workers(0)
    assert ms > 0
    for r, a in zip(batch, alone):
        _same(r, a, newton)
    return batch


@pytest.mark.parametrize("precision", PRECISIONS)
def test_batch_supertile_round(precision):
    """nuv0 = 128: 16 x 16 tiles per side, the two-level (supertile) screen."""
    import jsi_cad_next_versions_b200 as J
    with J.Context(0) as ctx:
        tasks = _upload_pairs(ctx, _hard_wave_pairs(10), 128)
        _check_batch(ctx, tasks, precision=precision)


@pytest.mark.parametrize("precision", PRECISIONS)
@pytest.mark.parametrize("k,rounds", [(8, 4), (3, 2), (1, 5)])
def test_batch_single_level_round(precision, k, rounds):
    """nuv0 = 64: 8 x 8 tiles per side, tile pairs screened directly."""
    import jsi_cad_next_versions_b200 as J
    with J.Context(0) as ctx:
        tasks = _upload_pairs(ctx, _sine_pairs(9), 64)
        _check_batch(ctx, tasks, k=k, rounds=rounds, precision=precision, lanes=1)


@pytest.mark.parametrize("precision", ["fp64", "fp32_screen"])
def test_batch_newton(precision):
    import jsi_cad_next_versions_b200 as J
    with J.Context(0) as ctx:
        tasks = _upload_pairs(ctx, _sine_pairs(6, seed0=300), 48)
        _check_batch(ctx, tasks, precision=precision, newton=True)


def test_batch_mixed_shapes_grouped():
    """Queries of several shapes in one call: grouped per shape, results in
    the caller's order."""
    import jsi_cad_next_versions_b200 as J
    rng = synth.SplitMix64(91)
    with J.Context(0) as ctx:
        tasks = []
        for q in range(12):
            if q % 3 == 0:
                a, b = synth.distance_pair_sine(seed_a=400 + q, seed_b=500 + q)[:2]
                nuv = 64
            elif q % 3 == 1:
                a, b = synth.random_surface(rng), synth.random_surface(rng)
                nuv = 33
            else:
                a, b = synth.distance_pair_hard_wave(seed_a=600 + q, seed_b=700 + q)[:2]
                nuv = 96
            tasks += _upload_pairs(ctx, [(a, b)], nuv)
        _check_batch(ctx, tasks, precision="fp64", lanes=3)


def test_batch_chunk_zero_runs_per_query():
    import jsi_cad_next_versions_b200 as J
    with J.Context(0) as ctx:
        tasks = _upload_pairs(ctx, _sine_pairs(5, seed0=800), 40)
        ctx.workers(2)
        try:
            lock, _ = ctx.min_distance_batch(tasks, precision="fp32_screen", trace=True)
            ctx.batch_chunk(0)
            solo, _ = ctx.min_distance_batch(tasks, precision="fp32_screen", trace=True)
        finally:
            ctx.workers(0)
        for r, a in zip(lock, solo):
            _same(r, a)


@pytest.mark.parametrize("env", ["JSI_BATCH_CAND_CAP", "JSI_BATCH_SURV_CAP"])
def test_batch_overflow_reruns_alone(env):
    """A one-entry list overflows in every query (k = 8 needs at least 8
    candidates, and round 1 keeps more than one tile pair): each query is
    flagged in its record and re-run alone, with the same results."""
    import jsi_cad_next_versions_b200 as J
    os.environ[env] = "1"
    try:
        with J.Context(0) as ctx:
            tasks = _upload_pairs(ctx, _hard_wave_pairs(4, seed0=900), 128)
            _check_batch(ctx, tasks, precision="fp32_screen", lanes=1)
    finally:
        del os.environ[env]


def test_batch_overflow_counter():
    import jsi_cad_next_versions_b200 as J
    os.environ["JSI_BATCH_CAND_CAP"] = "1"
    try:
        with J.Context(0) as ctx:
            tasks = _upload_pairs(ctx, _hard_wave_pairs(3, seed0=950), 128)
            ctx.workers(1)
            try:
                ctx.min_distance_batch(tasks, precision="fp64")
                assert ctx.batch_reruns() == len(tasks)
            finally:
                ctx.workers(0)
    finally:
        del os.environ["JSI_BATCH_CAND_CAP"]


def test_batch_full_size_screen():
    """The headline shape (hard-wave pair, nuv0 = 512) in one batch of 6."""
    import jsi_cad_next_versions_b200 as J
    with J.Context(0) as ctx:
        tasks = _upload_pairs(ctx, _hard_wave_pairs(6, seed0=1000), 512)
        batch = _check_batch(ctx, tasks, precision="fp32_screen", lanes=1)
        assert all(r.rounds == 4 for r in batch)


def test_bulk_domains_tasks_release():
    """surface_domains gives each surface's get_ubegin/get_vbegin/get_uend/
    get_vend; TaskBatch.from_arrays over them gives the same batch results as
    tasks built one by one (vectorised fields agree with the per-query
    records); release_many returns every block."""
    import jsi_cad_next_versions_b200 as J
    pairs = _sine_pairs(6, seed0=1300)
    flat = [x for pr in pairs for x in pr]
    with J.Context(0) as ctx:
        base = ctx.resident_bytes()
        ids = np.asarray(ctx.upload_many(flat), np.int32)
        dom = ctx.surface_domains(ids)
        assert np.array_equal(dom, np.stack([rect32(s) for s in flat]))
        one = [(ctx.task(int(ids[2 * q]), rect32(A), 48, 1), ctx.task(int(ids[2 * q + 1]), rect32(B), 48, 2))
               for q, (A, B) in enumerate(pairs)]
        packed = J.TaskBatch.from_arrays(ids[0::2], dom[0::2], 48, ids[1::2], dom[1::2], 48)
        ctx.workers(2)
        try:
            r1, _ = ctx.min_distance_batch(one, precision="fp64", trace=True)
            r2, _ = ctx.min_distance_batch(packed, precision="fp64", trace=True)
        finally:
            ctx.workers(0)
        for a, b in zip(r1, r2):
            _same(b, a)
        assert np.array_equal(r2.distance, np.array([r.distance for r in r2]))
        assert np.array_equal(r2.rounds, np.array([r.rounds for r in r2]))
        ctx.release_many(ids)
        assert ctx.resident_bytes() == base
        with pytest.raises(J.JsiError):
            ctx.surface_domains(ids[:1])


def test_packed_surface_set_uploads_in_chunks():
    """A SurfaceBatch uploaded in two slices gives the same domains and the
    same batch results as the surfaces uploaded one list at a time."""
    import jsi_cad_next_versions_b200 as J
    pairs = _hard_wave_pairs(3, seed0=1800) + _sine_pairs(3, seed0=1900)
    flat = [x for pr in pairs for x in pr]
    hostset = J.SurfaceBatch(flat)
    with J.Context(0) as ctx:
        base = ctx.resident_bytes()
        ids = np.asarray(ctx.upload_many(hostset[0:6]) + ctx.upload_many(hostset[6:12]), np.int32)
        ref_ids = np.asarray(ctx.upload_many(flat), np.int32)
        dom = ctx.surface_domains(ids)
        assert np.array_equal(dom, ctx.surface_domains(ref_ids))
        ctx.workers(2)
        try:
            for sl, nuv in ((slice(0, 3), 144), (slice(3, 6), 40)):
                got_ids, want_ids = ids.reshape(-1, 2)[sl], ref_ids.reshape(-1, 2)[sl]
                d = dom.reshape(-1, 2, 4)[sl]
                tb = J.TaskBatch.from_arrays(got_ids[:, 0], d[:, 0], nuv, got_ids[:, 1], d[:, 1], nuv)
                tr = J.TaskBatch.from_arrays(want_ids[:, 0], d[:, 0], nuv, want_ids[:, 1], d[:, 1], nuv)
                got, _ = ctx.min_distance_batch(tb, precision="fp32_screen", trace=True)
                want, _ = ctx.min_distance_batch(tr, precision="fp32_screen", trace=True)
                for a, b in zip(want, got):
                    _same(b, a)
        finally:
            ctx.workers(0)
        ctx.release_many(ids)
        ctx.release_many(ref_ids)
        assert ctx.resident_bytes() == base


def test_pinned_surface_set_uploads_by_dma():
    """A SurfaceBatch in the context's page-locked memory (uploaded by DMA
    straight from it, spanning several staging segments) gives the same
    resident surfaces as the same set in ordinary memory: same domains and
    the same batch results.  A slice taken out of order (records not in
    increasing address order) goes through the staged path."""
    import jsi_cad_next_versions_b200 as J
    pairs = _hard_wave_pairs(100, seed0=2100)  # 200 records x ~49 KB: more than one 8 MB segment
    flat = [x for pr in pairs for x in pr]
    with J.Context(0) as ctx:
        pinned = J.SurfaceBatch(flat, alloc=ctx.host_array)
        plain = J.SurfaceBatch(flat)
        ids = np.asarray(ctx.upload_many(pinned), np.int32)
        ref_ids = np.asarray(ctx.upload_many(plain), np.int32)
        dom = ctx.surface_domains(ids)
        assert np.array_equal(dom, ctx.surface_domains(ref_ids))
        # a slice of the same block again (a second DMA from it)
        ids2 = np.asarray(ctx.upload_many(pinned[10:30]), np.int32)
        assert np.array_equal(ctx.surface_domains(ids2), dom[10:30])
        # records of the pinned block in decreasing address order: staged path
        from types import SimpleNamespace
        rev = [SimpleNamespace(ivec=pinned.surface(q)[0], data=pinned.surface(q)[1]) for q in range(9, -1, -1)]
        ids3 = np.asarray(ctx.upload_many(rev), np.int32)
        assert np.array_equal(ctx.surface_domains(ids3), dom[9::-1])
        ctx.workers(2)
        try:
            sl = slice(0, 16)
            got_ids, want_ids = ids.reshape(-1, 2)[sl], ref_ids.reshape(-1, 2)[sl]
            d = dom.reshape(-1, 2, 4)[sl]
            tb = J.TaskBatch.from_arrays(got_ids[:, 0], d[:, 0], 160, got_ids[:, 1], d[:, 1], 160)
            tr = J.TaskBatch.from_arrays(want_ids[:, 0], d[:, 0], 160, want_ids[:, 1], d[:, 1], 160)
            for form in ("fp32_screen", "v5_fp32"):
                got, _ = ctx.min_distance_batch(tb, precision=form, trace=True)
                want, _ = ctx.min_distance_batch(tr, precision=form, trace=True)
                for a, b in zip(want, got):
                    _same(b, a)
        finally:
            ctx.workers(0)
        ctx.release_many(ids)
        ctx.release_many(ids2)
        ctx.release_many(ids3)
        ctx.release_many(ref_ids)
        ctx.host_free(pinned.data)


def test_submit_wait_overlapping_batches():
    """Two batches in flight: the second's surfaces are uploaded after the
    first is submitted; each equals the same batch run synchronously."""
    import jsi_cad_next_versions_b200 as J
    first, second = _sine_pairs(5, seed0=1400), _hard_wave_pairs(3, seed0=1500)
    with J.Context(0) as ctx:
        ctx.workers(2)
        try:
            h = []
            for pairs, nuv in ((first, 40), (second, 144)):
                ids = np.asarray(ctx.upload_many([x for pr in pairs for x in pr]), np.int32)
                dom = ctx.surface_domains(ids)
                tb = J.TaskBatch.from_arrays(ids[0::2], dom[0::2], nuv, ids[1::2], dom[1::2], nuv)
                h.append((tb, ctx.submit_distance_batch(tb, precision="fp32_screen", trace=True)))
            got = [ctx.wait_distance_batch(x)[0] for _, x in reversed(h)][::-1]
            for (tb, _), g in zip(h, got):
                ref, _ = ctx.min_distance_batch(tb, precision="fp32_screen", trace=True)
                for a, b in zip(ref, g):
                    _same(b, a)
            with pytest.raises(J.JsiError):
                ctx.wait_distance_batch(h[0][1])  # already waited for
        finally:
            ctx.workers(0)


def test_three_lanes_with_uploads_alongside():
    """Three worker lanes run submitted batches while the calling thread
    uploads and releases other surfaces (the surface table changes while
    lanes look surfaces up); every batch equals the same batch run alone."""
    import jsi_cad_next_versions_b200 as J
    pairs = _hard_wave_pairs(9, seed0=1600)
    extra = [x for pr in _sine_pairs(24, seed0=1700) for x in pr]
    with J.Context(0) as ctx:
        ids = np.asarray(ctx.upload_many([x for pr in pairs for x in pr]), np.int32)
        dom = ctx.surface_domains(ids)
        tb = J.TaskBatch.from_arrays(ids[0::2], dom[0::2], 144, ids[1::2], dom[1::2], 144)
        ctx.workers(3)
        try:
            ref, _ = ctx.min_distance_batch(tb, precision="fp32_screen", trace=True)
            for _ in range(3):
                h = ctx.submit_distance_batch(tb, precision="fp32_screen", trace=True)
                more = ctx.upload_many(extra)
                ctx.release_many(more)
                got, _ = ctx.wait_distance_batch(h)
                for a, b in zip(ref, got):
                    _same(b, a)
        finally:
            ctx.workers(0)


def test_upload_many_release_reuse():
    """Surfaces uploaded in one call, released, and other surfaces uploaded
    into the recycled device blocks: every query sees its own surfaces."""
    import jsi_cad_next_versions_b200 as J
    with J.Context(0) as ctx:
        first = _hard_wave_pairs(4, seed0=1100)
        second = _sine_pairs(4, seed0=1200)
        ids = ctx.upload_many([x for pr in first for x in pr])
        t1 = [(ctx.task(a, rect32(A), 96, 1), ctx.task(b, rect32(B), 96, 2))
              for (a, b), (A, B) in zip(zip(ids[0::2], ids[1::2]), first)]
        r1 = [ctx.min_distance(ta, tb, precision="fp64") for ta, tb in t1]
        for sid in ids:
            ctx.release(sid)
        ids2 = ctx.upload_many([x for pr in second for x in pr])
        t2 = [(ctx.task(a, rect32(A), 40, 1), ctx.task(b, rect32(B), 40, 2))
              for (a, b), (A, B) in zip(zip(ids2[0::2], ids2[1::2]), second)]
        ctx.workers(2)
        try:
            batch, _ = ctx.min_distance_batch(t2, precision="fp64")
        finally:
            ctx.workers(0)
        # reference values from a fresh context
        with J.Context(0) as c2:
            for (A, B), r in zip(second, batch):
                ta = c2.task(c2.upload(A), rect32(A), 40, 1)
                tb = c2.task(c2.upload(B), rect32(B), 40, 2)
                assert c2.min_distance(ta, tb, precision="fp64").distance == r.distance
        with J.Context(0) as c3:
            for (A, B), r in zip(first, r1):
                ta = c3.task(c3.upload(A), rect32(A), 96, 1)
                tb = c3.task(c3.upload(B), rect32(B), 96, 2)
                assert c3.min_distance(ta, tb, precision="fp64").distance == r.distance


@pytest.mark.parametrize("precision", ["fp32_screen", "fp64"])
def test_batch_graph_replay(precision):
    """A repeated batch is captured as a CUDA graph on its second run and
    replayed from the third on: the replays give the eager results."""
    import jsi_cad_next_versions_b200 as J
    with J.Context(0) as ctx:
        tasks = _upload_pairs(ctx, _hard_wave_pairs(6, seed0=1300), 128)
        ctx.workers(1)
        try:
            ctx.batch_graphs(False)
            eager, _ = ctx.min_distance_batch(tasks, precision=precision, trace=True, newton=True)
            ctx.batch_graphs(True)
            runs = [ctx.min_distance_batch(tasks, precision=precision, trace=True, newton=True)[0] for _ in range(4)]
            replays = ctx.batch_graphs()
        finally:
            ctx.workers(0)
        assert replays >= 2
        for res in runs:
            for r, a in zip(res, eager):
                _same(r, a, newton=True)


def test_autotune_batch():
    """The autotuner picks a chunk among its candidates for the shape and
    later batches of that shape use it; results do not change."""
    import jsi_cad_next_versions_b200 as J
    with J.Context(0) as ctx:
        tasks = _upload_pairs(ctx, _hard_wave_pairs(24, seed0=1400), 128)
        ctx.workers(2)
        try:
            before, _ = ctx.min_distance_batch(tasks, precision="fp32_screen", trace=True)
            chunk, ms = ctx.autotune_batch(tasks, precision="fp32_screen")
            after, _ = ctx.min_distance_batch(tasks, precision="fp32_screen", trace=True)
        finally:
            ctx.workers(0)
        assert chunk in (8, 16) and ms > 0  # 24 queries over 2 lanes: candidates 8 and 16
        for r, a in zip(after, before):
            _same(r, a)
