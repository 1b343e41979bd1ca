"""Serving loop: admission by memory budget and continuous batching.

CPU tests drive the loop with a fake context (no GPU): admission order,
budget and slot limits, failures.  The GPU test serves a Poisson stream of
mixed distance / intersection queries and checks that every result equals the
same query run alone."""
from __future__ import annotations

import time

import numpy as np
import pytest

from jsi_cad_next_versions_b200 import serve


class FakeCtx:
    """Stands in for Context: every query 'runs' for a fixed time after
    submission (a distance batch as one job); wait() returns a marker once
    that time has passed.  Every fail_every-th submitted query fails."""

    def __init__(self, run_s=0.002, fail_every=0):
        self.run_s = run_s
        self.fail_every = fail_every
        self.n = 0
        self.nq = 0
        self.jobs = {}
        self.lanes = 0
        self.order = []      # (kind, task a, task b) in submission order
        self.batch_sizes = []

    def workers(self, n, lane_bytes=0):
        self.lanes = n

    def batch_chunk(self, n):
        pass

    def task(self, sid, rect, nuv, side):
        return (sid, nuv, side)

    def _fails(self):
        self.nq += 1
        return bool(self.fail_every) and self.nq % self.fail_every == 0

    def submit_intersect(self, ta, tb, **kw):
        self.n += 1
        self.jobs[self.n] = (time.perf_counter() + self.run_s, self._fails())
        self.order.append(("intersection", ta, tb))
        return self.n

    def submit_distance_batch(self, pairs, **kw):
        self.n += 1
        fails = []
        for ta, tb in pairs:
            self.order.append(("distance", ta, tb))
            fails.append(self._fails())
        self.jobs[self.n] = (time.perf_counter() + self.run_s, fails)
        self.batch_sizes.append(len(pairs))
        return {"ticket": self.n, "status": [0] * len(pairs)}

    def poll_distance_batch(self, h):
        return time.perf_counter() >= self.jobs[h["ticket"]][0]

    def wait_distance_batch(self, h):
        end, fails = self.jobs.pop(h["ticket"])
        time.sleep(max(0.0, end - time.perf_counter()))
        h["status"] = [-3 if f else 0 for f in fails]
        return [("done", h["ticket"], e) for e in range(len(fails))], 0.0

    def wait(self, t, timeout_ms=-1):
        end, fail = self.jobs[t]
        now = time.perf_counter()
        if now < end:
            if timeout_ms == 0:
                return None
            time.sleep(min(end - now, timeout_ms / 1e3 if timeout_ms > 0 else end - now))
            if time.perf_counter() < end:
                return None
        del self.jobs[t]
        if fail:
            raise RuntimeError("JSI_ERR_NOMEM: arena budget exhausted")
        return ("done", t)


class FakeCache:
    def __init__(self, n):
        self.n = n

    def __len__(self):
        return self.n

    def task(self, idx, nuv, side):
        return (idx, nuv, side)


def test_admission_respects_budget_and_order():
    qs = serve.poisson_queries(200, rate=50000.0, n_surfaces=30, seed=3, nuv_lo=64, nuv_hi=128)
    budget = 3 * serve.query_bytes("intersection", 128)
    ctx = FakeCtx(run_s=0.001)
    loop = serve.ServingLoop(ctx, FakeCache(30), lanes=4, budget_bytes=budget, max_inflight=6)
    st = loop.run(qs)
    assert st.completed == 200 and st.failed == 0
    assert st.peak_admitted_bytes <= budget
    assert st.peak_inflight <= 6
    # each kind is submitted in arrival order (distance queries in batches)
    for kind in ("distance", "intersection"):
        assert [o[1][0] for o in ctx.order if o[0] == kind] == [q.a for q in qs if q.kind == kind]
    assert all(q.latency >= 0 for q in qs)
    assert st.p50_ms <= st.p99_ms


def test_distance_queries_are_batched_over_the_window():
    # 400 queries at 200k/s arrive within about 2 ms: with a 1 ms window the
    # distance queries gather into a few batches instead of one job each
    qs = serve.poisson_queries(400, rate=200000.0, n_surfaces=50, seed=5, nuv_lo=64, nuv_hi=128)
    ctx = FakeCtx(run_s=0.003)
    st = serve.ServingLoop(ctx, FakeCache(50), lanes=4, window_ms=1.0, max_batch=512).run(qs)
    nd = sum(q.kind == "distance" for q in qs)
    assert st.completed == 400
    assert sum(ctx.batch_sizes) == nd
    assert len(ctx.batch_sizes) < nd / 10
    assert st.batches == len(ctx.batch_sizes)


def test_failures_are_reported_not_raised():
    qs = serve.poisson_queries(40, rate=1e5, n_surfaces=10, seed=4)
    st = serve.ServingLoop(FakeCtx(run_s=0.0005, fail_every=5), FakeCache(10), lanes=2).run(qs)
    assert st.failed == 8 and st.completed == 32
    assert sum(q.status.startswith("failed") for q in qs) == 8


def test_poisson_stream_is_seeded():
    a = serve.poisson_queries(50, 1000.0, 20, seed=9)
    b = serve.poisson_queries(50, 1000.0, 20, seed=9)
    assert [(q.kind, q.a, q.b, q.nuv0, q.arrival) for q in a] == [(q.kind, q.a, q.b, q.nuv0, q.arrival) for q in b]
    gaps = np.diff([q.arrival for q in a])
    assert (gaps > 0).all() and abs(gaps.mean() - 1e-3) < 5e-4


@pytest.mark.gpu
def test_served_results_equal_results_alone():
    import jsi_cad_next_versions_b200 as J
    with J.Context(0) as ctx:
        cache = serve.build_cache(ctx, 40, seed=21)
        qs = serve.poisson_queries(120, rate=5000.0, n_surfaces=len(cache), seed=22, nuv_lo=24, nuv_hi=64)
        loop = serve.ServingLoop(ctx, cache, lanes=4, precision="fp32_screen", inter_rounds=4, trace=True)
        st = loop.run(qs)
        assert st.completed == len(qs), [q.status for q in qs if q.status != "ok"][:3]
        for q in qs:
            ta, tb = cache.task(q.a, q.nuv0, 1), cache.task(q.b, q.nuv0, 2)
            if q.kind == "distance":
                alone = ctx.min_distance(ta, tb, k=8, precision="fp32_screen", trace=True)
                assert np.array_equal(q.result.kth_d2, alone.kth_d2)
                for r in range(alone.rounds):
                    assert np.array_equal(q.result.pairs[r], alone.pairs[r])
            else:
                alone = ctx.intersect(ta, tb, rounds=4, precision="fp32_screen", trace=True)
                assert np.array_equal(q.result.counts, alone.counts)
                for r in range(alone.rounds):
                    # traces beyond a buffer's capacity are dropped on either side
                    if alone.pairs[r] is not None and q.result.pairs[r] is not None:
                        assert np.array_equal(q.result.pairs[r], alone.pairs[r])
        assert st.p50_ms <= st.p99_ms
        cache.release()
