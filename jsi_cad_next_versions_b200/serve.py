"""Serving loop over the library's worker lanes.

* ``SurfaceCache``  keeps surfaces resident on the device, addressed by id.
* ``ServingLoop``   takes a stream of timestamped queries (surface ids, kind,
                    first-round nuv), admits them in arrival order while their
                    memory estimate fits the budget beside the queries in
                    flight, batches the admitted distance queries over a short
                    window into lockstep batches (``jsi_submit_distance_batch``)
                    and hands intersections to the C++ worker pool
                    (``jsi_submit_intersect``): queries that arrive while
                    others run on the GPU are batched and started as they come,
                    and their kernels overlap on the device (continuous
                    batching).  Latency is arrival to completion.
* ``poisson_queries`` builds a seeded arrival stream.

    python -m jsi_cad_next_versions_b200.serve --surfaces 10000 --queries 4000 \\
        --rates 1000,10000,100000 --forms fp32_screen,fp64

prints one JSON line per (form, rate): throughput, p50/p99 latency, admitted
memory peak.  The reference has no serving layer (its API runs one query at a
time and keeps mutable file statics, intersection.cu:36-39).
"""
from __future__ import annotations

import argparse
import json
import math
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np

from . import synth


@dataclass
class Query:
    kind: str          # "distance" or "intersection"
    a: int             # surface ids in the cache
    b: int
    nuv0: int
    arrival: float     # seconds from the start of the stream
    result: object = None
    latency: float = float("nan")
    status: str = "pending"


def query_bytes(kind: str, nuv0: int) -> int:
    """Device memory estimate of one query (arena high-water mark): round-1
    samples, cells and tile lists of both sides in FP64 plus refinement rounds;
    intersection queries also hold per-round pair lists."""
    base = 2 * nuv0 * nuv0 * 32 * 3 + (8 << 20)
    return base if kind == "distance" else 4 * base + (64 << 20)


class SurfaceCache:
    """Surfaces resident on the device, addressed by cache index."""

    def __init__(self, ctx):
        self.ctx = ctx
        self.ids: list[int] = []
        self.rects: list[np.ndarray] = []

    def add(self, surf) -> int:
        self.ids.append(self.ctx.upload(surf))
        self.rects.append(np.array(surf.rect(), np.float32))
        return len(self.ids) - 1

    def add_many(self, surfs) -> None:
        self.ids.extend(self.ctx.upload_many(surfs))
        self.rects.extend(np.array(s.rect(), np.float32) for s in surfs)

    def __len__(self):
        return len(self.ids)

    def task(self, idx: int, nuv: int, side: int):
        return self.ctx.task(self.ids[idx], self.rects[idx], nuv, side)

    def release(self):
        for sid in self.ids:
            self.ctx.release(sid)
        self.ids.clear()
        self.rects.clear()


def poisson_queries(n: int, rate: float, n_surfaces: int, seed: int = 11, nuv_lo: int = 64, nuv_hi: int = 512,
                    distance_share: float = 0.5) -> list[Query]:
    """Seeded Poisson arrivals at `rate` queries/s over random surface pairs."""
    rng = synth.SplitMix64(seed)
    t = 0.0
    out = []
    for _ in range(n):
        t += -math.log(1.0 - rng.uniform()) / rate
        a = rng.randint(0, n_surfaces - 1)
        b = rng.randint(0, n_surfaces - 1)
        if b == a:
            b = (a + 1) % n_surfaces
        kind = "distance" if rng.uniform() < distance_share else "intersection"
        out.append(Query(kind, a, b, rng.randint(nuv_lo, nuv_hi), t))
    return out


@dataclass
class ServeStats:
    queries: int
    completed: int
    failed: int
    wall_s: float
    throughput: float
    p50_ms: float
    p99_ms: float
    peak_admitted_bytes: int
    peak_inflight: int
    latencies_ms: list = field(default_factory=list)


class ServingLoop:
    """Admission by memory budget + continuous batching over worker lanes.

    Arrived queries are admitted in arrival order while their memory
    estimate fits the budget beside the queries in flight.  Admitted distance
    queries wait at most ``window_ms`` (or until ``max_batch`` have gathered,
    or until the device would otherwise idle) and are then submitted together
    as one distance batch (``jsi_submit_distance_batch``: lockstep batches
    grouped by first-round nuv, one launch per stage for each group);
    intersection queries are submitted as lane jobs at once.  Queries that
    arrive while others run on the GPU are batched and started as they come,
    and their kernels overlap on the device.  Latency is arrival to the
    moment the loop sees the result."""

    def __init__(self, ctx, cache: SurfaceCache, *, lanes: int = 8, budget_bytes: int = 120 << 30,
                 max_inflight: int | None = None, precision: str = "fp32_screen", k: int = 8,
                 inter_rounds: int = 6, inter_precision: str | None = None, trace: bool = False,
                 window_ms: float = 2.0, max_batch: int = 512, chunk: int = 64):
        self.ctx = ctx
        self.cache = cache
        self.lanes = lanes
        self.budget = budget_bytes
        self.max_inflight = max_inflight or 8192
        self.precision = precision
        # both query kinds run the same form (the intersection's FP32 screen
        # re-checks its candidates in FP64, like the distance screen)
        self.inter_precision = inter_precision or precision
        self.k = k
        self.inter_rounds = inter_rounds
        self.trace = trace
        self.window = window_ms / 1e3
        self.max_batch = max_batch
        self.chunk = chunk

    def _submit_intersection(self, q: Query) -> int:
        ta = self.cache.task(q.a, q.nuv0, 1)
        tb = self.cache.task(q.b, q.nuv0, 2)
        return self.ctx.submit_intersect(ta, tb, rounds=self.inter_rounds, precision=self.inter_precision,
                                         trace=self.trace)

    def _submit_distances(self, qs: list[Query]):
        pairs = [(self.cache.task(q.a, q.nuv0, 1), self.cache.task(q.b, q.nuv0, 2)) for q in qs]
        return self.ctx.submit_distance_batch(pairs, k=self.k, precision=self.precision, trace=self.trace)

    def run(self, queries: list[Query], *, poll_ms: int = 1) -> ServeStats:
        self.ctx.workers(self.lanes)
        self.ctx.batch_chunk(self.chunk)
        pending = deque(queries)
        staged: list[tuple[Query, int, float]] = []     # admitted distance queries, admission time
        batches: list[tuple[dict, list[tuple[Query, int]]]] = []
        inter: dict[int, tuple[Query, int]] = {}
        used = 0
        peak_used = 0
        peak_inflight = 0
        n_batches = 0
        batch_sizes = []
        t0 = time.perf_counter()

        def finish(q: Query, r, need: int):
            nonlocal used
            used -= need
            q.latency = time.perf_counter() - t0 - q.arrival
            if isinstance(r, Exception):
                q.status = f"failed: {r}"
            else:
                q.result = r
                q.status = "ok"

        def inflight() -> int:
            return len(staged) + len(inter) + sum(len(b[1]) for b in batches)

        while pending or staged or batches or inter:
            now = time.perf_counter() - t0
            # admission in arrival order, memory and slots permitting
            while pending and pending[0].arrival <= now and inflight() < self.max_inflight:
                q = pending[0]
                need = query_bytes(q.kind, q.nuv0)
                if used + need > self.budget and inflight():
                    break
                pending.popleft()
                used += need
                peak_used = max(peak_used, used)
                if q.kind == "distance":
                    staged.append((q, need, now))
                    continue
                try:
                    inter[self._submit_intersection(q)] = (q, need)
                except Exception as exc:  # rejected at submission
                    finish(q, exc, need)
            peak_inflight = max(peak_inflight, inflight())
            # the batching window: flush when the oldest staged query has
            # waited window_ms, when max_batch have gathered, or when nothing
            # else is running on the device
            idle = not batches and not inter
            if staged and (now - staged[0][2] >= self.window or len(staged) >= self.max_batch or idle):
                group = staged[:self.max_batch]
                del staged[:len(group)]
                try:
                    h = self._submit_distances([q for q, _, _ in group])
                    batches.append((h, [(q, need) for q, need, _ in group]))
                    n_batches += 1
                    batch_sizes.append(len(group))
                except Exception as exc:
                    for q, need, _ in group:
                        finish(q, exc, need)
            progressed = False
            for entry in list(batches):
                h, members = entry
                if not self.ctx.poll_distance_batch(h):
                    continue
                try:
                    res, _ = self.ctx.wait_distance_batch(h)
                    st = list(h["status"])
                    for e, (q, need) in enumerate(members):
                        finish(q, res[e] if st[e] == 0 else RuntimeError(f"status {st[e]}"), need)
                except Exception as exc:
                    for q, need in members:
                        finish(q, exc, need)
                batches.remove(entry)
                progressed = True
            for t in list(inter):
                try:
                    r = self.ctx.wait(t, 0)
                except Exception as exc:
                    r = exc
                if r is None:
                    continue
                q, need = inter.pop(t)
                finish(q, r, need)
                progressed = True
            if not progressed:
                if pending and not staged and not batches and not inter:
                    time.sleep(max(0.0, min(pending[0].arrival - (time.perf_counter() - t0), 0.001)))
                elif inter and not staged:
                    t = next(iter(inter))
                    try:
                        r = self.ctx.wait(t, poll_ms)
                    except Exception as exc:
                        r = exc
                    if r is not None:
                        q, need = inter.pop(t)
                        finish(q, r, need)
                else:
                    time.sleep(50e-6)
        wall = time.perf_counter() - t0
        self.ctx.workers(0)
        lat = sorted(q.latency * 1e3 for q in queries if q.status == "ok")
        ok = len(lat)

        def pct(p):
            return lat[min(len(lat) - 1, int(p * len(lat)))] if lat else float("nan")
        st = ServeStats(queries=len(queries), completed=ok, failed=len(queries) - ok, wall_s=wall,
                        throughput=ok / wall if wall > 0 else 0.0, p50_ms=pct(0.5), p99_ms=pct(0.99),
                        peak_admitted_bytes=peak_used, peak_inflight=peak_inflight, latencies_ms=lat)
        st.batches = n_batches
        st.mean_batch = float(np.mean(batch_sizes)) if batch_sizes else 0.0
        return st


def build_cache(ctx, n: int, seed: int = 7) -> SurfaceCache:
    """n resident surfaces from the mixed-batch distribution (degrees 2..5,
    nets 4..64 log-uniform, 30% rational, random-phase height fields)."""
    rng = synth.SplitMix64(seed)
    cache = SurfaceCache(ctx)
    for q0 in range(0, n, 1024):
        cache.add_many([synth.random_surface(rng, name=f"cache{q}") for q in range(q0, min(n, q0 + 1024))])
    return cache


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--surfaces", type=int, default=10000)
    ap.add_argument("--queries", type=int, default=2000)
    ap.add_argument("--rates", default="1000,10000,100000")
    ap.add_argument("--forms", default="fp32_screen,fp64")
    ap.add_argument("--lanes", type=int, default=16)
    ap.add_argument("--budget-gb", type=float, default=120.0)
    ap.add_argument("--nuv-lo", type=int, default=64)
    ap.add_argument("--nuv-hi", type=int, default=512)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--window-ms", type=float, default=2.0, help="batching window of the distance queries")
    ap.add_argument("--profile", action="store_true", help="print the per-kernel device time of each run")
    args = ap.parse_args(argv)
    from .api import Context
    with Context(args.device) as ctx:
        t = time.perf_counter()
        cache = build_cache(ctx, args.surfaces)
        load_s = time.perf_counter() - t
        seen: dict[float, dict] = {}
        for form in args.forms.split(","):
            for rate in [float(x) for x in args.rates.split(",")]:
                qs = poisson_queries(args.queries, rate, len(cache), nuv_lo=args.nuv_lo, nuv_hi=args.nuv_hi)
                loop = ServingLoop(ctx, cache, lanes=args.lanes, budget_bytes=int(args.budget_gb * (1 << 30)),
                                   precision=form, window_ms=args.window_ms)
                if args.profile:
                    ctx.kernel_timing(True)
                st = loop.run(qs)
                kt = {}
                if args.profile:
                    kt = {k: round(v[0], 2) for k, v in sorted(ctx.kernel_times().items(), key=lambda kv: -kv[1][0])[:12]}
                    ctx.kernel_timing(False)
                reasons = sorted({q.status for q in qs if q.status != "ok"})[:3]
                # the same stream in another form: distances and overlap counts compared query by query
                rel = None
                prev = seen.get(rate)
                if prev is not None:
                    rel = 0.0
                    for q, o in zip(qs, prev["queries"]):
                        if q.status != "ok" or o.status != "ok":
                            continue
                        if q.kind == "distance":
                            a, b = float(q.result.distance), float(o.result.distance)
                            rel = max(rel, abs(a - b) / max(abs(b), 1e-300))
                        elif not np.array_equal(q.result.counts, o.result.counts):
                            rel = float("inf")
                seen.setdefault(rate, {"form": form, "queries": qs})
                print(json.dumps({
                    "form": form, "offered_rate": rate, "queries": st.queries, "completed": st.completed,
                    "failure_reasons": reasons,
                    "failed": st.failed, "throughput_qps": st.throughput, "p50_ms": st.p50_ms, "p99_ms": st.p99_ms,
                    "distance_batches": st.batches, "mean_batch": st.mean_batch,
                    "max_rel_distance_diff_vs_" + seen[rate]["form"]: rel,
                    "peak_admitted_gb": st.peak_admitted_bytes / (1 << 30), "peak_inflight": st.peak_inflight,
                    "lanes": args.lanes, "window_ms": args.window_ms, "resident_surfaces": len(cache),
                    "resident_mb": ctx.resident_bytes() / 2**20,
                    "cache_load_s": load_s, "nuv0_range": [args.nuv_lo, args.nuv_hi],
                    **({"kernel_ms": kt} if kt else {})}), flush=True)
        cache.release()


if __name__ == "__main__":
    main()
