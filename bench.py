#!/usr/bin/env python
"""Throughput of the hard-wave minimum-distance query on B200.

Workload (one step = one batch): ``--batch`` hard-wave query pairs, each two
bicubic 64x64 B-spline patches (A: z = 0.05 sin(20 pi x) cos(20 pi y) +
N(0, 1e-3); B: the field phase-shifted by pi, lifted by 0.1; seeded
synthetic surfaces, a distinct seed pair per query), first round nuv = 512,
three refinement rounds at nuv = 16, k = 8: minimum_distance of the reference
(JSI_CAD_NEXT_VERSION5/src/distance_analysis/distance_analysis.cu:356-506).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

* ``value``  queries/s with the surfaces resident in HBM, CUDA events on the
             library's own stream, L2 flushed (256 MiB write) between steps.
* ``e2e``    the same metric through the C ABI with host buffers: upload of
             both surfaces, the query, the result read-back, release.
* ``roofline`` the dominant kernel, its algorithmic work per launch over its
             CUDA-event duration measured in the timed region.
* ``cpu_baseline`` the reference itself (oracle/_ref, built from its sources)
             on this host's cores, one full query.
Multi-GPU: one process per GPU (torchrun); each rank runs its own batch
(independent queries: weak scaling, no data-path collective); the step time is
the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "queries/s + p50/p99 latency: FP32-screen vs plain FP64 on B200 at ≤1e-9 rel err"
WORKLOAD = "hard-wave 64x64 bicubic pair, minimum distance, nuv0=512 + 3 rounds nuv=16, k=8"
NUV0, NUV_REFINE, K, ROUNDS = 512, 16, 8, 4
FORMS = ("fp32_screen", "fp64", "v5_fp32")  # headline form first

# Algorithmic work of the screening kernels, per unit (FMA = 2 flops):
#  dist_leaf: one cell-pair centre distance = 3 sub + 3 mul + 2 add = 8 flops,
#             reading 2 cell centres from shared memory (tile staged once);
#  dist_cull: one tile-pair box bound = 6 sub + 3 max + 3 mul + 2 add = 14 flops,
#             reading 4 Vec4 tile bounds (64 B FP32 / 128 B FP64).
FLOPS_PER_PAIR_TEST = 8

# Algorithmic work per unit of each kernel (jsi_kernel_units), bicubic
# surfaces: (flops, HBM bytes) with FMA = 2 flops; bytes for FP32 cells
# (FP64: x2).  samples: P contraction 2*3*(16+4) = 120 flops, one 16 B sample
# written.  basis: A2.3 for p = 3 with 2 derivatives ~ 100 flops, 3*4 values
# + span written (52 B).  cells: 24 min/max + 12 add/div ~ 36 flops, one
# sample read + one centre written (32 B).  dist_tau / dist_cull: one
# representative distance (8 flops) / one box-gap bound (14 flops) per tile
# pair, tile data L2-resident (0 B).  dist_leaf / inter_leaf: 8 / 9 flops per
# executed cell-pair test, operands in registers (0 B).
# cells_r1: the first round's fused cell build (no sample grid in HBM), per
# cell: the factored bicubic contraction amortised over a band column
# (5 net rows x 4 x 3 FMA per column / 8 cells + 4 x 3 FMA per sample, with
# 9/8 samples per cell) ~ 40 flops, plus 18 min/max + 6 add + 3 halvings for
# the centre and 6 min/max for the tile range ~ 33 flops: 73 flops; HBM: the
# 16 B centre written plus 2 x 16 B tile bounds per 64 cells = 16.5 B.
UNIT_WORK = {"samples": (120, 16), "basis": (100, 52), "cells": (36, 32), "cells_r1": (73, 16.5),
             "dist_tau": (8, 0),
             "dist_cull": (14, 0), "dist_leaf": (8, 0), "dist_head": (8, 0), "inter_cull": (14, 0),
             "inter_leaf": (9, 0)}
# DRAM traffic per unit measured by ncu (dram__bytes_read.sum + dram__bytes_write.sum
# of one launch / its units), for the form it was captured in: the band kernel of
# the FP32 screen over 128 x 511^2 cells wrote and read 516.8 MB, 15.46 B per cell.
MEASURED_TRAFFIC = {("cells_r1", "fp32_screen"): 15.46}
# What one timed "launch" of a kernel name covers.
LAUNCH_NOTE = {"cells_r1": "the first round's cell build of one batch: one k_cells_bandw launch per side, "
                           "back to back on one stream, timed together"}
NOMINAL_FP32_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12   # 74.4: 148 SMs x 128 lanes x FMA x 1.965 GHz
NOMINAL_FP64_TFLOPS = NOMINAL_FP32_TFLOPS / 2


def roofline(kernel, kt, form, peaks):
    """Roofline record of the dominant kernel from its live CUDA-event time and
    its work units; HBM bound against the measured copy bandwidth, plus the
    CUDA-core bound against the nominal FP32/FP64 peak."""
    ms, launches, units = kt[kernel]
    avg_s = ms / max(launches, 1) / 1e3
    flops_u, bytes_u = UNIT_WORK.get(kernel, (0, 0))
    fp64 = form == "fp64" or (form == "fp32_screen" and kernel in ("basis",))
    scale = 2 if fp64 else 1
    per_launch_units = units / max(launches, 1)
    gbs = per_launch_units * bytes_u * scale / avg_s / 1e9 if avg_s > 0 else 0.0
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    tflops = per_launch_units * flops_u / avg_s / 1e12 if avg_s > 0 else 0.0
    fp_peak = NOMINAL_FP64_TFLOPS if fp64 else NOMINAL_FP32_TFLOPS
    tb = MEASURED_TRAFFIC.get((kernel, form))
    traffic = per_launch_units * tb if tb else None
    return {"bound": "hbm", "kernel": kernel, "achieved": gbs, "peak": hbm_peak, "unit": "GB/s",
            "frac": gbs / hbm_peak, "traffic": traffic, "traffic_unit": "bytes per launch (ncu, scaled by units)",
            "peak_source": "measured (MEASURED_PEAKS.json hbm_gbs)" if "hbm_gbs" in peaks else "fallback 6650 GB/s",
            "avg_launch_ms": avg_s * 1e3, "units_per_launch": per_launch_units,
            "launch": LAUNCH_NOTE.get(kernel, "one kernel launch"),
            "compute": {"achieved": tflops, "peak": fp_peak, "unit": "TFLOP/s", "frac": tflops / fp_peak,
                        "peak_source": "nominal CUDA-core peak (148 SMs x 128 FP32 lanes x 2 x 1.965 GHz; FP64 half)"}}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", type=int, choices=[2, 3, 4], default=2,
                    help="2: hard-wave distance batch (default); 3: rational saddle / plane intersection at "
                         "nuv0 = 256; 4: the 4096-pair mixed batch (half distance, half intersection)")
    ap.add_argument("--queries", type=int, default=4096, help="config 4: pairs in the mixed batch")
    ap.add_argument("--batch", type=int, default=512, help="queries per step")
    ap.add_argument("--nuv0", type=int, default=NUV0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--forms", default=",".join(FORMS))
    ap.add_argument("--lanes", type=int, default=2, help="worker lanes (concurrent batches on the device)")
    ap.add_argument("--chunk", type=int, default=256,
                    help="queries per lockstep batch on a lane (0: one query per lane job)")
    ap.add_argument("--e2e-chunks", type=int, default=2,
                    help="end-to-end pass: submitted chunks per step (uploads overlap the previous chunk)")
    ap.add_argument("--e2e-host", choices=("pinned", "pageable"), default="pinned",
                    help="end-to-end pass: host surfaces in page-locked memory from the context "
                         "(uploaded by DMA straight from it) or in ordinary memory (staged)")
    ap.add_argument("--no-graphs", action="store_true",
                    help="launch every batch eagerly (the library's default; kept for older command lines)")
    ap.add_argument("--graphs", action="store_true", help="replay repeated batches as CUDA graphs")
    ap.add_argument("--autotune", action="store_true",
                    help="pick each form's chunk with the library's autotuner before timing it")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def shard_seeds(batch: int, rank: int):
    """Seed pairs of the queries one rank runs: ranks own disjoint queries
    (independent units, no data-path collective)."""
    return [(1000 + 2 * (rank * batch + q), 1001 + 2 * (rank * batch + q)) for q in range(batch)]


def make_pairs(batch: int, rank: int):
    from jsi_cad_next_versions_b200 import synth
    pairs = []
    for sa, sb in shard_seeds(batch, rank):
        A, B, _ = synth.distance_pair_hard_wave(seed_a=sa, seed_b=sb)
        pairs.append((A, B))
    return pairs


def reduce_max(x: float, dist, device: str) -> float:
    """Max over ranks of a per-rank device time (the step time of the job)."""
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.text = ""
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.text, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                self.text, _ = self.proc.communicate()

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in (getattr(self, "text", "") or "").splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_baseline(nuv0: int):
    """The reference (oracle/_ref) on this host: one full query, all cores."""
    ncores = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(ncores))
    os.environ.setdefault("OMP_PROC_BIND", "close")
    os.environ.setdefault("OMP_PLACES", "cores")
    import oracle
    from jsi_cad_next_versions_b200 import synth
    if not oracle.Reference.available():
        return None
    R = oracle.Reference()
    sa, sb = shard_seeds(1, 0)[0]
    A, B, _ = synth.distance_pair_hard_wave(seed_a=sa, seed_b=sb)
    ra, rb = np.array(A.rect(), np.float32), np.array(B.rect(), np.float32)
    t0 = time.perf_counter()
    v = R.minimum_distance(A, B, ra, rb, nuv0, NUV_REFINE, K, ROUNDS)
    el = time.perf_counter() - t0
    return {"value": 1.0 / el, "unit": "queries/s", "cores": int(os.environ["OMP_NUM_THREADS"]), "kind": "reference",
            "sample": f"1 full query (hard-wave seeds {sa}/{sb}, the first query of the GPU batch, nuv0={nuv0}) "
                      f"through the reference's minimum_distance, {el:.2f} s",
            "result": float(v)}


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    ncores = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(ncores))
    os.environ.setdefault("OMP_PROC_BIND", "close")
    os.environ.setdefault("OMP_PLACES", "cores")
    import oracle
    if not oracle.Reference.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libjsi_v5_ref.so was not built (needs "
                                                              "the reference checkout at build time)"}))
        return
    from jsi_cad_next_versions_b200 import synth
    R = oracle.Reference()
    # The first query of the GPU arm's batch (rank 0's first seed pair).
    sa, sb = shard_seeds(1, 0)[0]
    A, B, _ = synth.distance_pair_hard_wave(seed_a=sa, seed_b=sb)
    ra, rb = np.array(A.rect(), np.float32), np.array(B.rect(), np.float32)
    # Each step is one full query (a bounded sample of the batch); the CPU has
    # no device warm-up, so one untimed query suffices.
    for _ in range(min(args.warmup, 1)):
        R.minimum_distance(A, B, ra, rb, args.nuv0, NUV_REFINE, K, ROUNDS)
    times = []
    v = None
    for _ in range(args.steps):
        t0 = time.perf_counter()
        v = R.minimum_distance(A, B, ra, rb, args.nuv0, NUV_REFINE, K, ROUNDS)
        times.append(time.perf_counter() - t0)
    total = sum(times)
    value = args.steps / total
    lat = sorted(t * 1e3 for t in times)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "queries/s", "n_gpus": world,
        "steps": args.steps, "warmup": min(args.warmup, 1), "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "queries_per_step": 1, "nuv0": args.nuv0, "cores": int(os.environ["OMP_NUM_THREADS"]),
                   "query": f"hard-wave seeds {sa}/{sb}: the first query of the GPU arm's batch"},
        "result": None if v is None else float(v),
        "latency_ms": {"p50": lat[len(lat) // 2], "p99": lat[min(len(lat) - 1, int(0.99 * len(lat)))]},
        "cpu_baseline": {"value": value, "unit": "queries/s", "cores": int(os.environ["OMP_NUM_THREADS"]),
                         "kind": "reference",
                         "sample": f"one full query per step (hard-wave seeds {sa}/{sb}) through minimum_distance"},
        "e2e": {"value": value, "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def percentile(v, q):
    v = sorted(v)
    if not v:
        return None
    return v[min(len(v) - 1, int(q * len(v)))]


def run_ours(args):
    import torch
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist
    import jsi_cad_next_versions_b200 as J

    ctx = J.Context(local)
    ctx.workers(args.lanes)
    ctx.batch_chunk(args.chunk)
    ctx.batch_graphs(bool(args.graphs and not args.no_graphs))
    stream = torch.cuda.ExternalStream(ctx.stream_handle())
    pairs = make_pairs(args.batch, rank)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")
    forms = [f for f in args.forms.split(",") if f]

    def barrier():
        if pg:
            pg.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x: float) -> float:
        return reduce_max(x, pg, f"cuda:{local}") if pg else x

    results = {}
    # ---------------- device throughput, surfaces resident -----------------
    ids = [(ctx.upload(A), ctx.upload(B)) for A, B in pairs]
    tasks = [(ctx.task(a, np.array(A.rect(), np.float32), args.nuv0, 1),
              ctx.task(b, np.array(B.rect(), np.float32), args.nuv0, 2)) for (a, b), (A, B) in zip(ids, pairs)]
    packed = J.TaskBatch(tasks)  # the query descriptors, packed once like the resident surfaces
    ref_values = {}
    first_query = {}  # the query the reference arm and the CPU baseline time
    for form in forms:
        step_distances = []

        def step():
            res, _ = ctx.min_distance_batch(packed, k=K, rounds=ROUNDS, nuv_refine=NUV_REFINE, precision=form)
            step_distances[:] = res.distance.tolist()
            first_query[form] = {"v5_value": float(res.v5_value[0]), "distance": float(res.distance[0])}
            return res.device_ms.tolist(), res[-1]
        # Clocks are sampled from the warm-up on (all of it runs under load):
        # the timed steps alone are shorter than nvidia-smi's start-up.
        clk = ClockSampler(local)
        clk.__enter__()
        tuned = None
        if args.autotune and args.chunk > 0:
            tuned, _ = ctx.autotune_batch(tasks, k=K, rounds=ROUNDS, nuv_refine=NUV_REFINE, precision=form)
        for _ in range(args.warmup):
            step()
        reruns0 = ctx.batch_reruns()
        launches0 = ctx.launch_count()
        step_ms, lats = [], []
        for _ in range(args.steps):
            flush.zero_()
            barrier()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            l, last = step()
            e1.record(stream)
            torch.cuda.synchronize()
            barrier()
            step_ms.append(max_over_ranks(e0.elapsed_time(e1)))
            lats += l
        launches = ctx.launch_count() - launches0
        reruns = ctx.batch_reruns() - reruns0
        # Per-kernel breakdown in separate steps (events around every launch
        # would perturb the timed steps above), on one lane: with several
        # lanes a launch's events would also span the other lanes' kernels.
        ctx.workers(1)
        ctx.kernel_timing(True)
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            step()
        ktimes = ctx.kernel_times()
        ctx.kernel_timing(False)
        ctx.workers(args.lanes)
        clk.__exit__(None, None, None)
        total_ms = sum(step_ms)
        results[form] = {
            "value": world * args.batch * args.steps / (total_ms / 1e3), "ms_per_step": total_ms / args.steps,
            "p50_ms": percentile(lats, 0.5), "p99_ms": percentile(lats, 0.99), "clocks": clk.summary(),
            "gpu_launches": launches, "kernels": ktimes, "last": last, "reruns": reruns, "tuned_chunk": tuned}
        ref_values[form] = last.v5_value if form == "v5_fp32" else last.distance
        results[form]["distances"] = step_distances

    # ---------------- the plain per-query FP64 path --------------------------
    # One query per call (jsi_min_distance: no batching, the host reads each
    # round's counts), on a bounded sample of the same queries.
    nq = min(24, len(tasks))
    for ta, tb in tasks[:2]:
        ctx.min_distance(ta, tb, k=K, rounds=ROUNDS, nuv_refine=NUV_REFINE, precision="fp64")
    flush.zero_()
    torch.cuda.synchronize()
    p0 = torch.cuda.Event(enable_timing=True)
    p1 = torch.cuda.Event(enable_timing=True)
    p0.record(stream)
    for ta, tb in tasks[:nq]:
        ctx.min_distance(ta, tb, k=K, rounds=ROUNDS, nuv_refine=NUV_REFINE, precision="fp64")
    p1.record(stream)
    torch.cuda.synchronize()
    fp64_per_query = nq / (p0.elapsed_time(p1) / 1e3)

    # ---------------- end to end through the C ABI, host buffers -----------
    form = forms[0]
    h0, d0 = ctx.transfer_bytes()
    for (a, b) in ids:
        ctx.release(a)
        ctx.release(b)

    # The host surfaces as one packed set (what a caller holding a model's
    # faces in memory passes); packing is done once, like building them.
    hostset = J.SurfaceBatch([x for pr in pairs for x in pr],
                             alloc=ctx.host_array if args.e2e_host == "pinned" else None)

    e2e_result = []
    per = max(1, -(-args.batch // max(1, args.e2e_chunks)))  # queries per submitted chunk

    def e2e_run(nsteps):
        # Host surfaces in, distances out, as one continuous stream of nsteps
        # steps of args.batch queries, in chunks: each chunk is uploaded
        # (bulk, each surface's full parameter domain as its rectangle, what
        # the reference's examples put in EvalAndConstructTask) and submitted
        # before the previous chunk is waited for, read back and released, so
        # that a chunk's host staging and upload overlap the queries of the
        # chunk before it, across step boundaries too.
        from collections import deque
        inflight = deque()
        out = []

        def drain_one():
            ids, h = inflight.popleft()
            res, _ = ctx.wait_distance_batch(h)
            out.append(res.distance.copy())
            ctx.release_many(ids)
        for _ in range(nsteps):
            for c0 in range(0, args.batch, per):
                ids = np.asarray(ctx.upload_many(hostset[2 * c0:2 * min(args.batch, c0 + per)]), np.int32)
                rects = ctx.surface_domains(ids)
                tb = J.TaskBatch.from_arrays(ids[0::2], rects[0::2], args.nuv0, ids[1::2], rects[1::2], args.nuv0)
                inflight.append((ids, ctx.submit_distance_batch(tb, k=K, rounds=ROUNDS, nuv_refine=NUV_REFINE,
                                                                precision=form)))
                while len(inflight) > 1:
                    drain_one()
        while inflight:
            drain_one()
        e2e_result[:] = out
    e2e_run(args.warmup)
    h0, d0 = ctx.transfer_bytes()
    rr0 = ctx.batch_reruns()
    barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    e2e_run(args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    e2e_total = max_over_ranks(e0.elapsed_time(e1))
    h1, d1 = ctx.transfer_bytes()
    e2e = {"value": world * args.batch * args.steps / (e2e_total / 1e3), "unit": "queries/s",
           "h2d_bytes_per_step": (h1 - h0) // args.steps, "d2h_bytes_per_step": (d1 - d0) // args.steps,
           "form": form, "chunks_per_step": -(-args.batch // per),
           "host_memory": ("page-locked (Context.host_array): uploaded by DMA straight from it"
                           if args.e2e_host == "pinned" else "pageable: staged into pinned memory"),
           "timing": f"{args.steps} steps as one continuous stream (chunks pipelined across steps); "
                     "the device working set per step (~4 GB of cells) exceeds L2",
           "reruns_per_step": (ctx.batch_reruns() - rr0) / args.steps}

    if rank != 0:
        ctx.close()
        if pg:
            pg.destroy_process_group()
        return

    head = results[forms[0]]
    rel_err = None
    if "fp64" in results and forms[0] != "fp64":
        a = np.array(head["distances"], np.float64)
        b = np.array(results["fp64"]["distances"], np.float64)
        rel_err = float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300)))
    # ---------------- roofline of the dominant kernel ----------------------
    kt = head["kernels"]
    dom = max(kt.items(), key=lambda kv: kv[1][0])[0] if kt else None
    peaks = {}
    try:
        peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
    except (OSError, ValueError):
        pass
    roof = roofline(dom, kt, forms[0], peaks) if dom else None
    cpu = None if args.no_cpu_baseline else cpu_baseline(args.nuv0)
    line = {
        "metric": METRIC, "value": head["value"], "unit": "queries/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": head["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": {"fp64": "f64", "v5_fp32": "f32", "fp32_screen": "f32+f64"}[forms[0]], "data": "synthetic",
        "config": {"workload": WORKLOAD, "form": forms[0], "queries_per_step_per_gpu": args.batch,
                   "lanes": args.lanes, "chunk": args.chunk,
                   "nuv0": args.nuv0, "l2": "flushed (256 MiB write) between steps", "parallelism": f"dp{world}"},
        "latency_ms": {"p50": head["p50_ms"], "p99": head["p99_ms"]},
        "forms": {f: {"queries_per_s": r["value"], "p50_ms": r["p50_ms"], "p99_ms": r["p99_ms"],
                      "result": ref_values[f], **({"tuned_chunk": r["tuned_chunk"]} if r["tuned_chunk"] else {})}
                  for f, r in results.items()},
        "first_query": {"seeds": list(shard_seeds(1, 0)[0]), "by_form": first_query,
                        "reference_result": cpu.get("result") if cpu else None},
        "rel_err_vs_fp64": rel_err,
        "speedup_vs_fp64": (head["value"] / results["fp64"]["value"]) if "fp64" in results else None,
        "fp64_per_query_qps": fp64_per_query,
        "speedup_vs_fp64_per_query": head["value"] / fp64_per_query,
        "e2e": e2e, "roofline": roof, "cpu_baseline": cpu, "clocks": head["clocks"],
        "gpu_launches": head["gpu_launches"],
        "batch_reruns": head["reruns"],
        "screen": {"pair_tests_per_round": [int(x) for x in last.pair_tests],
                   "candidates_per_round": [int(x) for x in last.candidates],
                   "tile_pairs_per_round": [int(x) for x in last.tile_pairs],
                   "tile_pairs_tested_per_round": [int(x) for x in last.tile_pairs_tested],
                   "supertile_pairs_per_round": [int(x) for x in last.supertile_pairs],
                   "kept_per_round": [int(x) for x in last.npairs]},
        "kernel_ms": {k: round(v[0] / args.steps, 4) for k, v in sorted(kt.items(), key=lambda kv: -kv[1][0])},
        "kernel_launches_per_step": {k: v[1] / args.steps for k, v in kt.items()},
    }
    print(json.dumps(line))
    ctx.close()
    if pg:
        pg.destroy_process_group()


# ---------------------------------------------------------------------------
# Config 3: rational saddle / plane intersection (32 x 32 rational bicubic
# NURBS, nuv0 = 256, curvature padding on and off, points refined in FP64).
# Config 4: the mixed batch (4096 seeded pairs: degrees 2-5, nets 4-64, 30%
# rational, half distance, half intersection, nuv0 64-512) in one call.
# ---------------------------------------------------------------------------

NOMINAL_FP64_NOTE = "nominal CUDA-core FP64 peak (148 SMs x 64 FP64 lanes x 2 x 1.965 GHz)"


def _peaks():
    try:
        return json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
    except (OSError, ValueError):
        return {}


def sample_roofline(ctx, kt, form):
    """Roofline of the intersection's sample kernel: the algorithmic flops the
    library counted for the timed launches (full records: every derivative
    combination within the degrees, FMA = 2) over their event time, against
    the CUDA-core peak of the form's arithmetic; HBM: 16 / 32 B per sample
    written (FP32 / FP64 samples)."""
    ms, launches, units = kt["samples"]
    flops = ctx.kernel_units("samples:flops")
    s = ms / 1e3
    fp64 = form != "v5_fp32" and form != "fp32_screen"
    peak_f = NOMINAL_FP64_TFLOPS if fp64 else NOMINAL_FP32_TFLOPS
    peaks = _peaks()
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    gbs = units * (32 if fp64 else 16) / s / 1e9 if s > 0 else 0.0
    tf = flops / s / 1e12 if s > 0 else 0.0
    return {"bound": "hbm", "kernel": "samples", "achieved": gbs, "peak": hbm_peak, "unit": "GB/s",
            "frac": gbs / hbm_peak, "traffic": None,
            "peak_source": "measured (MEASURED_PEAKS.json hbm_gbs)" if "hbm_gbs" in peaks else "fallback 6650 GB/s",
            "avg_launch_ms": ms / max(launches, 1), "units_per_launch": units / max(launches, 1),
            "launch": "one sample-kernel launch (one side of one round of one query)",
            "compute": {"achieved": tf, "peak": peak_f, "unit": "TFLOP/s", "frac": tf / peak_f,
                        "peak_source": NOMINAL_FP64_NOTE if fp64 else
                        "nominal CUDA-core FP32 peak (148 SMs x 128 FP32 lanes x 2 x 1.965 GHz)"}}


def region_roofline(ctx, kt, form):
    """Roofline of the refinement rounds' fused region kernel
    (k_region_cells): HBM bytes the library counted for the timed launches
    (region records, pads, every cell's centre and half span, three bound
    vectors per tile; the control net stays in L2) and the algorithmic flops
    of its samples (full records, FMA = 2), over their event time.  The
    refinement rounds run in FP64 in the FP64 and FP32-screen forms."""
    ms, launches, units = kt["region_cells"]
    flops = ctx.kernel_units("region_cells:flops")
    nbytes = ctx.kernel_units("region_cells:bytes")
    s = ms / 1e3
    fp64 = form != "v5_fp32"
    peak_f = NOMINAL_FP64_TFLOPS if fp64 else NOMINAL_FP32_TFLOPS
    peaks = _peaks()
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    gbs = nbytes / s / 1e9 if s > 0 else 0.0
    tf = flops / s / 1e12 if s > 0 else 0.0
    return {"bound": "hbm", "kernel": "region_cells", "achieved": gbs, "peak": hbm_peak, "unit": "GB/s",
            "frac": gbs / hbm_peak, "traffic": None,
            "peak_source": "measured (MEASURED_PEAKS.json hbm_gbs)" if "hbm_gbs" in peaks else "fallback 6650 GB/s",
            "avg_launch_ms": ms / max(launches, 1), "units_per_launch": units / max(launches, 1),
            "unit_name": "samples", "bytes_per_launch": nbytes / max(launches, 1),
            "launch": "one fused region-kernel launch (one side of one refinement round of one query)",
            "compute": {"achieved": tf, "peak": peak_f, "unit": "TFLOP/s", "frac": tf / peak_f,
                        "peak_source": NOMINAL_FP64_NOTE if fp64 else
                        "nominal CUDA-core FP32 peak (148 SMs x 128 FP32 lanes x 2 x 1.965 GHz)"}}


def dominant_roofline(ctx, kt, form, n_queries):
    """The dominant kernel's roofline when it is the region kernel or the
    sample kernel (the intersection's evaluation), else the sample kernel's."""
    dom = max(kt.items(), key=lambda kv: kv[1][0])[0] if kt else None
    if dom == "region_cells" and ctx.kernel_units("region_cells:bytes") > 0:
        return dom, region_roofline(ctx, kt, form)
    roof = sample_roofline(ctx, kt, form) if "samples" in kt else None
    return dom, roof


def _timed_steps(args, flush, stream, barrier, step):
    import torch
    for _ in range(args.warmup):
        step()
    times = []
    for _ in range(args.steps):
        flush.zero_()
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        step()
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        times.append(e0.elapsed_time(e1))
    return times


CFG3_WORKLOAD = ("rational saddle / plane intersection: two 32x32 rational bicubic NURBS (w ~ U[0.5, 2]), "
                 "nuv0=256, 6 rounds from nuv 16 (halved above 512 pairs, min 4), curvature padding on, "
                 "FP64 Newton points from every final pair")


def run_cfg3(args):
    import torch
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    import jsi_cad_next_versions_b200 as J
    from jsi_cad_next_versions_b200 import synth
    ctx = J.Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream_handle())
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")
    C, D, _ = synth.intersection_pair_saddle_plane()
    rc, rd = np.array(C.rect(), np.float32), np.array(D.rect(), np.float32)
    sc, sd = ctx.upload(C), ctx.upload(D)
    ta, tb = ctx.task(sc, rc, 256, 1), ctx.task(sd, rd, 256, 2)
    forms = [f for f in args.forms.split(",") if f]
    results = {}
    pts_ref = {}
    for use_k in (True, False):
        for form in forms:
            last = []

            def step():
                last[:] = [ctx.intersect(ta, tb, use_k=use_k, precision=form, points=True, points_cap=1 << 20)]
            clk = ClockSampler(local)
            clk.__enter__()
            launches0 = ctx.launch_count()
            times = _timed_steps(args, flush, stream, lambda: torch.cuda.synchronize(), step)
            launches = (ctx.launch_count() - launches0) / (args.steps + args.warmup)
            ctx.kernel_timing(True)
            for _ in range(args.steps):
                flush.zero_()
                torch.cuda.synchronize()
                step()
            kt = ctx.kernel_times()
            dom, roof = dominant_roofline(ctx, kt, form, 1)
            ctx.kernel_timing(False)
            clk.__exit__(None, None, None)
            r = last[0]
            key = f"{form}/k{int(use_k)}"
            pts_ref[key] = r.points
            results[key] = {"queries_per_s": 1e3 * args.steps / sum(times), "ms_per_query": sum(times) / args.steps,
                            "p50_ms": percentile(times, 0.5), "p99_ms": percentile(times, 0.99),
                            "counts": r.counts.tolist(), "points": int(r.points.shape[0]),
                            "points_converged": int(r.points_converged), "screen_candidates": r.screen_written,
                            "kmax_rechecked": r.kmax_rechecked, "gpu_launches": launches, "clocks": clk.summary(),
                            "dominant_kernel": dom, "roofline": roof,
                            "kernel_ms": {k: round(v[0] / args.steps, 4)
                                          for k, v in sorted(kt.items(), key=lambda kv: -kv[1][0])}}
    # point error of each form against the FP64 form (same pairs: the same points)
    for key, pts in pts_ref.items():
        ref = pts_ref.get("fp64/" + key.split("/")[1])
        if ref is not None and pts.shape == ref.shape and pts.size:
            d = np.abs(pts[:, :3] - ref[:, :3]).max() / max(1.0, float(np.abs(ref[:, :3]).max()))
            results[key]["max_rel_point_err_vs_fp64"] = float(d)
        elif ref is not None:
            results[key]["max_rel_point_err_vs_fp64"] = None
            results[key]["points_differ_from_fp64"] = [int(pts.shape[0]), int(ref.shape[0])]
    # Queries in flight: 16 independent copies of the query (padding on, the
    # headline form, points from every final pair) in one query_batch call on
    # 4 worker lanes, so one query's host round trips overlap another's kernels.
    form = forms[0]
    n_inflight, inflight_lanes = 16, 4
    ctx.workers(inflight_lanes)
    inflight_q = [("intersection", ta, tb)] * n_inflight
    inflight_last = []

    def inflight_step():
        inflight_last[:] = [ctx.query_batch(inflight_q, precision=form, newton=True, points=True,
                                            points_cap=1 << 20)]
    inflight_t = _timed_steps(args, flush, stream, lambda: torch.cuda.synchronize(), inflight_step)
    ires, ist, _ = inflight_last[0]
    inflight = {"queries": n_inflight, "lanes": inflight_lanes, "form": form,
                "queries_per_s": 1e3 * n_inflight * args.steps / sum(inflight_t),
                "failed": int(sum(1 for x in ist if x != 0)),
                "same_counts_as_alone": all(r is not None and r.counts.tolist() == results[f"{form}/k1"]["counts"]
                                            for r in ires)}
    ctx.workers(0)
    # end to end through the C ABI: both host surfaces uploaded, the query,
    # the points read back, both released
    ctx.release(sc)
    ctx.release(sd)

    def e2e_step():
        a, b = ctx.upload_many([C, D])
        ctx.intersect(ctx.task(a, rc, 256, 1), ctx.task(b, rd, 256, 2), use_k=True, precision=form, points=True,
                      points_cap=1 << 20)
        ctx.release_many([a, b])
    h0, d0 = ctx.transfer_bytes()
    e2e_t = _timed_steps(args, flush, stream, lambda: torch.cuda.synchronize(), e2e_step)
    h1, d1 = ctx.transfer_bytes()
    nrun = args.steps + args.warmup
    e2e = {"value": 1e3 * args.steps / sum(e2e_t), "unit": "queries/s", "h2d_bytes_per_step": (h1 - h0) // nrun,
           "d2h_bytes_per_step": (d1 - d0) // nrun, "form": form}
    head = results[f"{form}/k1"]
    cpu = None if args.no_cpu_baseline else cpu_baseline_cfg3()
    line = {
        "metric": METRIC, "value": head["queries_per_s"], "unit": "queries/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": head["ms_per_query"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": {"fp64": "f64", "v5_fp32": "f32", "fp32_screen": "f32+f64"}[form],
        "data": "synthetic",
        "config": {"workload": CFG3_WORKLOAD, "form": form, "queries_per_step": 1, "nuv0": 256,
                   "l2": "flushed (256 MiB write) between steps", "parallelism": f"dp{world}"},
        "latency_ms": {"p50": head["p50_ms"], "p99": head["p99_ms"]},
        "forms": results,
        "speedup_vs_fp64": head["queries_per_s"] / results["fp64/k1"]["queries_per_s"] if "fp64/k1" in results else None,
        "e2e": e2e, "roofline": head["roofline"], "cpu_baseline": cpu, "clocks": head["clocks"],
        "gpu_launches": head["gpu_launches"], "in_flight": inflight,
    }
    print(json.dumps(line))
    ctx.close()


def cpu_baseline_cfg3():
    ncores = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(ncores))
    os.environ.setdefault("OMP_PROC_BIND", "close")
    os.environ.setdefault("OMP_PLACES", "cores")
    import oracle
    from jsi_cad_next_versions_b200 import synth
    if not oracle.Reference.available():
        return None
    R = oracle.Reference()
    C, D, _ = synth.intersection_pair_saddle_plane()
    rc, rd = np.array(C.rect(), np.float32), np.array(D.rect(), np.float32)
    t0 = time.perf_counter()
    res = R.intersection(C, D, rc, rd, 256, 16, 1)
    el = time.perf_counter() - t0
    return {"value": 1.0 / el, "unit": "queries/s", "cores": int(os.environ["OMP_NUM_THREADS"]), "kind": "reference",
            "sample": f"1 full query through the reference's intersection (nuv0=256, padding on), {el:.2f} s, "
                      f"counts {res['counts'].tolist()}"}


def run_reference_cfg3(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    cpu = cpu_baseline_cfg3() if True else None
    if cpu is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libjsi_v5_ref.so was not built"}))
        return
    times = [1.0 / cpu["value"]]
    for _ in range(max(0, args.steps - 1)):
        times.append(1.0 / cpu_baseline_cfg3()["value"])
    value = len(times) / sum(times)
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": "queries/s", "n_gpus": world,
        "steps": len(times), "warmup": 0, "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": CFG3_WORKLOAD, "queries_per_step": 1, "nuv0": 256, "cores": cpu["cores"]},
        "cpu_baseline": {**cpu, "value": value}, "e2e": {"value": value, "unit": "queries/s",
                                                          "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))


CFG4_WORKLOAD = ("mixed batch: {n} seeded pairs, degrees 2-5 per direction, nets 4-64 (log-uniform), 30% rational "
                 "(w ~ U[0.5, 2]), random-phase sinusoid heights (amplitude 0.01-0.2), half distance (k=8, 4 rounds, "
                 "FP64 Newton closest points) and half intersection (6 rounds, padding on, FP64 Newton points), "
                 "nuv0 uniform in 64-512 per pair, one query_batch call per step")


def run_cfg4(args):
    import torch
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        pg = dist
    import jsi_cad_next_versions_b200 as J
    from jsi_cad_next_versions_b200 import synth
    ctx = J.Context(local)
    ctx.workers(args.lanes)
    ctx.batch_chunk(args.chunk)
    stream = torch.cuda.ExternalStream(ctx.stream_handle())
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")
    batch = synth.mixed_batch(args.queries, seed=7 + 1000 * rank)
    surfaces = [x for a, b, _ in batch for x in (a, b)]
    ids = ctx.upload_many(surfaces)
    queries = [(m["kind"], ctx.task(ids[2 * q], np.array(a.rect(), np.float32), m["nuv0"], 1),
                ctx.task(ids[2 * q + 1], np.array(b.rect(), np.float32), m["nuv0"], 2))
               for q, (a, b, m) in enumerate(batch)]
    forms = [f for f in args.forms.split(",") if f and f != "v5_fp32"]
    points_cap = 4096

    def barrier():
        if pg:
            pg.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        return reduce_max(x, pg, f"cuda:{local}") if pg else x
    results = {}
    outs = {}
    for form in forms:
        last = []

        def step():
            res, status, ms = ctx.query_batch(queries, precision=form, newton=True, points=True,
                                              points_cap=points_cap)
            last[:] = [res, status, ms]
        clk = ClockSampler(local)
        clk.__enter__()
        launches0 = ctx.launch_count()
        times = [max_over_ranks(t) for t in _timed_steps(args, flush, stream, barrier, step)]
        launches = (ctx.launch_count() - launches0) / (args.steps + args.warmup)
        ctx.workers(1)
        ctx.kernel_timing(True)
        step()
        kt = ctx.kernel_times()
        dom, roof = dominant_roofline(ctx, kt, form, len(queries))
        ctx.kernel_timing(False)
        ctx.workers(args.lanes)
        clk.__exit__(None, None, None)
        res, status, _ = last
        lat = [r.device_ms for r in res if r is not None]
        outs[form] = res
        results[form] = {"queries_per_s": world * len(queries) * args.steps / (sum(times) / 1e3),
                         "ms_per_step": sum(times) / args.steps, "p50_ms": percentile(lat, 0.5),
                         "p99_ms": percentile(lat, 0.99), "failed": int(sum(1 for s_ in status if s_ != 0)),
                         "failed_status": sorted({int(s_) for s_ in status if s_ != 0}),
                         "failed_queries": [q for q, s_ in enumerate(status) if s_ != 0][:8],
                         "gpu_launches": launches, "clocks": clk.summary(), "dominant_kernel": dom,
                         "roofline": roof,
                         "kernel_ms": {k: round(v[0], 3) for k, v in sorted(kt.items(), key=lambda kv: -kv[1][0])}}
    # distance / point agreement of the forms (query by query)
    err = None
    if "fp64" in outs and forms[0] != "fp64":
        e = 0.0
        for a, b in zip(outs[forms[0]], outs["fp64"]):
            if a is None or b is None:
                continue
            if hasattr(a, "kth_d2"):
                d = abs(a.newton_distance - b.newton_distance) / max(abs(b.newton_distance), 1e-300)
            else:
                d = 0.0 if np.array_equal(a.points, b.points) else float(
                    np.abs(a.points[:, :3] - b.points[:, :3]).max()) if a.points.shape == b.points.shape else 1.0
            e = max(e, d)
        err = e
    # end to end: host surfaces packed once, uploaded per step, the batch,
    # results read back (distances, up to points_cap points per intersection),
    # surfaces released
    form = forms[0]
    ctx.release_many(ids)
    hostset = J.SurfaceBatch(surfaces)

    def e2e_step():
        sid = np.asarray(ctx.upload_many(hostset), np.int32)
        rects = ctx.surface_domains(sid)
        qs = [(m["kind"], ctx.task(int(sid[2 * q]), rects[2 * q], m["nuv0"], 1),
               ctx.task(int(sid[2 * q + 1]), rects[2 * q + 1], m["nuv0"], 2)) for q, (_, _, m) in enumerate(batch)]
        ctx.query_batch(qs, precision=form, newton=True, points=True, points_cap=points_cap)
        ctx.release_many(sid)
    h0, d0 = ctx.transfer_bytes()
    e2e_t = [max_over_ranks(t) for t in _timed_steps(args, flush, stream, barrier, e2e_step)]
    h1, d1 = ctx.transfer_bytes()
    nrun = args.steps + args.warmup
    e2e = {"value": world * len(queries) * args.steps / (sum(e2e_t) / 1e3), "unit": "queries/s",
           "h2d_bytes_per_step": (h1 - h0) // nrun, "d2h_bytes_per_step": (d1 - d0) // nrun, "form": form,
           "points_copied_per_intersection": f"up to {points_cap}"}
    if rank != 0:
        ctx.close()
        if pg:
            pg.destroy_process_group()
        return
    head = results[form]
    cpu = None if args.no_cpu_baseline else cpu_baseline_cfg4(batch)
    line = {
        "metric": METRIC, "value": head["queries_per_s"], "unit": "queries/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": head["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": {"fp64": "f64", "fp32_screen": "f32+f64"}[form], "data": "synthetic",
        "config": {"workload": CFG4_WORKLOAD.format(n=len(queries)), "form": form,
                   "queries_per_step_per_gpu": len(queries), "lanes": args.lanes, "chunk": args.chunk,
                   "l2": "flushed (256 MiB write) between steps", "parallelism": f"dp{world}"},
        "latency_ms": {"p50": head["p50_ms"], "p99": head["p99_ms"],
                       "note": "per-query device time inside the batch"},
        "forms": results, "max_rel_err_vs_fp64": err,
        "speedup_vs_fp64": head["queries_per_s"] / results["fp64"]["queries_per_s"] if "fp64" in results else None,
        "e2e": e2e, "roofline": head["roofline"], "cpu_baseline": cpu, "clocks": head["clocks"],
        "gpu_launches": head["gpu_launches"],
    }
    print(json.dumps(line))
    ctx.close()
    if pg:
        pg.destroy_process_group()


def cpu_baseline_cfg4(batch, budget_s: float = 20.0):
    """The reference on the batch's first queries, alternating kinds, until
    about budget_s of host time: queries/s = queries run / time."""
    ncores = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(ncores))
    os.environ.setdefault("OMP_PROC_BIND", "close")
    os.environ.setdefault("OMP_PLACES", "cores")
    import oracle
    if not oracle.Reference.available():
        return None
    R = oracle.Reference()
    t0 = time.perf_counter()
    done = {"distance": 0, "intersection": 0}
    for a, b, m in batch:
        ra, rb = np.array(a.rect(), np.float32), np.array(b.rect(), np.float32)
        if m["kind"] == "distance":
            R.minimum_distance(a, b, ra, rb, m["nuv0"], 16, 8, 4)
        else:
            R.intersection(a, b, ra, rb, m["nuv0"], 16, 1)
        done[m["kind"]] += 1
        if time.perf_counter() - t0 > budget_s:
            break
    el = time.perf_counter() - t0
    n = sum(done.values())
    return {"value": n / el, "unit": "queries/s", "cores": int(os.environ["OMP_NUM_THREADS"]), "kind": "reference",
            "sample": f"the batch's first {n} queries ({done['distance']} distance, {done['intersection']} "
                      f"intersection) through the reference, {el:.1f} s"}


def run_reference_cfg4(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from jsi_cad_next_versions_b200 import synth
    batch = synth.mixed_batch(args.queries, seed=7)
    cpu = cpu_baseline_cfg4(batch)
    if cpu is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libjsi_v5_ref.so was not built"}))
        return
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": cpu["value"], "unit": "queries/s", "n_gpus": world,
        "steps": 1, "warmup": 0, "ms_per_step": 1e3 / cpu["value"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": CFG4_WORKLOAD.format(n=args.queries), "cores": cpu["cores"]},
        "cpu_baseline": cpu, "e2e": {"value": cpu["value"], "unit": "queries/s", "h2d_bytes_per_step": 0,
                                      "d2h_bytes_per_step": 0}}))


def main():
    args = parse()
    if args.config == 3:
        (run_reference_cfg3 if args.impl == "reference" else run_cfg3)(args)
    elif args.config == 4:
        (run_reference_cfg4 if args.impl == "reference" else run_cfg4)(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
