"""Python host mirror of the VERSION5 query API over the C ABI.

Two layers:

* ``Context`` - explicit context (device, arena, resident surfaces) with
  ``upload``, ``min_distance``, ``intersect`` and ``eval_grid``.
* The reference's own names (include/jsi_cad.hpp:11-46): ``init_cad``,
  ``deinit_cad``, ``EvalAndConstructTask``, ``minimum_distance``,
  ``intersection`` and ``evalWithCuda``, bound to a module-level default
  context, so code written against the reference reads the same.

Errors raise ``JsiError`` carrying the C status; nothing falls back to the CPU.
"""
from __future__ import annotations

import ctypes
from collections.abc import Sequence
from dataclasses import dataclass, field

import numpy as np

from . import _capi as C


class JsiError(RuntimeError):
    def __init__(self, status: int, message: str):
        self.status = status
        super().__init__(f"{C.STATUS_NAMES.get(status, status)}: {message}")


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def _shrink_points(buf: np.ndarray, written: int) -> np.ndarray:
    """The first ``written`` 8-double point records of a point buffer, in
    place: the buffer is shrunk (a realloc, which for a large block remaps
    its pages without copying them) instead of the records being copied."""
    buf.resize(written * 8, refcheck=False)
    return buf.reshape(-1, 8)


@dataclass
class DistanceResult:
    v5_value: float
    distance: float
    newton_distance: float
    uv1: tuple
    uv2: tuple
    point1: tuple
    point2: tuple
    rounds: int
    npairs: np.ndarray
    kth_d2: np.ndarray
    pair_tests: np.ndarray
    candidates: np.ndarray
    device_ms: float
    pairs: list = field(default_factory=list)  # per round (n, 3) int32 (slot, i, j) if traced
    tile_pairs: np.ndarray = None  # tile pairs that passed the bound screen, per round
    tile_pairs_tested: np.ndarray = None  # tile pairs whose bound or representative was evaluated, per round
    supertile_pairs: np.ndarray = None  # supertile pairs that passed their bound, per round
    # first round's screen candidates (cand_trace=True): (m, 3) int32 (slot, i, j) and their FP64 d2
    cand_pairs: np.ndarray | None = None
    cand_d2: np.ndarray | None = None


def _struct_dtype(st) -> np.dtype:
    """numpy dtype with the byte layout of a ctypes Structure (pointers as
    uint64), for zero-copy views of result arrays."""
    names, formats, offsets = [], [], []
    for name, ct in st._fields_:
        if hasattr(ct, "_length_"):
            f = (np.dtype(ct._type_), (ct._length_,))
        elif issubclass(ct, ctypes._Pointer):
            f = np.dtype(np.uint64)
        else:
            f = np.dtype(ct)
        names.append(name)
        formats.append(f)
        offsets.append(getattr(st, name).offset)
    return np.dtype({"names": names, "formats": formats, "offsets": offsets, "itemsize": ctypes.sizeof(st)})


_DIST_DTYPE = _struct_dtype(C.DistResult)


class DistanceBatch(Sequence):
    """Results of min_distance_batch.  Indexing gives the DistanceResult of
    one query (built on access); the fields of all queries are also numpy
    arrays over the C result records (``distance``, ``v5_value``,
    ``device_ms``, ``newton_distance``, ``rounds``, ``npairs``, ``kth_d2``,
    ``pair_tests``, ``candidates``, ``tile_pairs``; per-round fields are
    (n, JSI_MAX_ROUNDS))."""

    def __init__(self, res, bufs, k: int):
        self._res, self._bufs, self._k = res, bufs, k
        self.records = np.frombuffer(res, dtype=_DIST_DTYPE, count=len(res))

    def __len__(self) -> int:
        return len(self._res)

    def __getitem__(self, q):
        if isinstance(q, slice):
            return [self[i] for i in range(*q.indices(len(self)))]
        n = len(self._res)
        if q < 0:
            q += n
        if not 0 <= q < n:
            raise IndexError(q)
        return Context._dist_result(self._res[q], self._bufs[q], self._k)

    def __getattr__(self, name):
        names = {"rounds": "rounds_run"}
        key = names.get(name, name)
        if key in _DIST_DTYPE.names and key not in ("trace_pairs", "trace_cap"):
            return self.records[key]
        raise AttributeError(name)


_TASK_DTYPE = _struct_dtype(C.Task)


class TaskBatch:
    """Query pairs packed once for repeated min_distance_batch calls."""

    def __init__(self, pairs=None):
        if pairs is None:
            return
        self.n = len(pairs)
        self.a = (C.Task * self.n)(*[x[0] for x in pairs])
        self.b = (C.Task * self.n)(*[x[1] for x in pairs])

    @classmethod
    def from_arrays(cls, ids_a, rects_a, nuv_a, ids_b, rects_b, nuv_b, side_a: int = 1, side_b: int = 2):
        """Tasks from arrays: ids (n,), rects (n, 4) (ustart, vstart, ustop,
        vstop), nuv scalars or (n,) arrays."""
        tb = cls()
        n = len(ids_a)
        tb.n = n
        for name, ids, rects, nuv, side in (("a", ids_a, rects_a, nuv_a, side_a), ("b", ids_b, rects_b, nuv_b, side_b)):
            arr = (C.Task * n)()
            v = np.frombuffer(arr, dtype=_TASK_DTYPE, count=n)
            r = np.asarray(rects, np.float32)
            v["surface"] = ids
            v["ustart"], v["vstart"], v["ustop"], v["vstop"] = r[:, 0], r[:, 1], r[:, 2], r[:, 3]
            v["nuv"] = nuv
            v["side"] = side
            setattr(tb, name, arr)
        return tb

    def __len__(self) -> int:
        return self.n


class SurfaceBatch:
    """Host surfaces packed once for repeated bulk uploads.

    One contiguous float32 buffer holds every surface's EGADS data, each
    record starting on a 64-byte boundary, beside the arrays
    ``jsi_surface_upload_many`` takes: (n, 7) headers, data pointers and
    lengths. ``batch[a:b]`` is a view of surfaces a..b-1 (no copy), so a
    caller that uploads the same host set in chunks, again and again, pays no
    per-surface Python work per upload."""

    _ALIGN = 16  # floats (64 bytes)

    def __init__(self, surfaces=None, alloc=None):
        """``alloc(n)``, when given, supplies the float32 buffer (for example
        ``Context.host_array``: page-locked memory, which the bulk upload then
        reads by DMA without a staging copy)."""
        if surfaces is None:
            return
        n = len(surfaces)
        iv = [np.asarray(x.ivec, np.int32).reshape(-1) for x in surfaces]
        if any(v.shape[0] != 7 for v in iv):
            raise ValueError("every surface header has 7 entries")
        nd = np.fromiter((np.asarray(x.data).shape[0] for x in surfaces), dtype=np.int64, count=n)
        stride = -(-nd // self._ALIGN) * self._ALIGN
        off = np.zeros(n, np.int64)
        np.cumsum(stride[:-1], out=off[1:])
        total = int(stride.sum()) + self._ALIGN
        if alloc is None:
            self.data = np.zeros(total, np.float32)
        else:
            self.data = alloc(total)
            self.data[:] = 0.0
        base = (-(self.data.ctypes.data // 4)) % self._ALIGN  # first 64-byte boundary in the buffer
        off += base
        for x, o, k in zip(surfaces, off.tolist(), nd.tolist()):
            self.data[o:o + k] = np.asarray(x.data, np.float32).reshape(-1)
        self.ivec = np.ascontiguousarray(np.stack(iv), dtype=np.int32) if n else np.zeros((0, 7), np.int32)
        self.ndata = nd.astype(np.int32)
        self.offsets = off
        self.ptrs = (self.data.ctypes.data + 4 * off).astype(np.uintp)

    def __len__(self) -> int:
        return int(self.ndata.shape[0])

    def __getitem__(self, key):
        if not isinstance(key, slice) or key.step not in (None, 1):
            raise TypeError("SurfaceBatch takes contiguous slices")
        sub = SurfaceBatch()
        sub.data = self.data
        sub.ivec, sub.ndata = self.ivec[key], self.ndata[key]
        sub.offsets, sub.ptrs = self.offsets[key], self.ptrs[key]
        return sub

    def surface(self, q: int):
        """(ivec, data) views of surface q."""
        o = int(self.offsets[q])
        return self.ivec[q], self.data[o:o + int(self.ndata[q])]


@dataclass
class IntersectionCurves:
    """Polylines through the refined intersection points: curves[k] is an
    (m, 7) array of (x, y, z, u, v, s, t) in curve order."""
    points_found: int
    link_tol: float
    curves: list
    closed: list
    device_ms: float


@dataclass
class DistanceBounds:
    """Certified interval lb <= min distance <= ub (bounds mode)."""
    lb: float
    ub: float
    certified: bool
    rounds: int
    kept: np.ndarray
    pair_tests: np.ndarray
    lb_round: np.ndarray
    uv1: tuple
    uv2: tuple
    point1: tuple
    point2: tuple
    device_ms: float


@dataclass
class IntersectionResult:
    rounds: int
    counts: np.ndarray
    pair_tests: np.ndarray
    regions1: np.ndarray
    regions2: np.ndarray
    pad: tuple
    device_ms: float
    pairs: list = field(default_factory=list)  # per round (n, 3) int32 if traced
    points: np.ndarray | None = None  # (n, 8): x, y, z, u, v, s, t, residual
    points_converged: int = 0
    # FP32_SCREEN: the first round's FP32 candidates (count; (m, 3) (slot, i, j)
    # in key order when screen_trace=True) and the samples re-evaluated in FP64
    # for the exact compute_K maxima
    screen_written: int = 0
    screen_pairs: np.ndarray | None = None
    kmax_rechecked: int = 0


class Context:
    """A device context: one stream, one arena, resident surfaces."""

    def __init__(self, device: int = 0, arena_bytes: int = 0, hbm_budget_bytes: int = 0):
        self.lib = C.load()
        cfg = C.Config(device, arena_bytes, hbm_budget_bytes)
        h = ctypes.c_void_p()
        st = self.lib.jsi_create(ctypes.byref(cfg), ctypes.byref(h))
        if st != C.JSI_OK:
            raise JsiError(st, "jsi_create failed")
        self.handle = h
        self._surfaces = {}
        self._pending = {}

    def close(self):
        if getattr(self, "handle", None):
            self.lib.jsi_destroy(self.handle)
            self.handle = None
            getattr(self, "_host_blocks", {}).clear()

    def host_array(self, n: int, dtype=np.float32) -> np.ndarray:
        """A host array of n elements in page-locked memory owned by the
        context (``jsi_host_alloc``): surface records packed in it are
        uploaded by DMA straight from it.  It stays valid until
        ``host_free`` or ``close``."""
        nbytes = int(n) * np.dtype(dtype).itemsize
        p = ctypes.c_void_p()
        self._check(self.lib.jsi_host_alloc(self.handle, nbytes, ctypes.byref(p)))
        buf = (ctypes.c_char * nbytes).from_address(p.value)
        arr = np.frombuffer(buf, dtype=dtype, count=int(n))
        if not hasattr(self, "_host_blocks"):
            self._host_blocks = {}
        self._host_blocks[p.value] = buf
        return arr

    def host_free(self, arr: np.ndarray):
        """Frees an array from ``host_array`` (the array must not be used
        afterwards)."""
        ptr = arr.__array_interface__["data"][0]
        self._check(self.lib.jsi_host_free(self.handle, ctypes.c_void_p(ptr)))
        getattr(self, "_host_blocks", {}).pop(ptr, None)

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st: int):
        if st != C.JSI_OK:
            msg = self.lib.jsi_last_error(self.handle)
            raise JsiError(st, msg.decode() if msg else "")

    # -- surfaces ---------------------------------------------------------
    def upload(self, surface=None, *, ivec=None, data=None) -> int:
        """Upload a surface (``synth.Surface`` or ivec/data arrays); returns its id."""
        if surface is not None:
            ivec, data = surface.ivec, surface.data
        iv = np.ascontiguousarray(ivec, dtype=np.int32)
        da = np.ascontiguousarray(data, dtype=np.float32)
        sid = ctypes.c_int(0)
        self._check(self.lib.jsi_surface_upload(self.handle, _p(iv), _p(da), int(da.shape[0]), ctypes.byref(sid)))
        return sid.value

    def upload_many(self, surfaces) -> list[int]:
        """Upload several surfaces in one call (a sequence of surfaces, or a
        ``SurfaceBatch`` or slice of one); returns their ids."""
        n = len(surfaces)
        if n == 0:
            return []
        if isinstance(surfaces, SurfaceBatch):
            ids = np.zeros(n, np.int32)
            self._check(self.lib.jsi_surface_upload_many(self.handle, n, surfaces.ivec.ctypes.data,
                                                         surfaces.ptrs.ctypes.data, surfaces.ndata.ctypes.data,
                                                         ids.ctypes.data))
            return ids.tolist()
        iv = np.ascontiguousarray(np.stack([np.asarray(x.ivec, np.int32) for x in surfaces]), dtype=np.int32)
        keep = [np.ascontiguousarray(x.data, dtype=np.float32) for x in surfaces]
        ptrs = np.fromiter((k.ctypes.data for k in keep), dtype=np.uintp, count=n)
        nd = np.fromiter((k.shape[0] for k in keep), dtype=np.int32, count=n)
        ids = np.zeros(n, np.int32)
        self._check(self.lib.jsi_surface_upload_many(self.handle, n, iv.ctypes.data, ptrs.ctypes.data, nd.ctypes.data,
                                                     ids.ctypes.data))
        return ids.tolist()

    def release_many(self, ids):
        """Release several surfaces in one call."""
        a = np.ascontiguousarray(ids, dtype=np.int32)
        self._check(self.lib.jsi_surface_release_many(self.handle, a.size, a.ctypes.data))

    def surface_domains(self, ids) -> np.ndarray:
        """(n, 4) float32 full parameter domains (ustart, vstart, ustop, vstop)
        of resident surfaces."""
        a = np.ascontiguousarray(ids, dtype=np.int32)
        out = np.zeros((a.size, 4), np.float32)
        self._check(self.lib.jsi_surface_domains(self.handle, a.size, a.ctypes.data, out.ctypes.data))
        return out

    def release(self, sid: int):
        self._check(self.lib.jsi_surface_release(self.handle, sid))

    def resident_bytes(self) -> int:
        v = ctypes.c_ulonglong(0)
        self._check(self.lib.jsi_resident_bytes(self.handle, ctypes.byref(v)))
        return v.value

    # -- instrumentation --------------------------------------------------
    def stream_handle(self) -> int:
        """The context's cudaStream_t as an integer (for external CUDA events)."""
        v = ctypes.c_void_p()
        self._check(self.lib.jsi_context_stream(self.handle, ctypes.byref(v)))
        return v.value or 0

    def transfer_bytes(self):
        h2d, d2h = ctypes.c_ulonglong(0), ctypes.c_ulonglong(0)
        self._check(self.lib.jsi_transfer_bytes(self.handle, ctypes.byref(h2d), ctypes.byref(d2h)))
        return h2d.value, d2h.value

    def kernel_timing(self, enable: bool):
        """Bracket every kernel launch with CUDA events (resets the totals)."""
        self._check(self.lib.jsi_kernel_timing(self.handle, 1 if enable else 0))

    def kernel_times(self) -> dict:
        """{kernel name: (total ms, launches, work units)} since kernel_timing(True)."""
        names = self.lib.jsi_kernel_names(self.handle).decode()
        out = {}
        for n in filter(None, names.split(",")):
            ms, cnt, units = ctypes.c_double(0), ctypes.c_longlong(0), ctypes.c_double(0)
            self._check(self.lib.jsi_kernel_time(self.handle, n.encode(), ctypes.byref(ms), ctypes.byref(cnt)))
            self._check(self.lib.jsi_kernel_units(self.handle, n.encode(), ctypes.byref(units)))
            out[n] = (ms.value, cnt.value, units.value)
        return out

    def kernel_units(self, name: str) -> float:
        """Work units counted under a name since kernel_timing(True) (also
        the algorithmic flops of a kernel, as "<kernel>:flops")."""
        units = ctypes.c_double(0)
        self._check(self.lib.jsi_kernel_units(self.handle, name.encode(), ctypes.byref(units)))
        return units.value

    def launch_count(self) -> int:
        v = ctypes.c_ulonglong(0)
        self._check(self.lib.jsi_launch_count(ctypes.byref(v)))
        return v.value

    # -- queries ----------------------------------------------------------
    @staticmethod
    def task(sid: int, rect, nuv: int, side: int) -> C.Task:
        return C.Task(sid, float(rect[0]), float(rect[1]), float(rect[2]), float(rect[3]), int(nuv), int(side))

    @staticmethod
    def _dist_params(k, rounds, nuv_refine, precision, newton):
        prec = C.PRECISIONS[precision] if isinstance(precision, str) else int(precision)
        return C.DistParams(nuv_refine, k, rounds, prec, 1 if newton else 0)

    @staticmethod
    def _dist_result(r: C.DistResult, buf, k: int) -> DistanceResult:
        n = r.rounds_run
        npairs = np.array(r.npairs[:n], dtype=np.int64)
        pairs = []
        if buf is not None:
            for q in range(n):
                pairs.append(buf[q * k * 3:(q * k + int(npairs[q])) * 3].reshape(-1, 3).copy())
        return DistanceResult(
            v5_value=float(np.float32(r.v5_value)), distance=r.distance, newton_distance=r.newton_distance,
            uv1=tuple(r.uv1), uv2=tuple(r.uv2), point1=tuple(r.point1), point2=tuple(r.point2), rounds=n,
            npairs=npairs, kth_d2=np.array(r.kth_d2[:n]), pair_tests=np.array(r.pair_tests[:n], dtype=np.int64),
            candidates=np.array(r.candidates[:n], dtype=np.int64), device_ms=r.device_ms, pairs=pairs,
            tile_pairs=np.array(r.tile_pairs[:n], dtype=np.int64),
            tile_pairs_tested=np.array(r.tile_pairs_tested[:n], dtype=np.int64),
            supertile_pairs=np.array(r.supertile_pairs[:n], dtype=np.int64))

    def min_distance(self, a: C.Task, b: C.Task, *, k: int = 8, rounds: int = 4, nuv_refine: int = 16,
                     precision: str | int = "v5_fp32", newton: bool = False, trace: bool = False,
                     cand_trace: bool = False, cand_cap: int = 1 << 22) -> DistanceResult:
        p = self._dist_params(k, rounds, nuv_refine, precision, newton)
        r = C.DistResult()
        buf = None
        if trace:
            buf = np.full(rounds * k * 3, -1, dtype=np.int32)
            r.trace_pairs = buf.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
            r.trace_cap = rounds * k
        cbuf = cd2 = None
        if cand_trace:
            cbuf = np.full(cand_cap * 3, -1, dtype=np.int32)
            cd2 = np.full(cand_cap, np.nan, dtype=np.float64)
            r.cand_pairs = cbuf.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
            r.cand_d2 = cd2.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
            r.cand_cap = cand_cap
        self._check(self.lib.jsi_min_distance(self.handle, ctypes.byref(a), ctypes.byref(b), ctypes.byref(p),
                                              ctypes.byref(r)))
        res = self._dist_result(r, buf, k)
        if cand_trace:
            m = int(r.cand_written)
            if m > cand_cap:
                raise JsiError(-4, f"{m} screen candidates exceed cand_cap {cand_cap}")
            res.cand_pairs = cbuf[:3 * m].reshape(-1, 3).copy()
            res.cand_d2 = cd2[:m].copy()
        return res

    # -- worker lanes: queued / batched queries ----------------------------
    def workers(self, n: int, lane_bytes: int = 0):
        """Start n worker lanes (stream + arena + host thread each); 0 stops them."""
        self._check(self.lib.jsi_workers(self.handle, int(n), int(lane_bytes)))

    def submit_distance(self, a: C.Task, b: C.Task, *, k: int = 8, rounds: int = 4, nuv_refine: int = 16,
                        precision: str | int = "v5_fp32", newton: bool = False, trace: bool = False):
        """Queue a distance query; returns a ticket for wait()."""
        p = self._dist_params(k, rounds, nuv_refine, precision, newton)
        buf = np.full(rounds * k * 3, -1, dtype=np.int32) if trace else None
        t = ctypes.c_longlong(0)
        ptr = buf.ctypes.data_as(ctypes.POINTER(ctypes.c_int)) if trace else None
        self._check(self.lib.jsi_submit_distance(self.handle, ctypes.byref(a), ctypes.byref(b), ctypes.byref(p),
                                                 ptr, rounds * k if trace else 0, ctypes.byref(t)))
        self._pending[t.value] = ("d", buf, k, None)
        return t.value

    def submit_intersect(self, a: C.Task, b: C.Task, *, nuv_refine: int = 16, use_k: bool = True, rounds: int = 6,
                         halve_threshold: int = 512, min_nuv: int = 4, precision: str | int = "v5_fp32",
                         trace: bool = False, trace_cap: int = 1 << 22):
        prec = C.PRECISIONS[precision] if isinstance(precision, str) else int(precision)
        p = C.InterParams(nuv_refine, 1 if use_k else 0, rounds, halve_threshold, min_nuv, prec, 0)
        buf = np.full(trace_cap * 3, -1, dtype=np.int32) if trace else None
        t = ctypes.c_longlong(0)
        ptr = buf.ctypes.data_as(ctypes.POINTER(ctypes.c_int)) if trace else None
        self._check(self.lib.jsi_submit_intersect(self.handle, ctypes.byref(a), ctypes.byref(b), ctypes.byref(p),
                                                  ptr, trace_cap if trace else 0, ctypes.byref(t)))
        self._pending[t.value] = ("i", buf, trace_cap, None)
        return t.value

    def wait(self, ticket: int, timeout_ms: int = -1):
        """Result of a queued query, or None if not done within timeout_ms."""
        kind, buf, cap, _ = self._pending[ticket]
        d, i = C.DistResult(), C.InterResult()
        st = self.lib.jsi_wait(self.handle, ticket, int(timeout_ms), ctypes.byref(d), ctypes.byref(i))
        if st == -6:
            return None
        del self._pending[ticket]
        self._check(st)
        if kind == "d":
            return self._dist_result(d, buf, cap)
        return self._inter_result(i, buf, cap)

    def queue_depth(self):
        q, r = ctypes.c_int(0), ctypes.c_int(0)
        self._check(self.lib.jsi_queue_depth(self.handle, ctypes.byref(q), ctypes.byref(r)))
        return q.value, r.value

    def batch_chunk(self, chunk: int) -> None:
        """Queries per lockstep batch of min_distance_batch (0: one query per
        lane job)."""
        self._check(self.lib.jsi_batch_chunk(self.handle, int(chunk)))

    def batch_graphs(self, enable: bool | None = None) -> int:
        """Switch CUDA-graph replay of repeated lockstep batches (None: leave
        it); returns the number of replays so far."""
        v = ctypes.c_longlong(0)
        flag = -1 if enable is None else (1 if enable else 0)
        self._check(self.lib.jsi_batch_graphs(self.handle, flag, ctypes.byref(v)))
        return v.value

    def autotune_batch(self, pairs, *, k: int = 8, rounds: int = 4, nuv_refine: int = 16,
                       precision: str | int = "v5_fp32", newton: bool = False) -> tuple[int, float]:
        """Pick the lockstep chunk size for the shape of these queries (all of
        one shape) by timing them; returns (chunk, batch device ms)."""
        n = len(pairs)
        p = self._dist_params(k, rounds, nuv_refine, precision, newton)
        ta = (C.Task * n)(*[x[0] for x in pairs])
        tb = (C.Task * n)(*[x[1] for x in pairs])
        chunk, ms = ctypes.c_int(0), ctypes.c_float(0)
        self._check(self.lib.jsi_autotune_batch(self.handle, n, ta, tb, ctypes.byref(p), ctypes.byref(chunk),
                                                ctypes.byref(ms)))
        return chunk.value, ms.value

    def batch_reruns(self) -> int:
        """Batch items re-run alone after an internal list overflowed."""
        v = ctypes.c_longlong(0)
        self._check(self.lib.jsi_batch_reruns(self.handle, ctypes.byref(v)))
        return v.value

    def min_distance_batch(self, pairs, *, k: int = 8, rounds: int = 4, nuv_refine: int = 16,
                           precision: str | int = "v5_fp32", trace: bool = False, newton: bool = False):
        """Distance queries [(task_a, task_b), ...] over the worker lanes
        (lockstep batches per shape, see batch_chunk).
        ``pairs`` is a list of (task_a, task_b) or a TaskBatch.
        Returns (DistanceBatch, device_ms of the whole batch)."""
        return self.wait_distance_batch(self.submit_distance_batch(pairs, k=k, rounds=rounds, nuv_refine=nuv_refine,
                                                                   precision=precision, trace=trace, newton=newton))

    def submit_distance_batch(self, pairs, *, k: int = 8, rounds: int = 4, nuv_refine: int = 16,
                              precision: str | int = "v5_fp32", trace: bool = False, newton: bool = False):
        """Queue a batch (as min_distance_batch) and return at once; pass the
        returned handle to wait_distance_batch.  Uploads issued before the
        submit are visible to the batch, so the next batch's surfaces can be
        uploaded while this one runs."""
        tasks = pairs if isinstance(pairs, TaskBatch) else TaskBatch(pairs)
        n = tasks.n
        p = self._dist_params(k, rounds, nuv_refine, precision, newton)
        res = (C.DistResult * n)()
        bufs = [None] * n
        if trace:
            for q in range(n):
                buf = np.full(rounds * k * 3, -1, dtype=np.int32)
                res[q].trace_pairs = buf.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
                res[q].trace_cap = rounds * k
                bufs[q] = buf
        status = (ctypes.c_int * n)()
        t = ctypes.c_longlong(0)
        self._check(self.lib.jsi_submit_distance_batch(self.handle, n, tasks.a, tasks.b, ctypes.byref(p), res, status,
                                                       ctypes.byref(t)))
        # everything the C side writes into or reads from stays alive here
        return {"ticket": t.value, "tasks": tasks, "res": res, "bufs": bufs, "status": status, "k": k}

    def poll_distance_batch(self, handle) -> bool:
        """True when every lane job of a submitted batch has finished."""
        d = ctypes.c_int(0)
        self._check(self.lib.jsi_poll_distance_batch(self.handle, handle["ticket"], ctypes.byref(d)))
        return bool(d.value)

    def wait_distance_batch(self, handle):
        """Wait for a submitted batch: (DistanceBatch, device_ms)."""
        ms = ctypes.c_float(0)
        self._check(self.lib.jsi_wait_distance_batch(self.handle, handle["ticket"], ctypes.byref(ms)))
        return DistanceBatch(handle["res"], handle["bufs"], handle["k"]), ms.value

    def query_batch(self, queries, *, precision: str | int = "v5_fp32", k: int = 8, rounds: int = 4,
                    nuv_refine: int = 16, newton: bool = False, use_k: bool = True, inter_rounds: int = 6,
                    halve_threshold: int = 512, min_nuv: int = 4, points: bool = False, points_cap: int = 1 << 20,
                    trace: bool = False, trace_cap: int = 1 << 20):
        """Mixed queries [(kind, task_a, task_b), ...] (kind "distance" or
        "intersection") in one call over the worker lanes: distance queries in
        lockstep batches grouped by first-round nuv, intersection queries as
        lane jobs, largest first.  Returns (results, statuses, device_ms):
        results[q] is a DistanceResult or an IntersectionResult."""
        n = len(queries)
        kinds = (ctypes.c_int * n)(*[0 if q[0] in ("distance", 0) else 1 for q in queries])
        ta = (C.Task * n)(*[q[1] for q in queries])
        tb = (C.Task * n)(*[q[2] for q in queries])
        dp = self._dist_params(k, rounds, nuv_refine, precision, newton)
        prec = C.PRECISIONS[precision] if isinstance(precision, str) else int(precision)
        ip = C.InterParams(nuv_refine, 1 if use_k else 0, inter_rounds, halve_threshold, min_nuv, prec,
                           1 if points else 0)
        dres = (C.DistResult * n)()
        ires = (C.InterResult * n)()
        pbufs, tbufs = {}, {}
        for q in range(n):
            if kinds[q] == 1:
                if points:
                    pbufs[q] = np.empty(points_cap * 8, dtype=np.float64)
                    ires[q].points = pbufs[q].ctypes.data_as(ctypes.POINTER(ctypes.c_double))
                    ires[q].points_cap = points_cap
                if trace:
                    tbufs[q] = np.full(trace_cap * 3, -1, dtype=np.int32)
                    ires[q].trace_pairs = tbufs[q].ctypes.data_as(ctypes.POINTER(ctypes.c_int))
                    ires[q].trace_cap = trace_cap
        status = (ctypes.c_int * n)()
        ms = ctypes.c_float(0)
        st = self.lib.jsi_query_batch(self.handle, n, kinds, ta, tb, ctypes.byref(dp), ctypes.byref(ip), dres, ires,
                                      status, ctypes.byref(ms))
        out = []
        for q in range(n):
            if status[q] != 0:
                out.append(None)
            elif kinds[q] == 0:
                out.append(self._dist_result(dres[q], None, k))
            else:
                r = self._inter_result(ires[q], tbufs.get(q), trace_cap)
                if points:
                    r.points = _shrink_points(pbufs.pop(q), int(ires[q].points_written))
                    r.points_converged = int(ires[q].points_converged)
                r.screen_written = int(ires[q].screen_written)
                r.kmax_rechecked = int(ires[q].kmax_rechecked)
                out.append(r)
        if st != 0 and all(s == 0 for s in status):
            self._check(st)
        return out, list(status), ms.value

    def intersection_curves(self, a: C.Task, b: C.Task, *, nuv_refine: int = 16, use_k: bool = True, rounds: int = 6,
                            halve_threshold: int = 512, min_nuv: int = 4, link_tol: float = 0.0,
                            vertex_cap: int = 1 << 18, curve_cap: int = 1 << 12) -> IntersectionCurves:
        """Intersection curves of two surface rectangles (FP64 query, Newton
        points linked into polylines)."""
        ip = C.InterParams(nuv_refine, 1 if use_k else 0, rounds, halve_threshold, min_nuv, C.PRECISIONS["fp64"], 1)
        for _ in range(2):
            p = C.CurveParams(ip, link_tol)
            verts = np.zeros((vertex_cap, 7), np.float64)
            starts = np.zeros(curve_cap + 1, np.int64)
            closed = np.zeros(curve_cap, np.int32)
            r = C.CurveResult(0, 0, 0, 0.0, verts.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), vertex_cap,
                              starts.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong)),
                              closed.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), curve_cap, 0.0)
            st = self.lib.jsi_intersection_curves(self.handle, ctypes.byref(a), ctypes.byref(b), ctypes.byref(p),
                                                  ctypes.byref(r))
            if st == -4 and (r.vertices > vertex_cap or r.curves > curve_cap):
                vertex_cap, curve_cap = max(vertex_cap, r.vertices), max(curve_cap, r.curves)
                continue
            self._check(st)
            n = r.curves
            curves = [verts[starts[k]:starts[k + 1]].copy() for k in range(n)]
            return IntersectionCurves(r.points_found, r.link_tol, curves, [bool(x) for x in closed[:n]], r.device_ms)
        self._check(st)

    def distance_bounds(self, a: C.Task, b: C.Task, *, nuv_refine: int = 8, max_rounds: int = 10,
                        rel_tol: float = 1e-6, max_pairs: int = 1 << 22) -> DistanceBounds:
        """Rigorous interval for the minimum distance between two non-rational
        surface rectangles (the FP64 Newton pair as ub, branch and bound on
        padded cell boxes of a covering grid for lb)."""
        p = C.BoundsParams(nuv_refine, max_rounds, rel_tol, max_pairs)
        r = C.BoundsResult()
        self._check(self.lib.jsi_distance_bounds(self.handle, ctypes.byref(a), ctypes.byref(b), ctypes.byref(p),
                                                 ctypes.byref(r)))
        n = r.rounds_run
        return DistanceBounds(r.lb, r.ub, bool(r.certified), n, np.array(r.kept[:n], np.int64),
                              np.array(r.pair_tests[:n], np.int64), np.array(r.lb_round[:n], np.float64),
                              tuple(r.uv1), tuple(r.uv2), tuple(r.point1), tuple(r.point2), r.device_ms)

    def intersect(self, a: C.Task, b: C.Task, *, nuv_refine: int = 16, use_k: bool = True, rounds: int = 6,
                  halve_threshold: int = 512, min_nuv: int = 4, precision: str | int = "v5_fp32",
                  trace: bool = False, trace_cap: int = 1 << 24, points: bool = False,
                  points_cap: int = 1 << 22, screen_trace: bool = False,
                  screen_cap: int = 1 << 24) -> IntersectionResult:
        prec = C.PRECISIONS[precision] if isinstance(precision, str) else int(precision)
        p = C.InterParams(nuv_refine, 1 if use_k else 0, rounds, halve_threshold, min_nuv, prec, 1 if points else 0)
        r = C.InterResult()
        buf = None
        if trace:
            buf = np.full(trace_cap * 3, -1, dtype=np.int32)
            r.trace_pairs = buf.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
            r.trace_cap = trace_cap
        pbuf = None
        if points:
            pbuf = np.empty(points_cap * 8, dtype=np.float64)
            r.points = pbuf.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
            r.points_cap = points_cap
        sbuf = None
        if screen_trace:
            sbuf = np.full(screen_cap * 3, -1, dtype=np.int32)
            r.screen_pairs = sbuf.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
            r.screen_cap = screen_cap
        self._check(self.lib.jsi_intersect(self.handle, ctypes.byref(a), ctypes.byref(b), ctypes.byref(p),
                                           ctypes.byref(r)))
        res = self._inter_result(r, buf, trace_cap)
        res.screen_written = int(r.screen_written)
        res.kmax_rechecked = int(r.kmax_rechecked)
        if screen_trace:
            m = int(r.screen_written)
            if m > screen_cap:
                raise JsiError(-4, f"{m} screen candidates exceed screen_cap {screen_cap}")
            res.screen_pairs = sbuf[:3 * m].reshape(-1, 3).copy()
        if points:
            res.points = _shrink_points(pbuf, int(r.points_written))
            res.points_converged = int(r.points_converged)
        return res

    @staticmethod
    def _inter_result(r: C.InterResult, buf, trace_cap: int) -> IntersectionResult:
        n = r.rounds_run
        counts = np.array(r.counts[:n], dtype=np.int64)
        pairs = []
        if buf is not None:
            off = 0
            for c in counts:
                c = int(c)
                pairs.append(buf[off * 3:(off + c) * 3].reshape(-1, 3).copy() if off + c <= trace_cap else None)
                off += c
        return IntersectionResult(
            rounds=n, counts=counts, pair_tests=np.array(r.pair_tests[:n], dtype=np.int64),
            regions1=np.array(r.regions1[:n], dtype=np.int64), regions2=np.array(r.regions2[:n], dtype=np.int64),
            pad=(r.pad[0], r.pad[1]), device_ms=r.device_ms, pairs=pairs)

    def eval_grid(self, ivec, data, ustep, vstep, ustart, vstart, nuv, dtype=np.float32) -> np.ndarray:
        iv = np.ascontiguousarray(ivec, dtype=np.int32)
        da = np.ascontiguousarray(data, dtype=np.float32)
        out = np.zeros(nuv * nuv * C.RECORD_SIZE, dtype=dtype)
        if dtype == np.float32:
            st = self.lib.jsi_eval_grid(self.handle, _p(iv), _p(da), int(da.shape[0]), float(np.float32(ustep)),
                                        float(np.float32(vstep)), float(np.float32(ustart)),
                                        float(np.float32(vstart)), nuv, _p(out))
        else:
            st = self.lib.jsi_eval_grid_f64(self.handle, _p(iv), _p(da), int(da.shape[0]), float(ustep),
                                            float(vstep), float(ustart), float(vstart), nuv, _p(out))
        self._check(st)
        return out


def curvature_bounds(surface=None, *, ivec=None, data=None, rect=None) -> tuple[np.ndarray, np.ndarray]:
    """Per-coordinate bounds (m2u, m2v) on |S_uu| and |S_vv| over the whole
    surface, or over the parameter rectangle ``rect`` = (u0, v0, u1, v1) as
    the bounds mode pads a region (host only: no device, no context)."""
    if surface is not None:
        ivec, data = surface.ivec, surface.data
    iv = np.ascontiguousarray(ivec, dtype=np.int32)
    da = np.ascontiguousarray(data, dtype=np.float32)
    mu = np.zeros(3, np.float64)
    mv = np.zeros(3, np.float64)
    rc = None if rect is None else np.ascontiguousarray(rect, dtype=np.float64)
    st = C.load().jsi_surface_curvature_bounds(_p(iv), _p(da), int(da.shape[0]), None if rc is None else _p(rc),
                                               mu.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                               mv.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    if st != C.JSI_OK:
        raise JsiError(st, C.STATUS_NAMES.get(st, str(st)))
    return mu, mv


# ---------------------------------------------------------------------------
# The reference's names over a default context
# ---------------------------------------------------------------------------

_default: Context | None = None

default_global_dist_nuv = 512     # include/jsi_cad.hpp:35
default_global_intersect_nuv = 16  # include/jsi_cad.hpp:36
ONE_UV_SIZE = C.RECORD_SIZE        # include/jsi_cad.hpp:45


def init_cad(device: int = 0):
    """init_cad() (common.cu:35-49): creates the default device context."""
    global _default
    if _default is None:
        _default = Context(device)
    return _default


def deinit_cad():
    """deinit_cad() (common.cu:51-61): releases the default context."""
    global _default
    if _default is not None:
        _default.close()
        _default = None


def _ctx() -> Context:
    if _default is None:
        raise JsiError(-1, "init_cad() has not been called")
    return _default


@dataclass
class EvalAndConstructTask:
    """include/jsi_cad.hpp:11-23, with host arrays in place of d_ivec / d_data."""

    d_ivec: np.ndarray
    d_data: np.ndarray
    d_ndata: int
    ustart: float
    vstart: float
    ustop: float
    vstop: float
    nuv: int
    eval_task_side: int


def _upload_task(ctx: Context, t: EvalAndConstructTask):
    sid = ctx.upload(ivec=t.d_ivec, data=np.asarray(t.d_data)[: t.d_ndata])
    return Context.task(sid, (t.ustart, t.vstart, t.ustop, t.vstop), t.nuv, t.eval_task_side), sid


def minimum_distance(t1: EvalAndConstructTask, t2: EvalAndConstructTask, **kw) -> float:
    """float minimum_distance(t1, t2) (distance_analysis.cu:356-506)."""
    ctx = _ctx()
    a, sa = _upload_task(ctx, t1)
    b, sb = _upload_task(ctx, t2)
    try:
        return ctx.min_distance(a, b, **kw).v5_value
    finally:
        ctx.release(sa)
        ctx.release(sb)


def intersection(t1: EvalAndConstructTask, t2: EvalAndConstructTask, verbose: bool = False, **kw):
    """void intersection(t1, t2) (intersection.cu:338-475).  The reference only
    prints "Round r: overlap pairs = N"; this returns the per-round counts
    (and prints them when verbose)."""
    ctx = _ctx()
    a, sa = _upload_task(ctx, t1)
    b, sb = _upload_task(ctx, t2)
    try:
        res = ctx.intersect(a, b, **kw)
    finally:
        ctx.release(sa)
        ctx.release(sb)
    if verbose:
        for r, c in enumerate(res.counts, 1):
            print(f"Round {r}: overlap pairs = {int(c)}")
    return res.counts


def evalWithCuda(ivec, data, ndata, ustep, vstep, ustart, vstart, nuv, results=None):
    """evalWithCuda (evaluation.cu:391-405): nuv*nuv records of 18 floats."""
    out = _ctx().eval_grid(ivec, np.asarray(data)[:ndata], ustep, vstep, ustart, vstart, nuv)
    if results is not None:
        results[: out.shape[0]] = out
        return results
    return out
