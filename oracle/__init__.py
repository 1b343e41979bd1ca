"""ctypes access to the CPU oracle and to the compiled reference.

TEST INFRASTRUCTURE ONLY.  Only tests/, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` import this package; the product
(``jsi_cad_next_versions_b200``) never does.

* ``Oracle``    - oracle/libjsi_oracle.so, our restatement of the reference
                  VERSION5 algorithm (float and double instantiations).
* ``Reference`` - oracle/_ref/libjsi_v5_ref.so, the reference itself compiled
                  from its own sources by oracle/Makefile (present where the
                  reference checkout was available at build time).
"""
from __future__ import annotations

import contextlib
import ctypes
import os
import re
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "libjsi_oracle.so"
REF_SO = HERE / "_ref" / "libjsi_v5_ref.so"

_P = ctypes.c_void_p
_I = ctypes.c_int
_LL = ctypes.c_longlong
_F = ctypes.c_float
_D = ctypes.c_double


def _p(a):
    return None if a is None else a.ctypes.data_as(_P)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class Oracle:
    """Our CPU restatement (see oracle/jsi_oracle.h)."""

    def __init__(self, path: Path | str = ORACLE_SO):
        self.lib = ctypes.CDLL(str(path))
        L = self.lib
        L.orc_eval_grid_f32.argtypes = [_P, _P, _F, _F, _F, _F, _I, _P]
        L.orc_eval_grid_f64.argtypes = [_P, _P, _D, _D, _D, _D, _I, _P]
        L.orc_compute_k_f32.argtypes = [_P, _I]
        L.orc_compute_k_f32.restype = _F
        L.orc_compute_k_f64.argtypes = [_P, _I]
        L.orc_compute_k_f64.restype = _D
        L.orc_dist_query_f32.argtypes = [_P, _P, _P, _P, _P, _P, _I, _I, _I, _I, _P, _P, _P, _P]
        L.orc_dist_query_f32.restype = _I
        L.orc_dist_query_f64.argtypes = [_P, _P, _P, _P, _P, _P, _I, _I, _I, _I, _P, _P, _P, _P]
        L.orc_dist_query_f64.restype = _I
        qargs = [_P, _P, _P, _P, _P, _P, _I, _I, _I, _I, _I, _I, _LL, _P, _P, _LL, _P, _P, _P, _LL]
        L.orc_inter_query_f32.argtypes = qargs
        L.orc_inter_query_f32.restype = _I
        L.orc_inter_query_f64.argtypes = qargs
        L.orc_inter_query_f64.restype = _I
        L.orc_newton_distance.argtypes = [_P, _P, _P, _P, _P, _P, _P]
        L.orc_newton_point.argtypes = [_P, _P, _P, _P, _P, _P, _P]
        L.orc_region_cells_f32.argtypes = [_P, _P, _P, _I, _F, _P, _P]
        L.orc_region_cells_f64.argtypes = [_P, _P, _P, _I, _D, _P, _P]

    def eval_grid(self, surf, ustep, vstep, ustart, vstart, nuv, dtype=np.float32):
        out = np.zeros(nuv * nuv * 18, dtype=dtype)
        fn = self.lib.orc_eval_grid_f32 if dtype == np.float32 else self.lib.orc_eval_grid_f64
        fn(_p(_i32(surf.ivec)), _p(_f32(surf.data)), ustep, vstep, ustart, vstart, nuv, _p(out))
        return out

    def compute_k(self, records, nuv):
        if records.dtype == np.float32:
            return np.float32(self.lib.orc_compute_k_f32(_p(_f32(records)), nuv))
        return np.float64(self.lib.orc_compute_k_f64(_p(_f64(records)), nuv))

    def dist_query(self, a, b, rect1, rect2, nuv0, nuv_refine=16, k=8, rounds=4, dtype=np.float32):
        lim = max(1, k)
        kth = np.zeros(rounds, dtype=dtype)
        npairs = np.zeros(rounds, dtype=np.int32)
        pairs = np.full(rounds * lim * 3, -1, dtype=np.int32)
        starts = np.zeros(lim * 4, dtype=np.float64)
        conv = _f32 if dtype == np.float32 else _f64
        fn = self.lib.orc_dist_query_f32 if dtype == np.float32 else self.lib.orc_dist_query_f64
        nr = fn(_p(_i32(a.ivec)), _p(_f32(a.data)), _p(conv(rect1)), _p(_i32(b.ivec)), _p(_f32(b.data)),
                _p(conv(rect2)), nuv0, nuv_refine, k, rounds, _p(kth), _p(npairs), _p(pairs), _p(starts))
        per_round = [pairs[r * lim * 3:(r * lim + int(npairs[r])) * 3].reshape(-1, 3) for r in range(nr)]
        last = int(npairs[nr - 1]) if nr else 0
        return dict(rounds=nr, kth_d2=kth[:nr], npairs=npairs[:nr], pairs=per_round,
                    starts=starts[:last * 4].reshape(-1, 4))

    def inter_query(self, a, b, rect1, rect2, nuv0, nuv_refine=16, use_k=1, rounds=6, halve_threshold=512,
                    min_nuv=4, max_pairs=1 << 26, pair_cap=1 << 22, dtype=np.float32, starts_cap=0):
        counts = np.zeros(rounds, dtype=np.int64)
        pairs = np.zeros(pair_cap * 3, dtype=np.int32)
        written = ctypes.c_longlong(0)
        pads = np.zeros(2, dtype=dtype)
        starts = np.zeros(starts_cap * 4, dtype=np.float64) if starts_cap else None
        conv = _f32 if dtype == np.float32 else _f64
        fn = self.lib.orc_inter_query_f32 if dtype == np.float32 else self.lib.orc_inter_query_f64
        nr = fn(_p(_i32(a.ivec)), _p(_f32(a.data)), _p(conv(rect1)), _p(_i32(b.ivec)), _p(_f32(b.data)),
                _p(conv(rect2)), nuv0, nuv_refine, use_k, rounds, halve_threshold, min_nuv, max_pairs,
                _p(counts), _p(pairs), pair_cap, ctypes.byref(written), _p(pads), _p(starts), starts_cap)
        if nr < 0:
            raise RuntimeError("oracle intersection exceeded max_pairs")
        per_round = []
        off = 0
        for r in range(nr):
            c = int(counts[r])
            if off + c <= pair_cap:
                per_round.append(pairs[off * 3:(off + c) * 3].reshape(-1, 3))
            else:
                per_round.append(None)
            off += c
        out = dict(rounds=nr, counts=counts[:nr], pairs=per_round, pads=pads)
        if starts_cap:
            last = min(int(counts[nr - 1]), starts_cap) if nr else 0
            out["starts"] = starts[:last * 4].reshape(-1, 4)
        return out

    def newton_distance(self, a, b, dom, x0):
        out = np.zeros(11, np.float64)
        self.lib.orc_newton_distance(_p(_i32(a.ivec)), _p(_f32(a.data)), _p(_i32(b.ivec)), _p(_f32(b.data)),
                                     _p(_f64(dom)), _p(_f64(x0)), _p(out))
        return out

    def newton_point(self, a, b, dom, x0):
        out = np.zeros(8, np.float64)
        self.lib.orc_newton_point(_p(_i32(a.ivec)), _p(_f32(a.data)), _p(_i32(b.ivec)), _p(_f32(b.data)),
                                  _p(_f64(dom)), _p(_f64(x0)), _p(out))
        return out

    def region_cells(self, surf, rect, nuv, padding=0.0, radii=True, dtype=np.float32):
        n = (nuv - 1) * (nuv - 1) * 3
        c = np.zeros(n, dtype=dtype)
        r = np.zeros(n, dtype=dtype) if radii else None
        conv = _f32 if dtype == np.float32 else _f64
        fn = self.lib.orc_region_cells_f32 if dtype == np.float32 else self.lib.orc_region_cells_f64
        fn(_p(_i32(surf.ivec)), _p(_f32(surf.data)), _p(conv(rect)), nuv, padding, _p(c), _p(r))
        return c, r


@contextlib.contextmanager
def capture_stdout():
    """Capture what C code writes to file descriptor 1."""
    libc = ctypes.CDLL(None)
    libc.fflush(None)
    saved = os.dup(1)
    with tempfile.TemporaryFile(mode="w+b") as tmp:
        os.dup2(tmp.fileno(), 1)
        box = {}
        try:
            yield box
        finally:
            libc.fflush(None)
            os.dup2(saved, 1)
            os.close(saved)
            tmp.seek(0)
            box["text"] = tmp.read().decode(errors="replace")


class Reference:
    """The reference VERSION5 compiled from its own sources (oracle/_ref)."""

    def __init__(self, path: Path | str = REF_SO):
        self.lib = ctypes.CDLL(str(path))
        L = self.lib
        L.refp_minimum_distance.argtypes = [_P, _P, _I, _P, _P, _P, _I, _P, _I, _I, _I, _I]
        L.refp_minimum_distance.restype = _F
        L.refp_dist_round1.argtypes = [_P, _P, _I, _P, _P, _P, _I, _P, _I, _I, _P, _P, _P, _I, _P, _P]
        L.refp_dist_round1.restype = _I
        L.refp_eval_grid.argtypes = [_P, _P, _F, _F, _F, _F, _I, _P]
        L.refp_eval_with_cuda.argtypes = [_P, _P, _I, _F, _F, _F, _F, _I, _P]
        L.refp_compute_k.argtypes = [_P, _I]
        L.refp_compute_k.restype = _F
        L.refp_intersection.argtypes = [_P, _P, _I, _P, _P, _P, _I, _P, _I, _I, _I]
        L.refp_inter_round1.argtypes = [_P, _P, _I, _P, _P, _P, _I, _P, _I, _I, _P, _P, _I, _P, _P, _P, _P]
        L.refp_inter_round1.restype = _I

    @staticmethod
    def available(path: Path | str = REF_SO) -> bool:
        return Path(path).exists()

    def face(self, name: str):
        """(ivec int32[7], data float32) of a compiled reference input such as
        ``inter_case3_obj1`` (struct NurbsFace, include/nurbs_data.hpp:1-10)."""
        class _Face(ctypes.Structure):
            _fields_ = [("ivec", ctypes.POINTER(ctypes.c_int)), ("ndata", ctypes.c_int),
                        ("data", ctypes.POINTER(ctypes.c_float))]
        f = _Face.in_dll(self.lib, name)
        ivec = np.ctypeslib.as_array(f.ivec, shape=(7,)).astype(np.int32).copy()
        data = np.ctypeslib.as_array(f.data, shape=(f.ndata,)).astype(np.float32).copy()
        return ivec, data

    def minimum_distance(self, a, b, rect1, rect2, nuv0, nuv_refine=16, k=8, rounds=4, quiet=True):
        args = (_p(_i32(a.ivec)), _p(_f32(a.data)), a.ndata, _p(_f32(rect1)), _p(_i32(b.ivec)), _p(_f32(b.data)),
                b.ndata, _p(_f32(rect2)), nuv0, nuv_refine, k, rounds)
        if quiet:
            with capture_stdout():
                return np.float32(self.lib.refp_minimum_distance(*args))
        return np.float32(self.lib.refp_minimum_distance(*args))

    def dist_round1(self, a, b, rect1, rect2, nuv0, k=8):
        ncell = (nuv0 - 1) ** 2
        cap = max(1, k)
        d2 = np.zeros(cap, np.float32)
        ii = np.zeros(cap, np.int32)
        jj = np.zeros(cap, np.int32)
        c1 = np.zeros(3 * ncell, np.float32)
        c2 = np.zeros(3 * ncell, np.float32)
        n = self.lib.refp_dist_round1(_p(_i32(a.ivec)), _p(_f32(a.data)), a.ndata, _p(_f32(rect1)),
                                      _p(_i32(b.ivec)), _p(_f32(b.data)), b.ndata, _p(_f32(rect2)), nuv0, k,
                                      _p(d2), _p(ii), _p(jj), cap, _p(c1), _p(c2))
        return dict(d2=d2[:n], i=ii[:n], j=jj[:n], centers1=c1, centers2=c2)

    def eval_grid(self, surf, ustep, vstep, ustart, vstart, nuv):
        out = np.zeros(nuv * nuv * 18, np.float32)
        self.lib.refp_eval_grid(_p(_i32(surf.ivec)), _p(_f32(surf.data)), ustep, vstep, ustart, vstart, nuv, _p(out))
        return out

    def eval_with_cuda(self, surf, ustep, vstep, ustart, vstart, nuv):
        out = np.zeros(nuv * nuv * 18, np.float32)
        self.lib.refp_eval_with_cuda(_p(_i32(surf.ivec)), _p(_f32(surf.data)), surf.ndata, ustep, vstep, ustart,
                                     vstart, nuv, _p(out))
        return out

    def compute_k(self, records, nuv):
        return np.float32(self.lib.refp_compute_k(_p(_f32(records)), nuv))

    def intersection(self, a, b, rect1, rect2, nuv0, nuv_refine=16, use_k=1):
        """Runs the unmodified intersection(); returns per-round counts and
        the two printed initial paddings (from its stdout)."""
        with capture_stdout() as box:
            self.lib.refp_intersection(_p(_i32(a.ivec)), _p(_f32(a.data)), a.ndata, _p(_f32(rect1)),
                                       _p(_i32(b.ivec)), _p(_f32(b.data)), b.ndata, _p(_f32(rect2)), nuv0,
                                       nuv_refine, use_k)
        text = box["text"]
        counts = [int(m.group(2)) for m in re.finditer(r"Round (\d+): overlap pairs = (\d+)", text)]
        pads = [float(m.group(1)) for m in re.finditer(r"Compute_K initial side\d raw=\S+ scale=\S+ padding=(\S+)", text)]
        return dict(counts=np.array(counts, dtype=np.int64), pads=pads, text=text)

    def inter_round1(self, a, b, rect1, rect2, nuv0, use_k=1, cap=1 << 22):
        ncell = (nuv0 - 1) ** 2
        ii = np.zeros(cap, np.int32)
        jj = np.zeros(cap, np.int32)
        c1 = np.zeros(3 * ncell, np.float32)
        r1 = np.zeros(3 * ncell, np.float32)
        c2 = np.zeros(3 * ncell, np.float32)
        r2 = np.zeros(3 * ncell, np.float32)
        n = self.lib.refp_inter_round1(_p(_i32(a.ivec)), _p(_f32(a.data)), a.ndata, _p(_f32(rect1)),
                                       _p(_i32(b.ivec)), _p(_f32(b.data)), b.ndata, _p(_f32(rect2)), nuv0, use_k,
                                       _p(ii), _p(jj), cap, _p(c1), _p(r1), _p(c2), _p(r2))
        return dict(i=ii[:min(n, cap)], j=jj[:min(n, cap)], n=n, centers1=c1, radii1=r1, centers2=c2, radii2=r2)


def parse_reference_face(path: Path | str):
    """Read a reference ``examples/data/inter_case*_data.cu`` array file as
    text (ivec, ndata, data) and return (ivec int32[7], data float32)."""
    text = Path(path).read_text()
    iv = re.search(r"ivec\[7\]\s*=\s*\{([^}]*)\}", text)
    da = re.search(r"data\[\d+\]\s*=\s*\{([^}]*)\}", text, re.S)
    ivec = np.array([int(x) for x in iv.group(1).split(",")], dtype=np.int32)
    vals = [x.strip().rstrip("f") for x in da.group(1).split(",") if x.strip()]
    data = np.array([float(x) for x in vals], dtype=np.float64).astype(np.float32)
    return ivec, data
