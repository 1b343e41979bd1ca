"""Surface ingestion: the reference's interchange format and a binary cache.

* C-array source (what the reference's EGADS/IGES converter writes,
  JSI_CAD_NEXT_VERSION5/utils/nurbs_tool.cpp:95-118, and what its
  examples/data/*_data.cu files hold): ``static int ivec[7] = {...};
  static int ndata = N; static float data[N] = {...};`` followed by a
  ``struct NurbsFace`` definition.  ``read_face_source`` parses it with each
  decimal literal rounded once, correctly, to float32 (as the C compiler does);
  ``write_face_source`` emits it with 9 significant digits (float32
  round-trip exact).
* Binary cache (``save_cache`` / ``load_cache``): b"JSIS", version 1, count,
  then per surface int32 ivec[7], int32 ndata, float32 data[ndata], all
  little-endian: the resident set of a serving process in one file.
"""
from __future__ import annotations

import re
import struct
from fractions import Fraction
from pathlib import Path

import numpy as np

from .synth import Surface

_IVEC = re.compile(r"ivec\s*\[\s*7\s*\]\s*=\s*\{([^}]*)\}")
_DATA = re.compile(r"data\s*\[\s*(\d+)\s*\]\s*=\s*\{([^}]*)\}", re.S)
_NAME = re.compile(r"struct\s+NurbsFace\s+(\w+)")
_MAGIC = b"JSIS"


def _float32_exact(token: str) -> np.float32:
    """Decimal literal -> nearest float32, ties to even (one rounding, as a C
    compiler converts a float literal).  The double-then-float conversion is
    at most one float32 ulp off; the exact value decides between neighbours."""
    x = np.float32(float(token))
    if not np.isfinite(x):
        return x
    exact = Fraction(token)
    fx = Fraction(float(x))
    if fx == exact:
        return x
    nb = np.nextafter(x, np.float32(np.inf) if exact > fx else np.float32(-np.inf), dtype=np.float32)
    fn = Fraction(float(nb))
    dx, dn = abs(exact - fx), abs(exact - fn)
    if dn < dx or (dn == dx and (int(nb.view(np.uint32)) & 1) == 0):
        return nb
    return x


def read_face_source(text: str) -> Surface:
    """Parse one surface from C-array source text."""
    iv = _IVEC.search(text)
    da = _DATA.search(text)
    if not iv or not da:
        raise ValueError("no ivec[7] / data[N] arrays in the source")
    ivec = np.array([int(x) for x in iv.group(1).replace("\n", " ").split(",") if x.strip()], dtype=np.int32)
    if ivec.shape[0] != 7:
        raise ValueError("ivec must have 7 entries")
    tokens = [t.strip().rstrip("fF") for t in da.group(2).split(",") if t.strip()]
    n = int(da.group(1))
    if len(tokens) != n:
        raise ValueError(f"data[{n}] has {len(tokens)} values")
    data = np.array([_float32_exact(t) for t in tokens], dtype=np.float32)
    name = _NAME.search(text)
    return Surface(ivec=ivec, data=data, name=name.group(1) if name else "")


def read_face_file(path: str | Path) -> Surface:
    return read_face_source(Path(path).read_text())


def write_face_source(s: Surface, name: str = "face") -> str:
    """C-array source of one surface (the reference's interchange format)."""
    iv = ", ".join(str(int(x)) for x in s.ivec)
    vals = ",\n    ".join(", ".join(f"{float(v):.9g}f" for v in s.data[i:i + 6]) for i in range(0, s.ndata, 6))
    return (f'#include "nurbs_data.hpp"\n\nstatic int ivec[7] = {{{iv}}};\nstatic int ndata = {s.ndata};\n'
            f"static float data[{s.ndata}] = {{\n    {vals}\n}};\n\n"
            f"struct NurbsFace {name} = {{\n    .ivec = ivec,\n    .ndata = ndata,\n    .data = data\n}};\n")


def save_cache(path: str | Path, surfaces) -> None:
    with open(path, "wb") as f:
        f.write(_MAGIC + struct.pack("<II", 1, len(surfaces)))
        for s in surfaces:
            f.write(np.ascontiguousarray(s.ivec, "<i4").tobytes())
            f.write(struct.pack("<i", s.ndata))
            f.write(np.ascontiguousarray(s.data, "<f4").tobytes())


def load_cache(path: str | Path) -> list[Surface]:
    raw = Path(path).read_bytes()
    if raw[:4] != _MAGIC:
        raise ValueError("not a surface cache file")
    version, count = struct.unpack_from("<II", raw, 4)
    if version != 1:
        raise ValueError(f"unsupported cache version {version}")
    off = 12
    out = []
    for _ in range(count):
        ivec = np.frombuffer(raw, "<i4", 7, off).astype(np.int32)
        off += 28
        (n,) = struct.unpack_from("<i", raw, off)
        off += 4
        data = np.frombuffer(raw, "<f4", n, off).astype(np.float32)
        off += 4 * n
        out.append(Surface(ivec=ivec, data=data))
    if off != len(raw):
        raise ValueError("trailing bytes in the cache file")
    return out
