"""C-ABI library checks that need no GPU: it loads, exports every symbol
include/jsi_b200.h declares, and fails loudly (no CPU fallback) without a
device."""
from __future__ import annotations

import ctypes
import re

import pytest

from conftest import ROOT


def _declared_symbols():
    text = (ROOT / "include" / "jsi_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(jsi_[a-z0-9_]+)\s*\(", text)))


def test_header_and_binding_agree():
    from jsi_cad_next_versions_b200 import _capi
    assert sorted(_capi.EXPORTED) == _declared_symbols()


def test_library_exports_every_declared_symbol():
    from jsi_cad_next_versions_b200 import _capi
    lib = ctypes.CDLL(str(_capi.LIB_PATH))
    missing = [s for s in _declared_symbols() if not hasattr(lib, s)]
    assert not missing


def test_library_is_sm100a_build():
    data = (ROOT / "jsi_cad_next_versions_b200" / "libjsi_b200.so").read_bytes()
    assert b"sm_100a" in data


def test_status_strings_and_abi():
    from jsi_cad_next_versions_b200 import _capi
    lib = _capi.load()
    assert lib.jsi_abi_version() == 3
    assert lib.jsi_status_string(0) == b"ok"
    assert lib.jsi_status_string(-4) == b"capacity exceeded"


def test_defaults_match_reference_statics():
    """k_of_topk=8, max_layers=4, next_nuv=16 (distance_analysis.cu:33-36);
    global_nuv=16, 6 rounds, halve above 512 down to 4 (intersection.cu:36,368-370)."""
    from jsi_cad_next_versions_b200 import _capi
    lib = _capi.load()
    d = _capi.DistParams()
    lib.jsi_dist_params_default(ctypes.byref(d))
    assert (d.nuv_refine, d.k, d.rounds, d.precision, d.newton) == (16, 8, 4, 0, 0)
    i = _capi.InterParams()
    lib.jsi_inter_params_default(ctypes.byref(i))
    assert (i.nuv_refine, i.use_k, i.rounds, i.halve_threshold, i.min_nuv, i.precision) == (16, 1, 6, 512, 4, 0)


def test_no_device_is_an_error_not_a_fallback():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    import jsi_cad_next_versions_b200 as J
    with pytest.raises(J.JsiError) as e:
        J.Context(0)
    assert e.value.status == -8


def test_null_arguments_rejected():
    from jsi_cad_next_versions_b200 import _capi
    lib = _capi.load()
    assert lib.jsi_create(None, None) == -1
    assert lib.jsi_destroy(None) == -1
    assert lib.jsi_min_distance(None, None, None, None, None) == -1
    assert lib.jsi_intersect(None, None, None, None, None) == -1
    # the bulk, asynchronous and interval entry points
    assert lib.jsi_surface_upload_many(None, 0, None, None, None, None) == -1
    assert lib.jsi_surface_release_many(None, 0, None) == -1
    assert lib.jsi_surface_domains(None, 0, None, None) == -1
    assert lib.jsi_min_distance_batch(None, 0, None, None, None, None, None, None) == -1
    assert lib.jsi_submit_distance_batch(None, 0, None, None, None, None, None, None) == -1
    assert lib.jsi_wait_distance_batch(None, 0, None) == -1
    assert lib.jsi_distance_bounds(None, None, None, None, None) == -1
    assert lib.jsi_intersection_curves(None, None, None, None, None) == -1


def test_ctypes_layouts_match_the_header(tmp_path):
    """Every structure the Python mirror passes through the C ABI has the
    header's size and field offsets (a mismatch would let the library write
    past the caller's buffers)."""
    import shutil
    import subprocess
    from jsi_cad_next_versions_b200 import _capi as C
    if not shutil.which("gcc"):
        pytest.skip("no C compiler")
    structs = {"jsi_task": C.Task, "jsi_dist_params": C.DistParams, "jsi_dist_result": C.DistResult,
               "jsi_inter_params": C.InterParams, "jsi_inter_result": C.InterResult,
               "jsi_bounds_params": C.BoundsParams, "jsi_bounds_result": C.BoundsResult,
               "jsi_curve_params": C.CurveParams, "jsi_curve_result": C.CurveResult, "jsi_config": C.Config}
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "jsi_b200.h"', "int main(void) {"]
    for cname, st in structs.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in st._fields_:
            lines.append(f'  printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", f"-I{ROOT / 'include'}", str(src), "-o", str(exe)], check=True)
    got = {}
    for ln in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.splitlines():
        cname, fname, val = ln.split()
        got[(cname, fname)] = int(val)
    for cname, st in structs.items():
        assert got[(cname, "size")] == ctypes.sizeof(st), cname
        for fname, _ in st._fields_:
            assert got[(cname, fname)] == getattr(st, fname).offset, (cname, fname)
