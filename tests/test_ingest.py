"""Surface ingestion: the reference's C-array interchange format and the
binary cache."""
from __future__ import annotations

import os
from pathlib import Path

import numpy as np
import pytest

from jsi_cad_next_versions_b200 import ingest, synth

# The reference checkout (its data files are read where present, else skipped).
REF_DATA = (Path(os.environ.get("JSI_REFERENCE_ROOT", str(Path(__file__).resolve().parents[2] / "reference")))
            / "JSI_CAD_NEXT_VERSION5" / "examples" / "data")


def test_source_round_trip_is_exact():
    rng = synth.SplitMix64(8)
    for q in range(5):
        s = synth.random_surface(rng)
        back = ingest.read_face_source(ingest.write_face_source(s, f"f{q}"))
        assert np.array_equal(back.ivec, s.ivec)
        assert np.array_equal(back.data.view(np.uint32), s.data.view(np.uint32))
        assert back.name == f"f{q}"


def test_float_literals_round_once():
    # 1 + 2^-24 sits exactly between two float32 values: ties to even (1.0);
    # a hair above rounds up.
    assert ingest._float32_exact("1.000000059604644775390625") == np.float32(1.0)
    assert ingest._float32_exact("1.0000000596046447753906251") == np.nextafter(np.float32(1), np.float32(2))
    assert ingest._float32_exact("-0.85") == np.float32(-0.85)


def test_cache_round_trip(tmp_path):
    rng = synth.SplitMix64(9)
    surfs = [synth.random_surface(rng) for _ in range(7)]
    path = tmp_path / "cache.jsis"
    ingest.save_cache(path, surfs)
    back = ingest.load_cache(path)
    assert len(back) == 7
    for a, b in zip(surfs, back):
        assert np.array_equal(a.ivec, b.ivec) and np.array_equal(a.data.view(np.uint32), b.data.view(np.uint32))
    raw = path.read_bytes()
    (tmp_path / "bad").write_bytes(b"XXXX" + raw[4:])
    with pytest.raises(ValueError):
        ingest.load_cache(tmp_path / "bad")


@pytest.mark.parametrize("case,obj", [(3, 1), (3, 2), (4, 1), (4, 2), (1, 1)])
def test_reads_the_reference_data_files(ref, case, obj):
    """The reference's own examples/data files parse to the same float32 data
    its compiler produced (oracle/_ref holds the compiled arrays)."""
    path = REF_DATA / f"inter_case{case}-{obj}_data.cu"
    if not path.exists():
        pytest.skip("reference checkout absent")
    s = ingest.read_face_file(path)
    ivec, data = ref.face(f"inter_case{case}_obj{obj}")
    assert np.array_equal(s.ivec, ivec)
    assert np.array_equal(s.data.view(np.uint32), data.view(np.uint32))
