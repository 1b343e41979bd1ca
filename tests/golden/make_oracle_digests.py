"""Per-round pair-list digests of the oracle's intersection query on the
full-size saddle / plane configuration (two rational bicubic 32 x 32 NURBS,
nuv0 = 256, curvature padding on and off), FP32 and FP64 instantiations.

    python tests/golden/make_oracle_digests.py

The lists themselves (1.3 M first-round pairs with padding on) are too large
to commit, so oracle_inter_n256.json holds, per round, the count and the
SHA-256 of the (slot, i, j) int32 triples in (slot, i, j) order.  The oracle
is test infrastructure (oracle/jsi_oracle.cpp, pinned to the reference); the
FP32 counts are checked here against the reference's own counts
(ref_inter_synth.npz) before anything is written.
"""
from __future__ import annotations

import hashlib
import json
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402
from jsi_cad_next_versions_b200 import synth  # noqa: E402

OUT = Path(__file__).resolve().parent


def digest_pairs(p: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(p, dtype=np.int32).tobytes()).hexdigest()


def main():
    O = oracle.Oracle()
    ref = dict(np.load(OUT / "ref_inter_synth.npz"))
    C, D, _ = synth.intersection_pair_saddle_plane()
    out = {}
    for dt, name in ((np.float32, "f32"), (np.float64, "f64")):
        rc, rd = np.array(C.rect(), np.float32).astype(dt), np.array(D.rect(), np.float32).astype(dt)
        for use_k in (1, 0):
            t0 = time.time()
            r = O.inter_query(C, D, rc, rd, 256, 16, use_k, dtype=dt, pair_cap=1 << 22)
            if dt == np.float32:
                assert np.array_equal(r["counts"], ref[f"n256/k{use_k}/counts"]), (r["counts"], use_k)
            out[f"{name}/k{use_k}"] = {"counts": [int(c) for c in r["counts"]],
                                       "sha256": [digest_pairs(p) for p in r["pairs"]],
                                       "pads": [float(x) for x in r["pads"]]}
            print(name, use_k, r["counts"].tolist(), f"{time.time() - t0:.1f}s", flush=True)
    (OUT / "oracle_inter_n256.json").write_text(json.dumps(out, indent=1))


if __name__ == "__main__":
    main()
