"""Shared fixtures.  GPU tests carry @pytest.mark.gpu; the CPU suite runs with
-m "not gpu".  Tests compare the CUDA path (through the C ABI) with the CPU
oracle (oracle/), which is pinned against the reference's golden vectors."""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = Path(__file__).resolve().parent / "golden"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")
    config.addinivalue_line("markers", "slow: long-running parity case")


@pytest.fixture(scope="session")
def orc():
    import oracle
    if not oracle.ORACLE_SO.exists():
        import subprocess
        subprocess.run(["make", "-C", str(ROOT / "oracle")], check=True)
    return oracle.Oracle()


@pytest.fixture(scope="session")
def ref():
    import oracle
    if not oracle.Reference.available():
        pytest.skip("reference build oracle/_ref is absent (needs the reference checkout at build time)")
    return oracle.Reference()


@pytest.fixture(scope="session")
def gpu_ctx():
    import jsi_cad_next_versions_b200 as J
    ctx = J.Context(0)
    yield ctx
    ctx.close()


def load_npz(name: str):
    return dict(np.load(GOLDEN / name))


def surface_from(ivec, data):
    from jsi_cad_next_versions_b200 import synth
    return synth.Surface(np.asarray(ivec, np.int32), np.asarray(data, np.float32))


def rect32(s):
    return np.array(s.rect(), np.float32)
