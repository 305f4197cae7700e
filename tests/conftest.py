"""Shared test set-up: import paths for the engine binding, the generators and the CPU oracle, and the `gpu` marker.

GPU tests are marked ``@pytest.mark.gpu``; everything else runs on a CPU-only machine."""
import json
import os
import shutil
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
PKG = ROOT / "taral-lp_b200"
GOLDEN = ROOT / "tests" / "golden"
for p in (PKG, ROOT / "oracle"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def engine_lib():
    """The built engine library (built in-tree if missing)."""
    import pdhg
    if not pdhg.LIB_PATH.exists() or not pdhg.CLI_PATH.exists():
        sys.path.insert(0, str(PKG))
        import build
        build.build()
    return pdhg.lib()


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle
    oracle.build()
    return oracle.lib()


def golden(name):
    p = GOLDEN / name
    return json.loads(p.read_text()) if p.suffix == ".json" else np.load(p)


def rel(a, b):
    return abs(a - b) / max(1.0, abs(b))


class _BoundedPdhg:
    """The pdhg binding with a 120 s default time limit on whole solves, so a regression fails instead of
    running to the engine's 3600 s default."""

    def __getattr__(self, name):
        import pdhg
        return getattr(pdhg, name)

    @staticmethod
    def solve(lp, **kw):
        import pdhg
        kw.setdefault("time_limit", 120.0)
        return pdhg.solve(lp, **kw)


bounded_pdhg = _BoundedPdhg()
