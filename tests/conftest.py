"""Shared setup: import paths, the ``gpu`` marker, golden fixtures.

Tests marked ``gpu`` need a CUDA device and the built library
(``make -C bit-physics_b200/csrc``); they fail -- never skip -- without one,
because the engine has no CPU fallback.  Everything else runs on the CPU.
"""

from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
for p in (ROOT / "bit-physics_b200", ROOT / "oracle", ROOT / "tests"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built liblbm_d3q19.so")


def load_npz(name: str) -> dict[str, np.ndarray]:
    with np.load(GOLDEN / name) as z:
        return {k: z[k] for k in z.files}


@pytest.fixture(scope="session")
def golden_pure():
    return load_npz("pure_functions.npz")


@pytest.fixture(scope="session")
def golden_equilibrium():
    return json.loads((GOLDEN / "equilibrium.json").read_text())


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle

    oracle.build()
    return oracle
