"""Shared fixtures.  `-m "not gpu"` runs everywhere; `-m gpu` needs a B200."""
from __future__ import annotations

import importlib.util
import json
import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
PKG_DIR = ROOT / "matrix-permanent-calculator_b200"
GOLDEN = ROOT / "tests" / "golden" / "golden.json"
# reference sources: $REF_SRC, else a `reference` directory beside this repository
REF_SRC = Path(os.environ.get("REF_SRC", ROOT.parent / "reference"))

sys.path.insert(0, str(ROOT / "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (runs the sm_100a kernels)")
    config.addinivalue_line("markers", "slow: takes more than a few seconds")


def load_package():
    """Import the engine's Python mirror (its directory name is not an identifier)."""
    if "perman_b200" in sys.modules:
        return sys.modules["perman_b200"]
    spec = importlib.util.spec_from_file_location("perman_b200", PKG_DIR / "__init__.py")
    mod = importlib.util.module_from_spec(spec)
    sys.modules["perman_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="session")
def pb():
    mod = load_package()
    if not mod.LIB_PATH.exists():
        sys.path.insert(0, str(PKG_DIR))
        import build  # noqa: F401  (matrix-permanent-calculator_b200/build.py)
        build.build()
    return mod


@pytest.fixture(scope="session")
def orc():
    from oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def ref():
    from oracle import Reference
    try:
        return Reference()
    except (FileNotFoundError, OSError) as e:
        pytest.skip(f"reference build unavailable: {e}")


@pytest.fixture(scope="session")
def golden():
    if not GOLDEN.exists():
        pytest.skip("tests/golden/golden.json not generated yet")
    with open(GOLDEN) as f:
        data = json.load(f)
    for c in data["cases"]:
        c["A"] = np.array(c["matrix"], dtype=np.float64)
    return {c["name"]: c for c in data["cases"]}


@pytest.fixture(scope="session")
def engine(pb):
    eng = pb.Engine(0)
    yield eng
    eng.close()


def rel_err(got: float, want: float) -> float:
    if want == 0:
        return abs(got)
    return abs(got - want) / abs(want)


def bernoulli(rng, n, d):
    while True:
        m = (rng.random((n, n)) < d).astype(np.float64)
        if m.any(axis=0).all() and m.any(axis=1).all():
            return m
