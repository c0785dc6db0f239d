"""Shared test set-up: markers, import path, built artefacts, fixtures."""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an NVIDIA B200 (sm_100a); runs through the C-ABI library")


@pytest.fixture(scope="session", autouse=True)
def _built():
    from egsolver_b200 import build

    build.build()
    from oracle import oracle

    oracle.ensure_built()
    yield


def load_solution(path: Path) -> dict[int, int]:
    import gzip

    text = gzip.open(path, "rt").read() if path.suffix == ".gz" else path.read_text()
    out = {}
    for line in text.splitlines():
        k, v = line.split()
        out[int(k)] = int(v)
    return out


def by_ext(game, credits: np.ndarray) -> dict[int, int]:
    """Credits keyed by external vertex id (as the reference prints them)."""
    ext = game.ext_id if game.ext_id is not None else np.arange(game.num_nodes)
    return {int(e): int(c) for e, c in zip(ext, credits)}


def to_top32(f: np.ndarray) -> np.ndarray:
    """64-bit credits with TOP mapped to the reference's INT_MAX."""
    out = f.astype(np.int64).copy()
    out[f == np.iinfo(np.int64).max] = 2147483647
    return out


@pytest.fixture(scope="session")
def golden_clique():
    import egsolver_b200 as eg

    g = eg.read_game(str(GOLDEN / "clique_500_cp4.txt.gz"))
    return g, load_solution(GOLDEN / "clique_500_cp4.sol")


@pytest.fixture(scope="session")
def golden_fig2():
    import egsolver_b200 as eg

    g = eg.read_game(str(GOLDEN / "eg_fig2.txt"))
    return g, load_solution(GOLDEN / "eg_fig2.sol")


@pytest.fixture(scope="session")
def golden_ieee1394():
    """The reference's 571,378-vertex model-checking game with the solution
    its own driver prints."""
    import egsolver_b200 as eg

    g = eg.read_game(str(GOLDEN / "ieee1394_p4.txt.gz"))
    return g, load_solution(GOLDEN / "ieee1394_p4.sol.gz")
