"""Full-size parity on the GPU: the n = 2^20 benchmark game (cfg2) against
the digest of the oracle's solve (tests/golden/cfg2_full_size.json, made by
tests/golden/make_full_size_golden.py), with the default schedule (dense
rounds) and with frontier rounds only."""
from __future__ import annotations

import json

import numpy as np
import pytest

import egsolver_b200 as eg
from egsolver_b200 import workloads
from tests.conftest import GOLDEN
from tests.golden.make_full_size_golden import digest

pytestmark = pytest.mark.gpu

PIN = GOLDEN / "cfg2_full_size.json"


@pytest.fixture(scope="module")
def cfg2_resident():
    game = workloads.cfg2()
    with eg.ResidentGame(game) as r:
        yield game, r


@pytest.mark.parametrize("kw", [dict(), dict(direction=eg.DIRECTION_SPARSE)], ids=["default", "frontier"])
def test_cfg2_full_size_matches_the_pin(cfg2_resident, kw):
    if not PIN.exists():
        pytest.skip("no full-size pin committed (tests/golden/make_full_size_golden.py makes it)")
    pin = json.loads(PIN.read_text())
    game, r = cfg2_resident
    assert pin["n"] == game.num_nodes and pin["m"] == game.num_edges
    r.solve(**kw)
    got = digest(r.credits(64))
    for key in ("num_top", "sum_finite", "max_finite", "sha256"):
        assert got[key] == pin[key], key
