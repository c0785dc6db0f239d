"""The ports of the reference's fixture generators (script/multi: mkclique,
mkladder, multi) against the reference's own output, byte for byte: its
shipped copies of the example game (tests/golden/ref_eg_fig2*.txt) and, where
`make -C oracle fixtures` has compiled them from the reference tree, the
reference tools themselves (oracle/_ref)."""
from __future__ import annotations

import subprocess
from pathlib import Path

import numpy as np
import pytest

import egsolver_b200 as eg
from oracle import oracle as O

GOLDEN = Path(__file__).resolve().parent / "golden"
REF = Path(O.__file__).resolve().parent / "_ref"


def test_copies_reproduce_the_shipped_fixtures():
    fig = (GOLDEN / "ref_eg_fig2.txt").read_text()
    assert eg.copies_text(fig, 2) == (GOLDEN / "ref_eg_fig2_duecopie.txt").read_text()
    assert eg.copies_text(fig, 4) == (GOLDEN / "ref_eg_fig2_quattrocopie.txt").read_text()
    two = eg.copies_text(fig, 2)
    assert eg.copies_text(two, 2) == (GOLDEN / "ref_eg_fig2_duecopie_di_duecopie.txt").read_text()


def _ref_tool(name: str) -> Path:
    p = REF / name
    if not p.exists():
        pytest.skip(f"{p} not built (make -C oracle fixtures needs the reference tree)")
    return p


@pytest.mark.parametrize("number", [1, 2, 3, 10, 250])
def test_clique_and_ladder_equal_the_reference_tools(number):
    out = subprocess.run([str(_ref_tool("mkclique")), str(number)], capture_output=True, check=True).stdout
    assert eg.clique_text(number).encode() == out
    out = subprocess.run([str(_ref_tool("mkladder")), str(number)], capture_output=True, check=True).stdout
    assert eg.ladder_text(number).encode() == out


@pytest.mark.parametrize("copies", [2, 3, 8])
def test_copies_equal_the_reference_tool(copies):
    text = eg.clique_text(40) + ""
    out = subprocess.run([str(_ref_tool("multi")), "--copies", str(copies)], input=text.encode(), capture_output=True,
                         check=True).stdout
    assert eg.copies_text(text, copies).encode() == out
    lad = eg.ladder_text(30)
    out = subprocess.run([str(_ref_tool("multi")), "--copies", str(copies)], input=lad.encode(), capture_output=True,
                         check=True).stdout
    assert eg.copies_text(lad, copies).encode() == out


def test_generated_games_solve_like_the_oracle_on_the_cpu():
    """The fixture games read back through the library's reader are ordinary
    games: the oracle solves them (clique with copies, ladder)."""
    g = eg.read_game_text(eg.copies_text(eg.clique_text(30), 2))
    assert g.num_nodes == 60
    f, st = O.eg_solve(g, bits=32)
    assert st["finished"]
    lad = eg.read_game_text(eg.ladder_text(50))
    f2, st2 = O.eg_solve(lad, bits=32)
    assert st2["finished"] and lad.num_nodes == 100
    assert O.count_inconsistent(lad, f2) == 0
    # the first player circles its own vertices at no cost; the second
    # player's vertices chain -1 steps around the ladder forever
    own = lad.owners()
    assert np.all(f2[own == 0] == 0) and np.all(f2[own == 1] == O.TOP32)
