"""The game reader (reference text format) and writer, on the CPU."""
from __future__ import annotations

import gzip

import numpy as np
import pytest

import egsolver_b200 as eg
from tests.conftest import GOLDEN


def test_golden_clique_shape(golden_clique):
    g, _ = golden_clique
    assert g.num_nodes == 2000 and g.num_edges == 1746500
    assert g.num_nodes0 == 1000
    assert g.max_abs_weight == 1
    deg = np.diff(g.row_ptr)
    assert deg.min() == 499 and deg.max() == 1996  # reference sol.txt:21-22


def test_owner_sorted_layout(golden_fig2):
    g, _ = golden_fig2
    # file: 0 MIN, 1 MAX, 2 MIN, 3 MAX, 4 MAX -> player 0 (MAX) first: 1, 3, 4
    assert g.num_nodes0 == 3
    assert list(g.ext_id) == [1, 3, 4, 0, 2]
    # vertex "1 MAX 3:-3,4:1" -> internal 0 with successors ext 3, 4
    b, e = g.row_ptr[0], g.row_ptr[1]
    assert [int(g.ext_id[s]) for s in g.succ[b:e]] == [3, 4]
    assert list(g.weight[b:e]) == [-3, 1]


def test_text_roundtrip_random_games():
    for seed in range(5):
        g = eg.generate(2, 300, 50, 40, 11 + seed)
        h = eg.read_game_text(eg.game_to_text(g))
        np.testing.assert_array_equal(h.row_ptr, g.row_ptr)
        np.testing.assert_array_equal(h.succ, g.succ)
        np.testing.assert_array_equal(h.weight, g.weight)
        assert h.num_nodes0 == g.num_nodes0


def test_comments_names_arena_header_and_blanks():
    text = """arena 2 5;   # header with "arena" and NUMEDGES
    // a comment line
    0 MAX 1:-2,2:3 "v zero";
    % another comment
    1 MIN 0:1;
    2 MAX 2:0 ;
    """
    g = eg.read_game_text(text)
    assert g.num_nodes == 3 and g.num_edges == 4
    assert g.num_nodes0 == 2
    assert sorted(g.ext_id.tolist()) == [0, 1, 2]


def test_gzip_file(tmp_path):
    p = tmp_path / "g.txt.gz"
    with gzip.open(p, "wt") as f:
        f.write("1;\n0 MAX 1:-1;\n1 MIN 0:2;\n")
    g = eg.read_game(str(p))
    assert g.num_nodes == 2 and list(np.diff(g.row_ptr)) == [1, 1]


@pytest.mark.parametrize("text,fragment", [
    ("1;\n0 MAX 1:1;\n0 MIN 1:1;\n", "Repeated node identifier"),
    ("1;\n0 MAX 1:1;\n5 MIN 1:1;\n", "Unexpected node identifier"),
    ("1;\n0 MAX 7:1;\n1 MIN 0:1;\n", "Unexpected successor identifier"),
    ("2;\n0 MAX 1:1;\n1 MIN 0:1;\n", "Expecting 3 nodes, read 2"),
    ("1;\n0 MAX 1 1;\n1 MIN 0:1;\n", "syntax error"),
    ("1;\n0 MAX 1:1\n1 MIN 0:1;\n", "syntax error"),
    ("1;\n0 MAX 1:99999999999;\n1 MIN 0:1;\n", "out-of-range"),
    ("1;\n0 XX 1:1;\n1 MIN 0:1;\n", "syntax error"),
    ("", "syntax error"),
])
def test_reader_errors(text, fragment):
    with pytest.raises(eg.EGError) as ei:
        eg.read_game_text(text)
    assert ei.value.name == "EG_ERR_IO"
    assert fragment in str(ei.value)


def test_missing_file():
    with pytest.raises(eg.EGError) as ei:
        eg.read_game(str(GOLDEN / "does_not_exist.txt"))
    assert ei.value.name == "EG_ERR_IO"


def test_unit_and_random_weight_modes():
    text = "2;\n0 MAX 1:-5,2:7;\n1 MIN 0:3;\n2 MIN 1:-1;\n"
    g = eg.read_game_text(text, weight_mode=1)
    assert set(g.weight.tolist()) == {1}
    a = eg.read_game_text(text, weight_mode=3, rnd_lo=-4, rnd_hi=4, rnd_seed=9)
    b = eg.read_game_text(text, weight_mode=3, rnd_lo=-4, rnd_hi=4, rnd_seed=9)
    np.testing.assert_array_equal(a.weight, b.weight)
    assert a.weight.min() >= -4 and a.weight.max() <= 4


def test_binary_cache_round_trip(tmp_path):
    """The binary CSR cache gives back the game the text reader gave, and is
    used (and kept fresh) by the cached reader."""
    import os
    import time

    src = tmp_path / "g.txt"
    src.write_text(eg.copies_text(eg.clique_text(25), 3))
    want = eg.read_game(str(src))
    binf = tmp_path / "g.egb"
    eg.write_game_binary(want, str(binf))
    got = eg.read_game_binary(str(binf))
    for a in ("row_ptr", "succ", "weight", "ext_id"):
        np.testing.assert_array_equal(getattr(got, a), getattr(want, a))
    assert got.num_nodes0 == want.num_nodes0 and got.max_abs_weight == want.max_abs_weight
    # options recorded with the file must match when asked for
    with pytest.raises(eg.EGError):
        eg.read_game_binary(str(binf), weight_mode=1)
    # the cached reader writes the cache on first use and reads it afterwards
    cache = tmp_path / "c.egb"
    g1 = eg.read_game(str(src), cache=str(cache))
    assert cache.exists()
    np.testing.assert_array_equal(g1.succ, want.succ)
    # a cache that is newer than the text is trusted: prove it by a planted
    # difference in the text that the cached read does not see
    src.write_text(eg.clique_text(7))
    os.utime(cache, (time.time() + 5, time.time() + 5))
    g2 = eg.read_game(str(src), cache=str(cache))
    assert g2.num_nodes == want.num_nodes
    # a newer text replaces the cache
    os.utime(src, (time.time() + 20, time.time() + 20))
    g3 = eg.read_game(str(src), cache=str(cache))
    assert g3.num_nodes == 7


def test_binary_file_corruption_is_detected(tmp_path):
    g = eg.read_game_text(eg.ladder_text(40))
    p = tmp_path / "x.egb"
    eg.write_game_binary(g, str(p))
    raw = bytearray(p.read_bytes())
    raw[-5] ^= 0x40
    p.write_bytes(bytes(raw))
    with pytest.raises(eg.EGError) as ei:
        eg.read_game_binary(str(p))
    assert ei.value.name == "EG_ERR_IO"
    p.write_bytes(bytes(raw[:100]))
    with pytest.raises(eg.EGError):
        eg.read_game_binary(str(p))
