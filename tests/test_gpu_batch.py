"""GPU parity of the batched solver: every (game, threshold) of a batch equals
the oracle's solve of the energy game with weights w*d - p."""
from __future__ import annotations

import numpy as np
import pytest

import egsolver_b200 as eg
from egsolver_b200 import workloads
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def small_batch(num=18, seed=5):
    rng = np.random.default_rng(seed)
    games = []
    for i in range(num):
        n = int(rng.integers(40, 1500))
        kind = [1, 2, 4, 5][i % 4]
        deg = {1: 3, 2: min(n - 1, 64), 4: 16, 5: 30}[kind]
        games.append(eg.generate(kind, n, deg, int(rng.integers(3, 60)), 77 + i, param=2 if kind == 4 else 6))
    return games


def check_batch(b, games, p, d):
    for g, game in enumerate(games):
        got = b.credits(g)
        for k in range(p.shape[1]):
            want, st = O.eg_solve(eg.threshold_game(game, int(p[g, k]), d), bits=64)
            assert st["finished"]
            np.testing.assert_array_equal(got[k], want, err_msg=f"game {g} threshold {k} (p={p[g, k]})")


@pytest.mark.parametrize("K", [1, 3, 8, 32])
def test_small_batch_all_thresholds(K):
    games = small_batch()
    rng = np.random.default_rng(K)
    d = 4
    p = rng.integers(-60, 61, size=(len(games), K)).astype(np.int32)
    with eg.Batch(games, thresholds=K, scale=d) as b:
        b.set_thresholds(p)
        _, st = b.solve()
        assert st.games_failed == 0 and st.num_games == len(games)
        check_batch(b, games, p, d)


def test_cfg4_games_subset():
    games = [g for g in workloads.cfg4_games(64) if g.num_nodes <= 2600][:6]
    p_all, d = workloads.cfg4_thresholds(64)
    p = p_all[: len(games)]
    with eg.Batch(games, thresholds=8, scale=d) as b:
        b.set_thresholds(p)
        _, st = b.solve()
        assert st.edges > 0
        check_batch(b, games, p, d)


def test_graph_replay_with_new_thresholds():
    games = small_batch(10, seed=9)
    d = 2
    with eg.Batch(games, thresholds=4, scale=d, use_graph=True) as b:
        for rep in range(3):
            p = np.random.default_rng(rep).integers(-30, 31, size=(len(games), 4)).astype(np.int32)
            b.set_thresholds(p)
            _, st = b.solve()
            assert st.graph_replayed == (1 if rep > 0 else 0)
            check_batch(b, games, p, d)


def test_autotuner_then_solve():
    games = small_batch(12, seed=2)
    p = np.random.default_rng(1).integers(-40, 41, size=(len(games), 8)).astype(np.int32)
    with eg.Batch(games, thresholds=8, scale=3) as b:
        b.set_thresholds(p)
        blk = b.tune()
        assert blk in (512, 1024)
        _, st = b.solve()
        assert st.block == blk
        assert st.num_units == len(games)     # K = 8: the group size stays at eight
        check_batch(b, games, p, 3)


def test_unit_variants_match_the_oracle():
    """Every kind of work unit: 32- and 64-bit credits, 4- and 8-byte slots,
    groups of 8/4/2/1 thresholds (K = 15 splits into 8 + 4 + 2 + 1), and
    hybrid credits (shared memory plus global scratch) for a game too large
    for one CTA's shared memory."""
    rng = np.random.default_rng(21)
    games = [
        eg.generate(4, 900, 9, 60, 301, param=2),        # narrow slots, 32-bit credits
        eg.generate(4, 700, 6, 20000, 302, param=2),     # |w| > 32766 -> 8-byte slots
        eg.generate(1, 600, 3, 3, 303),                  # tiny weights, big thresholds -> 64-bit credits
        eg.generate(4, 66000, 3, 5, 304, param=2),       # > 65534 rows: 8-byte slots; hybrid credits
    ]
    d = 3
    K = 15
    p = np.zeros((len(games), K), dtype=np.int32)
    p[0] = rng.integers(-150, 151, K)
    p[1] = rng.integers(-40000, 40001, K)
    p[2] = rng.integers(-(1 << 29), 1 << 29, K)         # MG far above 2^30 for positive p
    p[3] = rng.integers(-14, -2, K)                     # short climbs: the test stays quick
    with eg.Batch(games, thresholds=K, scale=d) as b:
        b.set_thresholds(p)
        _, st = b.solve()
        assert st.games_failed == 0
        # 8+4+2+1 groups per small game; the large one (credits beyond one
        # CTA's shared memory) as 15 hybrid units of one threshold
        assert st.num_units == 3 * 4 + 15
        for g, game in enumerate(games):
            got = b.credits(g)
            for k in range(K):
                tg = eg.threshold_game(game, int(p[g, k]), d)
                if game.num_nodes > 10_000:
                    assert O.count_inconsistent(tg, got[k]) == 0, f"game {g} threshold {k}"
                else:
                    want, _ = O.eg_solve(tg, bits=64)
                    np.testing.assert_array_equal(got[k], want, err_msg=f"game {g} threshold {k}")


@pytest.mark.parametrize("group_max", [1, 2, 4, 8])
def test_group_sizes_give_identical_credits(group_max):
    games = small_batch(8, seed=31)
    p = np.random.default_rng(4).integers(-50, 51, size=(len(games), 8)).astype(np.int32)
    with eg.Batch(games, thresholds=8, scale=2, group_max=group_max) as b:
        b.set_thresholds(p)
        b.solve()
        check_batch(b, games, p, 2)


def test_round_cap_marks_games():
    games = [workloads.cfg1()]
    p = np.array([[40]], dtype=np.int32)  # strongly negative weights: long climb to TOP
    with eg.Batch(games, thresholds=1, scale=1, max_rounds=2) as b:
        b.set_thresholds(p)
        status, st = b.solve(raise_on_error=False)
        assert eg._ffi.STATUS_NAMES[status] == "EG_ERR_LOOPCAP"
        rounds, gst = b.game_result(0)
        assert rounds == 2 and eg._ffi.STATUS_NAMES[gst] == "EG_ERR_LOOPCAP"


def test_owner_arrays_in_a_batch():
    g = workloads.cfg1(300)
    own = g.owners().copy()
    h = eg.Game(row_ptr=g.row_ptr, succ=g.succ, weight=g.weight, owner=own)
    p = np.array([[0, 5], [0, 5]], dtype=np.int32)
    with eg.Batch([g, h], thresholds=2, scale=1) as b:
        b.set_thresholds(p)
        b.solve()
        np.testing.assert_array_equal(b.credits(0), b.credits(1))
        check_batch(b, [g], p[:1], 1)  # the oracle takes the split convention of g


def test_cfg4_game_near_the_top_of_the_size_range():
    """A cfg4 game of 17,931 vertices at all 8 thresholds (one of them
    drives every credit to TOP, which runs into the cluster tail): two
    thresholds against the oracle's worklist solve, all eight by the
    oracle's fixed-point check."""
    games = workloads.cfg4_games(64)
    p_all, d = workloads.cfg4_thresholds(64)
    g = games[34]
    assert g.num_nodes == 17931
    with eg.Batch([g], thresholds=8, scale=d) as b:
        b.set_thresholds(p_all[34:35])
        _, st = b.solve()
        assert st.games_failed == 0
        got = b.credits(0)
    for k in range(8):
        tg = eg.threshold_game(g, int(p_all[34, k]), d)
        assert O.count_inconsistent(tg, got[k]) == 0, f"threshold {k}"
    for k in (0, 2):
        want, _ = O.eg_solve(eg.threshold_game(g, int(p_all[34, k]), d), bits=64)
        np.testing.assert_array_equal(got[k], want)


@pytest.mark.parametrize("tail_sweeps,tail_cluster", [(1, 16), (4, 8), (2, 2)])
def test_tail_shapes_give_identical_credits(tail_sweeps, tail_cluster):
    """Every (game, threshold) straight to the cluster tail, at several
    sweeps per cluster barrier and cluster sizes (CTAs past the rows of a
    small game hold empty ranges)."""
    games = small_batch(6, seed=41)
    p = np.random.default_rng(7).integers(-50, 51, size=(len(games), 4)).astype(np.int32)
    with eg.Batch(games, thresholds=4, scale=2, tail_rows=1, tail_sweeps=tail_sweeps,
                  tail_cluster=tail_cluster) as b:
        b.set_thresholds(p)
        _, st = b.solve()
        assert st.games_failed == 0 and st.tail_entries == len(games) * 4
        check_batch(b, games, p, 2)
