"""The oracle itself: pinned against the reference's golden output and
against the reference's own cpu_solver.c compiled unmodified (oracle/_ref)."""
from __future__ import annotations

import numpy as np
import pytest

import egsolver_b200 as eg
from egsolver_b200 import workloads
from oracle import oracle as O
from tests.conftest import by_ext, to_top32

TOP32 = O.TOP32


def small_games():
    """Seeded small games covering the generator kinds and owner mixes."""
    out = []
    for seed in range(6):
        out.append(eg.generate(1, 60 + 7 * seed, 3, 5 + seed, 100 + seed))
        out.append(eg.generate(2, 200 + 30 * seed, 40, 50, 200 + seed))
        out.append(eg.generate(4, 150, 12, 20, 300 + seed, param=2))
        out.append(eg.generate(5, 180, 30, 9, 400 + seed, param=6))
    out.append(eg.generate(3, 40, 39, 7, 500))
    return out


def test_golden_clique_eg_int32(golden_clique):
    game, sol = golden_clique
    f, st = O.eg_solve(game, bits=32)
    assert by_ext(game, f) == sol
    assert st["finished"]


def test_golden_clique_eg_int64(golden_clique):
    game, sol = golden_clique
    f, _ = O.eg_solve(game, bits=64)
    assert by_ext(game, to_top32(f)) == sol


def test_golden_clique_eg0_serial(golden_clique):
    """EG0 (Jacobi) reproduces the reference's recorded run: 2011 sweeps."""
    game, sol = golden_clique
    f, st = O.eg0_solve(game, threads=0)
    assert by_ext(game, f) == sol
    assert st["loops"] == 2011


def test_golden_fig2(golden_fig2):
    game, sol = golden_fig2
    f, st = O.eg_solve(game, bits=32)
    assert by_ext(game, f) == sol
    assert st["mg"] == 7


def test_ominus_edges():
    mg = 10
    for bits in (32, 64):
        top = TOP32 if bits == 32 else O.TOP64
        assert O.ominus(0, 5, mg, bits) == 0          # max(0, a - b)
        assert O.ominus(3, -4, mg, bits) == 7
        assert O.ominus(6, -4, mg, bits) == 10        # a - b == MG is still finite
        assert O.ominus(7, -4, mg, bits) == top       # a - b > MG saturates
        assert O.ominus(top, 3, mg, bits) == top      # TOP stays TOP
        assert O.ominus(top, -3, mg, bits) == top


def test_mg_and_max_loop_match_reference_formulas(golden_clique):
    game, _ = golden_clique
    assert O.mg(game) == 1992  # reference sol.txt:32 prints MG_pesi=1992
    assert O.max_loop(game.num_edges, game.num_nodes, 1992) == 6958056000001  # sol.txt:32 max_loop
    assert eg.compute_mg(game) == 1992
    assert eg.default_max_loop(game.num_edges, game.num_nodes, 1992) == 6958056000001
    assert O.max_loop(10**9, 10**9, 10**9) == 2**63 - 2


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built (needs the reference tree once)")
def test_restatement_equals_reference_cpu_solver():
    """Same credits AND the same number of worklist pops as the unmodified
    reference EG_cpu_solver, on every small game."""
    for g in small_games():
        ref_f, ref_st = O.ref_cpu_solve(g, "eg")
        f32, st32 = O.eg_solve(g, bits=32)
        f64, _ = O.eg_solve(g, bits=64)
        np.testing.assert_array_equal(f32, ref_f)
        np.testing.assert_array_equal(to_top32(f64), ref_f)
        assert st32["processed"] == ref_st["processed"]
        assert st32["mg"] == ref_st["mg"]


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")
def test_eg0_equals_reference_eg0_single_thread():
    for g in small_games()[:8]:
        ref_f, ref_st = O.ref_cpu_solve(g, "eg0", threads=1)
        f, st = O.eg0_solve(g, threads=0)
        np.testing.assert_array_equal(f, ref_f)
        assert st["processed"] == ref_st["processed"]
        fo, _ = O.eg0_solve(g, threads=4)
        np.testing.assert_array_equal(fo, ref_f)


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")
def test_csr2csc_equals_reference_host_csr2csc():
    rng = np.random.default_rng(7)
    for nrow, ncol, nnz in ((4, 5, 9), (50, 30, 400), (300, 1000, 5000), (7, 7, 0)):
        counts = rng.multinomial(nnz, np.ones(nrow) / nrow)
        rp = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
        col = rng.integers(0, ncol, nnz).astype(np.int32)
        val = rng.integers(-99, 99, nnz).astype(np.int32)
        a = O.csr2csc(nrow, ncol, rp, col, val)
        b = O.ref_host_csr2csc(nrow, ncol, rp, col, val)
        for x, y in zip(a, b):
            np.testing.assert_array_equal(x, y)


def test_cfg1_oracle_is_a_fixed_point():
    g = workloads.cfg1()
    f, st = O.eg_solve(g, bits=64)
    assert st["finished"]
    assert O.count_inconsistent(g, f) == 0
    # the least fixed point is below any other: lifting from f changes nothing
    f32, _ = O.eg_solve(g, bits=32)
    np.testing.assert_array_equal(to_top32(f), f32)


def test_count_inconsistent_detects_a_planted_error():
    g = workloads.cfg1()
    f, _ = O.eg_solve(g, bits=64)
    bad = f.copy()
    i = int(np.flatnonzero(bad < O.TOP64)[0])
    bad[i] += 1
    assert O.count_inconsistent(g, bad) >= 1


def test_ieee1394_model_checking_game_matches_the_reference_driver(golden_ieee1394):
    game, sol = golden_ieee1394
    assert game.num_nodes == 571378 and game.num_edges == 996970
    f, st = O.eg_solve(game, bits=32)
    assert st["finished"] and st["loops"] == 64725026  # the reference driver's own pop count
    assert by_ext(game, f) == sol


@pytest.mark.parametrize("args", [(1, 500, 4, 10, 7, 0), (2, 4096, 4095, 1000, 0xE6 + 2, 0), (3, 60, 59, 500, 9, 0),
                                  (4, 700, 16, 100, 11, 2), (5, 900, 256, 40, 12, 6)])
def test_restated_generator_equals_the_library_generator(args):
    """The reference arm builds its games with the oracle's restated generator;
    it must produce the library's games exactly."""
    kind, n, deg, wmax, seed, param = args
    a = eg.generate(kind, n, deg, wmax, seed, param=param)
    b = O.generate(kind, n, deg, wmax, seed, param=param)
    assert a.num_nodes0 == b.num_nodes0
    np.testing.assert_array_equal(a.row_ptr, b.row_ptr)
    np.testing.assert_array_equal(a.succ, b.succ)
    np.testing.assert_array_equal(a.weight, b.weight)


def test_oracle_workloads_equal_the_package_workloads():
    from egsolver_b200 import workloads

    for name, n in (("cfg1", 0), ("cfg2", 1 << 12), ("cfg3", 0)):
        a = getattr(workloads, name)(n) if n else getattr(workloads, name)()
        b = O.workload(name, n)
        np.testing.assert_array_equal(a.row_ptr, b.row_ptr)
        np.testing.assert_array_equal(a.succ, b.succ)
        np.testing.assert_array_equal(a.weight, b.weight)
