"""GPU parity: the CUDA solver, called through the C-ABI, against the oracle
(bit-exact credits, TOP set and winning region) on golden fixtures, the
benchmark configurations at oracle-friendly sizes, and edge cases."""
from __future__ import annotations

import subprocess

import numpy as np
import pytest

import egsolver_b200 as eg
from egsolver_b200 import workloads
from oracle import oracle as O
from tests.conftest import GOLDEN, ROOT, by_ext, load_solution, to_top32

pytestmark = pytest.mark.gpu

VARIANTS = [
    dict(variant=eg.VARIANT_AUTO),
    dict(variant=eg.VARIANT_THREAD),
    dict(variant=eg.VARIANT_WARP, lanes_per_vertex=2),
    dict(variant=eg.VARIANT_WARP, lanes_per_vertex=4),
    dict(variant=eg.VARIANT_WARP, lanes_per_vertex=8),
    dict(variant=eg.VARIANT_WARP, lanes_per_vertex=16),
    dict(variant=eg.VARIANT_WARP, lanes_per_vertex=32),
    dict(variant=eg.VARIANT_CTA),
    dict(variant=eg.VARIANT_SMEM),
]


def vid(v):
    return "-".join(f"{k}{x}" for k, x in v.items())


def assert_exact(game, gpu: np.ndarray, bits: int):
    ref, st = O.eg_solve(game, bits=64)
    assert st["finished"]
    if bits == 32:
        np.testing.assert_array_equal(gpu.astype(np.int64), to_top32(ref))
    else:
        np.testing.assert_array_equal(gpu, ref)
    # winning region of player 0 = finite credits
    np.testing.assert_array_equal(gpu < (2**31 - 1 if bits == 32 else 2**63 - 1), ref < O.TOP64)


@pytest.mark.parametrize("v", VARIANTS, ids=vid)
@pytest.mark.parametrize("bits", [32, 64])
def test_fig2_known_answer(golden_fig2, v, bits):
    game, sol = golden_fig2
    f, st = eg.solve(game, credit_bits=bits, **v)
    assert by_ext(game, to_top32(f) if bits == 64 else f) == sol
    assert st.mg == 7


@pytest.mark.parametrize("v", [VARIANTS[0], VARIANTS[6], VARIANTS[7], VARIANTS[1], VARIANTS[8]], ids=vid)
def test_golden_clique_500_cp4(golden_clique, v):
    game, sol = golden_clique
    f, st = eg.solve(game, credit_bits=32, **v)
    assert by_ext(game, f) == sol
    assert st.num_top == 1000
    assert st.mg == 1992


@pytest.mark.parametrize("v", VARIANTS, ids=vid)
def test_cfg1_all_variants(v):
    game = workloads.cfg1()
    for bits in (32, 64):
        f, st = eg.solve(game, credit_bits=bits, **v)
        assert_exact(game, f, bits)
        assert st.edges >= st.lifts * 4


@pytest.mark.parametrize("v", [VARIANTS[0], VARIANTS[5], VARIANTS[6], VARIANTS[7]], ids=vid)
def test_cfg3_clique_2000(v):
    game = workloads.cfg3()
    f, _ = eg.solve(game, credit_bits=32, **v)
    assert_exact(game, f, 32)


@pytest.mark.parametrize("n", [1 << 12, 1 << 14])
def test_cfg2_scaled_int64(n):
    game = workloads.cfg2(n)
    f, st = eg.solve(game, credit_bits=64)
    assert_exact(game, f, 64)
    assert st.rounds > 1


def test_cfg2_scaled_variants_and_buckets():
    game = workloads.cfg2(1 << 12)
    ref, _ = O.eg_solve(game, bits=64)
    for v in VARIANTS[1:] + [dict(small_max_deg=2, large_min_deg=40), dict(small_max_deg=64, large_min_deg=65)]:
        f, _ = eg.solve(game, credit_bits=64, **v)
        np.testing.assert_array_equal(f, ref, err_msg=str(v))


# Round kinds of the lean grid layout.  With dense_permille=1 and
# sparse_permille=1000 every frontier round with a few raises hands over to
# the dense kernel, whose next round records and hands back through a seed
# step, so every transition runs many times in one solve.
DIRECTIONS = [
    dict(direction=eg.DIRECTION_SPARSE),
    dict(direction=eg.DIRECTION_DENSE),
    dict(direction=eg.DIRECTION_SWITCH),
    dict(direction=eg.DIRECTION_SWITCH, dense_permille=1, sparse_permille=1000),
    dict(direction=eg.DIRECTION_SWITCH, dense_permille=1, sparse_permille=1),
]


@pytest.fixture(scope="module")
def cfg2_2e14():
    game = workloads.cfg2(1 << 14)
    ref, _ = O.eg_solve(game, bits=64)
    return game, ref


@pytest.mark.parametrize("d", DIRECTIONS, ids=vid)
@pytest.mark.parametrize("bits", [32, 64])
def test_round_kinds_give_identical_credits(cfg2_2e14, d, bits):
    game, ref = cfg2_2e14
    f, st = eg.solve(game, credit_bits=bits, **d)
    if bits == 32:
        np.testing.assert_array_equal(f.astype(np.int64), to_top32(ref))
    else:
        np.testing.assert_array_equal(f, ref)
    assert st.grid > 1  # the grid kernel, not the one-CTA one
    sweeps = 4  # default sweeps per dense round; dense_rounds counts sweeps
    if d["direction"] == eg.DIRECTION_SPARSE:
        assert st.dense_rounds == 0
    elif d["direction"] == eg.DIRECTION_DENSE:
        assert st.dense_rounds == sweeps * st.rounds
    elif d.get("sparse_permille") == 1000:
        # frontier, dense, recording dense, seed + frontier, ...
        assert st.rounds // 3 <= st.dense_rounds // sweeps < st.rounds


# Data paths of the dense rounds: 64-bit credits with a shuffle scan, or
# (narrow, when MG + max|w| fits) 32-bit credits with warp reductions; 8-byte
# or 16-byte edge pairs.
DENSE_PATHS = [dict(), dict(wide_pairs=True), dict(narrow=True), dict(narrow=True, wide_pairs=True),
               dict(dense_depth=1), dict(dense_depth=1, narrow=True, wide_pairs=True), dict(dense_sweeps=2),
               dict(dense_sweeps=2, narrow=True, dense_depth=1), dict(dense_sweeps=3), dict(dense_sweeps=4),
               dict(dense_sweeps=4, narrow=True, dense_depth=1)]


@pytest.mark.parametrize("d", DENSE_PATHS, ids=lambda d: vid(d) or "default")
@pytest.mark.parametrize("direction", [eg.DIRECTION_SWITCH, eg.DIRECTION_DENSE])
def test_dense_data_paths_give_identical_credits(cfg2_2e14, d, direction):
    game, ref = cfg2_2e14
    f, st = eg.solve(game, credit_bits=64, direction=direction, **d)
    np.testing.assert_array_equal(f, ref)
    assert st.credit_bits == (32 if d.get("narrow") else 64)
    assert st.dense_rounds > 0 and st.dense_launches >= 1


def big_weight_game():
    """cfg2 at n = 2^14 with weights scaled so that MG fits 31 bits but
    MG + max|w| does not: 32-bit credits must take the 64-bit difference."""
    g = workloads.cfg2(1 << 14)
    w = g.weight.astype(np.int64) * 302
    deg = np.diff(g.row_ptr)
    src = np.repeat(np.arange(g.num_nodes), deg)
    worst = np.zeros(g.num_nodes, np.int64)
    np.maximum.at(worst, src, np.maximum(0, -w))
    v = int(np.argmax(worst))
    j = g.row_ptr[v] + int(np.argmin(w[g.row_ptr[v]:g.row_ptr[v + 1]]))
    w[j] = -(worst[v] + (2**31 - 1) - 150000 - worst.sum())
    return eg.Game(row_ptr=g.row_ptr, succ=g.succ, weight=w.astype(np.int32), num_nodes0=g.num_nodes0)


def test_dense_rounds_with_mg_near_the_32_bit_limit():
    game = big_weight_game()
    mg = eg.compute_mg(game, 64)
    assert mg <= 2**31 - 1 < mg + int(np.abs(game.weight).max())
    ref, _ = O.eg_solve(game, bits=64)
    f32, st32 = eg.solve(game, credit_bits=32)
    assert st32.credit_bits == 32 and st32.dense_rounds > 0
    np.testing.assert_array_equal(f32.astype(np.int64), to_top32(ref))
    f64, st64 = eg.solve(game, credit_bits=64, narrow=True)
    assert st64.credit_bits == 64  # no narrowing: MG + max|w| does not fit
    np.testing.assert_array_equal(f64, ref)


@pytest.mark.parametrize("d", DIRECTIONS[1:4], ids=vid)
def test_round_kinds_on_heavy_only_clique(d):
    game = workloads.cfg3()
    f, st = eg.solve(game, credit_bits=32, **d)
    assert_exact(game, f, 32)


def test_random_small_games_bit_exact():
    kinds = [(1, 3), (2, 60), (4, 16), (5, 40)]
    for seed in range(12):
        kind, deg = kinds[seed % 4]
        g = eg.generate(kind, 64 + 37 * seed, deg, 3 + 5 * seed, 1000 + seed, param=2 if kind == 4 else 5)
        for v in (VARIANTS[0], VARIANTS[1], VARIANTS[4], VARIANTS[7], VARIANTS[8]):
            f, _ = eg.solve(g, credit_bits=64, **v)
            assert_exact(g, f, 64)


def test_owner_array_equals_split_convention():
    g = workloads.cfg1()
    ref, _ = eg.solve(g)
    # same game with vertices shuffled and owners given per vertex
    rng = np.random.default_rng(3)
    n = g.num_nodes
    perm = rng.permutation(n)  # new -> old
    inv = np.empty(n, np.int64)
    inv[perm] = np.arange(n)
    deg = np.diff(g.row_ptr)[perm]
    rp = np.concatenate([[0], np.cumsum(deg)])
    succ = np.concatenate([inv[g.succ[g.row_ptr[o]:g.row_ptr[o + 1]]] for o in perm]).astype(np.int32)
    w = np.concatenate([g.weight[g.row_ptr[o]:g.row_ptr[o + 1]] for o in perm])
    h = eg.Game(row_ptr=rp, succ=succ, weight=w, owner=g.owners()[perm])
    f, _ = eg.solve(h)
    np.testing.assert_array_equal(f, ref[perm])


def test_single_vertex_self_loops():
    # player 0 with only a negative self-loop: credit climbs past MG -> TOP
    g = eg.Game(row_ptr=[0, 1], succ=[0], weight=[-1], num_nodes0=1)
    f, st = eg.solve(g)
    assert f[0] == eg.EG_TOP64 and st.mg == 1
    # player 1 with a positive self-loop: credit 0
    g = eg.Game(row_ptr=[0, 1], succ=[0], weight=[5], num_nodes0=0)
    f, _ = eg.solve(g, credit_bits=32)
    assert f[0] == 0


def test_mg_beyond_int32_needs_64_bit_credits():
    n = 4
    w = [-(2**30), -(2**30), -(2**30), 7]
    g = eg.Game(row_ptr=np.arange(n + 1), succ=[1, 2, 3, 0], weight=w, num_nodes0=2)
    with pytest.raises(eg.EGError) as ei:
        eg.solve(g, credit_bits=32)
    assert ei.value.name == "EG_ERR_OVERFLOW"
    f, st = eg.solve(g, credit_bits=64)
    assert st.mg == 3 * 2**30
    ref, _ = O.eg_solve(g, bits=64)
    np.testing.assert_array_equal(f, ref)


def test_sink_rejected():
    g = eg.Game(row_ptr=[0, 1, 1], succ=[1], weight=[1], num_nodes0=1)
    with pytest.raises(eg.EGError) as ei:
        eg.solve(g)
    assert ei.value.name == "EG_ERR_INVALID"


def test_round_cap_gives_a_lower_bound():
    g = workloads.cfg1()
    ref, _ = O.eg_solve(g, bits=64)
    with eg.ResidentGame(g) as r:
        status, st = r.solve(raise_on_error=False, max_rounds=3)
        assert eg._ffi.STATUS_NAMES[status] == "EG_ERR_LOOPCAP"
        assert st.rounds == 3
        part = r.credits()
        assert np.all(part <= ref)
        assert np.any(part < ref)


def test_cancel_flag_stops_the_solve():
    g = workloads.cfg2(1 << 14)
    flag = eg.CancelFlag()
    try:
        flag.set(1)
        with eg.ResidentGame(g) as r:
            status, st = r.solve(raise_on_error=False, cancel=flag)
            assert eg._ffi.STATUS_NAMES[status] == "EG_ERR_CANCELLED"
            assert st.rounds == 1
            flag.set(0)
            status, _ = r.solve(raise_on_error=False, cancel=flag)
            assert status == 0
    finally:
        flag.free()


def test_timeout_stops_the_solve():
    g = workloads.cfg2(1 << 14)
    with eg.ResidentGame(g) as r:
        status, st = r.solve(raise_on_error=False, timeout_ms=0.001)
        assert eg._ffi.STATUS_NAMES[status] == "EG_ERR_TIMEOUT"
        status, _ = r.solve(raise_on_error=False)
        assert status == 0


def test_resident_game_resolve_and_keep_layout():
    g = workloads.cfg2(1 << 13)
    ref, _ = O.eg_solve(g, bits=64)
    with eg.ResidentGame(g) as r:
        r.solve()
        np.testing.assert_array_equal(r.credits(), ref)
        _, st2 = r.solve(keep_layout=True)
        np.testing.assert_array_equal(r.credits(), ref)
        _, st3 = r.solve(credit_bits=32, keep_layout=True)
        np.testing.assert_array_equal(r.credits(32).astype(np.int64), to_top32(ref))
        assert st2.kernel_launches < st3.kernel_launches + 1
        assert r.device_bytes > 0


def test_from_device_pointers_with_torch():
    torch = pytest.importorskip("torch")
    g = workloads.cfg1()
    ref, _ = eg.solve(g)
    rp = torch.from_numpy(g.row_ptr).cuda()
    sc = torch.from_numpy(g.succ).cuda()
    wt = torch.from_numpy(g.weight).cuda()
    r = eg.ResidentGame.from_device(g.num_nodes, g.num_edges, g.num_nodes0, rp.data_ptr(), sc.data_ptr(), wt.data_ptr())
    r.solve()
    ptr, bits = r.credits_device()
    assert bits == 64 and ptr != 0
    np.testing.assert_array_equal(r.credits(), ref)
    r.free()


def test_csr2csc_equals_host_csr2csc():
    rng = np.random.default_rng(11)
    for nrow, ncol, nnz in ((4, 5, 9), (100, 70, 3000), (2000, 5000, 100000), (9, 9, 0)):
        counts = rng.multinomial(nnz, np.ones(nrow) / nrow)
        rp = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
        col = rng.integers(0, ncol, nnz).astype(np.int32)
        val = rng.integers(-1000, 1000, nnz).astype(np.int32)
        got = eg.csr2csc(nrow, ncol, rp, col, val)
        want = O.csr2csc(nrow, ncol, rp, col, val)
        for a, b in zip(got, want):
            np.testing.assert_array_equal(a, b)


def test_csr2csc_of_cfg2_is_a_permutation_with_stable_columns():
    g = workloads.cfg2(1 << 18)
    cp, cr, cv = eg.csr2csc(g.num_nodes, g.num_nodes, g.row_ptr, g.succ, g.weight)
    assert cp[-1] == g.num_edges
    for c in range(0, g.num_nodes, 9973):  # rows ascending inside every column
        seg = cr[cp[c]:cp[c + 1]]
        assert np.all(np.diff(seg) >= 0)
    want = O.csr2csc(g.num_nodes, g.num_nodes, g.row_ptr, g.succ, g.weight)
    for a, b in zip((cp, cr, cv), want):
        np.testing.assert_array_equal(a, b)


@pytest.mark.skipif(not O.REF_BIN.exists(), reason="reference driver not built")
@pytest.mark.parametrize("shuffling", ["1", "32"])
def test_reference_driver_runs_unchanged_on_the_gpu(shuffling):
    """The reference's own egsolver.c, linked against this library through the
    reference-ABI shim, solves the golden game on the GPU."""
    out = subprocess.run([str(O.REF_BIN), "--gpu", "--eg", "--shuffling", shuffling, "--input",
                          str(GOLDEN / "clique_500_cp4.txt.gz")], capture_output=True, text=True, timeout=300,
                         cwd=str(ROOT))
    assert out.returncode == 0, out.stderr[-2000:]
    sol = {}
    seen = False
    for line in out.stdout.splitlines():
        if line.startswith("Solution:"):
            seen = True
            continue
        if seen and ")" in line and line.split(")")[0].isdigit():
            k, v = line.split(")")
            sol[int(k)] = int(v)
    assert sol == load_solution(GOLDEN / "clique_500_cp4.sol")


def test_ieee1394_model_checking_game(golden_ieee1394):
    """A real game from the reference's dataset (571,378 vertices, mostly
    out-degree 1 and 2) against the solution the reference's driver prints."""
    game, sol = golden_ieee1394
    f, _ = eg.solve(game, credit_bits=32)
    assert by_ext(game, f) == sol


def test_autotuner_keeps_credits_and_caches_by_shape(cfg2_2e14):
    """Tuned knobs give the oracle's credits; a second game of the same shape
    takes the cached choice without timing."""
    game, ref = cfg2_2e14
    with eg.ResidentGame(game) as r:
        knobs, rep = r.tune(rounds=120)
        assert rep["candidates"] >= 5 and not rep["from_cache"]
        assert rep["best_rate"] >= rep["default_rate"] > 0
        r.solve(**knobs)
        np.testing.assert_array_equal(r.credits(64), ref)
    with eg.ResidentGame(game) as r2:
        knobs2, rep2 = r2.tune(rounds=120)
        assert rep2["from_cache"] and knobs2 == knobs


def test_autotuner_on_a_game_without_heavy_vertices():
    """A threshold game of the batched workload (out-degree at most 16, so
    no heavy tasks; lean kernel and dense rounds) under tuned knobs."""
    g = workloads.cfg4_games(64)[13]
    p, d = workloads.cfg4_thresholds(64)
    tg = eg.threshold_game(g, int(p[13, 0]), d)
    want, _ = O.eg_solve(tg, bits=64)
    with eg.ResidentGame(tg) as r:
        f0, st0 = r.solve()
        np.testing.assert_array_equal(r.credits(64), want)
        knobs, rep = r.tune(rounds=200)
        r.solve(**knobs)
        np.testing.assert_array_equal(r.credits(64), want)
