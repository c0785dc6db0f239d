"""Seeded workloads of the benchmark configurations (shared by tests and bench).

seed = 0xE6 + configuration number; splitmix64 inside the library's
generator (eg_generate).  Sizes:
  cfg1  n=1000, 4 distinct successors, w in [-10,10]
  cfg2  n=2^20, out-degree floor(power law x^-2 on [1,4097)) in [1,4096]
        (mean 7.9), w in [-1000,1000]
  cfg3  complete digraph n=2000, w in [-500,500]
"""
from __future__ import annotations

from . import generate

SEED = 0xE6


def cfg1(n: int = 1000):
    return generate(1, n, 4, 10, SEED + 1)


def cfg2(n: int = 1 << 20):
    return generate(2, n, min(4096, n - 1), 1000, SEED + 2)


def cfg3(n: int = 2000):
    return generate(3, n, n - 1, 500, SEED + 3)


def cfg4_games(num_games: int = 4096, seed: int = SEED + 4):
    """Batched workload: games with n log-uniform in [1024, 65536], out-degree
    uniform in {2..16}, owners 50/50, weights uniform in [-100, 100]."""
    import numpy as np

    rng = np.random.default_rng(seed)
    ns = np.rint(np.exp(rng.uniform(np.log(1024), np.log(65536), num_games))).astype(int)
    return [generate(4, int(n), 16, 100, seed * 1_000_003 + i, param=2) for i, n in enumerate(ns)]


def cfg4_thresholds(num_games: int = 4096, k: int = 8, seed: int = SEED + 4):
    """K = 8 mean-payoff thresholds p/d per game, d = 8, p uniform in [-800, 800]."""
    import numpy as np

    rng = np.random.default_rng(seed + 1)
    return rng.integers(-800, 801, size=(num_games, k)).astype(np.int32), 8


def cfg5_requests(num: int, n_max: int = 1 << 22, seed: int = SEED + 5):
    """Served workload: request games with n log-uniform in [1000, n_max]
    (4M in the configuration), out-degree 1 + geometric (mean 6), owners
    50/50, weights uniform in [-W, W] with W log-uniform in [10, 10^4]; each
    request carries K in {4..32} thresholds p uniform in [-8W, 8W] at d = 8."""
    import numpy as np

    rng = np.random.default_rng(seed)
    out = []
    for i in range(num):
        n = int(round(float(np.exp(rng.uniform(np.log(1000), np.log(n_max))))))
        W = int(round(float(np.exp(rng.uniform(np.log(10), np.log(10_000))))))
        K = int(rng.integers(4, 33))
        p = rng.integers(-8 * W, 8 * W + 1, size=K).astype(np.int32)
        g = generate(5, n, min(256, n - 1), W, seed * 7_919 + i, param=6)
        out.append((g, p, 8))
    return out
