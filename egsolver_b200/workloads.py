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
