"""CPU model of the dense-round kernel's slice walk (eg_dense.cu: dense_slice,
compute_chunk, dense_report, k_dense_setup).

The kernel cuts the edge-pair stream into equal slices, walks each slice 32
pairs at a time with a segmented scan, carries a vertex that runs on into
the next chunk, and reports a vertex cut by a slice edge to a shared
accumulator whose last reporter finalizes it.  This test restates those
rules lane by lane and checks, for random degree sequences with padding
slots and heavy vertices and for many slice sizes, that every vertex is
finalized exactly once, with the minimum over all of its pairs, and that the
reporter count of k_dense_setup is the number of reports."""
from __future__ import annotations

import numpy as np

TOP = 10**9


def walk(P: np.ndarray, val: np.ndarray, slice_: int, nwarps: int) -> dict[int, int]:
    npairs = int(P[-1])
    n = len(P) - 1
    owner = np.repeat(np.arange(n), np.diff(P))
    end = np.zeros(npairs, bool)
    for u in range(n):
        if P[u + 1] > P[u]:
            end[P[u + 1] - 1] = True
    # k_dense_setup: slices overlapping the vertex's pairs
    nrep = {u: (P[u + 1] - 1) // slice_ - P[u] // slice_ + 1 for u in range(n) if P[u + 1] > P[u]}
    acc, rem, got = {}, dict(nrep), {}

    def report(u: int, v: int) -> None:
        acc[u] = min(acc.get(u, TOP), v)
        rem[u] -= 1
        if rem[u] == 0:
            assert u not in got
            got[u] = acc.pop(u)

    for w in range(nwarps):
        s0, s1 = min(w * slice_, npairs), min(w * slice_ + slice_, npairs)
        if s0 >= s1:
            continue
        carry_on = s0 > 0 and not end[s0 - 1]
        carry_cut, carry, u_last = carry_on, TOP, -1
        for c0 in range(s0, s1, 32):
            lanes = range(32)
            inn = [c0 + l < s1 for l in lanes]
            en = [bool(end[c0 + l]) if inn[l] else True for l in lanes]  # lanes past the end count as ends
            u = [int(owner[c0 + l]) if inn[l] else -1 for l in lanes]
            x = [int(val[c0 + l]) if inn[l] else TOP for l in lanes]
            ends = sum(1 << l for l in lanes if en[l])
            heads = ((ends << 1) | 1) & 0xFFFFFFFF
            head = [max(j for j in range(l + 1) if heads >> j & 1) for l in lanes]
            o = 1
            while o < 32:  # shuffle-up scan restricted to the lane's run
                y = [x[l - o] if l >= o else x[l] for l in lanes]
                x = [min(x[l], y[l]) if l - o >= head[l] else x[l] for l in lanes]
                o <<= 1
            if carry_on:
                x = [min(x[l], carry) if head[l] == 0 else x[l] for l in lanes]
            for l in lanes:
                if inn[l] and en[l]:
                    if head[l] == 0 and carry_cut:
                        report(u[l], x[l])
                    else:
                        assert nrep[u[l]] == 1 and u[l] not in got
                        got[u[l]] = x[l]
            open_ = not (ends >> 31 & 1)
            carry_cut = open_ and carry_cut and (ends & 0x7FFFFFFF) == 0
            carry_on, carry, u_last = open_, x[31], u[31]
        if carry_on:
            report(u_last, carry)
    # every cut vertex heard from all of its slices; the others never reported
    assert not acc and all(rem[u] == (0 if nrep[u] > 1 else 1) for u in rem)
    return got


def test_every_vertex_is_finalized_once_with_its_minimum():
    rng = np.random.default_rng(5)
    for trial in range(120):
        n = int(rng.integers(1, 250))
        deg = rng.integers(1, 6, size=n)
        for _ in range(int(rng.integers(0, 4))):
            deg[rng.integers(0, n)] = int(rng.integers(30, 400))
        deg[rng.random(n) < 0.05] = 0  # padding slots own no pairs
        P = np.concatenate([[0], np.cumsum((deg + 1) // 2)])
        npairs = int(P[-1])
        if npairs == 0:
            continue
        val = rng.integers(0, 1000, size=npairs)
        want = {u: int(val[P[u]:P[u + 1]].min()) for u in range(n) if P[u + 1] > P[u]}
        nwarps = int(rng.integers(1, 40))
        per = -(-npairs // nwarps)
        slice_ = max(32, -(-per // 32) * 32)  # as eg_dgame_solve sizes it
        assert walk(P, val, slice_, nwarps + 3) == want, trial

