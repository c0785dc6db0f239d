"""Pins the full-size benchmark games with the reference's own CPU solver.

    python tests/golden/make_full_size_golden.py WORKLOAD WHICH OUT.json

WORKLOAD is cfg2 (n = 2^20 sparse game) or cfg3 (2000-vertex clique);
WHICH is "reference" (the reference's EG_cpu_solver compiled unmodified,
oracle/_ref/libegref.so, int32 credits), "port" (the int64 worklist
restatement in oracle/eg_oracle.c), or "eg0-omp" (the restatement of the
reference's EG0 Jacobi sweeps with its thread-safety defects fixed, int32
credits, all host cores).  Every schedule reaches the same least fixed
point.  The serial worklist takes hours on cfg2 and the Jacobi sweeps tens of
minutes on eight cores, which is why the result is committed as a digest
rather than recomputed by the tests.

OUT.json records: the SHA-256 of the credits as little-endian int64 in
vertex order with TOP written as INT64_MAX, the number of TOP vertices, the
sum of finite credits, MG, worklist pops, and the solve time.  The GPU test
tests/test_gpu_full_size.py recomputes the digest from the GPU credits.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from egsolver_b200 import workloads  # noqa: E402
from oracle import oracle as O  # noqa: E402

TOP64 = np.iinfo(np.int64).max


def digest(credits64: np.ndarray) -> dict:
    c = np.ascontiguousarray(credits64, dtype="<i8")
    finite = c[c != TOP64]
    return {"sha256": hashlib.sha256(c.tobytes()).hexdigest(), "num_top": int((c == TOP64).sum()),
            "sum_finite": int(finite.sum()), "max_finite": int(finite.max()) if finite.size else 0}


def main(workload: str, which: str, out: str) -> None:
    game = getattr(workloads, workload)()
    t0 = time.time()
    if which == "reference":
        f32, st = O.ref_cpu_solve(game, "eg", threads=1)
        f = f32.astype(np.int64)
        f[f32 == O.TOP32] = TOP64
        info = {"pops": st["processed"], "mg": st["mg"], "reference_seconds": st["seconds"]}
    elif which == "eg0-omp":
        threads = os.cpu_count() or 1
        f32, st = O.eg0_solve(game, threads=threads)
        f = f32.astype(np.int64)
        f[f32 == O.TOP32] = TOP64
        info = {"sweeps": st["loops"], "mg": st["mg"], "edges": st["edges"], "finished": st["finished"],
                "threads": threads}
    else:
        f, st = O.eg_solve(game, bits=64)
        info = {"pops": st["processed"], "mg": st["mg"], "edges": st["edges"], "finished": st["finished"]}
    rec = {"workload": workload, "which": which, "n": game.num_nodes, "m": game.num_edges,
           "wall_seconds": time.time() - t0, **info, **digest(f)}
    Path(out).write_text(json.dumps(rec, indent=1) + "\n")
    print(json.dumps(rec))


if __name__ == "__main__":
    main(sys.argv[1], sys.argv[2], sys.argv[3])
