"""ctypes wrapper of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() (as the checker) and bench.py's
cpu_baseline / reference arm may use this module.  The product never imports
it.

  liboracle.so   C restatement of the reference solver (oracle/eg_oracle.c)
  _ref/libegref.so   the reference's own cpu_solver.c / host_csr2csc.c,
                     compiled unmodified from the reference tree
  _ref/egsolver      the reference's own driver (egsolver.c) linked against
                     the solver's reference-ABI shim

Build with `make -C oracle` (and `make -C oracle ref` where the reference
tree is present); ensure_built() does that on demand.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
REF_LIB = HERE / "_ref" / "libegref.so"
REF_BIN = HERE / "_ref" / "egsolver"
# the reference checkout: $EG_REFERENCE_TREE, else a directory named "reference"
# beside this repository
REF_TREE = Path(os.environ.get("EG_REFERENCE_TREE", str(HERE.parent.parent / "reference")))

TOP32 = 2147483647
TOP64 = 9223372036854775807
ALGOR_EG, ALGOR_EG0 = 6, 7


class OracleStats(C.Structure):
    _fields_ = [("loops", C.c_int64), ("processed", C.c_int64), ("edges", C.c_int64), ("finished", C.c_int64)]


_lib = None
_ref = None


def ensure_built() -> None:
    if not LIB.exists() or LIB.stat().st_mtime < (HERE / "eg_oracle.c").stat().st_mtime:
        subprocess.run(["make", "-C", str(HERE), "all"], check=True, capture_output=True)
    if (REF_TREE / "src" / "cpu_solver.c").exists():
        # incremental: relinks the reference driver whenever the solver library changed
        subprocess.run(["make", "-C", str(HERE), "ref", f"REF={REF_TREE}"], check=True, capture_output=True)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        ensure_built()
        L = C.CDLL(str(LIB))
        P, I32, I64 = C.c_void_p, C.c_int32, C.c_int64
        for name in ("oracle_eg_solve_i32", "oracle_eg_solve_i64", "oracle_eg0_solve_i32"):
            getattr(L, name).argtypes = [I32, I32, I64, P, P, P, I64, I64, P, C.POINTER(OracleStats)]
            getattr(L, name).restype = C.c_int
        L.oracle_eg0_omp_i32.argtypes = [I32, I32, I64, P, P, P, I64, I64, P, C.POINTER(OracleStats), I32]
        L.oracle_eg0_omp_i32.restype = C.c_int
        L.oracle_mg.argtypes = [I32, P, P, I32]
        L.oracle_mg.restype = I64
        L.oracle_max_loop.argtypes = [I64, I64, I64, I64]
        L.oracle_max_loop.restype = I64
        L.oracle_ominus.argtypes = [I64, I64, I64, I32]
        L.oracle_ominus.restype = I64
        L.oracle_csr2csc.argtypes = [I32, I32, I64, P, P, P, P, P, P]
        L.oracle_csr2csc.restype = None
        L.oracle_count_inconsistent_i64.argtypes = [I32, I32, P, P, P, I64, P]
        L.oracle_count_inconsistent_i64.restype = I64
        L.oracle_generate.argtypes = [I32, I32, I32, I32, I32, C.c_uint64, C.POINTER(C.POINTER(C.c_int64)),
                                      C.POINTER(C.POINTER(C.c_int32)), C.POINTER(C.POINTER(C.c_int32)),
                                      C.POINTER(C.c_int64), C.POINTER(C.c_int32)]
        L.oracle_generate.restype = C.c_int
        L.oracle_free.argtypes = [P]
        L.oracle_free.restype = None
        _lib = L
    return _lib


def ref_available() -> bool:
    ensure_built()
    return REF_LIB.exists()


def ref_lib() -> C.CDLL:
    global _ref
    if _ref is None:
        ensure_built()
        if not REF_LIB.exists():
            raise RuntimeError(f"{REF_LIB} not built (the reference tree is needed once, to compile it)")
        L = C.CDLL(str(REF_LIB))
        P = C.c_void_p
        L.ref_cpu_solve.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, P, P, P, C.c_long, C.c_int, P,
                                    C.POINTER(C.c_long), C.POINTER(C.c_int), C.POINTER(C.c_double)]
        L.ref_cpu_solve.restype = C.c_int
        L.host_csr2csc.argtypes = [C.c_int, C.c_int, C.c_int, P, P, P, P, P, P]
        L.host_csr2csc.restype = None
        _ref = L
    return _ref


def _arrs(game):
    ptr = np.ascontiguousarray(game.row_ptr, dtype=np.int64)
    succ = np.ascontiguousarray(game.succ, dtype=np.int32)
    w = np.ascontiguousarray(game.weight, dtype=np.int32)
    return ptr, succ, w


def mg(game, limit_bits: int = 64) -> int:
    ptr, succ, w = _arrs(game)
    return int(lib().oracle_mg(game.num_nodes, ptr.ctypes.data, w.ctypes.data, limit_bits))


def max_loop(m: int, n: int, mgv: int, ml: int = -1) -> int:
    return int(lib().oracle_max_loop(m, n, mgv, ml))


def ominus(a: int, b: int, mgv: int, bits: int) -> int:
    return int(lib().oracle_ominus(a, b, mgv, bits))


def eg_solve(game, bits: int = 64, max_loop_: int = -1):
    """The reference's EG worklist solver restated (int32 exact or int64)."""
    ptr, succ, w = _arrs(game)
    n = game.num_nodes
    mgv = mg(game, 32 if bits == 32 else 64)
    if mgv < 0:
        raise OverflowError("MG overflows 32-bit credits")
    f = np.zeros(n, dtype=np.int32 if bits == 32 else np.int64)
    st = OracleStats()
    fn = lib().oracle_eg_solve_i32 if bits == 32 else lib().oracle_eg_solve_i64
    rc = fn(n, game.num_nodes0, game.num_edges, ptr.ctypes.data, succ.ctypes.data, w.ctypes.data, mgv, max_loop_,
            f.ctypes.data, C.byref(st))
    if rc != 0:
        raise MemoryError("oracle allocation failed")
    return f, {"loops": st.loops, "processed": st.processed, "edges": st.edges, "finished": bool(st.finished),
               "mg": mgv}


def eg0_solve(game, threads: int = 0, max_loop_: int = -1):
    """Jacobi sweeps (serial restatement when threads == 0, fixed OpenMP otherwise)."""
    ptr, succ, w = _arrs(game)
    n = game.num_nodes
    mgv = mg(game, 32)
    if mgv < 0:
        raise OverflowError("MG overflows 32-bit credits")
    f = np.zeros(n, dtype=np.int32)
    st = OracleStats()
    if threads == 0:
        rc = lib().oracle_eg0_solve_i32(n, game.num_nodes0, game.num_edges, ptr.ctypes.data, succ.ctypes.data,
                                        w.ctypes.data, mgv, max_loop_, f.ctypes.data, C.byref(st))
    else:
        rc = lib().oracle_eg0_omp_i32(n, game.num_nodes0, game.num_edges, ptr.ctypes.data, succ.ctypes.data,
                                      w.ctypes.data, mgv, max_loop_, f.ctypes.data, C.byref(st), threads)
    if rc != 0:
        raise MemoryError("oracle allocation failed")
    return f, {"loops": st.loops, "processed": st.processed, "edges": st.edges, "finished": bool(st.finished),
               "mg": mgv}


def csr2csc(nrow: int, ncol: int, row_ptr, col, val):
    row_ptr = np.ascontiguousarray(row_ptr, dtype=np.int64)
    col = np.ascontiguousarray(col, dtype=np.int32)
    val = np.ascontiguousarray(val, dtype=np.int32)
    nnz = col.shape[0]
    cp = np.zeros(ncol + 1, dtype=np.int64)
    cr = np.zeros(max(nnz, 1), dtype=np.int32)
    cv = np.zeros(max(nnz, 1), dtype=np.int32)
    lib().oracle_csr2csc(nrow, ncol, nnz, val.ctypes.data, col.ctypes.data, row_ptr.ctypes.data, cv.ctypes.data,
                         cr.ctypes.data, cp.ctypes.data)
    return cp, cr[:nnz], cv[:nnz]


def count_inconsistent(game, f: np.ndarray, mgv: int | None = None) -> int:
    """Vertices whose lift differs from f (0: f is a fixed point)."""
    ptr, succ, w = _arrs(game)
    f64 = np.ascontiguousarray(f, dtype=np.int64).copy()
    if f.dtype == np.int32:
        f64[f == TOP32] = TOP64
    mgv = mg(game, 64) if mgv is None else mgv
    return int(lib().oracle_count_inconsistent_i64(game.num_nodes, game.num_nodes0, ptr.ctypes.data,
                                                   succ.ctypes.data, w.ctypes.data, mgv, f64.ctypes.data))


def ref_cpu_solve(game, algo: str = "eg", threads: int = 1, max_loop_: int = -1):
    """The reference's own cpu_solver() on the game (int32, TOP = INT_MAX)."""
    L = ref_lib()
    ptr = np.ascontiguousarray(game.row_ptr, dtype=np.int32)
    succ = np.ascontiguousarray(game.succ, dtype=np.int32)
    w = np.ascontiguousarray(game.weight, dtype=np.int32)
    n = game.num_nodes
    out = np.zeros(n, dtype=np.int32)
    processed = C.c_long()
    mgv = C.c_int()
    secs = C.c_double()
    a = ALGOR_EG if algo == "eg" else ALGOR_EG0
    rc = L.ref_cpu_solve(a, n, game.num_nodes0, game.num_edges, ptr.ctypes.data, succ.ctypes.data, w.ctypes.data,
                         max_loop_, threads, out.ctypes.data, C.byref(processed), C.byref(mgv), C.byref(secs))
    if rc == -1:
        raise OverflowError("MG overflows int (the reference exits here)")
    if rc != 0:
        raise MemoryError("reference allocation failed")
    return out, {"processed": processed.value, "mg": mgv.value, "seconds": secs.value}


def ref_host_csr2csc(nrow: int, ncol: int, row_ptr, col, val):
    L = ref_lib()
    row_ptr = np.ascontiguousarray(row_ptr, dtype=np.int32)
    col = np.ascontiguousarray(col, dtype=np.int32)
    val = np.ascontiguousarray(val, dtype=np.int32)
    nnz = col.shape[0]
    cp = np.zeros(ncol + 1, dtype=np.int32)
    cr = np.zeros(max(nnz, 1), dtype=np.int32)
    cv = np.zeros(max(nnz, 1), dtype=np.int32)
    L.host_csr2csc(nrow, ncol, nnz, val.ctypes.data, col.ctypes.data, row_ptr.ctypes.data, cv.ctypes.data,
                   cr.ctypes.data, cp.ctypes.data)
    return cp.astype(np.int64), cr[:nnz], cv[:nnz]


class OracleGame:
    """A generated game in the same CSR form as the solver's Game (host
    arrays, owner-sorted: vertices [0, num_nodes0) belong to player 0)."""

    def __init__(self, row_ptr, succ, weight, num_nodes0):
        self.row_ptr, self.succ, self.weight, self.num_nodes0 = row_ptr, succ, weight, int(num_nodes0)
        self.owner = None
        self.max_abs_weight = int(np.abs(weight.astype(np.int64)).max()) if weight.size else 0

    @property
    def num_nodes(self) -> int:
        return int(self.row_ptr.shape[0] - 1)

    @property
    def num_edges(self) -> int:
        return int(self.succ.shape[0])


def generate(kind: int, n: int, deg: int, wmax: int, seed: int, param: int = 0) -> OracleGame:
    """The benchmark's seeded generator, restated in eg_oracle.c (same games as
    the solver library's eg_generate, without loading that library)."""
    L = lib()
    pp, sp, wp = C.POINTER(C.c_int64)(), C.POINTER(C.c_int32)(), C.POINTER(C.c_int32)()
    m, n0 = C.c_int64(), C.c_int32()
    rc = L.oracle_generate(kind, n, deg, wmax, param, seed & (2**64 - 1), C.byref(pp), C.byref(sp), C.byref(wp),
                           C.byref(m), C.byref(n0))
    if rc != 0:
        raise ValueError(f"oracle_generate failed ({rc})")
    try:
        ptr = np.ctypeslib.as_array(pp, shape=(n + 1,)).copy()
        succ = np.ctypeslib.as_array(sp, shape=(max(m.value, 1),))[: m.value].copy()
        w = np.ctypeslib.as_array(wp, shape=(max(m.value, 1),))[: m.value].copy()
    finally:
        for q in (pp, sp, wp):
            L.oracle_free(C.cast(q, C.c_void_p))
    return OracleGame(ptr, succ, w, n0.value)


SEED = 0xE6  # seed base of the benchmark workloads: SEED + configuration number


def workload(name: str, n: int = 0) -> OracleGame:
    """The single-game benchmark workloads (configurations 1-3) built by the
    restated generator, with the same kinds, bounds and seeds as the solver
    package's workloads module."""
    if name == "cfg1":
        return generate(1, n or 1000, 4, 10, SEED + 1)
    if name == "cfg2":
        n = n or (1 << 20)
        return generate(2, n, min(4096, n - 1), 1000, SEED + 2)
    if name == "cfg3":
        n = n or 2000
        return generate(3, n, n - 1, 500, SEED + 3)
    raise ValueError(f"unknown workload {name}")
