"""egsolver_b200 -- energy-game solver for one NVIDIA B200 (sm_100a).

Python mirror of the C-ABI in include/egsolver_b200.h.  Every call goes
through the in-tree CUDA library libegsolver_b200.so; there is no CPU or
eager-framework fallback, and a missing library raises on first use.

Conventions follow the reference solver (fvella/EGSolver): player 0 is the
file format's MAX and minimises the credit, player 1 (MIN) maximises it;
vertices [0, num_nodes0) belong to player 0 unless an owner array is given;
TOP (an unbounded credit) is INT32_MAX / INT64_MAX.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import _ffi
from ._ffi import (DIRECTION_DENSE, DIRECTION_SPARSE, DIRECTION_SWITCH, EG_TOP32, EG_TOP64,  # noqa: F401
                   VARIANT_AUTO, VARIANT_CTA, VARIANT_SMEM, VARIANT_THREAD, VARIANT_WARP)

__all__ = ["Game", "EGError", "Stats", "solve", "ResidentGame", "Batch", "BatchStats", "Server", "threshold_game",
           "generate", "read_game", "read_game_text", "read_game_binary", "write_game_binary", "clique_text", "ladder_text", "copies_text",
           "csr2csc", "compute_mg", "default_max_loop", "device_count", "CancelFlag", "EG_TOP32", "EG_TOP64",
           "lib"]


class EGError(RuntimeError):
    """A non-OK eg_status, with the library's message."""

    def __init__(self, status: int, message: str):
        self.status = status
        self.name = _ffi.STATUS_NAMES.get(status, str(status))
        super().__init__(f"{self.name}: {message}")


def lib() -> C.CDLL:
    return _ffi.load()


def _check(status: int) -> None:
    if status != _ffi.EG_OK:
        raise EGError(status, lib().eg_last_error().decode(errors="replace"))


def _ptr(a: Optional[np.ndarray]) -> Optional[int]:
    return None if a is None else a.ctypes.data


@dataclass
class Game:
    """A game in CSR form (host arrays).

    row_ptr: int64[n+1]; succ, weight: int32[m]; owner: optional uint8[n];
    num_nodes0: split index used when owner is None; ext_id: optional
    external names of the vertices (as read from a file).
    """

    row_ptr: np.ndarray
    succ: np.ndarray
    weight: np.ndarray
    num_nodes0: int = 0
    owner: Optional[np.ndarray] = None
    ext_id: Optional[np.ndarray] = None
    max_abs_weight: int = field(default=-1)

    def __post_init__(self):
        self.row_ptr = np.ascontiguousarray(self.row_ptr, dtype=np.int64)
        self.succ = np.ascontiguousarray(self.succ, dtype=np.int32)
        self.weight = np.ascontiguousarray(self.weight, dtype=np.int32)
        if self.owner is not None:
            self.owner = np.ascontiguousarray(self.owner, dtype=np.uint8)
        if self.max_abs_weight < 0:
            self.max_abs_weight = int(np.abs(self.weight.astype(np.int64)).max()) if self.weight.size else 0

    @property
    def num_nodes(self) -> int:
        return int(self.row_ptr.shape[0] - 1)

    @property
    def num_edges(self) -> int:
        return int(self.succ.shape[0])

    def owners(self) -> np.ndarray:
        if self.owner is not None:
            return self.owner
        o = np.ones(self.num_nodes, dtype=np.uint8)
        o[: self.num_nodes0] = 0
        return o

    def c_struct(self) -> _ffi.EgGame:
        g = _ffi.EgGame()
        g.num_nodes = self.num_nodes
        g.num_nodes0 = int(self.num_nodes0)
        g.num_edges = self.num_edges
        g.row_ptr = _ptr(self.row_ptr)
        g.succ = _ptr(self.succ)
        g.weight = _ptr(self.weight)
        g.owner = _ptr(self.owner)
        return g


@dataclass
class Stats:
    mg: int
    rounds: int
    lifts: int
    edges: int
    num_top: int
    solve_ms: float
    lift_ms: float
    kernel_launches: int
    credit_bits: int
    variant_small: int
    variant_mid: int
    variant_large: int
    small_max_deg: int
    large_min_deg: int
    changes: int
    pushes: int
    grid: int
    block: int
    dense_rounds: int
    dense_launches: int
    phase_heavy_ns: float
    phase_light_ns: float
    phase_wait_ns: float
    dense_ms: float
    dense_changes: int

    @classmethod
    def from_c(cls, s: _ffi.EgStats) -> "Stats":
        return cls(**s.as_dict())

    @property
    def gteps(self) -> float:
        return self.edges / (self.solve_ms * 1e6) if self.solve_ms > 0 else 0.0


def make_opts(credit_bits: int = 64, variant: int = VARIANT_AUTO, max_rounds: int = -1, timeout_ms: float = 0.0,
              device: int = 0, lanes_per_vertex: int = 0, small_max_deg: int = 0, large_min_deg: int = 0,
              keep_layout: bool = False, cancel: Optional["CancelFlag"] = None, grid_ctas: int = 0,
              task_edges: int = 0, schedule: int = 0, profile: bool = False, ctas_per_sm: int = 0,
              direction: int = 0, dense_permille: int = 0, sparse_permille: int = 0, narrow: bool = False,
              wide_pairs: bool = False, dense_depth: int = 0, dense_sweeps: int = 0) -> _ffi.EgOpts:
    o = _ffi.EgOpts()
    lib().eg_opts_default(C.byref(o))
    o.credit_bits = credit_bits
    o.variant = variant
    o.max_rounds = max_rounds
    o.timeout_ms = timeout_ms
    o.device = device
    o.lanes_per_vertex = lanes_per_vertex
    o.small_max_deg = small_max_deg
    o.large_min_deg = large_min_deg
    o.keep_layout = 1 if keep_layout else 0
    o.grid_ctas = grid_ctas
    o.task_edges = task_edges
    o.schedule = schedule
    o.profile = 1 if profile else 0
    o.ctas_per_sm = ctas_per_sm
    o.direction = direction
    o.dense_permille = dense_permille
    o.sparse_permille = sparse_permille
    o.narrow = 1 if narrow else 0
    o.wide_pairs = 1 if wide_pairs else 0
    o.dense_depth = dense_depth
    o.dense_sweeps = dense_sweeps
    o.cancel = cancel.ptr if cancel is not None else None
    return o


def solve(game: Game, credit_bits: int = 64, **kw) -> tuple[np.ndarray, Stats]:
    """One-call solve with host buffers (eg_solve_i32 / eg_solve_i64)."""
    opts = make_opts(credit_bits=credit_bits, **kw)
    st = _ffi.EgStats()
    cg = game.c_struct()
    if credit_bits == 32:
        out = np.zeros(game.num_nodes, dtype=np.int32)
        _check(lib().eg_solve_i32(C.byref(cg), C.byref(opts), out.ctypes.data, C.byref(st)))
    else:
        out = np.zeros(game.num_nodes, dtype=np.int64)
        _check(lib().eg_solve_i64(C.byref(cg), C.byref(opts), out.ctypes.data, C.byref(st)))
    return out, Stats.from_c(st)


class ResidentGame:
    """A game kept in device memory (eg_dgame_*)."""

    def __init__(self, game: Game, **kw):
        self._h = C.c_void_p()
        opts = make_opts(**kw)
        cg = game.c_struct()
        _check(lib().eg_dgame_upload(C.byref(cg), C.byref(opts), C.byref(self._h)))
        self.num_nodes = game.num_nodes

    @classmethod
    def from_device(cls, n: int, m: int, n0: int, row_ptr_dev: int, succ_dev: int, weight_dev: int,
                    owner_dev: Optional[int] = None, **kw) -> "ResidentGame":
        self = cls.__new__(cls)
        self._h = C.c_void_p()
        g = _ffi.EgGame(n, n0, m, row_ptr_dev, succ_dev, weight_dev, owner_dev)
        opts = make_opts(**kw)
        _check(lib().eg_dgame_from_device(C.byref(g), C.byref(opts), C.byref(self._h)))
        self.num_nodes = n
        return self

    def solve(self, raise_on_error: bool = True, **kw) -> tuple[int, Stats]:
        opts = make_opts(**kw)
        st = _ffi.EgStats()
        status = lib().eg_dgame_solve(self._h, C.byref(opts), C.byref(st))
        if raise_on_error:
            _check(status)
        return status, Stats.from_c(st)

    def credits(self, bits: int = 64) -> np.ndarray:
        if bits == 32:
            out = np.zeros(self.num_nodes, dtype=np.int32)
            _check(lib().eg_dgame_credits_i32(self._h, out.ctypes.data))
        else:
            out = np.zeros(self.num_nodes, dtype=np.int64)
            _check(lib().eg_dgame_credits_i64(self._h, out.ctypes.data))
        return out

    def credits_device(self) -> tuple[int, int]:
        p = C.c_void_p()
        bits = C.c_int32()
        _check(lib().eg_dgame_credits_device(self._h, C.byref(p), C.byref(bits)))
        return int(p.value), int(bits.value)

    @property
    def device_bytes(self) -> int:
        return int(lib().eg_dgame_device_bytes(self._h))

    TUNED_KNOBS = ("large_min_deg", "task_edges", "small_max_deg", "dense_sweeps", "dense_depth")

    def tune(self, rounds: int = 300, **kw) -> tuple[dict, dict]:
        """Autotunes the AUTO layout on capped solves (eg_dgame_tune); returns
        the chosen knobs (keyword arguments of solve) and the report."""
        base = make_opts(**kw)
        out = _ffi.EgOpts()
        rep = _ffi.EgTuneReport()
        _check(lib().eg_dgame_tune(self._h, C.byref(base), rounds, C.byref(out), C.byref(rep)))
        knobs = {k: int(getattr(out, k)) for k in self.TUNED_KNOBS}
        return knobs, {"candidates": rep.candidates, "from_cache": bool(rep.from_cache),
                       "default_rate": rep.default_rate, "best_rate": rep.best_rate}

    def free(self) -> None:
        if self._h:
            lib().eg_dgame_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.free()


class CancelFlag:
    """A flag in mapped pinned host memory that running solves poll."""

    def __init__(self):
        p = C.c_void_p()
        _check(lib().eg_cancel_flag_alloc(C.byref(p)))
        self.ptr = p.value
        self._view = C.cast(p, C.POINTER(C.c_int32))

    def set(self, value: int = 1) -> None:
        self._view[0] = value

    def free(self) -> None:
        if self.ptr:
            lib().eg_cancel_flag_free(self.ptr)
            self.ptr = None


@dataclass
class BatchStats:
    num_games: int
    thresholds: int
    total_nodes: int
    total_edges: int
    rounds_max: int
    rounds_sum: int
    lifts: int
    edges: int
    num_top: int
    solve_ms: float
    block: int
    grid: int
    games_failed: int
    graph_replayed: int
    num_units: int = 0
    smem_bytes: int = 0
    tail_entries: int = 0
    phase1_ms: float = 0.0
    tail_ms: float = 0.0

    @property
    def gteps(self) -> float:
        return self.edges / (self.solve_ms * 1e6) if self.solve_ms > 0 else 0.0


class Batch:
    """Many games x K mean-payoff thresholds solved in one persistent launch
    (eg_batch_*).  Threshold p of game g turns every weight w into w*d - p."""

    def __init__(self, games: list[Game], thresholds: int, scale: int = 1, block: int = 0, device: int = 0,
                 max_rounds: int = -1, timeout_ms: float = 0.0, use_graph: bool = False, group_max: int = 0,
                 tail_rows: int = 0, park_percent: int = 0, tail_sweeps: int = 0, tail_cluster: int = 0):
        self._h = C.c_void_p()
        self._keep = [g.c_struct() for g in games]
        arr = (_ffi.EgGame * len(games))(*self._keep)
        o = _ffi.EgBatchOpts()
        o.thresholds = thresholds
        o.scale = scale
        o.block = block
        o.device = device
        o.max_rounds = max_rounds
        o.timeout_ms = timeout_ms
        o.use_graph = 1 if use_graph else 0
        o.group_max = group_max
        o.tail_rows = tail_rows
        o.park_percent = park_percent
        o.tail_sweeps = tail_sweeps
        o.tail_cluster = tail_cluster
        _check(lib().eg_batch_create(arr, len(games), C.byref(o), C.byref(self._h)))
        self.sizes = [g.num_nodes for g in games]
        self.K = thresholds

    def set_thresholds(self, p) -> None:
        a = np.ascontiguousarray(p, dtype=np.int32).reshape(-1)
        if a.size != len(self.sizes) * self.K:
            raise ValueError("need num_games * K thresholds")
        _check(lib().eg_batch_set_thresholds(self._h, a.ctypes.data))

    def solve(self, raise_on_error: bool = True) -> tuple[int, BatchStats]:
        st = _ffi.EgBatchStats()
        status = lib().eg_batch_solve(self._h, C.byref(st))
        if raise_on_error:
            _check(status)
        return status, BatchStats(**st.as_dict())

    def credits(self, game: int) -> np.ndarray:
        """Credits of one game as a (K, n) int64 array (TOP = EG_TOP64)."""
        n = self.sizes[game]
        out = np.zeros(self.K * n, dtype=np.int64)
        _check(lib().eg_batch_credits(self._h, game, out.ctypes.data))
        return out.reshape(self.K, n)

    def game_result(self, game: int) -> tuple[int, int]:
        r = C.c_int64()
        s = C.c_int32()
        _check(lib().eg_batch_game_result(self._h, game, C.byref(r), C.byref(s)))
        return int(r.value), int(s.value)

    def tune(self) -> int:
        b = C.c_int32()
        _check(lib().eg_batch_tune(self._h, C.byref(b)))
        return int(b.value)

    @property
    def device_bytes(self) -> int:
        return int(lib().eg_batch_device_bytes(self._h))

    def free(self) -> None:
        if self._h:
            lib().eg_batch_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.free()


class Server:
    """Serving loop for mean-payoff threshold queries (eg_serve_*): games are
    registered once, queries are submitted at any time and run in
    continuously formed micro-batches."""

    def __init__(self, device: int = 0, max_inflight: int = 0, streams: int = 0, block: int = 0,
                 hbm_reserve_bytes: int = 0, max_rounds: int = -1, large_ctas: int = 0):
        o = _ffi.EgServeOpts()
        o.device, o.max_inflight, o.streams, o.block = device, max_inflight, streams, block
        o.hbm_reserve_bytes, o.max_rounds, o.large_ctas = hbm_reserve_bytes, max_rounds, large_ctas
        self._h = C.c_void_p()
        _check(lib().eg_serve_create(C.byref(o), C.byref(self._h)))
        self._sizes: dict[int, int] = {}
        self._qk: dict[int, tuple[int, int]] = {}

    def add_game(self, game: Game) -> int:
        gid = C.c_int64()
        cg = game.c_struct()
        _check(lib().eg_serve_add_game(self._h, C.byref(cg), C.byref(gid)))
        self._sizes[gid.value] = game.num_nodes
        return int(gid.value)

    def remove_game(self, gid: int) -> None:
        _check(lib().eg_serve_remove_game(self._h, gid))

    def submit(self, gid: int, p, d: int = 1) -> int:
        a = np.ascontiguousarray(p, dtype=np.int32).reshape(-1)
        qid = C.c_int64()
        _check(lib().eg_serve_submit(self._h, gid, a.ctypes.data, a.size, d, C.byref(qid)))
        self._qk[qid.value] = (gid, a.size)
        return int(qid.value)

    def poll(self, qid: int) -> tuple[int, float]:
        st = C.c_int32()
        lat = C.c_double()
        _check(lib().eg_serve_poll(self._h, qid, C.byref(st), C.byref(lat)))
        return int(st.value), float(lat.value)

    def wait(self, qid: int, timeout_ms: float = -1.0) -> None:
        _check(lib().eg_serve_wait(self._h, qid, timeout_ms))

    def result(self, qid: int) -> tuple[np.ndarray, int]:
        gid, k = self._qk[qid]
        out = np.zeros(k * self._sizes[gid], dtype=np.int64)
        r = C.c_int64()
        _check(lib().eg_serve_result(self._h, qid, out.ctypes.data, C.byref(r)))
        del self._qk[qid]
        return out.reshape(k, -1), int(r.value)

    def stats(self) -> dict:
        s = _ffi.EgServeStats()
        _check(lib().eg_serve_stats_get(self._h, C.byref(s)))
        return s.as_dict()

    def trace(self) -> list[dict]:
        """Device-clock spans of the finished micro-batches (eg_serve_trace)."""
        n = C.c_int32()
        _check(lib().eg_serve_trace(self._h, None, 0, C.byref(n)))
        arr = (_ffi.EgServeSpan * max(n.value, 1))()
        _check(lib().eg_serve_trace(self._h, arr, n.value, C.byref(n)))
        return [{"batch": a.batch, "queries": a.queries, "units": a.units, "begin_ms": a.begin_ms,
                 "end_ms": a.end_ms} for a in arr[:n.value]]

    def close(self) -> None:
        if self._h:
            _check(lib().eg_serve_destroy(self._h))
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def threshold_game(game: Game, p: int, d: int) -> Game:
    """The energy game of the mean-payoff query (weights w*d - p), for checking."""
    w = game.weight.astype(np.int64) * d - p
    if w.min() < -2**31 or w.max() >= 2**31:
        raise OverflowError("shifted weights do not fit int32")
    return Game(row_ptr=game.row_ptr, succ=game.succ, weight=w.astype(np.int32), num_nodes0=game.num_nodes0,
                owner=game.owner, ext_id=game.ext_id)


def _own_to_game(og_ptr) -> Game:
    og = og_ptr.contents
    n = og.game.num_nodes
    m = og.game.num_edges

    def arr(addr, count, ctype, dtype):
        if count == 0:
            return np.zeros(0, dtype=dtype)
        return np.ctypeslib.as_array(C.cast(addr, C.POINTER(ctype)), shape=(count,)).astype(dtype, copy=True)

    g = Game(row_ptr=arr(og.row_ptr, n + 1, C.c_int64, np.int64), succ=arr(og.succ, m, C.c_int32, np.int32),
             weight=arr(og.weight, m, C.c_int32, np.int32), num_nodes0=og.game.num_nodes0,
             ext_id=arr(og.ext_id, n, C.c_int32, np.int32), max_abs_weight=og.max_abs_weight)
    lib().eg_owned_game_free(og_ptr)
    return g


def _take_text(fn, *args) -> str:
    buf, ln = C.c_void_p(), C.c_size_t()
    _check(fn(*args, C.byref(buf), C.byref(ln)))
    try:
        return C.string_at(buf, ln.value).decode()
    finally:
        lib().eg_free_text(buf)


def clique_text(number: int) -> str:
    """The reference's mkclique game text (eg_fixture_clique_text)."""
    return _take_text(lib().eg_fixture_clique_text, number)


def ladder_text(number: int) -> str:
    """The reference's mkladder game text (eg_fixture_ladder_text)."""
    return _take_text(lib().eg_fixture_ladder_text, number)


def copies_text(text: str, copies: int) -> str:
    """The reference's multi rewrite of a game text (eg_fixture_copies_text)."""
    raw = text.encode()
    return _take_text(lib().eg_fixture_copies_text, raw, len(raw), copies)


def generate(kind: int, n: int, deg: int, wmax: int, seed: int, param: int = 0) -> Game:
    """Seeded random game (eg_generate); owner-sorted like the reference layout."""
    out = C.POINTER(_ffi.EgOwnedGame)()
    _check(lib().eg_generate(kind, n, deg, wmax, param, seed & (2**64 - 1), C.byref(out)))
    return _own_to_game(out)


def _read_opts(weight_mode: int, rnd_lo: int, rnd_hi: int, rnd_seed: int) -> _ffi.EgReadOpts:
    return _ffi.EgReadOpts(weight_mode, rnd_lo, rnd_hi, rnd_seed)


def read_game(path: str, weight_mode: int = 0, rnd_lo: int = -1, rnd_hi: int = 1, rnd_seed: int = 0,
              cache: Optional[str] = None) -> Game:
    """Reads a game in the reference text format (gzip or plain); with cache,
    through the binary CSR cache file at that path (eg_read_game_file_cached)."""
    out = C.POINTER(_ffi.EgOwnedGame)()
    ro = _read_opts(weight_mode, rnd_lo, rnd_hi, rnd_seed)
    if cache is None:
        _check(lib().eg_read_game_file(str(path).encode(), C.byref(ro), C.byref(out)))
    else:
        _check(lib().eg_read_game_file_cached(str(path).encode(), C.byref(ro), str(cache).encode(), C.byref(out)))
    return _own_to_game(out)


def write_game_binary(game: Game, path: str, weight_mode: int = 0, rnd_lo: int = -1, rnd_hi: int = 1,
                      rnd_seed: int = 0) -> None:
    """Writes the game to the binary CSR file format (eg_write_game_binary);
    the reader options are recorded with it.  The game must be owner-sorted
    (no owner array), as the reader returns it."""
    if game.owner is not None:
        raise ValueError("the binary format holds owner-sorted games (num_nodes0 split)")
    ext = game.ext_id if game.ext_id is not None else np.arange(game.num_nodes, dtype=np.int32)
    ext = np.ascontiguousarray(ext, dtype=np.int32)
    og = _ffi.EgOwnedGame()
    og.game = game.c_struct()
    og.row_ptr, og.succ, og.weight, og.ext_id = _ptr(game.row_ptr), _ptr(game.succ), _ptr(game.weight), _ptr(ext)
    og.max_abs_weight = game.max_abs_weight
    ro = _read_opts(weight_mode, rnd_lo, rnd_hi, rnd_seed)
    _check(lib().eg_write_game_binary(str(path).encode(), C.byref(og), C.byref(ro)))


def read_game_binary(path: str, weight_mode: Optional[int] = None, rnd_lo: int = -1, rnd_hi: int = 1,
                     rnd_seed: int = 0) -> Game:
    """Reads a binary CSR file; with weight_mode given, only if it was written
    with those reader options."""
    out = C.POINTER(_ffi.EgOwnedGame)()
    ro = None if weight_mode is None else C.byref(_read_opts(weight_mode, rnd_lo, rnd_hi, rnd_seed))
    _check(lib().eg_read_game_binary(str(path).encode(), ro, C.byref(out)))
    return _own_to_game(out)


def read_game_text(text: str | bytes, weight_mode: int = 0, rnd_lo: int = -1, rnd_hi: int = 1,
                   rnd_seed: int = 0) -> Game:
    b = text.encode() if isinstance(text, str) else text
    out = C.POINTER(_ffi.EgOwnedGame)()
    ro = _read_opts(weight_mode, rnd_lo, rnd_hi, rnd_seed)
    _check(lib().eg_read_game_buffer(b, len(b), C.byref(ro), C.byref(out)))
    return _own_to_game(out)


def game_to_text(game: Game) -> str:
    """The game in the reference text format, one line per vertex in
    increasing external id: `MAX;` then `v MAX|MIN s:w,...;` (player 0 is
    MAX), using game.ext_id as the external names when present."""
    n = game.num_nodes
    ext = game.ext_id if game.ext_id is not None else np.arange(n, dtype=np.int32)
    own = game.owners()
    order = np.argsort(ext, kind="stable")
    lines = [f"{int(ext.max())} {game.num_edges};"]
    rp, sc, wt = game.row_ptr, game.succ, game.weight
    for v in order:
        b, e = int(rp[v]), int(rp[v + 1])
        edges = ",".join(f"{int(ext[s])}:{int(x)}" for s, x in zip(sc[b:e], wt[b:e]))
        lines.append(f"{int(ext[v])} {'MAX' if own[v] == 0 else 'MIN'} {edges};")
    return "\n".join(lines) + "\n"


def write_game_text(game: Game, path: str) -> None:
    """Writes game_to_text(game) to path, gzip-compressed when it ends in .gz."""
    import gzip

    data = game_to_text(game).encode()
    if str(path).endswith(".gz"):
        with gzip.open(path, "wb", compresslevel=9) as f:
            f.write(data)
    else:
        with open(path, "wb") as f:
            f.write(data)


def csr2csc(num_rows: int, num_cols: int, row_ptr: np.ndarray, col: np.ndarray, val: np.ndarray):
    """Device counting-sort transpose (eg_csr2csc_i32): returns (csc_ptr, csc_row, csc_val)."""
    row_ptr = np.ascontiguousarray(row_ptr, dtype=np.int64)
    col = np.ascontiguousarray(col, dtype=np.int32)
    val = np.ascontiguousarray(val, dtype=np.int32)
    nnz = col.shape[0]
    cp = np.zeros(num_cols + 1, dtype=np.int64)
    cr = np.zeros(max(nnz, 1), dtype=np.int32)
    cv = np.zeros(max(nnz, 1), dtype=np.int32)
    _check(lib().eg_csr2csc_i32(num_rows, num_cols, nnz, row_ptr.ctypes.data, col.ctypes.data, val.ctypes.data,
                                cp.ctypes.data, cr.ctypes.data, cv.ctypes.data))
    return cp, cr[:nnz], cv[:nnz]


def compute_mg(game: Game, limit_bits: int = 64) -> int:
    cg = game.c_struct()
    mg = C.c_int64()
    _check(lib().eg_compute_mg(C.byref(cg), limit_bits, C.byref(mg)))
    return int(mg.value)


def default_max_loop(m: int, n: int, mg: int, max_loop: int = -1) -> int:
    return int(lib().eg_default_max_loop(m, n, mg, max_loop))


def validate(game: Game) -> None:
    cg = game.c_struct()
    _check(lib().eg_validate(C.byref(cg)))


def device_count() -> int:
    c = C.c_int32()
    status = lib().eg_device_count(C.byref(c))
    return int(c.value) if status == _ffi.EG_OK else 0
