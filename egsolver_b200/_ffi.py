"""ctypes declarations of the C-ABI in include/egsolver_b200.h.

The library is loaded from this package's directory; importing this module
on a machine where it has not been built raises immediately (there is no
fallback implementation).
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libegsolver_b200.so"

EG_OK = 0
STATUS_NAMES = {
    0: "EG_OK", 1: "EG_ERR_INVALID", 2: "EG_ERR_CUDA", 3: "EG_ERR_OOM", 4: "EG_ERR_TIMEOUT",
    5: "EG_ERR_OVERFLOW", 6: "EG_ERR_LOOPCAP", 7: "EG_ERR_CANCELLED", 8: "EG_ERR_NO_DEVICE",
    9: "EG_ERR_BUSY", 10: "EG_ERR_NOT_FOUND", 11: "EG_ERR_IO",
}
EG_TOP32 = 2147483647
EG_TOP64 = 9223372036854775807

VARIANT_AUTO, VARIANT_THREAD, VARIANT_WARP, VARIANT_CTA, VARIANT_SMEM = 0, 1, 2, 3, 4
DIRECTION_SWITCH, DIRECTION_SPARSE, DIRECTION_DENSE = 0, 1, 2


class EgGame(C.Structure):
    _fields_ = [
        ("num_nodes", C.c_int32),
        ("num_nodes0", C.c_int32),
        ("num_edges", C.c_int64),
        ("row_ptr", C.c_void_p),
        ("succ", C.c_void_p),
        ("weight", C.c_void_p),
        ("owner", C.c_void_p),
    ]


class EgOpts(C.Structure):
    _fields_ = [
        ("credit_bits", C.c_int32),
        ("variant", C.c_int32),
        ("small_max_deg", C.c_int32),
        ("large_min_deg", C.c_int32),
        ("max_rounds", C.c_int64),
        ("timeout_ms", C.c_double),
        ("cancel", C.c_void_p),
        ("device", C.c_int32),
        ("lanes_per_vertex", C.c_int32),
        ("keep_layout", C.c_int32),
        ("grid_ctas", C.c_int32),
        ("task_edges", C.c_int32),
        ("schedule", C.c_int32),
        ("profile", C.c_int32),
        ("ctas_per_sm", C.c_int32),
        ("direction", C.c_int32),
        ("dense_permille", C.c_int32),
        ("sparse_permille", C.c_int32),
        ("narrow", C.c_int32),
        ("wide_pairs", C.c_int32),
        ("dense_depth", C.c_int32),
        ("dense_sweeps", C.c_int32),
    ]


class EgStats(C.Structure):
    _fields_ = [
        ("mg", C.c_int64),
        ("rounds", C.c_int64),
        ("lifts", C.c_int64),
        ("edges", C.c_int64),
        ("num_top", C.c_int64),
        ("solve_ms", C.c_double),
        ("lift_ms", C.c_double),
        ("kernel_launches", C.c_int64),
        ("credit_bits", C.c_int32),
        ("variant_small", C.c_int32),
        ("variant_mid", C.c_int32),
        ("variant_large", C.c_int32),
        ("small_max_deg", C.c_int32),
        ("large_min_deg", C.c_int32),
        ("changes", C.c_int64),
        ("pushes", C.c_int64),
        ("grid", C.c_int32),
        ("block", C.c_int32),
        ("dense_rounds", C.c_int32),
        ("dense_launches", C.c_int32),
        ("phase_heavy_ns", C.c_double),
        ("phase_light_ns", C.c_double),
        ("phase_wait_ns", C.c_double),
        ("dense_ms", C.c_double),
        ("dense_changes", C.c_int64),
    ]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


class EgOwnedGame(C.Structure):
    _fields_ = [
        ("game", EgGame),
        ("row_ptr", C.c_void_p),
        ("succ", C.c_void_p),
        ("weight", C.c_void_p),
        ("ext_id", C.c_void_p),
        ("max_abs_weight", C.c_int32),
    ]


class EgReadOpts(C.Structure):
    _fields_ = [
        ("weight_mode", C.c_int32),
        ("rnd_lo", C.c_int32),
        ("rnd_hi", C.c_int32),
        ("rnd_seed", C.c_uint64),
    ]


class EgBatchOpts(C.Structure):
    _fields_ = [
        ("thresholds", C.c_int32),
        ("scale", C.c_int32),
        ("block", C.c_int32),
        ("device", C.c_int32),
        ("max_rounds", C.c_int64),
        ("timeout_ms", C.c_double),
        ("use_graph", C.c_int32),
        ("group_max", C.c_int32),
        ("tail_rows", C.c_int32),
        ("park_percent", C.c_int32),
        ("tail_sweeps", C.c_int32),
        ("tail_cluster", C.c_int32),
        ("reserved", C.c_int32 * 2),
    ]


class EgBatchStats(C.Structure):
    _fields_ = [
        ("num_games", C.c_int32),
        ("thresholds", C.c_int32),
        ("total_nodes", C.c_int64),
        ("total_edges", C.c_int64),
        ("rounds_max", C.c_int64),
        ("rounds_sum", C.c_int64),
        ("lifts", C.c_int64),
        ("edges", C.c_int64),
        ("num_top", C.c_int64),
        ("solve_ms", C.c_double),
        ("block", C.c_int32),
        ("grid", C.c_int32),
        ("games_failed", C.c_int32),
        ("graph_replayed", C.c_int32),
        ("num_units", C.c_int32),
        ("smem_bytes", C.c_int32),
        ("tail_entries", C.c_int32),
        ("reserved", C.c_int32 * 1),
        ("phase1_ms", C.c_double),
        ("tail_ms", C.c_double),
    ]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


class EgServeOpts(C.Structure):
    _fields_ = [
        ("device", C.c_int32),
        ("max_inflight", C.c_int32),
        ("streams", C.c_int32),
        ("block", C.c_int32),
        ("hbm_reserve_bytes", C.c_int64),
        ("max_rounds", C.c_int64),
        ("large_ctas", C.c_int32),
        ("reserved", C.c_int32 * 5),
    ]


class EgServeStats(C.Structure):
    _fields_ = [
        ("submitted", C.c_int64), ("admitted", C.c_int64), ("completed", C.c_int64), ("failed", C.c_int64),
        ("games_registered", C.c_int64), ("games_resident", C.c_int64), ("game_uploads", C.c_int64),
        ("evictions", C.c_int64), ("micro_batches", C.c_int64), ("threshold_solves", C.c_int64),
        ("latency_p50_ms", C.c_double), ("latency_p99_ms", C.c_double), ("latency_mean_ms", C.c_double),
        ("latency_max_ms", C.c_double), ("elapsed_s", C.c_double), ("queries_per_s", C.c_double),
        ("solves_per_s", C.c_double), ("device_bytes", C.c_int64), ("reserved", C.c_int32 * 6),
    ]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


class EgTuneReport(C.Structure):
    _fields_ = [("candidates", C.c_int32), ("from_cache", C.c_int32), ("default_rate", C.c_double),
                ("best_rate", C.c_double), ("reserved", C.c_int32 * 4)]


class EgServeSpan(C.Structure):
    _fields_ = [("batch", C.c_int64), ("queries", C.c_int32), ("units", C.c_int32), ("begin_ms", C.c_double),
                ("end_ms", C.c_double)]


# every symbol the header declares, with (restype, argtypes)
_P = C.c_void_p
_I32, _I64 = C.c_int32, C.c_int64
SIGNATURES = {
    "eg_last_error": (C.c_char_p, []),
    "eg_abi_version": (_I32, []),
    "eg_opts_default": (None, [C.POINTER(EgOpts)]),
    "eg_device_count": (_I32, [C.POINTER(_I32)]),
    "eg_compute_mg": (_I32, [C.POINTER(EgGame), _I32, C.POINTER(_I64)]),
    "eg_default_max_loop": (_I64, [_I64, _I64, _I64, _I64]),
    "eg_validate": (_I32, [C.POINTER(EgGame)]),
    "eg_solve_i32": (_I32, [C.POINTER(EgGame), C.POINTER(EgOpts), _P, C.POINTER(EgStats)]),
    "eg_solve_i64": (_I32, [C.POINTER(EgGame), C.POINTER(EgOpts), _P, C.POINTER(EgStats)]),
    "eg_dgame_upload": (_I32, [C.POINTER(EgGame), C.POINTER(EgOpts), C.POINTER(_P)]),
    "eg_dgame_from_device": (_I32, [C.POINTER(EgGame), C.POINTER(EgOpts), C.POINTER(_P)]),
    "eg_dgame_solve": (_I32, [_P, C.POINTER(EgOpts), C.POINTER(EgStats)]),
    "eg_dgame_credits_i32": (_I32, [_P, _P]),
    "eg_dgame_credits_i64": (_I32, [_P, _P]),
    "eg_dgame_credits_device": (_I32, [_P, C.POINTER(_P), C.POINTER(_I32)]),
    "eg_dgame_device_bytes": (_I64, [_P]),
    "eg_dgame_tune": (_I32, [_P, C.POINTER(EgOpts), _I64, C.POINTER(EgOpts), C.POINTER(EgTuneReport)]),
    "eg_dgame_free": (None, [_P]),
    "eg_csr2csc_i32": (_I32, [_I32, _I32, _I64, _P, _P, _P, _P, _P, _P]),
    "eg_cancel_flag_alloc": (_I32, [C.POINTER(_P)]),
    "eg_cancel_flag_free": (None, [_P]),
    "eg_read_game_file": (_I32, [C.c_char_p, C.POINTER(EgReadOpts), C.POINTER(C.POINTER(EgOwnedGame))]),
    "eg_read_game_buffer": (_I32, [C.c_char_p, C.c_size_t, C.POINTER(EgReadOpts), C.POINTER(C.POINTER(EgOwnedGame))]),
    "eg_owned_game_free": (None, [C.POINTER(EgOwnedGame)]),
    "eg_write_game_binary": (_I32, [C.c_char_p, C.POINTER(EgOwnedGame), C.POINTER(EgReadOpts)]),
    "eg_read_game_binary": (_I32, [C.c_char_p, C.POINTER(EgReadOpts), C.POINTER(C.POINTER(EgOwnedGame))]),
    "eg_read_game_file_cached": (_I32, [C.c_char_p, C.POINTER(EgReadOpts), C.c_char_p,
                                        C.POINTER(C.POINTER(EgOwnedGame))]),
    "eg_parse_text": (_I32, [C.c_char_p, C.c_size_t, _P]),
    "eg_read_file_bytes": (_I32, [C.c_char_p, C.POINTER(C.c_void_p), C.POINTER(C.c_size_t)]),
    "eg_generate": (_I32, [_I32, _I32, _I32, _I32, _I32, C.c_uint64, C.POINTER(C.POINTER(EgOwnedGame))]),
    "eg_batch_create": (_I32, [C.POINTER(EgGame), _I32, C.POINTER(EgBatchOpts), C.POINTER(_P)]),
    "eg_batch_set_thresholds": (_I32, [_P, _P]),
    "eg_batch_solve": (_I32, [_P, C.POINTER(EgBatchStats)]),
    "eg_batch_credits": (_I32, [_P, _I32, _P]),
    "eg_batch_game_result": (_I32, [_P, _I32, C.POINTER(_I64), C.POINTER(_I32)]),
    "eg_batch_tune": (_I32, [_P, C.POINTER(_I32)]),
    "eg_batch_device_bytes": (_I64, [_P]),
    "eg_batch_free": (None, [_P]),
    "eg_csr2csc_device_noalloc": (_I32, [_I32, _I32, _I64, _P, _P, _P, _P, _P, _P, _P]),
    "eg_fixture_clique_text": (_I32, [_I32, C.POINTER(C.c_void_p), C.POINTER(C.c_size_t)]),
    "eg_fixture_ladder_text": (_I32, [_I32, C.POINTER(C.c_void_p), C.POINTER(C.c_size_t)]),
    "eg_fixture_copies_text": (_I32, [C.c_char_p, C.c_size_t, _I32, C.POINTER(C.c_void_p), C.POINTER(C.c_size_t)]),
    "eg_free_text": (None, [C.c_void_p]),
    "eg_serve_create": (_I32, [C.POINTER(EgServeOpts), C.POINTER(_P)]),
    "eg_serve_add_game": (_I32, [_P, C.POINTER(EgGame), C.POINTER(_I64)]),
    "eg_serve_remove_game": (_I32, [_P, _I64]),
    "eg_serve_submit": (_I32, [_P, _I64, _P, _I32, _I32, C.POINTER(_I64)]),
    "eg_serve_poll": (_I32, [_P, _I64, C.POINTER(_I32), C.POINTER(C.c_double)]),
    "eg_serve_wait": (_I32, [_P, _I64, C.c_double]),
    "eg_serve_result": (_I32, [_P, _I64, _P, C.POINTER(_I64)]),
    "eg_serve_stats_get": (_I32, [_P, C.POINTER(EgServeStats)]),
    "eg_serve_trace": (_I32, [_P, C.POINTER(EgServeSpan), _I32, C.POINTER(_I32)]),
    "eg_serve_destroy": (_I32, [_P]),
}

_lib = None


def load() -> C.CDLL:
    """Loads the solver library (once); raises if it has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python -m egsolver_b200.build` "
                "(the solver has no CPU fallback)")
        lib = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib
