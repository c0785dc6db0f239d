"""The C-ABI library on the CPU: it loads, exports every declared symbol, and
its host-side logic (validation, MG, round cap, generators, error paths)
behaves; nothing here launches a kernel."""
from __future__ import annotations

import re
import subprocess

import numpy as np
import pytest

import egsolver_b200 as eg
from egsolver_b200 import _ffi, workloads
from oracle import oracle as O
from tests.conftest import ROOT

HEADERS = [ROOT / "include" / "egsolver_b200.h", ROOT / "include" / "egsolver_b200_serve.h"]

REFERENCE_ABI = ["alloca_memoria_host", "alloca_memoria_device", "copia_dati_su_device", "gpu_solver",
                 "dealloca_memoria_host", "dealloca_memoria_device", "checkDevice", "checkCUDAError"]


def declared_functions(path) -> set[str]:
    text = re.sub(r"/\*.*?\*/", "", path.read_text(), flags=re.S)
    names = set()
    for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b(eg_\w+)\s*\(", text, flags=re.M):
        names.add(m.group(1))
    return names


def exported(lib_path) -> set[str]:
    out = subprocess.run(["nm", "-D", "--defined-only", str(lib_path)], capture_output=True, text=True, check=True)
    return {line.split()[-1] for line in out.stdout.splitlines() if " T " in line}


def test_every_declared_function_is_exported_and_bound():
    decl = set().union(*(declared_functions(h) for h in HEADERS))
    assert len(decl) >= 25, decl
    exp = exported(_ffi.LIB_PATH)
    missing = decl - exp
    assert not missing, f"declared but not exported: {sorted(missing)}"
    unbound = decl - set(_ffi.SIGNATURES)
    assert not unbound, f"declared but not bound in _ffi: {sorted(unbound)}"
    lib = eg.lib()
    for name in decl:
        assert getattr(lib, name) is not None


def test_reference_abi_shim_exports_the_reference_symbols():
    out = subprocess.run(["nm", "--defined-only", str(ROOT / "egsolver_b200" / "libegrefabi.a")],
                         capture_output=True, text=True, check=True).stdout
    defined = {line.split()[-1] for line in out.splitlines() if " T " in line}
    assert set(REFERENCE_ABI) <= defined


def test_abi_version_and_defaults():
    assert eg.lib().eg_abi_version() == 1
    o = eg.make_opts()
    assert o.credit_bits == 64 and o.variant == eg.VARIANT_AUTO and o.max_rounds == -1


def test_validate_rejects_malformed_games():
    ok = eg.Game(row_ptr=[0, 1, 2], succ=[1, 0], weight=[1, -1], num_nodes0=1)
    eg.validate(ok)
    bad = [
        eg.Game(row_ptr=[0, 1, 1], succ=[1], weight=[1], num_nodes0=1),          # sink
        eg.Game(row_ptr=[0, 1, 2], succ=[1, 2], weight=[1, 1], num_nodes0=1),     # successor out of range
        eg.Game(row_ptr=[0, 2, 1], succ=[1, 0], weight=[1, 1], num_nodes0=1),     # not monotone
        eg.Game(row_ptr=[0, 1, 2], succ=[1, 0], weight=[1, 1], num_nodes0=3),     # split out of range
        eg.Game(row_ptr=[0, 1, 2], succ=[1, 0], weight=[1, 1], owner=np.array([0, 2], np.uint8)),
    ]
    for g in bad:
        with pytest.raises(eg.EGError) as ei:
            eg.validate(g)
        assert ei.value.name == "EG_ERR_INVALID"


def test_mg_overflow_check_mirrors_reference():
    n = 3
    g = eg.Game(row_ptr=np.arange(n + 1), succ=[1, 2, 0], weight=[-2**31 + 1, -2**31 + 1, -5], num_nodes0=1)
    with pytest.raises(eg.EGError) as ei:
        eg.compute_mg(g, 32)
    assert ei.value.name == "EG_ERR_OVERFLOW"
    assert eg.compute_mg(g, 64) == 2 * (2**31 - 1) + 5
    assert O.mg(g, 32) == -1


def test_generators_are_deterministic_and_shaped():
    a = workloads.cfg1()
    b = workloads.cfg1()
    np.testing.assert_array_equal(a.succ, b.succ)
    np.testing.assert_array_equal(a.weight, b.weight)
    assert a.num_nodes == 1000 and a.num_edges == 4000
    assert np.all(np.diff(a.row_ptr) == 4)
    assert a.weight.min() >= -10 and a.weight.max() <= 10
    c3 = workloads.cfg3()
    assert c3.num_edges == 2000 * 1999
    # no self-loops, no duplicate successors
    for g in (a, workloads.cfg2(1 << 14)):
        src = np.repeat(np.arange(g.num_nodes), np.diff(g.row_ptr))
        assert not np.any(src == g.succ)
        pairs = src.astype(np.int64) * g.num_nodes + g.succ
        assert np.unique(pairs).size == pairs.size
    # owners are fair coins
    assert 400 < a.num_nodes0 < 600


def test_cfg2_degree_law():
    g = workloads.cfg2(1 << 16)
    deg = np.diff(g.row_ptr)
    assert deg.min() >= 1 and deg.max() <= 4096
    assert 7.0 < deg.mean() < 8.8
    # P(deg >= k) ~ 1/k for the continuous x^-2 law
    assert abs((deg >= 10).mean() - 0.1) < 0.01


def test_solve_without_device_fails_loudly():
    if eg.device_count() > 0:
        pytest.skip("a device is present")
    g = workloads.cfg1()
    with pytest.raises(eg.EGError) as ei:
        eg.solve(g)
    assert ei.value.name in ("EG_ERR_NO_DEVICE", "EG_ERR_CUDA")


def test_bad_options_rejected_before_any_device_work():
    g = workloads.cfg1()
    with pytest.raises(eg.EGError) as ei:
        eg.solve(g, credit_bits=16)
    assert ei.value.name == "EG_ERR_INVALID"
    with pytest.raises(eg.EGError):
        eg.solve(g, variant=eg.VARIANT_WARP, lanes_per_vertex=3)
    for bad in (dict(direction=3), dict(direction=-1), dict(dense_permille=1001), dict(sparse_permille=-1),
                dict(dense_depth=3), dict(dense_depth=-1), dict(dense_sweeps=5), dict(dense_sweeps=-1)):
        with pytest.raises(eg.EGError) as ei:
            eg.solve(g, **bad)
        assert ei.value.name == "EG_ERR_INVALID"


def test_bad_batch_options_rejected_before_any_device_work():
    games = [workloads.cfg1()]
    for bad in (dict(group_max=3), dict(tail_sweeps=17), dict(tail_sweeps=-1), dict(tail_cluster=3),
                dict(tail_cluster=32), dict(block=48)):
        with pytest.raises(eg.EGError) as ei:
            eg.Batch(games, thresholds=2, scale=1, **bad)
        assert ei.value.name == "EG_ERR_INVALID"
