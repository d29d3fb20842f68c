"""The C ABI without a GPU: the library loads, exports every function include/drmppi.h
declares, the ctypes structures have the C layout, and argument validation rejects bad
configurations before touching a device (the reference throws std::runtime_error for
the same cases: src/mppi_controller.cu:27-29, src/config.cpp:10-21,39-46)."""
from __future__ import annotations

import ctypes as C
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

from conftest import ROOT, drb
from helpers import small_mppi

abi = drb.abi
HEADER = ROOT / "include" / "drmppi.h"


def declared_functions() -> list[str]:
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(dr_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_function():
    lib = abi.lib()
    names = declared_functions()
    assert len(names) > 40
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    nm = subprocess.run(["nm", "-D", "--defined-only", str(abi.LIB_PATH)], capture_output=True, text=True).stdout
    for n in names:
        assert re.search(rf"\bT {n}$", nm, flags=re.M), n
    # every declared function has a ctypes prototype
    assert set(names) <= set(abi.EXPORTED), sorted(set(names) - set(abi.EXPORTED))


def test_struct_layouts_match_c(tmp_path: Path):
    structs = {"dr_opp_config": abi.dr_opp_config, "dr_env_config": abi.dr_env_config, "dr_sim_state": abi.dr_sim_state,
               "dr_mppi_config": abi.dr_mppi_config, "dr_prmppi_config": abi.dr_prmppi_config, "dr_mppi_info": abi.dr_mppi_info,
               "dr_prmppi_info": abi.dr_prmppi_info, "dr_pid_config": abi.dr_pid_config, "dr_gate_env_config": abi.dr_gate_env_config,
               "dr_gate_state": abi.dr_gate_state}
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void){"]
    for sname, st in structs.items():
        lines.append(f'printf("{sname} size %zu\\n", sizeof({sname}));')
        for fname, _ in st._fields_:
            lines.append(f'printf("{sname}.{fname} %zu\\n", offsetof({sname}, {fname}));')
    lines.append("return 0;}")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    got = {}
    for ln in out:
        if ln.strip():
            k, v = ln.rsplit(" ", 1)
            got[k] = int(v)
    for sname, st in structs.items():
        assert got[f"{sname} size"] == C.sizeof(st), sname
        for fname, _ in st._fields_:
            assert got[f"{sname}.{fname}"] == getattr(st, fname).offset, f"{sname}.{fname}"


def _create(sc, cfg=None):
    h = C.c_void_p()
    rc = abi.lib().dr_mppi_create(C.byref(sc.env), C.byref(cfg or sc.mppi), 1, None, 0, None, C.byref(h))
    if rc == abi.DR_OK:
        abi.lib().dr_mppi_destroy(h)
    return rc


def test_invalid_configs_are_rejected_before_any_device_work():
    sc = small_mppi(True, K=64, T=20, M=6)
    bad = []
    c = type(sc.mppi).from_buffer_copy(sc.mppi)
    c.n_knots = 70
    bad.append(c)  # more knots than DR_MAX_KNOTS (config.cpp:39-41)
    c = type(sc.mppi).from_buffer_copy(sc.mppi)
    c.knots[2] = c.knots[1]
    bad.append(c)  # knots not increasing
    c = type(sc.mppi).from_buffer_copy(sc.mppi)
    c.knots[c.n_knots - 1] = c.n_timesteps - 1
    bad.append(c)  # tau_{M-1} > T-2 (utils.py:497 requirement)
    c = type(sc.mppi).from_buffer_copy(sc.mppi)
    c.n_samples = 0
    bad.append(c)
    c = type(sc.mppi).from_buffer_copy(sc.mppi)
    c.verif_horizon = c.n_timesteps + 1
    bad.append(c)  # the reference kernel would index failCount out of range
    c = type(sc.mppi).from_buffer_copy(sc.mppi)
    c.inv_temperature = float("nan")
    bad.append(c)
    for c in bad:
        assert _create(sc, c) == abi.DR_ERR_INVALID_ARG
        assert abi.lib().dr_last_error()
    env = abi.dr_env_config.from_buffer_copy(sc.env)
    env.n_theta = 3  # not compiled in
    h = C.c_void_p()
    assert abi.lib().dr_mppi_create(C.byref(env), C.byref(sc.mppi), 1, None, 0, None, C.byref(h)) == abi.DR_ERR_UNSUPPORTED
    env = abi.dr_env_config.from_buffer_copy(sc.env)
    env.p_grid = None
    assert abi.lib().dr_mppi_create(C.byref(env), C.byref(sc.mppi), 1, None, 0, None, C.byref(h)) == abi.DR_ERR_INVALID_ARG
    nan_grid = sc.grids.kappa_grid.copy()
    nan_grid[17] = np.nan
    env = abi.dr_env_config.from_buffer_copy(sc.env)
    env.kappa_grid = abi.fptr(nan_grid)
    assert abi.lib().dr_mppi_create(C.byref(env), C.byref(sc.mppi), 1, None, 0, None, C.byref(h)) == abi.DR_ERR_INVALID_ARG
    # a valid configuration either succeeds (GPU present) or reports the missing device
    assert _create(sc) in (abi.DR_OK, abi.DR_ERR_NO_DEVICE)


def test_wrong_nominal_size_raises_like_the_reference():
    sc = small_mppi(False, K=64, T=20)
    with pytest.raises(ValueError, match="expected nominal size"):
        drb.controllers.MPPIController(sc.env, sc.mppi, 1, nominal=np.zeros(5, np.float32))


def test_status_strings():
    for s in range(8):
        assert abi.lib().dr_status_string(s)
    assert abi.lib().dr_abi_version() == abi.DR_ABI_VERSION == 2
    assert abi.lib().dr_supported(1, 2) == 1 and abi.lib().dr_supported(1, 3) == 0


def test_invalid_track_samples_and_cp_arguments_are_rejected():
    """dr_track_grids refuses non-finite samples and repeated consecutive samples (the
    arc-length spline parameter must increase strictly, as scipy's CubicSpline requires
    in the reference), before any device work; the test hooks refuse bad sizes."""
    n = abi.DR_N_TRACK_SAMPLES
    ang = np.arange(n) * 2 * np.pi / n
    q = np.ascontiguousarray(np.stack([6 * np.cos(ang), 6 * np.sin(ang)], axis=1)[None], np.float64)
    out = [np.zeros((1, n, 2), np.float32), np.zeros((1, n, 2), np.float32), np.zeros((1, n, 2), np.float32), np.zeros((1, n), np.float32),
           np.zeros(1, np.float32)]
    ptrs = [abi.fptr(a) for a in out]
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    bad = q.copy()
    bad[0, 7, 1] = np.nan
    assert abi.lib().dr_track_grids(dp(bad), 1, *ptrs) == abi.DR_ERR_INVALID_ARG
    bad = q.copy()
    bad[0, 8] = bad[0, 7]
    assert abi.lib().dr_track_grids(dp(bad), 1, *ptrs) == abi.DR_ERR_INVALID_ARG
    assert abi.lib().dr_track_grids(dp(q), 0, *ptrs) == abi.DR_ERR_INVALID_ARG
    k = np.zeros(1, np.uint32)
    assert abi.lib().dr_debug_cp_host(abi.uptr(k), 0, 10, 0.05, 1, dp(np.zeros(1))) == abi.DR_ERR_INVALID_ARG
