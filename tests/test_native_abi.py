"""The C ABI library: it loads, exports every symbol that include/lbm_d3q19.h
declares, and its argument checks answer without touching a GPU."""

from __future__ import annotations

import ctypes as C
import re

import numpy as np
import pytest
from conftest import ROOT

from lattice_boltzmann_d3q19_b200 import _native as N

HEADER = ROOT / "include" / "lbm_d3q19.h"


def declared_functions() -> list[str]:
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(lbm_[a-z0-9_]+)\s*\(", text)))


def test_header_declarations_are_bound():
    names = declared_functions()
    assert len(names) >= 30
    assert set(names) == set(N.SIGNATURES), set(names) ^ set(N.SIGNATURES)


def test_library_exports_every_declared_symbol():
    lib = N.lib()
    for name in declared_functions():
        assert hasattr(lib, name), name


def test_desc_defaults():
    d = N.LbmDesc()
    assert N.lib().lbm_desc_init(C.byref(d)) == N.LBM_OK
    assert (d.nx, d.ny, d.nz) == (1, 1, 1)
    assert d.periodic == 7 and d.tau == 1.0 and d.inflow_rho == 1.0
    assert N.lib().lbm_version() >= 10000


def test_desc_layout_matches_header():
    # 6 int32, tau, 18 + 3 doubles, drag_k, inflow_rho, 3 doubles, 4 int32,
    # 3 doubles (storage_ref_u)
    assert C.sizeof(N.LbmDesc) == 6 * 4 + 8 + 21 * 8 + 8 + 8 + 24 + 16 + 24


@pytest.mark.parametrize(
    "field,value",
    [("nx", 0), ("storage", 9), ("force_mode", 7), ("tau", 0.5), ("periodic", 8), ("block_size", 48),
     ("cells_per_thread", 3), ("staging", 5)],
)
def test_create_rejects_bad_descriptors(field, value):
    d = N.LbmDesc()
    N.lib().lbm_desc_init(C.byref(d))
    d.nx = d.ny = d.nz = 4
    setattr(d, field, value)
    h = C.c_void_p()
    rc = N.lib().lbm_create(C.byref(d), C.byref(h))
    assert rc == N.LBM_ERR_INVALID
    assert not h.value
    assert N.lib().lbm_last_error()


def test_create_too_many_cells():
    d = N.LbmDesc()
    N.lib().lbm_desc_init(C.byref(d))
    d.nx, d.ny, d.nz = 2048, 2048, 1024
    h = C.c_void_p()
    assert N.lib().lbm_create(C.byref(d), C.byref(h)) == N.LBM_ERR_INVALID


def test_null_arguments():
    lib = N.lib()
    assert lib.lbm_create(None, None) == N.LBM_ERR_INVALID
    assert lib.lbm_step(None, 1) == N.LBM_ERR_INVALID
    assert lib.lbm_destroy(None) == N.LBM_OK
    assert lib.lbm_step_count(None) == -1


def test_no_device_is_reported_not_faked():
    """Without a GPU the library says so; there is no CPU fallback."""
    if N.device_count() > 0:
        pytest.skip("a CUDA device is present")
    d = N.LbmDesc()
    N.lib().lbm_desc_init(C.byref(d))
    h = C.c_void_p()
    assert N.lib().lbm_create(C.byref(d), C.byref(h)) == N.LBM_ERR_NO_DEVICE
    f = np.zeros((19, 2, 2, 2))
    out = np.empty_like(f)
    rc = N.lib().lbm_stream(N.ptr(f), N.ptr(out), 2, 2, 2)
    assert rc == N.LBM_ERR_NO_DEVICE
    from lattice_boltzmann_d3q19_b200 import reference as R

    with pytest.raises(N.LbmError):
        R.stream(f)


def _dev_calls_with(ptrs, shape=(3, 2, 2)):
    """Every stateless device-pointer entry point called with the given
    pointers (ptrs[k] for its k-th array argument)."""
    lib = N.lib()
    p = [C.c_void_p(a.ctypes.data) for a in ptrs]
    nx, ny, nz = shape
    return {
        "feq_field": lib.lbm_feq_field_dev(p[0], p[1], p[2], nx, ny, nz, None),
        "density_field": lib.lbm_density_field_dev(p[0], p[1], nx, ny, nz, None),
        "momentum_field": lib.lbm_momentum_field_dev(p[0], p[1], nx, ny, nz, None),
        "macroscopic_velocity": lib.lbm_macroscopic_velocity_dev(p[0], None, p[1], nx, ny, nz, None),
        "stream": lib.lbm_stream_dev(p[0], p[1], nx, ny, nz, None),
        "bgk_step": lib.lbm_bgk_step_dev(p[0], p[1], 0.7, None, nx, ny, nz, None),
        "bounce_back": lib.lbm_bounce_back_y_walls_dev(p[0], p[1], nx, ny, nz, None, None, None),
        "conservation_noalloc": lib.lbm_conservation_noalloc(p[0], None, nx, ny, nz, p[1], None),
    }


def test_dev_entry_points_refuse_host_pointers_without_a_device():
    """Host NumPy pointers handed to the device-pointer entry points come
    back as an error status (no device here: before any kernel could run)."""
    if N.device_count() > 0:
        pytest.skip("a CUDA device is present (the gpu-marked test covers it)")
    arrs = [np.zeros(19 * 12) for _ in range(3)]
    for name, rc in _dev_calls_with(arrs).items():
        assert rc < 0, name


@pytest.mark.gpu
def test_dev_entry_points_reject_host_pointers():
    """On a GPU, host memory passed where device memory is required is
    rejected with LBM_ERR_INVALID before any launch (a kernel would fault)."""
    arrs = [np.zeros(19 * 12) for _ in range(3)]
    for name, rc in _dev_calls_with(arrs).items():
        assert rc == N.LBM_ERR_INVALID, (name, rc, N.lib().lbm_last_error())
