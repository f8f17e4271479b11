"""ctypes binding of liblbm_d3q19.so (the C ABI declared in include/lbm_d3q19.h).

The library is built in-tree by ``bit-physics_b200/csrc/Makefile``.  There is
no CPU fallback: importing the package without the built library, or calling
into it without a CUDA device, raises.
"""

from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

PKG_DIR = Path(__file__).resolve().parent
LIB_PATH = PKG_DIR / "liblbm_d3q19.so"

LBM_OK = 0
LBM_ERR_INVALID = -1
LBM_ERR_CUDA = -2
LBM_ERR_NOMEM = -3
LBM_ERR_STATE = -4
LBM_ERR_NONFINITE = -5
LBM_ERR_UNSUPPORTED = -6
LBM_ERR_NO_DEVICE = -7

STORAGE = {"f64": 0, "f32": 1, "f16": 2, "bf16": 3}
FORCE = {"none": 0, "uniform": 1, "field": 2, "drag": 3}
FACES = {"x-": 0, "x+": 1, "y-": 2, "y+": 3, "z-": 4, "z+": 5}
STAGING = {"auto": 0, "registers": 1, "tma": 2, "pipelined": 3, "persistent": 4}
SCHEDULES = {"single": 0, "pair_scalar": 1, "pair_mixed": 2, "branches": 3}
CELL_FLUID, CELL_SOLID, CELL_INFLOW, CELL_OUTFLOW = 0, 1, 2, 3


class LbmError(RuntimeError):
    """A C-ABI call returned a negative status."""

    def __init__(self, code: int, message: str):
        super().__init__(f"[{code}] {message}")
        self.code = code


class LbmDesc(C.Structure):
    _fields_ = [
        ("nx", C.c_int32),
        ("ny", C.c_int32),
        ("nz", C.c_int32),
        ("storage", C.c_int32),
        ("periodic", C.c_int32),
        ("force_mode", C.c_int32),
        ("tau", C.c_double),
        ("wall_velocity", C.c_double * 18),
        ("body_force", C.c_double * 3),
        ("drag_k", C.c_double),
        ("inflow_rho", C.c_double),
        ("inflow_u", C.c_double * 3),
        ("device", C.c_int32),
        ("block_size", C.c_int32),
        ("cells_per_thread", C.c_int32),
        ("staging", C.c_int32),
        ("storage_ref_u", C.c_double * 3),
    ]


# Every symbol declared in include/lbm_d3q19.h, with its ctypes signature.
_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)
_u8p = C.POINTER(C.c_uint8)
_h = C.c_void_p
_i = C.c_int32
SIGNATURES: dict[str, tuple[list, object]] = {
    "lbm_desc_init": ([C.POINTER(LbmDesc)], C.c_int),
    "lbm_create": ([C.POINTER(LbmDesc), C.POINTER(_h)], C.c_int),
    "lbm_destroy": ([_h], C.c_int),
    "lbm_set_stream": ([_h, C.c_void_p], C.c_int),
    "lbm_synchronize": ([_h], C.c_int),
    "lbm_set_populations": ([_h, _dp], C.c_int),
    "lbm_get_populations": ([_h, _dp], C.c_int),
    "lbm_set_equilibrium": ([_h, _dp, _dp], C.c_int),
    "lbm_set_flags": ([_h, _u8p], C.c_int),
    "lbm_set_force_field": ([_h, _dp], C.c_int),
    "lbm_set_porosity": ([_h, _fp], C.c_int),
    "lbm_set_tau": ([_h, C.c_double], C.c_int),
    "lbm_set_wall_velocity": ([_h, _i, _dp], C.c_int),
    "lbm_set_body_force": ([_h, _dp], C.c_int),
    "lbm_step": ([_h, _i], C.c_int),
    "lbm_step_count": ([_h], C.c_int64),
    "lbm_step_planes": ([_h, _i, _i], C.c_int),
    "lbm_step_commit": ([_h], C.c_int),
    "lbm_set_rule_blocks": ([_h, _i], C.c_int),
    "lbm_get_rule_blocks": ([_h, C.POINTER(C.c_int32), C.POINTER(C.c_int32)], C.c_int),
    "lbm_get_rho_u": ([_h, _dp, _dp], C.c_int),
    "lbm_run_capture": ([_h, _i, _i, _dp, _dp], C.c_int),
    "lbm_step_monitor": ([_h, _i, _dp], C.c_int),
    "lbm_conservation": ([_h, _dp], C.c_int),
    "lbm_check_health": ([_h], C.c_int),
    "lbm_feq_field": ([_dp, _dp, _dp, _i, _i, _i], C.c_int),
    "lbm_density_field": ([_dp, _dp, _i, _i, _i], C.c_int),
    "lbm_momentum_field": ([_dp, _dp, _i, _i, _i], C.c_int),
    "lbm_macroscopic_velocity": ([_dp, _dp, _dp, _i, _i, _i], C.c_int),
    "lbm_stream": ([_dp, _dp, _i, _i, _i], C.c_int),
    "lbm_bgk_step": ([_dp, _dp, C.c_double, _dp, _i, _i, _i], C.c_int),
    "lbm_bounce_back_y_walls": ([_dp, _dp, _i, _i, _i, _dp, _dp], C.c_int),
    "lbm_feq_field_dev": ([_h, _h, _h, _i, _i, _i, _h], C.c_int),
    "lbm_density_field_dev": ([_h, _h, _i, _i, _i, _h], C.c_int),
    "lbm_momentum_field_dev": ([_h, _h, _i, _i, _i, _h], C.c_int),
    "lbm_macroscopic_velocity_dev": ([_h, _h, _h, _i, _i, _i, _h], C.c_int),
    "lbm_stream_dev": ([_h, _h, _i, _i, _i, _h], C.c_int),
    "lbm_bgk_step_dev": ([_h, _h, C.c_double, _h, _i, _i, _i, _h], C.c_int),
    "lbm_bounce_back_y_walls_dev": ([_h, _h, _i, _i, _i, _dp, _dp, _h], C.c_int),
    "lbm_batch_create": ([C.POINTER(LbmDesc), _i, C.POINTER(_h)], C.c_int),
    "lbm_batch_destroy": ([_h], C.c_int),
    "lbm_batch_count": ([_h], C.c_int),
    "lbm_batch_lattice": ([_h, _i, C.POINTER(_h)], C.c_int),
    "lbm_batch_set_schedule": ([_h, _i, _i, _i], C.c_int),
    "lbm_batch_get_schedule": ([_h, C.POINTER(_i), C.POINTER(_i), C.POINTER(_i)], C.c_int),
    "lbm_batch_step": ([_h, _i], C.c_int),
    "lbm_batch_step_unbatched": ([_h, _i], C.c_int),
    "lbm_batch_autotune": ([_h, _i, _dp], C.c_int),
    "lbm_batch_synchronize": ([_h], C.c_int),
    "lbm_conservation_noalloc": ([_h, _h, _i, _i, _i, _h, _h], C.c_int),
    "lbm_plane_get": ([_h, _i, C.c_uint32, _h], C.c_int),
    "lbm_plane_put": ([_h, _i, C.c_uint32, _h], C.c_int),
    "lbm_conservation_planes": ([_h, _i, _i, _dp], C.c_int),
    "lbm_get_rho_u_dev": ([_h, _h, _h], C.c_int),
    "lbm_diagnostics": ([_h, C.c_double, _dp], C.c_int),
    "lbm_test_barrier_limit": ([_h, C.c_int32, C.c_int64], C.c_int),
    "lbm_moment16_basis": ([_dp, _dp], C.c_int),
    "lbm_moment16_calibrate": ([_h, C.c_int32, C.c_double, _dp, _dp], C.c_int),
    "lbm_moment16_step": ([_h, _dp, _dp, C.c_int32], C.c_int),
    "lbm_set_porosity_dev": ([_h, _h], C.c_int),
    "lbm_tape_forward": ([_h, _i, _i, C.POINTER(_h)], C.c_int),
    "lbm_tape_backward": ([_h, _h, _h, _h, _h], C.c_int),
    "lbm_tape_bytes": ([_h], C.c_int64),
    "lbm_tape_destroy": ([_h], C.c_int),
    "lbm_last_error": ([], C.c_char_p),
    "lbm_version": ([], C.c_int),
    "lbm_device_count": ([], C.c_int),
    "lbm_release_workspace": ([], C.c_int),
}

_lib: C.CDLL | None = None


def lib() -> C.CDLL:
    """Load the native library once; raise if it has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `make -C bit-physics_b200/csrc` "
                "(or __graft_entry__.build()); there is no CPU fallback"
            )
        lib_ = C.CDLL(str(LIB_PATH))
        for name, (args, res) in SIGNATURES.items():
            fn = getattr(lib_, name)
            fn.argtypes = args
            fn.restype = res
        _lib = lib_
    return _lib


def check(rc: int) -> None:
    if rc != LBM_OK:
        msg = lib().lbm_last_error()
        raise LbmError(int(rc), msg.decode() if msg else "")


def device_count() -> int:
    return int(lib().lbm_device_count())


def require_device() -> None:
    if device_count() == 0:
        raise LbmError(LBM_ERR_NO_DEVICE, "no CUDA device available (the engine has no CPU fallback)")


def f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def ptr(a: np.ndarray | None, ctype=_dp):
    return None if a is None else a.ctypes.data_as(ctype)


_MADV_HUGEPAGE = 14
_libc = None


def fresh_host_array(shape) -> np.ndarray:
    """np.empty(shape) float64 with transparent huge pages requested for it
    (Linux madvise): a readback of ~100 MB into a fresh array then takes
    ~50 page faults instead of ~25,000.  Only for arrays allocated here;
    caller-owned output arrays are never advised.  A hint: failures are
    ignored."""
    global _libc
    a = np.empty(shape)
    try:
        if _libc is None:
            _libc = C.CDLL(None, use_errno=True)
            _libc.madvise.argtypes = [C.c_void_p, C.c_size_t, C.c_int]
            _libc.madvise.restype = C.c_int
        page = 4096
        lo = (a.ctypes.data + page - 1) & ~(page - 1)
        hi = (a.ctypes.data + a.nbytes) & ~(page - 1)
        if hi > lo:
            _libc.madvise(C.c_void_p(lo), C.c_size_t(hi - lo), _MADV_HUGEPAGE)
    except (OSError, AttributeError):
        pass
    return a

