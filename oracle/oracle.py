"""CPU oracle for the D3Q19 BGK hot path -- TEST INFRASTRUCTURE ONLY.

ctypes front end of ``liblbm_oracle.so`` (built from ``lbm_oracle.c`` by the
``Makefile`` beside it).  Only ``tests/``, ``__graft_entry__.smoke()`` and
``bench.py`` (its ``cpu_baseline`` leg and the ``--impl reference`` arm) may
import this module; the product package never does.

Two layers, as in ``lbm_oracle.c``:

* reference-exact f64 functions with the signatures of the Stack-E Warp module
  ``packages/lattice-boltzmann-d3q19-stack-e/lattice_boltzmann_d3q19_stack_e/
  reference/d3q19_warp.py`` (``feq_field`` :253, ``density_field`` :283,
  ``momentum_field`` :295, ``stream`` :308, ``bgk_step`` :321,
  ``macroscopic_velocity`` :371, ``apply_bounce_back_y_walls`` :386);
* ``OracleLattice``: the generalised step (flags, walled faces, inflow /
  outflow, drag, reduced-precision storage) that the GPU engine implements.
"""

from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
_LIB_PATH = _HERE / "liblbm_oracle.so"

CELL_FLUID, CELL_SOLID, CELL_INFLOW, CELL_OUTFLOW = 0, 1, 2, 3
FORCE_NONE, FORCE_UNIFORM, FORCE_FIELD, FORCE_DRAG = 0, 1, 2, 3
STORE_F64, STORE_F32, STORE_F16_SHIFT, STORE_BF16_SHIFT = 0, 1, 2, 3
PERIODIC_X, PERIODIC_Y, PERIODIC_Z = 1, 2, 4
FACE_XM, FACE_XP, FACE_YM, FACE_YP, FACE_ZM, FACE_ZP = range(6)

_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)
_u8p = C.POINTER(C.c_uint8)


class _OrcLattice(C.Structure):
    _fields_ = [
        ("nx", C.c_int32),
        ("ny", C.c_int32),
        ("nz", C.c_int32),
        ("periodic", C.c_int32),
        ("force_mode", C.c_int32),
        ("storage", C.c_int32),
        ("tau", C.c_double),
        ("wall_u", C.c_double * 18),
        ("body_force", C.c_double * 3),
        ("drag_k", C.c_double),
        ("inflow_rho", C.c_double),
        ("inflow_u", C.c_double * 3),
        ("flags", _u8p),
        ("force", _dp),
        ("porosity", _fp),
        ("storage_ref_u", C.c_double * 3),
    ]


def build() -> Path:
    """Compile the oracle library with its Makefile (gcc, -ffp-contract=off)."""
    import subprocess

    subprocess.run(["make", "-s", "-C", str(_HERE)], check=True)
    return _LIB_PATH


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not _LIB_PATH.exists():
            build()
        _lib = C.CDLL(str(_LIB_PATH))
        i, d = C.c_int, C.c_double
        L = C.POINTER(_OrcLattice)
        _lib.orc_feq_field.argtypes = [_dp, _dp, _dp, i, i, i]
        _lib.orc_density_field.argtypes = [_dp, _dp, i, i, i]
        _lib.orc_momentum_field.argtypes = [_dp, _dp, i, i, i]
        _lib.orc_macroscopic_velocity.argtypes = [_dp, _dp, _dp, i, i, i]
        _lib.orc_collide.argtypes = [_dp, _dp, _dp, d, i, i, i]
        _lib.orc_stream.argtypes = [_dp, _dp, i, i, i]
        _lib.orc_bgk_step.argtypes = [_dp, _dp, d, _dp, i, i, i]
        _lib.orc_bounce_back_y_walls.argtypes = [_dp, _dp, i, i, i, _dp, _dp]
        _lib.orc_engine_collide_local.argtypes = [L, _dp, _dp, _dp, _dp]
        _lib.orc_engine_step.argtypes = [L, _dp, _dp, _dp, _dp]
        _lib.orc_engine_reconstruct.argtypes = [L, _dp, _dp, _dp, _dp]
        _lib.orc_engine_moments_local.argtypes = [L, _dp, _dp, _dp]
        _lib.orc_engine_run.argtypes = [L, _dp, i]
        _lib.orc_engine_run.restype = i
        _lib.orc_conservation.argtypes = [L, _dp, _dp]
        _lib.orc_store_round.argtypes = [i, _dp, _dp, C.c_int64]
        _lib.orc_constants.argtypes = [_dp, _dp]
        _lib.orc_num_threads.restype = i
        _lib.orc_set_num_threads.argtypes = [i]
        _lib.orc_f32_to_f16.argtypes = [C.c_float]
        _lib.orc_f32_to_f16.restype = C.c_uint16
        _lib.orc_f16_to_f32.argtypes = [C.c_uint16]
        _lib.orc_f16_to_f32.restype = C.c_float
        _lib.orc_f32_to_bf16.argtypes = [C.c_float]
        _lib.orc_f32_to_bf16.restype = C.c_uint16
        _lib.orc_bf16_to_f32.argtypes = [C.c_uint16]
        _lib.orc_bf16_to_f32.restype = C.c_float
    return _lib


def _ptr(a: np.ndarray | None, ctype=_dp):
    if a is None:
        return None
    return a.ctypes.data_as(ctype)


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def set_num_threads(n: int) -> None:
    lib().orc_set_num_threads(int(n))


def num_threads() -> int:
    return int(lib().orc_num_threads())


def constants() -> tuple[np.ndarray, np.ndarray]:
    w = np.empty(19)
    cs = np.empty(5)
    lib().orc_constants(_ptr(w), _ptr(cs))
    return w, cs


# --------------------------------------------------------------------------
# Reference-exact f64 surface (same names / argument meaning as d3q19_warp.py)
# --------------------------------------------------------------------------
def feq_field(rho, u) -> np.ndarray:
    rho, u = _f64(rho), _f64(u)
    nx, ny, nz = rho.shape
    out = np.empty((19, nx, ny, nz))
    lib().orc_feq_field(_ptr(rho), _ptr(u), _ptr(out), nx, ny, nz)
    return out


def density_field(f) -> np.ndarray:
    f = _f64(f)
    _, nx, ny, nz = f.shape
    out = np.empty((nx, ny, nz))
    lib().orc_density_field(_ptr(f), _ptr(out), nx, ny, nz)
    return out


def momentum_field(f) -> np.ndarray:
    f = _f64(f)
    _, nx, ny, nz = f.shape
    out = np.empty((3, nx, ny, nz))
    lib().orc_momentum_field(_ptr(f), _ptr(out), nx, ny, nz)
    return out


def macroscopic_velocity(f, force_lattice=None) -> np.ndarray:
    f = _f64(f)
    _, nx, ny, nz = f.shape
    F = None if force_lattice is None else _f64(force_lattice)
    out = np.empty((3, nx, ny, nz))
    lib().orc_macroscopic_velocity(_ptr(f), _ptr(F), _ptr(out), nx, ny, nz)
    return out


def collide(f, tau, force_lattice=None) -> np.ndarray:
    f = _f64(f)
    _, nx, ny, nz = f.shape
    F = None if force_lattice is None else _f64(force_lattice)
    out = np.empty_like(f)
    lib().orc_collide(_ptr(f), _ptr(out), _ptr(F), float(tau), nx, ny, nz)
    return out


def stream(f_post) -> np.ndarray:
    f = _f64(f_post)
    _, nx, ny, nz = f.shape
    out = np.empty_like(f)
    lib().orc_stream(_ptr(f), _ptr(out), nx, ny, nz)
    return out


def bgk_step(f, tau, force_lattice=None) -> np.ndarray:
    f = _f64(f)
    _, nx, ny, nz = f.shape
    F = None if force_lattice is None else _f64(force_lattice)
    out = np.empty_like(f)
    lib().orc_bgk_step(_ptr(f), _ptr(out), float(tau), _ptr(F), nx, ny, nz)
    return out


def apply_bounce_back_y_walls(f, wall_velocity_top=(0.0, 0.0, 0.0), wall_velocity_bottom=(0.0, 0.0, 0.0)):
    f = _f64(f)
    _, nx, ny, nz = f.shape
    top = _f64(wall_velocity_top)
    bot = _f64(wall_velocity_bottom)
    out = np.empty_like(f)
    lib().orc_bounce_back_y_walls(_ptr(f), _ptr(out), nx, ny, nz, _ptr(top), _ptr(bot))
    return out


# --------------------------------------------------------------------------
# Half / bfloat16 round-to-nearest-even conversions (scalar; for tests)
# --------------------------------------------------------------------------
def f32_to_f16_bits(x: float) -> int:
    return int(lib().orc_f32_to_f16(float(x)))


def f16_bits_to_f32(h: int) -> float:
    return float(lib().orc_f16_to_f32(int(h)))


def f32_to_bf16_bits(x: float) -> int:
    return int(lib().orc_f32_to_bf16(float(x)))


def bf16_bits_to_f32(h: int) -> float:
    return float(lib().orc_bf16_to_f32(int(h)))


def store_round(storage: int, f, ref_u=(0.0, 0.0, 0.0)) -> np.ndarray:
    """f rounded to what the storage holds; the 16-bit storages hold the
    deviation from feq(1, ref_u)."""
    out = _f64(f).copy()
    n = out.size // 19
    lib().orc_store_round(int(storage), _ptr(_f64(ref_u)), _ptr(out), n)
    return out


# --------------------------------------------------------------------------
# Generalised lattice (mirror of the GPU engine's semantics)
# --------------------------------------------------------------------------
class OracleLattice:
    """CPU mirror of one GPU lattice: PRE state (f held directly) until the first
    step, then POST state (post-collision array held; f reconstructed)."""

    def __init__(
        self,
        shape,
        tau,
        *,
        periodic=PERIODIC_X | PERIODIC_Y | PERIODIC_Z,
        wall_velocity=None,
        storage=STORE_F64,
        flags=None,
        force_mode=FORCE_NONE,
        body_force=(0.0, 0.0, 0.0),
        force_field=None,
        porosity=None,
        drag_k=0.0,
        inflow_rho=1.0,
        inflow_u=(0.0, 0.0, 0.0),
        storage_ref_u=None,
    ):
        nx, ny, nz = (int(s) for s in shape)
        self.shape = (nx, ny, nz)
        # the 16-bit storages' reference velocity; default: the inflow
        # velocity, as the engine's Lattice
        self.storage_ref_u = tuple(float(v) for v in (inflow_u if storage_ref_u is None else storage_ref_u))
        self.n = nx * ny * nz
        self.storage = int(storage)
        self._flags = None if flags is None else np.ascontiguousarray(flags, dtype=np.uint8)
        self._force = None if force_field is None else _f64(force_field)
        self._poro = None if porosity is None else np.ascontiguousarray(porosity, dtype=np.float32)
        s = _OrcLattice()
        s.nx, s.ny, s.nz = nx, ny, nz
        s.periodic = int(periodic)
        s.force_mode = int(force_mode)
        s.storage = self.storage
        s.tau = float(tau)
        wu = np.zeros((6, 3)) if wall_velocity is None else _f64(wall_velocity).reshape(6, 3)
        for k in range(18):
            s.wall_u[k] = float(wu.reshape(-1)[k])
        for k in range(3):
            s.body_force[k] = float(body_force[k])
            s.inflow_u[k] = float(inflow_u[k])
        s.drag_k = float(drag_k)
        s.inflow_rho = float(inflow_rho)
        for k in range(3):
            s.storage_ref_u[k] = self.storage_ref_u[k]
        s.flags = _ptr(self._flags, _u8p)
        s.force = _ptr(self._force)
        s.porosity = _ptr(self._poro, _fp)
        self._s = s
        self._pre = True
        self._a = np.zeros((19, nx, ny, nz))
        self.step_count = 0

    @property
    def _L(self):
        return C.byref(self._s)

    def set_populations(self, f) -> None:
        self._a = store_round(self.storage, f, self.storage_ref_u).reshape((19, *self.shape))
        self._spare = None
        self._pre = True

    def step(self, n_steps: int = 1) -> None:
        for _ in range(int(n_steps)):
            b = self._spare if getattr(self, "_spare", None) is not None else np.empty_like(self._a)
            if self._pre:
                lib().orc_engine_collide_local(self._L, _ptr(self._a), _ptr(b), None, None)
                self._pre = False
            else:
                lib().orc_engine_step(self._L, _ptr(self._a), _ptr(b), None, None)
            self._spare, self._a = self._a, b
            self.step_count += 1

    def get_populations(self) -> np.ndarray:
        if self._pre:
            return self._a.copy()
        out = np.empty_like(self._a)
        lib().orc_engine_reconstruct(self._L, _ptr(self._a), _ptr(out), None, None)
        return out

    def rho_u(self) -> tuple[np.ndarray, np.ndarray]:
        rho = np.empty(self.shape)
        u = np.empty((3, *self.shape))
        if self._pre:
            lib().orc_engine_moments_local(self._L, _ptr(self._a), _ptr(rho), _ptr(u))
        else:
            lib().orc_engine_reconstruct(self._L, _ptr(self._a), None, _ptr(rho), _ptr(u))
        return rho, u

    def conservation(self) -> np.ndarray:
        out = np.empty(4)
        f = self.get_populations()
        lib().orc_conservation(self._L, _ptr(f), _ptr(out))
        return out

    def run(self, n_steps: int) -> None:
        """Advance n_steps with the library's own loop (used for timing)."""
        f = self.get_populations()
        rc = lib().orc_engine_run(self._L, _ptr(f), int(n_steps))
        if rc != 0:
            raise MemoryError("oracle run: allocation failed")
        self._a = f
        self._pre = True
        self.step_count += int(n_steps)


def reference_library_path() -> str:
    return os.fspath(_LIB_PATH)
