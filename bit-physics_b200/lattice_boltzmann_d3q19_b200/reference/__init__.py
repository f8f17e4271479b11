"""Drop-in for ``lattice_boltzmann_d3q19_stack_e.reference`` on the B200.

Same public names, argument meaning and return types as the reference's
re-export list (``lattice_boltzmann_d3q19_stack_e/reference/__init__.py:12-68``):
pure functions on NumPy f64 arrays of shape (19, nx, ny, nz) that return new
arrays.  The field functions run as sm_100a kernels through the C ABI
(``lbm_bgk_step``, ``lbm_stream``, ...); their f64 results are bit-identical
to the reference's.  The point-evaluation helpers ``feq``,
``density_moment`` and ``momentum_moment`` are host-only in the reference
(d3q19_warp.py:221-247) and stay host-side here.

Like the reference, inputs are copied and outputs are fresh arrays; unlike
it, shape errors are reported before any device work (ValueError).
"""

from __future__ import annotations

import numpy as np

from .. import _native as N
from ..constants import (
    CANONICAL_COUETTE_NX,
    CANONICAL_COUETTE_NY,
    CANONICAL_COUETTE_STEPS,
    CANONICAL_DESCRIPTOR_COUETTE,
    CANONICAL_DESCRIPTOR_POISEUILLE,
    CANONICAL_NZ,
    CANONICAL_POISEUILLE_NX,
    CANONICAL_POISEUILLE_NY,
    CANONICAL_POISEUILLE_STEPS,
    CANONICAL_SEED,
    CS2,
    VELOCITIES,
    WEIGHTS,
    C,
    W,
)


def _pop(f, name="f") -> np.ndarray:
    a = N.f64(f)
    if a.ndim != 4 or a.shape[0] != 19:
        raise ValueError(f"{name} must have shape (19, nx, ny, nz); got {a.shape}")
    return a


def _vec_field(a, shape, name) -> np.ndarray:
    a = N.f64(a)
    if a.shape != (3, *shape):
        raise ValueError(f"{name} must have shape {(3, *shape)}; got {a.shape}")
    return a


# --------------------------------------------------------------------------
# Point-evaluation surface (host-only, as in d3q19_warp.py:221-247)
# --------------------------------------------------------------------------
def feq(rho, u):
    """The 19 equilibrium values at one (rho, u), Qian et al. 1992 eq. 3a,
    in the division form of equilibrium.py:258-277 (the golden-table surface)."""
    ux, uy, uz = float(u[0]), float(u[1]), float(u[2])
    r = float(rho)
    u_sq = ux * ux + uy * uy + uz * uz
    values = []
    for (c0, c1, c2), w in zip(VELOCITIES, WEIGHTS, strict=True):
        cu = c0 * ux + c1 * uy + c2 * uz
        values.append(w * r * (1.0 + cu / CS2 + (cu * cu) / (2.0 * CS2 * CS2) - u_sq / (2.0 * CS2)))
    return values


def density_moment(f):
    """sum_i f_i."""
    return float(sum(f))


def momentum_moment(f):
    """sum_i c_i f_i as a 3-list, accumulated in lex order."""
    m = [0.0, 0.0, 0.0]
    for (c0, c1, c2), fi in zip(VELOCITIES, f, strict=False):
        v = float(fi)
        m[0] += c0 * v
        m[1] += c1 * v
        m[2] += c2 * v
    return m


# --------------------------------------------------------------------------
# Field surface (GPU, via the C ABI)
# --------------------------------------------------------------------------
def feq_field(rho, u):
    """Equilibrium on a grid: rho (nx,ny,nz), u (3,nx,ny,nz) -> (19,nx,ny,nz)."""
    rho = N.f64(rho)
    if rho.ndim != 3:
        raise ValueError(f"rho must have shape (nx, ny, nz); got {rho.shape}")
    u = _vec_field(u, rho.shape, "u")
    out = np.empty((19, *rho.shape))
    N.check(N.lib().lbm_feq_field(N.ptr(rho), N.ptr(u), N.ptr(out), *rho.shape))
    return out


def density_field(f):
    """sum over directions -> (nx, ny, nz)."""
    f = _pop(f)
    out = np.empty(f.shape[1:])
    N.check(N.lib().lbm_density_field(N.ptr(f), N.ptr(out), *f.shape[1:]))
    return out


def momentum_field(f):
    """sum_i c_i f_i -> (3, nx, ny, nz)."""
    f = _pop(f)
    out = np.empty((3, *f.shape[1:]))
    N.check(N.lib().lbm_momentum_field(N.ptr(f), N.ptr(out), *f.shape[1:]))
    return out


def stream(f_post):
    """Periodic streaming: out[d, x] = f_post[d, (x - c_d) mod n]."""
    f = _pop(f_post, "f_post")
    out = np.empty_like(f)
    N.check(N.lib().lbm_stream(N.ptr(f), N.ptr(out), *f.shape[1:]))
    return out


def bgk_step(f, tau, force_lattice=None):
    """One BGK collision (Guo forcing when force_lattice is given) + streaming."""
    f = _pop(f)
    F = None if force_lattice is None else _vec_field(force_lattice, f.shape[1:], "force_lattice")
    out = np.empty_like(f)
    N.check(N.lib().lbm_bgk_step(N.ptr(f), N.ptr(out), float(tau), N.ptr(F), *f.shape[1:]))
    return out


def macroscopic_velocity(f, force_lattice=None):
    """u = (m [+ 0.5 F]) / max(rho, 1e-30)."""
    f = _pop(f)
    F = None if force_lattice is None else _vec_field(force_lattice, f.shape[1:], "force_lattice")
    out = np.empty((3, *f.shape[1:]))
    N.check(N.lib().lbm_macroscopic_velocity(N.ptr(f), N.ptr(F), N.ptr(out), *f.shape[1:]))
    return out


def apply_bounce_back_y_walls(f, wall_velocity_top=(0.0, 0.0, 0.0), wall_velocity_bottom=(0.0, 0.0, 0.0)):
    """Bounce-back at y = 0 and y = ny - 1 with moving-wall injection.

    Sign convention (kept from the reference, bgk.py:198-215): the injection
    -2 w_i rho_w (c_i . u_w) / c_s^2 is added to the incoming direction i, so
    a top wall given velocity (+U, 0, 0) drives the adjacent fluid towards -x.
    """
    f = _pop(f)
    top = N.f64(wall_velocity_top)
    bot = N.f64(wall_velocity_bottom)
    if top.shape != (3,) or bot.shape != (3,):
        raise ValueError("wall velocities must be 3-vectors")
    out = np.empty_like(f)
    N.check(N.lib().lbm_bounce_back_y_walls(N.ptr(f), N.ptr(out), *f.shape[1:], N.ptr(top), N.ptr(bot)))
    return out


__all__ = [
    "CANONICAL_COUETTE_NX",
    "CANONICAL_COUETTE_NY",
    "CANONICAL_COUETTE_STEPS",
    "CANONICAL_DESCRIPTOR_COUETTE",
    "CANONICAL_DESCRIPTOR_POISEUILLE",
    "CANONICAL_NZ",
    "CANONICAL_POISEUILLE_NX",
    "CANONICAL_POISEUILLE_NY",
    "CANONICAL_POISEUILLE_STEPS",
    "CANONICAL_SEED",
    "CS2",
    "VELOCITIES",
    "WEIGHTS",
    "C",
    "W",
    "apply_bounce_back_y_walls",
    "bgk_step",
    "density_field",
    "density_moment",
    "feq",
    "feq_field",
    "macroscopic_velocity",
    "momentum_field",
    "momentum_moment",
    "stream",
]
