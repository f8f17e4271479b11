"""Small helpers shared by the tests (hashing, trajectories, the MMS case)."""

from __future__ import annotations

import hashlib
import math

import numpy as np

PURE_TAGS = ("a", "b", "c")  # 7x6x5, 4x1x3 (ny = 1), 1x2x1


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<f8").tobytes()).hexdigest()


def same_bytes(a: np.ndarray, b: np.ndarray) -> bool:
    a = np.ascontiguousarray(a, dtype="<f8")
    b = np.ascontiguousarray(b, dtype="<f8")
    return a.shape == b.shape and a.tobytes() == b.tobytes()


def max_abs(a, b) -> float:
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b)))) if np.size(a) else 0.0


# --------------------------------------------------------------------------
# Forced Taylor-Green manufactured solution (closed form; u, v, p and the
# source terms S_u, S_v of the 2-D incompressible Navier-Stokes equations on
# the unit square, nu = 0.01, rho = 1), as used by the reference's gate-4b
# test (tests/test_mms_convergence.py:176-239).
# --------------------------------------------------------------------------
TWO_PI = 2.0 * float(np.pi)
FOUR_PI = 4.0 * float(np.pi)
EIGHT_PI2 = 8.0 * float(np.pi) * float(np.pi)


def tg_velocity(x, y, t):
    sx, cxv = np.sin(TWO_PI * x), np.cos(TWO_PI * x)
    sy, cyv = np.sin(TWO_PI * y), np.cos(TWO_PI * y)
    ct = float(np.cos(t))
    return sx * cyv * ct, -cxv * sy * ct


def tg_source(x, y, t, nu=0.01):
    sx, cxv = np.sin(TWO_PI * x), np.cos(TWO_PI * x)
    sy, cyv = np.sin(TWO_PI * y), np.cos(TWO_PI * y)
    s4x, s4y = np.sin(FOUR_PI * x), np.sin(FOUR_PI * y)
    ct, st = float(np.cos(t)), float(np.sin(t))
    c2 = ct * ct
    su = -sx * cyv * st + TWO_PI * s4x * c2 + EIGHT_PI2 * nu * sx * cyv * ct
    sv = cxv * sy * st + TWO_PI * s4y * c2 - EIGHT_PI2 * nu * cxv * sy * ct
    return su, sv


def mms_case(n_grid, feq_field, bgk_step, macroscopic_velocity, cs2=1.0 / 3.0):
    """Run the forced Taylor-Green ladder point at N = n_grid with the given
    step functions; returns (error, final velocity field, n_steps)."""
    nu_lat = cs2 * (0.65 - 0.5)
    dx = 1.0 / n_grid
    n_steps = max(1, round(0.05 / (nu_lat * dx * dx / 0.01)))
    dt = 0.05 / n_steps
    tau = 0.5 + 0.01 * dt / (cs2 * dx * dx)
    idx = (np.arange(n_grid, dtype=np.float64) + 0.5) / n_grid
    gx, gy = np.meshgrid(idx, idx, indexing="ij")
    u0, v0 = tg_velocity(gx, gy, 0.0)
    sv = dt / dx
    u_lat = np.zeros((3, n_grid, n_grid, 3))
    u_lat[0] = (0.05 * u0 * sv)[:, :, None]
    u_lat[1] = (0.05 * v0 * sv)[:, :, None]
    f = feq_field(np.ones((n_grid, n_grid, 3)), u_lat)
    sf = dt * dt / dx

    def force_at(t):
        su, svv = tg_source(gx, gy, t)
        F = np.zeros((3, n_grid, n_grid, 3))
        F[0] = (0.05 * su * sf)[:, :, None]
        F[1] = (0.05 * svv * sf)[:, :, None]
        return F

    for step in range(n_steps):
        f = bgk_step(f, tau, force_lattice=force_at((step + 0.5) * dt))
    u_end = macroscopic_velocity(f, force_lattice=force_at(0.05))
    ua, va = tg_velocity(gx, gy, 0.05)
    eu = float(np.sqrt(np.mean((u_end[0][:, :, 0] / sv - 0.05 * ua) ** 2)))
    ev = float(np.sqrt(np.mean((u_end[1][:, :, 0] / sv - 0.05 * va) ** 2)))
    return math.sqrt(eu * eu + ev * ev), u_end, n_steps
