"""Lattice configurations for the adjoint tests: the same case built as a GPU
Lattice, a C-oracle lattice and a PyTorch-f64 restatement."""

from __future__ import annotations

import numpy as np

import oracle as O
import torch_lbm
from lattice_boltzmann_d3q19_b200 import geometry

FORCE = {"none": O.FORCE_NONE, "uniform": O.FORCE_UNIFORM, "field": O.FORCE_FIELD, "drag": O.FORCE_DRAG}


def _spheres(shape, flags, centres, r):
    X, Y, Z = np.meshgrid(*[np.arange(s) for s in shape], indexing="ij")
    for c in centres:
        flags[(X - c[0]) ** 2 + (Y - c[1]) ** 2 + (Z - c[2]) ** 2 <= r * r] = O.CELL_SOLID


def case(name: str, shape=None):
    """dict with the Lattice keyword arguments ("kw"), flags, porosity
    ("alpha"), force field and an initial state ("f0")."""
    rng = np.random.default_rng(11)
    if name == "drag_channel":
        # inflow x = 0, two outflow planes, spheres, walled y with moving
        # faces, periodic z, porosity drag with a body force
        shape = shape or (20, 12, 10)
        flags = np.zeros(shape, np.uint8)
        _spheres(shape, flags, [(7, 5, 4), (12, 8, 7)], 2.2)
        flags[0] = O.CELL_INFLOW
        flags[-2:] = O.CELL_OUTFLOW
        wall = np.zeros((6, 3))
        wall[3] = (0.02, 0.0, 0.01)
        wall[2] = (-0.01, 0.0, 0.0)
        kw = dict(periodic=5, wall_velocity=wall, force_mode="drag", body_force=(1e-5, 0.0, 2e-6), drag_k=0.1,
                  inflow_u=(0.04, 0.0, 0.0))
        alpha = geometry.smooth_porosity(shape, sigma=2.0, seed=3)
        tau, force = 0.6, None
    elif name == "cavity":
        # all six faces walled, lid on y+ and a moving z- face, no force
        shape = shape or (10, 9, 8)
        flags = None
        wall = np.zeros((6, 3))
        wall[3] = (0.05, 0.0, 0.0)
        wall[4] = (0.0, 0.01, 0.0)
        kw = dict(periodic=0, wall_velocity=wall, force_mode="none")
        alpha, tau, force = None, 0.7, None
    elif name == "field_periodic":
        # periodic box with a solid block and a per-cell force field
        shape = shape or (10, 8, 12)
        flags = np.zeros(shape, np.uint8)
        flags[4:6, 3:5, 5:8] = O.CELL_SOLID
        force = 1e-4 * rng.standard_normal((3, *shape))
        kw = dict(periodic=7, force_mode="field")
        alpha, tau = None, 0.8
    else:
        raise KeyError(name)
    rho0 = 1.0 + 0.01 * rng.standard_normal(shape)
    u0 = 0.02 * rng.standard_normal((3, *shape))
    f0 = O.feq_field(rho0, u0)
    return dict(shape=shape, tau=tau, kw=kw, flags=flags, alpha=alpha, force=force, f0=f0)


def torch_lattice(c, device="cpu"):
    kw = dict(c["kw"])
    return torch_lbm.TorchLattice(c["shape"], c["tau"], periodic=kw.pop("periodic"),
                                  wall_velocity=kw.pop("wall_velocity", None), force_mode=kw.pop("force_mode"),
                                  body_force=kw.pop("body_force", (0, 0, 0)), drag_k=kw.pop("drag_k", 0.0),
                                  inflow_u=kw.pop("inflow_u", (0, 0, 0)), flags=c["flags"], force=c["force"],
                                  device=device)


def oracle_lattice(c):
    kw = c["kw"]
    return O.OracleLattice(c["shape"], c["tau"], periodic=kw["periodic"], wall_velocity=kw.get("wall_velocity"),
                           flags=c["flags"], force_mode=FORCE[kw["force_mode"]],
                           body_force=kw.get("body_force", (0.0, 0.0, 0.0)), force_field=c["force"],
                           porosity=c["alpha"], drag_k=kw.get("drag_k", 0.0), inflow_u=kw.get("inflow_u", (0, 0, 0)))


def gpu_lattice(c, storage="f64"):
    from lattice_boltzmann_d3q19_b200 import Lattice

    lat = Lattice(c["shape"], c["tau"], storage=storage, **c["kw"])
    if c["flags"] is not None:
        lat.set_flags(c["flags"])
    if c["force"] is not None:
        lat.set_force_field(c["force"])
    if c["alpha"] is not None:
        lat.set_porosity(c["alpha"])
    return lat


def loss_fn(rho, u, box_x):
    """L = sum over x in box of 1/2 rho |u|^2 + 0.1 sum (rho - 1)^2 over
    non-solid cells (numpy or torch arrays)."""
    x0, x1 = box_x
    ke = 0.5 * (rho[x0:x1] * (u[:, x0:x1] ** 2).sum(0)).sum()
    mass = 0.1 * (((rho - 1.0) * (rho != 0)) ** 2).sum()
    return ke + mass


CASES = ("drag_channel", "cavity", "field_periodic")
