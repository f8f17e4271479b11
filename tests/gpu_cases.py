"""Matched GPU / oracle lattice pairs for the parity tests."""

from __future__ import annotations

import numpy as np

import oracle as O
from lattice_boltzmann_d3q19_b200 import Lattice, geometry

STORE = {"f64": O.STORE_F64, "f32": O.STORE_F32, "f16": O.STORE_F16_SHIFT, "bf16": O.STORE_BF16_SHIFT}
FORCE = {"none": O.FORCE_NONE, "uniform": O.FORCE_UNIFORM, "field": O.FORCE_FIELD, "drag": O.FORCE_DRAG}


def random_state(shape, seed, amp=0.03):
    rng = np.random.default_rng(seed)
    rho = 1.0 + 0.02 * rng.standard_normal(shape)
    u = amp * rng.standard_normal((3, *shape))
    return O.feq_field(rho, u)


def pair(shape, tau, storage="f64", *, periodic=(True, True, True), wall_velocity=None, flags=None,
         force_mode="none", body_force=(0.0, 0.0, 0.0), force_field=None, porosity=None, drag_k=0.0,
         inflow_rho=1.0, inflow_u=(0.0, 0.0, 0.0), block_size=0):
    """A GPU Lattice and an OracleLattice with identical parameters."""
    wu = Lattice._wall_array(wall_velocity)
    mask = (1 if periodic[0] else 0) | (2 if periodic[1] else 0) | (4 if periodic[2] else 0)
    gpu = Lattice(shape, tau, storage=storage, periodic=mask, wall_velocity=wu, force_mode=force_mode,
                  body_force=body_force, drag_k=drag_k, inflow_rho=inflow_rho, inflow_u=inflow_u,
                  block_size=block_size)
    cpu = O.OracleLattice(shape, tau, periodic=mask, wall_velocity=wu, storage=STORE[storage], flags=flags,
                          force_mode=FORCE[force_mode], body_force=body_force, force_field=force_field,
                          porosity=porosity, drag_k=drag_k, inflow_rho=inflow_rho, inflow_u=inflow_u)
    if flags is not None:
        gpu.set_flags(flags)
    if force_field is not None:
        gpu.set_force_field(force_field)
    if porosity is not None:
        gpu.set_porosity(porosity)
    return gpu, cpu


def cavity_case(shape=(12, 10, 9), lid=0.05, storage="f64"):
    kw = geometry.lid_driven_cavity(lid)
    return pair(shape, 0.6, storage, periodic=kw["periodic"], wall_velocity=kw["wall_velocity"])


def channel_case(shape=(40, 16, 14), storage="f64", seed=5):
    flags, _ = geometry.sphere_channel(shape, n_spheres=4, radius=(2.0, 4.0), seed=seed)
    return pair(shape, 0.56, storage, flags=flags, inflow_u=(0.04, 0.0, 0.0)), flags


def drag_case(shape=(24, 10, 12), storage="f64"):
    alpha = geometry.smooth_porosity(shape, sigma=2.0, seed=9)
    flags = np.zeros(shape, dtype=np.uint8)
    flags[0] = 2
    flags[-1] = 3
    return pair(shape, 0.7, storage, flags=flags, force_mode="drag", porosity=alpha, drag_k=0.05,
                body_force=(1e-6, 0.0, 0.0), inflow_u=(0.03, 0.0, 0.0))
