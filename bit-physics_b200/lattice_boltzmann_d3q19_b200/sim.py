"""Canonical runners: the reference's Poiseuille / Couette / diagnostic captures.

Mirror of ``lattice_boltzmann_d3q19_stack_e/sim.py:112-401`` on the GPU engine:
same lattices (64x32x3 x 1000 steps Poiseuille with F_x = 1e-5; 32x16x3 x
500 steps Couette with top wall (0.05, 0, 0); 16x8x3 x 50 diagnostic), same
tau 0.7, same cadence-1 rho/u frames and Tier-1/Tier-2 diagnostics.  With
f64 storage every frame is bit-identical to the reference's.

Captures are written as ``<descriptor>.npz`` with the reference's payload keys
``steps/{N}/state/{rho,u}`` and ``steps/{N}/diagnostics/{check}``
(common_warp/capture/model.py:36-43) plus a ``<descriptor>.json`` manifest
(sim.py:193-229); HDF5 is not used because h5py is not a dependency here.
"""

from __future__ import annotations

import json
import time
from pathlib import Path

import numpy as np

from .constants import (
    CANONICAL_COUETTE_NX,
    CANONICAL_COUETTE_NY,
    CANONICAL_COUETTE_STEPS,
    CANONICAL_COUETTE_WALL_VELOCITY,
    CANONICAL_DESCRIPTOR_COUETTE,
    CANONICAL_DESCRIPTOR_POISEUILLE,
    CANONICAL_NZ,
    CANONICAL_POISEUILLE_FORCE_X,
    CANONICAL_POISEUILLE_NX,
    CANONICAL_POISEUILLE_NY,
    CANONICAL_POISEUILLE_STEPS,
    CANONICAL_TAU,
)
from .engine import Lattice

Y_WALLS = (True, False, True)  # periodic x and z, walls at y = 0 and y = ny - 1


def health_check(rho: np.ndarray, u: np.ndarray) -> dict[str, float]:
    """Tier-1 diagnostics (sim.py:89-96)."""
    return {
        "check_health": 0.0 if (np.all(np.isfinite(rho)) and np.all(np.isfinite(u))) else 1.0,
        "rho_min": float(np.min(rho)),
        "rho_max": float(np.max(rho)),
        "u_max_lat": float(np.max(np.sqrt((u * u).sum(axis=0)))),
    }


def vector_field_diagnostics(u: np.ndarray, dx_phys: float) -> dict[str, float]:
    """Tier-2 diagnostics on the z = 0 slice (sim.py:99-109): max |div u| by
    central differences and the circulation proxy sum(u_x) dx^2."""
    ux = u[0, :, :, 0]
    uy = u[1, :, :, 0]
    half_inv = 0.5 / dx_phys
    div = (np.roll(ux, -1, axis=0) - np.roll(ux, 1, axis=0)) * half_inv + (
        np.roll(uy, -1, axis=1) - np.roll(uy, 1, axis=1)
    ) * half_inv
    return {
        "check_divergence_free": float(np.max(np.abs(div))),
        "check_circulation": float(np.sum(ux) * dx_phys * dx_phys),
    }


def poiseuille_lattice(nx, ny, nz, tau=CANONICAL_TAU, force_x=CANONICAL_POISEUILLE_FORCE_X, storage="f64") -> Lattice:
    """Body-forced channel between no-slip y walls, rest initial state (sim.py:119-139)."""
    lat = Lattice((nx, ny, nz), tau, storage=storage, periodic=Y_WALLS, force_mode="uniform",
                  body_force=(force_x, 0.0, 0.0))
    lat.set_equilibrium()
    return lat


def couette_lattice(nx, ny, nz, tau=CANONICAL_TAU, wall_velocity=CANONICAL_COUETTE_WALL_VELOCITY,
                    storage="f64") -> Lattice:
    """Moving top wall, resting bottom wall, rest initial state (sim.py:156-179)."""
    lat = Lattice((nx, ny, nz), tau, storage=storage, periodic=Y_WALLS,
                  wall_velocity={"y+": (wall_velocity, 0.0, 0.0), "y-": (0.0, 0.0, 0.0)})
    lat.set_equilibrium()
    return lat


def evolve(lat: Lattice, n_steps: int, capture_interval: int, dx_phys: float):
    """Frames (step, {rho, u}, diagnostics) at step 0, every capture_interval
    steps and the final step, as the reference's evolve loops yield them."""
    steps, rho, u = lat.run_capture(n_steps, capture_interval)
    frames = []
    for k, s in enumerate(steps):
        diag = {**health_check(rho[k], u[k]), **vector_field_diagnostics(u[k], dx_phys)}
        frames.append((int(s), {"rho": rho[k], "u": u[k]}, diag))
    return frames


def write_capture(frames, manifest: dict, out_dir: Path, descriptor: str) -> Path:
    payload = {}
    for step, state, diagnostics in frames:
        for name, arr in state.items():
            payload[f"steps/{step}/state/{name}"] = np.asarray(arr, dtype=np.float64)
        for check, val in diagnostics.items():
            payload[f"steps/{step}/diagnostics/{check}"] = np.float64(val)
    out_dir.mkdir(parents=True, exist_ok=True)
    np.savez(out_dir / f"{descriptor}.npz", **payload)
    manifest = dict(manifest)
    manifest["payload"] = {"format": "npz", "path": f"{descriptor}.npz"}
    path = out_dir / f"{descriptor}.json"
    path.write_text(json.dumps(manifest, indent=1) + "\n")
    return path


def _manifest(descriptor, tier, dims, seed, n_steps, capture_interval, wall, params, storage):
    return {
        "schema_version": "1.0.0",
        "sim": {"name": "lattice-boltzmann-d3q19", "category": "lattice", "variant": "bgk-d3q19-qian-1992"},
        "stack": {"name": "b200-cuda", "version": "0.1.0", "build_id": "lattice-boltzmann-d3q19-b200"},
        "config": {"tier": tier, "dims": list(dims), "dtype": storage, "seed": int(seed), "params": params},
        "run": {"step_count": int(n_steps), "capture_interval": int(capture_interval),
                "wall_clock_seconds": float(wall)},
        "determinism": {"claimed": "bit-exact-same-hw", "atomic_ops": False, "subgroup_ops": False},
    }


def _run(descriptor, tier, seed, out_dir, nx, ny, nz, n_steps, interval, kind, storage):
    t0 = time.perf_counter()
    if kind == "poiseuille":
        lat = poiseuille_lattice(nx, ny, nz, storage=storage)
        params = {"descriptor": descriptor, "tau": CANONICAL_TAU, "force_x_lattice": CANONICAL_POISEUILLE_FORCE_X,
                  "nz_convention": "depth-3-z-periodic-slab", "boundary": "bounce-back-y-walls-periodic-xz"}
    else:
        lat = couette_lattice(nx, ny, nz, storage=storage)
        params = {"descriptor": descriptor, "tau": CANONICAL_TAU,
                  "wall_velocity_top_lattice": CANONICAL_COUETTE_WALL_VELOCITY,
                  "nz_convention": "depth-3-z-periodic-slab",
                  "boundary": "bounce-back-y-walls-with-moving-top-plate-periodic-xz"}
    with lat:
        frames = evolve(lat, n_steps, interval, 1.0 / nx)
    wall = time.perf_counter() - t0
    manifest = _manifest(descriptor, tier, (nx, ny, nz), seed, n_steps, interval, wall, params, storage)
    return write_capture(frames, manifest, Path(out_dir), descriptor)


def sim_runner_seeded(seed: int, out_dir, storage: str = "f64") -> Path:
    """Canonical Poiseuille capture, 64x32x3 x 1000 steps, cadence 1 (sim.py:250-300)."""
    return _run(CANONICAL_DESCRIPTOR_POISEUILLE, "test", seed, out_dir, CANONICAL_POISEUILLE_NX,
                CANONICAL_POISEUILLE_NY, CANONICAL_NZ, CANONICAL_POISEUILLE_STEPS, 1, "poiseuille", storage)


def sim_runner_seeded_couette(seed: int, out_dir, storage: str = "f64") -> Path:
    """Canonical Couette capture, 32x16x3 x 500 steps, cadence 1 (sim.py:303-350)."""
    return _run(CANONICAL_DESCRIPTOR_COUETTE, "test", seed, out_dir, CANONICAL_COUETTE_NX, CANONICAL_COUETTE_NY,
                CANONICAL_NZ, CANONICAL_COUETTE_STEPS, 1, "couette", storage)


def sim_runner_diagnostic(seed: int, out_dir, storage: str = "f64") -> Path:
    """Small Poiseuille run, 16x8x3 x 50 steps, cadence 10 (sim.py:353-401)."""
    return _run("poiseuille-16x8-seed42-step50", "diagnostic", seed, out_dir, 16, 8, CANONICAL_NZ, 50, 10,
                "poiseuille", storage)


__all__ = [
    "couette_lattice",
    "evolve",
    "health_check",
    "poiseuille_lattice",
    "sim_runner_diagnostic",
    "sim_runner_seeded",
    "sim_runner_seeded_couette",
    "vector_field_diagnostics",
    "write_capture",
]
