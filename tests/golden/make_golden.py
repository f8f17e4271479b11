"""Regenerate the golden fixtures in this directory from the reference itself.

Runs only where the Bit-Physics reference tree is mounted; its root is
given by the ``BITPHYSICS_REF`` environment variable (required, e.g.
``BITPHYSICS_REF=/path/to/Bit-Physics python make_golden.py``).  It imports the
Phase-1 NumPy reference package ``packages/lattice-boltzmann-d3q19``
read-only -- the frozen parent that the Stack-E Warp port reproduces
byte-for-byte (docs/sim-specs/lattice/lattice-boltzmann-d3q19/
equivalence.md:219-243) -- and writes small ``.npz`` / ``.json`` fixtures.
The tests read only these fixtures, never the reference tree.

Fixtures:

* ``equilibrium.json`` -- the reference's golden table point
  (tools/testkit/golden/tables/lattice/d3q19-equilibrium.json, test point 0).
* ``pure_functions.npz`` -- seeded random inputs and the reference outputs of
  feq_field, density_field, momentum_field, macroscopic_velocity (with and
  without force), stream, bgk_step (with and without force) and
  apply_bounce_back_y_walls (moving top and bottom walls), on 7x6x5, a ny=1
  slab and a 1x2x1 lattice.
* ``couette_32x16x3.npz`` / ``poiseuille_64x32x3.npz`` -- the two canonical
  trajectories of the reference runner (Stack-E sim.py:119-190; tau 0.7,
  Couette top wall (0.05,0,0), Poiseuille F_x = 1e-5): sha256 of the f64
  bytes of rho and u at EVERY step, the full rho/u at a few steps, and the
  final populations.
* ``determinism_16x8x3.npz`` -- the random initial condition of
  tests/test_determinism.py:61-74 and one bgk_step of it.
* ``mms.json`` / ``mms_n32.npz`` -- the forced Taylor-Green MMS ladder of
  tests/test_mms_convergence.py:186-239 (errors for N=32,64,128) and the
  final velocity field at N=32.
"""

from __future__ import annotations

import hashlib
import importlib.util
import json
import math
import os
import sys
from pathlib import Path

import numpy as np

OUT = Path(__file__).resolve().parent
if not os.environ.get("BITPHYSICS_REF"):
    sys.exit("make_golden.py: set BITPHYSICS_REF to the root of the Bit-Physics reference tree")
REF = Path(os.environ["BITPHYSICS_REF"])


def _import_reference():
    sys.path.insert(0, str(REF / "packages" / "lattice-boltzmann-d3q19"))
    from lattice_boltzmann_d3q19.reference import bgk, constants, equilibrium

    return bgk, equilibrium, constants


def _mms_solution():
    # Loaded by file path: the testkit package __init__ imports h5py.
    path = (
        REF / "tools/testkit/code_verification/mms/solutions/incompressible_ns_2d/solution.py"
    )
    spec = importlib.util.spec_from_file_location("_mms_solution", path)
    mod = importlib.util.module_from_spec(spec)
    sys.modules["_mms_solution"] = mod
    spec.loader.exec_module(mod)
    return mod.IncompressibleNS2DSolution


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<f8").tobytes()).hexdigest()


def make_equilibrium() -> None:
    table = json.loads(
        (REF / "tools/testkit/golden/tables/lattice/d3q19-equilibrium.json").read_text()
    )
    tp = table["test_points"][0]
    out = {
        "source": "tools/testkit/golden/tables/lattice/d3q19-equilibrium.json test_points[0]",
        "tolerance_abs": table["tolerance"]["absolute"],
        "rho": tp["inputs"]["rho"],
        "u": tp["inputs"]["u"],
        "f_eq": tp["expected"]["f_eq"],
        "density_moment": tp["expected"]["density_moment"],
        "momentum": [
            tp["expected"]["momentum_x"],
            tp["expected"]["momentum_y"],
            tp["expected"]["momentum_z"],
        ],
    }
    (OUT / "equilibrium.json").write_text(json.dumps(out, indent=1) + "\n")


def make_pure(bgk, eq) -> None:
    rng = np.random.default_rng(20260525)
    arrays: dict[str, np.ndarray] = {}
    top = np.array([0.05, -0.01, 0.02])
    bot = np.array([-0.03, 0.004, 0.01])
    arrays["wall_top"] = top
    arrays["wall_bottom"] = bot
    arrays["tau"] = np.array(0.63)
    for tag, sh in (("a", (7, 6, 5)), ("b", (4, 1, 3)), ("c", (1, 2, 1))):
        rho = 1.0 + 0.05 * rng.standard_normal(sh)
        u = 0.05 * rng.standard_normal((3, *sh))
        f = eq.feq_field(rho, u) + 1e-3 * rng.standard_normal((19, *sh))
        F = 1e-4 * rng.standard_normal((3, *sh))
        arrays[f"{tag}_rho_in"] = rho
        arrays[f"{tag}_u_in"] = u
        arrays[f"{tag}_f"] = f
        arrays[f"{tag}_force"] = F
        arrays[f"{tag}_feq_field"] = eq.feq_field(rho, u)
        arrays[f"{tag}_density_field"] = eq.density_field(f)
        arrays[f"{tag}_momentum_field"] = eq.momentum_field(f)
        arrays[f"{tag}_macroscopic_velocity"] = bgk.macroscopic_velocity(f)
        arrays[f"{tag}_macroscopic_velocity_force"] = bgk.macroscopic_velocity(f, F)
        arrays[f"{tag}_stream"] = bgk.stream(f)
        arrays[f"{tag}_bgk_step"] = bgk.bgk_step(f, 0.63)
        arrays[f"{tag}_bgk_step_force"] = bgk.bgk_step(f, 0.63, F)
        arrays[f"{tag}_bounce"] = bgk.apply_bounce_back_y_walls(
            f, wall_velocity_top=tuple(top), wall_velocity_bottom=tuple(bot)
        )
    np.savez_compressed(OUT / "pure_functions.npz", **arrays)


def _trajectory(bgk, eq, name, nx, ny, nz, n_steps, force_x, wall_top, keep):
    f = eq.feq_field(np.ones((nx, ny, nz)), np.zeros((3, nx, ny, nz)))
    force = None
    if force_x is not None:
        force = np.zeros((3, nx, ny, nz))
        force[0] = force_x
    rho_h, u_h, frames = [], [], {}

    def record(step, f):
        rho = eq.density_field(f)
        u = bgk.macroscopic_velocity(f, force_lattice=force)
        rho_h.append(sha(rho))
        u_h.append(sha(u))
        if step in keep:
            frames[f"rho_{step}"] = rho
            frames[f"u_{step}"] = u

    record(0, f)
    for step in range(1, n_steps + 1):
        f = bgk.bgk_step(f, 0.7, force_lattice=force)
        if wall_top is None:
            f = bgk.apply_bounce_back_y_walls(f)
        else:
            f = bgk.apply_bounce_back_y_walls(
                f, wall_velocity_top=wall_top, wall_velocity_bottom=(0.0, 0.0, 0.0)
            )
        record(step, f)
    np.savez_compressed(
        OUT / f"{name}.npz",
        rho_sha256=np.array(rho_h),
        u_sha256=np.array(u_h),
        f_final=f,
        keep_steps=np.array(sorted(keep)),
        **frames,
    )


def make_trajectories(bgk, eq) -> None:
    # Stack-E sim.py:156-190 (Couette) and :119-153 (Poiseuille); sim.py:76-78.
    _trajectory(bgk, eq, "couette_32x16x3", 32, 16, 3, 500, None, (0.05, 0.0, 0.0), {1, 10, 100, 500})
    _trajectory(bgk, eq, "poiseuille_64x32x3", 64, 32, 3, 1000, 1.0e-5, None, {1, 1000})


def make_determinism(bgk, eq) -> None:
    # tests/test_determinism.py:61-74.
    rng = np.random.default_rng(42)
    rho0 = 1.0 + 0.01 * rng.standard_normal((16, 8, 3))
    u0 = 0.01 * rng.standard_normal((3, 16, 8, 3))
    f0 = eq.feq_field(rho0, u0)
    np.savez_compressed(
        OUT / "determinism_16x8x3.npz", rho0=rho0, u0=u0, f0=f0, f1=bgk.bgk_step(f0, 0.7)
    )


def make_mms(bgk, eq, constants) -> None:
    # tests/test_mms_convergence.py:176-239, restated with the reference functions.
    Sol = _mms_solution()
    sol = Sol(nu=0.01, L=1.0, rho=1.0)
    CS2 = constants.CS2
    results = []
    for n_grid in (32, 64, 128):
        nu_lat = CS2 * (0.65 - 0.5)
        dx = 1.0 / n_grid
        dt_nat = nu_lat * dx * dx / 0.01
        n_steps = max(1, round(0.05 / dt_nat))
        dt = 0.05 / n_steps
        tau = 0.5 + 0.01 * dt / (CS2 * dx * dx)
        idx = (np.arange(n_grid, dtype=np.float64) + 0.5) / n_grid
        gx, gy = np.meshgrid(idx, idx, indexing="ij")
        u0, v0, _ = sol.evaluate(gx, gy, 0.0)
        sv = dt / dx
        u_lat = np.zeros((3, n_grid, n_grid, 3))
        u_lat[0] = (0.05 * u0 * sv)[:, :, None]
        u_lat[1] = (0.05 * v0 * sv)[:, :, None]
        f = eq.feq_field(np.ones((n_grid, n_grid, 3)), u_lat)
        sf = dt * dt / dx
        for step in range(n_steps):
            su, svv = sol.source_term(gx, gy, (step + 0.5) * dt)
            F = np.zeros((3, n_grid, n_grid, 3))
            F[0] = (0.05 * su * sf)[:, :, None]
            F[1] = (0.05 * svv * sf)[:, :, None]
            f = bgk.bgk_step(f, tau, force_lattice=F)
        su, svv = sol.source_term(gx, gy, 0.05)
        F = np.zeros((3, n_grid, n_grid, 3))
        F[0] = (0.05 * su * sf)[:, :, None]
        F[1] = (0.05 * svv * sf)[:, :, None]
        u_end = bgk.macroscopic_velocity(f, force_lattice=F)
        ua, va, _ = sol.evaluate(gx, gy, 0.05)
        eu = float(np.sqrt(np.mean((u_end[0][:, :, 0] / sv - 0.05 * ua) ** 2)))
        ev = float(np.sqrt(np.mean((u_end[1][:, :, 0] / sv - 0.05 * va) ** 2)))
        results.append(
            {"N": n_grid, "n_steps": n_steps, "tau": tau, "err": math.sqrt(eu * eu + ev * ev)}
        )
        if n_grid == 32:
            np.savez_compressed(OUT / "mms_n32.npz", u_end=u_end, sha_u=np.array(sha(u_end)))
    dxs = np.array([1.0 / r["N"] for r in results])
    errs = np.array([r["err"] for r in results])
    slope = float(np.polyfit(np.log(dxs), np.log(errs), 1)[0])
    (OUT / "mms.json").write_text(json.dumps({"ladder": results, "slope": slope}, indent=1) + "\n")


def main() -> None:
    bgk, eq, constants = _import_reference()
    make_equilibrium()
    make_pure(bgk, eq)
    make_trajectories(bgk, eq)
    make_determinism(bgk, eq)
    make_mms(bgk, eq, constants)
    (OUT / "PROVENANCE.json").write_text(
        json.dumps(
            {
                "generator": "tests/golden/make_golden.py",
                "reference_package": "packages/lattice-boltzmann-d3q19 (Phase-1 NumPy reference)",
                "numpy": np.__version__,
            },
            indent=1,
        )
        + "\n"
    )


if __name__ == "__main__":
    main()
