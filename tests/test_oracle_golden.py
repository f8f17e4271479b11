"""Pin the CPU oracle to the reference: every golden vector, bit-exact.

The fixtures in tests/golden were produced by the reference's own NumPy
implementation (tests/golden/make_golden.py); the oracle must reproduce them
byte-for-byte before any GPU result is compared against it.
"""

from __future__ import annotations

import json

import numpy as np
import pytest
from conftest import GOLDEN, load_npz
from helpers import PURE_TAGS, mms_case, same_bytes, sha


@pytest.mark.parametrize("tag", PURE_TAGS)
def test_pure_functions_bit_exact(oracle_mod, golden_pure, tag):
    O, g = oracle_mod, golden_pure
    f, F = g[f"{tag}_f"], g[f"{tag}_force"]
    tau = float(g["tau"])
    assert same_bytes(O.feq_field(g[f"{tag}_rho_in"], g[f"{tag}_u_in"]), g[f"{tag}_feq_field"])
    assert same_bytes(O.density_field(f), g[f"{tag}_density_field"])
    assert same_bytes(O.momentum_field(f), g[f"{tag}_momentum_field"])
    assert same_bytes(O.macroscopic_velocity(f), g[f"{tag}_macroscopic_velocity"])
    assert same_bytes(O.macroscopic_velocity(f, F), g[f"{tag}_macroscopic_velocity_force"])
    assert same_bytes(O.stream(f), g[f"{tag}_stream"])
    assert same_bytes(O.bgk_step(f, tau), g[f"{tag}_bgk_step"])
    assert same_bytes(O.bgk_step(f, tau, F), g[f"{tag}_bgk_step_force"])
    out = O.apply_bounce_back_y_walls(f, tuple(g["wall_top"]), tuple(g["wall_bottom"]))
    assert same_bytes(out, g[f"{tag}_bounce"])


def test_equilibrium_golden_table(oracle_mod, golden_equilibrium):
    g = golden_equilibrium
    rho = np.full((1, 1, 1), g["rho"])
    u = np.array(g["u"], dtype=np.float64).reshape(3, 1, 1, 1)
    f = oracle_mod.feq_field(rho, u).reshape(19)
    assert np.max(np.abs(f - np.array(g["f_eq"]))) <= g["tolerance_abs"]
    w, cs = oracle_mod.constants()
    assert sum(float(x) for x in w) == 1.0 and cs[0] == 1.0 / 3.0


def _trajectory_hashes(O, nx, ny, n_steps, force_x, wall_top):
    lat_kw = {"periodic": O.PERIODIC_X | O.PERIODIC_Z}
    if force_x is not None:
        lat_kw.update(force_mode=O.FORCE_UNIFORM, body_force=(force_x, 0.0, 0.0))
    if wall_top is not None:
        wu = np.zeros((6, 3))
        wu[O.FACE_YP] = wall_top
        lat_kw["wall_velocity"] = wu
    lat = O.OracleLattice((nx, ny, 3), 0.7, **lat_kw)
    lat.set_populations(O.feq_field(np.ones((nx, ny, 3)), np.zeros((3, nx, ny, 3))))
    rho_h, u_h, frames = [], [], {}
    for step in range(n_steps + 1):
        if step:
            lat.step(1)
        rho, u = lat.rho_u()
        rho_h.append(sha(rho))
        u_h.append(sha(u))
        frames[step] = (rho, u)
    return rho_h, u_h, frames, lat.get_populations()


@pytest.mark.parametrize(
    "name,nx,ny,steps,force_x,wall_top",
    [
        ("couette_32x16x3", 32, 16, 500, None, (0.05, 0.0, 0.0)),
        ("poiseuille_64x32x3", 64, 32, 1000, 1.0e-5, None),
    ],
)
def test_canonical_trajectory_every_frame(oracle_mod, name, nx, ny, steps, force_x, wall_top):
    """Stack-E gate 14: rho and u identical at every captured step."""
    g = load_npz(f"{name}.npz")
    rho_h, u_h, frames, f_final = _trajectory_hashes(oracle_mod, nx, ny, steps, force_x, wall_top)
    assert rho_h == list(g["rho_sha256"])
    assert u_h == list(g["u_sha256"])
    for s in g["keep_steps"]:
        assert same_bytes(frames[int(s)][0], g[f"rho_{s}"])
        assert same_bytes(frames[int(s)][1], g[f"u_{s}"])
    assert same_bytes(f_final, g["f_final"])


def test_couette_sign_convention(oracle_mod):
    """A top wall moving at +0.05 x drives the top row to u_x = -0.05 (bgk.py:198-215)."""
    g = load_npz("couette_32x16x3.npz")
    u = g["u_500"]
    assert np.allclose(u[0, :, -1, :], -0.05, atol=1e-12)
    assert np.allclose(u[0, :, 0, :], 0.0, atol=1e-12)


def test_determinism_fixture(oracle_mod):
    g = load_npz("determinism_16x8x3.npz")
    assert same_bytes(oracle_mod.feq_field(g["rho0"], g["u0"]), g["f0"])
    assert same_bytes(oracle_mod.bgk_step(g["f0"], 0.7), g["f1"])


def test_mms_ladder(oracle_mod):
    """Gate 4b: forced Taylor-Green errors equal to the reference's; slope 2 +- 0.5."""
    O = oracle_mod
    ref = json.loads((GOLDEN / "mms.json").read_text())
    g32 = load_npz("mms_n32.npz")
    errs = []
    for entry in ref["ladder"]:
        err, u_end, n_steps = mms_case(entry["N"], O.feq_field, O.bgk_step, O.macroscopic_velocity)
        assert n_steps == entry["n_steps"]
        assert err == entry["err"]
        if entry["N"] == 32:
            assert same_bytes(u_end, g32["u_end"])
        errs.append(err)
    dx = np.array([1.0 / e["N"] for e in ref["ladder"]])
    slope = float(np.polyfit(np.log(dx), np.log(np.array(errs)), 1)[0])
    assert abs(slope - 2.0) <= 0.5
    assert slope == pytest.approx(ref["slope"], abs=1e-12)
