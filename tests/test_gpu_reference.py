"""GPU parity of the drop-in reference surface: bit-exact against the
reference's own outputs (golden fixtures) and against the CPU oracle."""

from __future__ import annotations

import json

import numpy as np
import pytest
from conftest import GOLDEN, load_npz
from helpers import PURE_TAGS, mms_case, same_bytes

from lattice_boltzmann_d3q19_b200 import reference as R

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("tag", PURE_TAGS)
def test_pure_functions_bit_exact(golden_pure, tag):
    g = golden_pure
    f, F = g[f"{tag}_f"], g[f"{tag}_force"]
    tau = float(g["tau"])
    assert same_bytes(R.feq_field(g[f"{tag}_rho_in"], g[f"{tag}_u_in"]), g[f"{tag}_feq_field"])
    assert same_bytes(R.density_field(f), g[f"{tag}_density_field"])
    assert same_bytes(R.momentum_field(f), g[f"{tag}_momentum_field"])
    assert same_bytes(R.macroscopic_velocity(f), g[f"{tag}_macroscopic_velocity"])
    assert same_bytes(R.macroscopic_velocity(f, F), g[f"{tag}_macroscopic_velocity_force"])
    assert same_bytes(R.stream(f), g[f"{tag}_stream"])
    assert same_bytes(R.bgk_step(f, tau), g[f"{tag}_bgk_step"])
    assert same_bytes(R.bgk_step(f, tau, F), g[f"{tag}_bgk_step_force"])
    out = R.apply_bounce_back_y_walls(f, tuple(g["wall_top"]), tuple(g["wall_bottom"]))
    assert same_bytes(out, g[f"{tag}_bounce"])


@pytest.mark.parametrize("shape", [(1, 1, 1), (2, 3, 1), (9, 7, 33), (33, 5, 2)])
def test_pure_functions_match_oracle(oracle_mod, shape):
    O = oracle_mod
    rng = np.random.default_rng(sum(shape))
    rho = 1.0 + 0.05 * rng.standard_normal(shape)
    u = 0.05 * rng.standard_normal((3, *shape))
    f = O.feq_field(rho, u) + 1e-3 * rng.standard_normal((19, *shape))
    F = 1e-4 * rng.standard_normal((3, *shape))
    assert same_bytes(R.feq_field(rho, u), O.feq_field(rho, u))
    assert same_bytes(R.bgk_step(f, 0.9, F), O.bgk_step(f, 0.9, F))
    assert same_bytes(R.bgk_step(f, 0.51), O.bgk_step(f, 0.51))
    assert same_bytes(R.stream(f), O.stream(f))
    top, bot = (0.01, 0.02, -0.03), (0.0, -0.01, 0.02)
    assert same_bytes(R.apply_bounce_back_y_walls(f, top, bot), O.apply_bounce_back_y_walls(f, top, bot))
    assert same_bytes(R.macroscopic_velocity(f, F), O.macroscopic_velocity(f, F))


def test_determinism_fixture():
    g = load_npz("determinism_16x8x3.npz")
    f0 = R.feq_field(g["rho0"], g["u0"])
    assert same_bytes(f0, g["f0"])
    a = R.bgk_step(f0, 0.7)
    b = R.bgk_step(f0, 0.7)
    assert same_bytes(a, g["f1"]) and same_bytes(a, b)


def test_mms_ladder_bit_exact():
    """Gate 4b on the GPU surface: same errors as the reference, slope 2 +- 0.5."""
    ref = json.loads((GOLDEN / "mms.json").read_text())
    g32 = load_npz("mms_n32.npz")
    errs = []
    for entry in ref["ladder"]:
        err, u_end, _ = mms_case(entry["N"], R.feq_field, R.bgk_step, R.macroscopic_velocity)
        assert err == entry["err"]
        if entry["N"] == 32:
            assert same_bytes(u_end, g32["u_end"])
        errs.append(err)
    dx = np.array([1.0 / e["N"] for e in ref["ladder"]])
    slope = float(np.polyfit(np.log(dx), np.log(errs), 1)[0])
    assert abs(slope - 2.0) <= 0.5


def test_shape_errors_raise_before_device_work():
    with pytest.raises(ValueError):
        R.stream(np.zeros((18, 2, 2, 2)))
    with pytest.raises(ValueError):
        R.bgk_step(np.zeros((19, 2, 2, 2)), 0.7, force_lattice=np.zeros((3, 2, 2, 1)))
