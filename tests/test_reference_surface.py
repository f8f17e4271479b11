"""Host-side reference surface: constants, descriptors, point-evaluation
equilibrium (the reference's gates 4a, 5 and 11), geometry builders."""

from __future__ import annotations

import numpy as np
import pytest
from hypothesis import given, settings
from hypothesis import strategies as st

from lattice_boltzmann_d3q19_b200 import geometry
from lattice_boltzmann_d3q19_b200 import reference as R
from lattice_boltzmann_d3q19_b200._native import CELL_FLUID, CELL_INFLOW, CELL_OUTFLOW, CELL_SOLID

U_BOUND = 0.1 * (1.0 / 3.0) ** 0.5


def test_velocity_set_is_d3q19():
    assert len(R.VELOCITIES) == 19 and len(R.WEIGHTS) == 19
    assert tuple(R.VELOCITIES[0]) == (0, 0, 0)
    c = np.asarray(R.VELOCITIES)
    from lattice_boltzmann_d3q19_b200.constants import OPP

    assert np.all(c[OPP] == -c)


def test_weights_normalised_and_sound_speed():
    assert sum(R.WEIGHTS) == 1.0
    assert R.CS2 == 1.0 / 3.0


def test_rest_equilibrium_recovers_weights():
    f = R.feq(rho=1.0, u=(0.0, 0.0, 0.0))
    for i, w in enumerate(R.WEIGHTS):
        assert f[i] == w
    assert abs(R.density_moment(f) - 1.0) <= 1e-14


def test_canonical_descriptors_lock():
    assert R.CANONICAL_DESCRIPTOR_POISEUILLE == "poiseuille-64x32-seed42-step1000"
    assert R.CANONICAL_DESCRIPTOR_COUETTE == "couette-32x16-seed42-step500"
    assert int(R.CANONICAL_NZ) == 3 and int(R.CANONICAL_SEED) == 42


def test_equilibrium_golden(golden_equilibrium):
    g = golden_equilibrium
    f = R.feq(rho=g["rho"], u=g["u"])
    for i, expected in enumerate(g["f_eq"]):
        assert f[i] == pytest.approx(expected, abs=1e-15)
    assert sum(f) == pytest.approx(g["density_moment"], abs=1e-14)
    m = R.momentum_moment(f)
    for a in range(3):
        assert m[a] == pytest.approx(g["momentum"][a], abs=1e-14)


_floats = dict(allow_nan=False, allow_infinity=False)


@given(
    rho=st.floats(min_value=0.5, max_value=1.5, **_floats),
    ux=st.floats(min_value=-U_BOUND, max_value=U_BOUND, **_floats),
    uy=st.floats(min_value=-U_BOUND, max_value=U_BOUND, **_floats),
    uz=st.floats(min_value=-U_BOUND, max_value=U_BOUND, **_floats),
)
@settings(max_examples=50, deadline=None)
def test_pbt_equilibrium_moments(rho, ux, uy, uz):
    """Gate 11: sum feq = rho and sum c feq = rho u to 1e-14 (invariants.py:44-95)."""
    if (ux * ux + uy * uy + uz * uz) ** 0.5 / R.CS2**0.5 >= 0.1:
        return
    f = R.feq(rho, (ux, uy, uz))
    assert abs(R.density_moment(f) - rho) <= 1e-14 * max(abs(rho), 1.0)
    m = R.momentum_moment(f)
    for a, ua in enumerate((ux, uy, uz)):
        assert abs(m[a] - rho * ua) <= 1e-14 * max(abs(rho * ua), 1.0)


def test_sphere_channel_geometry():
    flags, spheres = geometry.sphere_channel((64, 32, 32), n_spheres=6, radius=(3.0, 5.0), seed=3)
    assert flags.dtype == np.uint8 and flags.shape == (64, 32, 32)
    assert np.all(flags[0] == CELL_INFLOW) and np.all(flags[-1] == CELL_OUTFLOW)
    assert set(np.unique(flags)) <= {CELL_FLUID, CELL_SOLID, CELL_INFLOW, CELL_OUTFLOW}
    assert spheres.shape == (6, 4)
    assert np.all((spheres[:, 0] >= 0.2 * 64) & (spheres[:, 0] < 0.8 * 64))
    assert np.all((spheres[:, 3] >= 3.0) & (spheres[:, 3] <= 5.0))
    solid = (flags == CELL_SOLID).sum()
    assert 0 < solid < 6 * (4 / 3) * np.pi * 5.5**3
    flags2, _ = geometry.sphere_channel((64, 32, 32), n_spheres=6, radius=(3.0, 5.0), seed=3)
    assert np.array_equal(flags, flags2)


def test_smooth_porosity_range():
    a = geometry.smooth_porosity((16, 12, 10), sigma=2.0, seed=1)
    assert a.dtype == np.float32 and a.shape == (16, 12, 10)
    assert a.min() == 0.0 and a.max() == 1.0
    # smooth: neighbouring cells differ much less than the full range
    assert np.abs(np.diff(a, axis=0)).mean() < 0.2


def test_cavity_ensemble_ranges():
    ens = geometry.cavity_ensemble(64, seed=42)
    assert len(ens) == 64
    for shape, tau, lid in ens:
        assert all(32 <= s <= 128 for s in shape)
        assert 0.52 <= tau <= 0.9 and 0.02 <= lid <= 0.08
