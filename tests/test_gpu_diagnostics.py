"""Tier-1 / Tier-2 diagnostics reduced on the GPU (lbm_diagnostics) against
the reference's NumPy expressions (Stack-E sim.py:89-109, restated in
sim.health_check / sim.vector_field_diagnostics) on the same rho / u."""

from __future__ import annotations

import numpy as np
import pytest
from gpu_cases import random_state

from lattice_boltzmann_d3q19_b200 import Lattice, geometry, sim

pytestmark = pytest.mark.gpu


def _host(lat, dx):
    rho, u = lat.rho_u()
    return {**sim.health_check(rho, u), **sim.vector_field_diagnostics(u, dx)}


def _check(dev, host):
    for k in ("check_health", "rho_min", "rho_max", "u_max_lat", "check_divergence_free"):
        assert dev[k] == host[k], (k, dev[k], host[k])
    # the circulation is a sum: equal up to its order of summation
    assert abs(dev["check_circulation"] - host["check_circulation"]) <= 1e-12 * max(
        1e-30, abs(host["check_circulation"]) + 1e-9)


@pytest.mark.parametrize("storage", ["f64", "f32", "f16"])
def test_device_diagnostics_match_numpy_on_the_couette_run(storage):
    with sim.couette_lattice(32, 16, 3, storage=storage) as lat:
        for n in (0, 7, 40):
            lat.step(n)
            _check(lat.diagnostics(1.0 / 32), _host(lat, 1.0 / 32))


@pytest.mark.parametrize("storage", ["f64", "f16"])
def test_device_diagnostics_on_a_sphere_channel(storage):
    shape = (48, 20, 16)
    flags, _ = geometry.sphere_channel(shape, n_spheres=4, radius=(2.0, 4.0), seed=3)
    with Lattice(shape, 0.6, storage=storage, inflow_u=(0.04, 0.0, 0.0)) as lat:
        lat.set_flags(flags)
        lat.set_populations(random_state(shape, 5, amp=0.02))
        lat.step(9)
        dev = lat.diagnostics(0.5)
        _check(dev, _host(lat, 0.5))
        assert dev["rho_min"] == 0.0  # solid cells read back as 0
        assert dev["check_health"] == 0.0


def test_device_diagnostics_report_non_finite_states():
    shape = (8, 6, 4)
    f = random_state(shape, 6)
    f[3, 2, 1, 1] = np.nan
    with Lattice(shape, 0.7) as lat:
        lat.set_populations(f)
        dev = lat.diagnostics(1.0)
        assert dev["check_health"] == 1.0
        assert np.isnan(dev["rho_min"]) and np.isnan(dev["rho_max"])
