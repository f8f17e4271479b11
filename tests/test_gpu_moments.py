"""The 16-bit moment-encoded state (the reference's frontier format,
packages/lattice-boltzmann-d3q19-frontier-moment-encoded/src/lbm_me.cpp:71-138
and :212-250) on a B200: the basis, the codec's round-trip bound, calibrated
ranges that cover the run, and moment-encoded stepping against the f64 run
of the same lattice."""

from __future__ import annotations

import numpy as np
import pytest
from gpu_cases import random_state

from lattice_boltzmann_d3q19_b200 import Lattice, LbmError, geometry
from lattice_boltzmann_d3q19_b200 import _native as N
from lattice_boltzmann_d3q19_b200.constants import VELOCITIES

pytestmark = pytest.mark.gpu


def _basis():
    m = np.empty((19, 19))
    minv = np.empty((19, 19))
    assert N.lib().lbm_moment16_basis(N.ptr(m), N.ptr(minv)) == N.LBM_OK
    return m, minv


def test_basis_is_the_monomial_basis_and_inverts():
    m, minv = _basis()
    c = np.array(VELOCITIES, dtype=float)
    x, y, z = c[:, 0], c[:, 1], c[:, 2]
    mono = [np.ones(19), x, y, z, x * x, y * y, z * z, x * y, x * z, y * z, x * x * y, x * x * z, y * y * x,
            y * y * z, z * z * x, z * z * y, x * x * y * y, x * x * z * z, y * y * z * z]
    assert np.array_equal(m, np.array(mono))
    assert np.max(np.abs(m @ minv - np.eye(19))) < 1e-12


def _channel(shape, storage):
    flags, _ = geometry.sphere_channel(shape, n_spheres=3, radius=(2.0, 3.0), seed=2)
    lat = Lattice(shape, 0.6, storage=storage, inflow_u=(0.04, 0.0, 0.0))
    lat.set_flags(flags)
    return lat, flags


def test_moment16_run_tracks_the_f64_run():
    shape, steps = (32, 16, 12), 200
    f0 = random_state(shape, 3, amp=0.01)
    ref, flags = _channel(shape, "f64")
    with ref:
        ref.set_populations(f0)
        lo, hi = ref.moment16_calibrate(steps, margin=0.05)
        r64, u64 = ref.rho_u()
    assert np.all(hi > lo)
    out = {}
    for mode in ("moment16", "f32", "f16"):
        lat, _ = _channel(shape, "f32" if mode == "moment16" else mode)
        with lat:
            lat.set_populations(f0)
            if mode == "moment16":
                lat.moment16_step(lo, hi, steps)
            else:
                lat.step(steps)
            assert lat.step_count == steps
            out[mode] = lat.rho_u()
    fluid = flags != 1
    umax = np.abs(u64[:, fluid]).max()
    err = {k: float(np.abs(v[1] - u64)[:, fluid].max() / umax) for k, v in out.items()}
    print("u max-rel error against f64:", err)
    # 16-bit codes over calibrated ranges: far finer than f16 deviations here
    assert err["moment16"] < 1e-3
    assert err["moment16"] < err["f16"]
    assert np.all(np.isfinite(out["moment16"][0]))


def test_moment16_codes_roundtrip_within_half_a_step():
    """A state encoded and decoded once (a moment16 run of one step after an
    f32 step) differs from the f32 step by at most half a code step per
    moment, mapped through M^-1."""
    shape = (16, 12, 8)
    f0 = random_state(shape, 4, amp=0.02)
    ref = Lattice(shape, 0.7, storage="f32")
    with ref:
        ref.set_populations(f0)
        lo, hi = ref.moment16_calibrate(1, margin=0.1)
        f_ref = ref.get_populations()
    with Lattice(shape, 0.7, storage="f32") as lat:
        lat.set_populations(f0)
        lat.moment16_step(lo, hi, 1)
        f = lat.get_populations()
    _, minv = _basis()
    half_step = (hi - lo) / 65535.0 / 2.0
    bound = np.abs(minv) @ half_step + 1e-6
    assert np.all(np.abs(f - f_ref).reshape(19, -1).max(axis=1) <= bound)


def test_moment16_argument_checks():
    lo, hi = np.zeros(19), np.ones(19)
    with Lattice((4, 4, 4), 0.7, storage="f16") as lat:
        with pytest.raises(LbmError):
            lat.moment16_step(lo, hi, 1)  # needs f32 storage
    with Lattice((4, 4, 4), 0.7, storage="f32") as lat:
        with pytest.raises(LbmError):
            lat.moment16_step(hi, lo, 1)  # lo >= hi
