"""Many steps per cooperative launch (LBM_STAGING_PERSISTENT): the same bits
as a launch per step, bit-exact f64 against the oracle, and the bounded grid
barrier's failure path (a barrier that never opens ends the launch with the
error word raised, and the lattice stays usable)."""

from __future__ import annotations

import numpy as np
import pytest
from gpu_cases import cavity_case, random_state
from helpers import same_bytes

import oracle as O
from lattice_boltzmann_d3q19_b200 import Lattice, LbmError, geometry
from lattice_boltzmann_d3q19_b200 import _native as N

pytestmark = pytest.mark.gpu


def _cavity(shape, storage, staging):
    kw = geometry.lid_driven_cavity(0.05)
    return Lattice(shape, 0.6, storage=storage, staging=staging, **kw)


def test_f64_persistent_cavity_bit_exact_with_oracle():
    gpu, cpu = cavity_case((12, 10, 9))
    gpu.close()
    f0 = O.feq_field(np.ones(cpu.shape), np.zeros((3, *cpu.shape)))
    with _cavity((12, 10, 9), "f64", "persistent") as lat:
        lat.set_populations(f0)
        cpu.set_populations(f0)
        for n in (1, 2, 37):
            lat.step(n)
            cpu.step(n)
            assert same_bytes(lat.get_populations(), cpu.get_populations())


@pytest.mark.parametrize("storage", ["f64", "f32", "f16", "bf16"])
def test_persistent_matches_a_launch_per_step(storage):
    shape = (24, 20, 16)
    flags, _ = geometry.sphere_channel(shape, n_spheres=3, radius=(2.0, 3.0), seed=4)
    flags[0] = 2
    flags[-1] = 3
    f0 = random_state(shape, 8, amp=0.01)
    out = {}
    # the persistent kernel steps pairs: against a launch per step of the
    # two-cell kernel bit for bit, and of the default (16-bit: four-cell,
    # shift folded into the collision constants) within tolerance
    runs = [("auto", 0), ("persistent", 0)]
    if storage in ("f16", "bf16"):
        runs.append(("registers", 2))
    for staging, cpt in runs:
        with Lattice(shape, 0.58, storage=storage, staging=staging, cells_per_thread=cpt, inflow_u=(0.04, 0.0, 0.0),
                     periodic=(True, False, True), wall_velocity={"y+": (0.03, 0.0, 0.0)}) as lat:
            lat.set_flags(flags)
            lat.set_populations(f0)
            lat.step(1)
            lat.step(40)
            lat.step(3)
            out[staging] = (lat.get_populations(), lat.step_count)
    assert out["auto"][1] == out["persistent"][1] == 44
    same = out["registers" if storage in ("f16", "bf16") else "auto"][0]
    assert same_bytes(same, out["persistent"][0])
    tol = {"f64": 0.0, "f32": 0.0, "f16": 2e-4, "bf16": 2e-3}[storage]
    assert float(np.max(np.abs(out["auto"][0] - out["persistent"][0]))) <= tol


def test_barrier_that_never_opens_times_out_and_reports():
    shape = (16, 12, 8)
    f0 = random_state(shape, 9, amp=0.01)
    with _cavity(shape, "f32", "persistent") as lat:
        lat.set_populations(f0)
        lat.step(1)
        assert N.lib().lbm_test_barrier_limit(lat.handle, 1, 50_000_000) == N.LBM_OK
        lat.step(10)  # every block waits 50 ms at the first barrier, then leaves
        with pytest.raises(LbmError) as e:
            lat.synchronize()
        assert e.value.code == N.LBM_ERR_CUDA and "timed out" in str(e.value)
        # the context is usable and the lattice runs again from new populations
        assert N.lib().lbm_test_barrier_limit(lat.handle, 0, 0) == N.LBM_OK
        lat.set_populations(f0)
        lat.step(6)
        lat.synchronize()
        f_a = lat.get_populations()
    with _cavity(shape, "f32", "auto") as ref:
        ref.set_populations(f0)
        ref.step(6)
        assert same_bytes(f_a, ref.get_populations())


def test_barrier_hook_needs_persistent_staging():
    with Lattice((4, 4, 4), 0.7, storage="f32") as lat:
        assert N.lib().lbm_test_barrier_limit(lat.handle, 1, 1000) == N.LBM_ERR_STATE
