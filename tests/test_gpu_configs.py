"""Parity at the benchmark configurations' own sizes.

The other GPU parity tests run small lattices; these run the kernels the
benchmark numbers come from on the benchmark lattices themselves:

* the 256 x 128 x 128 sphere channel (40 spheres, r ~ U[4, 10], seed 42,
  tau 0.56, inflow u_x = 0.04, zero-gradient outflow): f64 bit-exact against
  the OpenMP oracle, f32 / f16 / bf16 within the stated tolerance of the
  oracle run with the same storage rounding;
* the 64^3 lid-driven cavity in its reference-exact form (x and z periodic,
  walls in y only, lid (0.05, 0, 0) on y = ny - 1, tau 0.6, 1000 steps from
  rest): f64 bit-exact against the oracle's restatement of the reference's
  own functions (bgk_step then apply_bounce_back_y_walls,
  d3q19_warp.py:321-415), f32 / f16 / bf16 within tolerance;
* 5000 steps of the sphere channel at tau 0.51 / 0.56 / 0.8 in every reduced
  storage against the f64 build of the same kernels, with the velocity
  errors bounded as stated below.
"""

from __future__ import annotations

import numpy as np
import pytest
from helpers import same_bytes

import oracle as O
from lattice_boltzmann_d3q19_b200 import Lattice, geometry

pytestmark = pytest.mark.gpu

C2 = (256, 128, 128)
C1 = (64, 64, 64)
STORE = {"f64": O.STORE_F64, "f32": O.STORE_F32, "f16": O.STORE_F16_SHIFT, "bf16": O.STORE_BF16_SHIFT}
# Max-abs tolerance on populations after the steps below (the oracle applies
# the same storage rounding in f64 arithmetic; the GPU computes in f32).
FAST_TOL = {"f32": 2e-6, "f16": 2e-4, "bf16": 2e-3}


@pytest.fixture(scope="module")
def c2_flags():
    flags, spheres = geometry.sphere_channel(C2, n_spheres=40, radius=(4.0, 10.0), seed=42)
    assert len(spheres) == 40 and (flags == 1).sum() > 0
    return flags


def _c2_pair(storage, flags):
    gpu = Lattice(C2, 0.56, storage=storage, inflow_u=(0.04, 0.0, 0.0))
    gpu.set_flags(flags)
    cpu = O.OracleLattice(C2, 0.56, storage=STORE[storage], flags=flags, inflow_u=(0.04, 0.0, 0.0))
    u0 = np.zeros((3, *C2))
    u0[0] = 0.04
    f0 = O.feq_field(np.ones(C2), u0)
    return gpu, cpu, f0


def test_c2_sphere_channel_f64_bit_exact(c2_flags):
    gpu, cpu, f0 = _c2_pair("f64", c2_flags)
    with gpu:
        gpu.set_populations(f0)
        cpu.set_populations(f0)
        for chunk in (1, 9):
            gpu.step(chunk)
            cpu.step(chunk)
            assert same_bytes(gpu.get_populations(), cpu.get_populations())
        rg, ug = gpu.rho_u()
        rc, uc = cpu.rho_u()
        assert same_bytes(rg, rc) and same_bytes(ug, uc)
        # the geometry's solid cells read back as rho = 0, u = 0
        assert np.all(rg[c2_flags == 1] == 0.0)


@pytest.mark.parametrize("storage", ["f32", "f16", "bf16"])
def test_c2_sphere_channel_reduced_storage(storage, c2_flags):
    gpu, cpu, f0 = _c2_pair(storage, c2_flags)
    with gpu:
        gpu.set_populations(f0)
        cpu.set_populations(f0)
        gpu.step(10)
        cpu.step(10)
        df = float(np.max(np.abs(gpu.get_populations() - cpu.get_populations())))
        rg, ug = gpu.rho_u()
        rc, uc = cpu.rho_u()
        dr, du = float(np.max(np.abs(rg - rc))), float(np.max(np.abs(ug - uc)))
        print(f"C2 {storage}, 10 steps: max|df|={df:.3e} max|drho|={dr:.3e} max|du|={du:.3e}")
        assert df <= FAST_TOL[storage] and dr <= 4 * FAST_TOL[storage] and du <= 4 * FAST_TOL[storage]
        # solid cells are identified exactly: zero readback there
        assert np.all(rg[c2_flags == 1] == 0.0)


def _c1_reference(steps: int) -> np.ndarray:
    """The reference's loop on the 64^3 proxy: bgk_step then the y-wall
    bounce-back with the lid on the top wall (sim.py:140-142 order)."""
    f = O.feq_field(np.ones(C1), np.zeros((3, *C1)))
    for _ in range(steps):
        f = O.apply_bounce_back_y_walls(O.bgk_step(f, 0.6), wall_velocity_top=(0.05, 0.0, 0.0))
    return f


@pytest.fixture(scope="module")
def c1_reference():
    return _c1_reference(1000)


def _c1_lattice(storage):
    return Lattice(C1, 0.6, storage=storage, periodic=(True, False, True), wall_velocity={"y+": (0.05, 0.0, 0.0)})


def test_c1_cavity_proxy_f64_bit_exact_1000_steps(c1_reference):
    with _c1_lattice("f64") as lat:
        lat.set_equilibrium()
        lat.step(1000)
        f = lat.get_populations()
        rho, u = lat.rho_u()
    assert same_bytes(f, c1_reference)
    assert same_bytes(rho, O.density_field(c1_reference))
    assert same_bytes(u, O.macroscopic_velocity(c1_reference))


# After 1000 steps: max-abs on rho and u against the f64 reference run.
C1_TOL = {"f32": (2e-6, 2e-6), "f16": (5e-4, 1e-3), "bf16": (5e-3, 2e-2)}


@pytest.mark.parametrize("storage", ["f32", "f16", "bf16"])
def test_c1_cavity_proxy_reduced_storage_1000_steps(storage, c1_reference):
    with _c1_lattice(storage) as lat:
        lat.set_equilibrium()
        lat.step(1000)
        rho, u = lat.rho_u()
    dr = float(np.max(np.abs(rho - O.density_field(c1_reference))))
    du = float(np.max(np.abs(u - O.macroscopic_velocity(c1_reference))))
    print(f"C1 proxy {storage}, 1000 steps: max|drho|={dr:.3e} max|du|={du:.3e}")
    assert dr <= C1_TOL[storage][0] and du <= C1_TOL[storage][1]


# 5000 steps of the headline channel: u error over fluid cells, L2 of the
# error field relative to the L2 of the f64 field, and the largest error
# magnitude relative to the largest f64 speed.  Bounds: (L2-rel, max-rel).
# The 16-bit storages hold deviations from feq(1, inflow velocity); f16 is
# held to the 1e-3 L2-relative target at every tau (measured on a B200 at
# 2000 steps: 1.1e-4, 5.4e-5, 1.2e-4 at tau 0.51 / 0.56 / 0.8).  f32 and
# bf16: about twice the values measured.
PRECISION_BOUND = {
    "f32": {0.51: (2.5e-4, 2e-3), 0.56: (5e-5, 1e-4), 0.8: (1.5e-4, 2e-4)},
    "f16": {0.51: (1e-3, 1e-2), 0.56: (1e-3, 1e-2), 0.8: (1e-3, 1e-2)},
    "bf16": {0.51: (2.5e-2, 2.5e-1), 0.56: (2.5e-2, 1e-1), 0.8: (4.5e-2, 1.3e-1)},
}


@pytest.mark.parametrize("tau", [0.51, 0.56, 0.8])
def test_c2_5000_steps_reduced_storage_against_f64(tau, c2_flags):
    import torch

    fluid = torch.from_numpy(c2_flags != 1).cuda()

    def run(storage):
        with Lattice(C2, tau, storage=storage, inflow_u=(0.04, 0.0, 0.0)) as lat:
            lat.set_flags(c2_flags)
            lat.set_equilibrium(1.0, (0.04, 0.0, 0.0))
            lat.step(5000)
            assert lat.check_health()
            rho = torch.empty(C2, dtype=torch.float64, device="cuda")
            u = torch.empty((3, *C2), dtype=torch.float64, device="cuda")
            lat.rho_u_device(rho.data_ptr(), u.data_ptr())
            lat.synchronize()
        return rho, u

    _, u64 = run("f64")
    ref = u64[:, fluid]
    umax = torch.sqrt((ref * ref).sum(0)).max()
    for storage in ("f32", "f16", "bf16"):
        _, u = run(storage)
        du = (u - u64)[:, fluid]
        l2 = float(torch.linalg.vector_norm(du) / torch.linalg.vector_norm(ref))
        mx = float(torch.sqrt((du * du).sum(0)).max() / umax)
        print(f"tau {tau} {storage}: u L2-rel {l2:.3e}, max-rel {mx:.3e}")
        b = PRECISION_BOUND[storage][tau]
        assert l2 <= b[0] and mx <= b[1], (storage, tau, l2, mx)
