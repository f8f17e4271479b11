"""GPU engine vs the CPU oracle on the extended boundary semantics.

f64 storage: bit-exact (masks, flags, walls, inflow / outflow, drag, force
fields, edge shapes).  f32 / f16 / bf16: within stated tolerances of the
oracle run with the same storage rounding.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest
from gpu_cases import cavity_case, channel_case, drag_case, pair, random_state
from helpers import same_bytes

import oracle as O
from lattice_boltzmann_d3q19_b200 import Lattice, LbmError
from lattice_boltzmann_d3q19_b200 import _native as N

pytestmark = pytest.mark.gpu


def _advance_and_compare(gpu, cpu, f0, steps, exact=True, tol=None):
    gpu.set_populations(f0)
    cpu.set_populations(f0)
    # PRE-state readback first
    rg, ug = gpu.rho_u()
    rc, uc = cpu.rho_u()
    for k, n in enumerate(steps):
        gpu.step(n)
        cpu.step(n)
        fg, fc = gpu.get_populations(), cpu.get_populations()
        rg, ug = gpu.rho_u()
        rc, uc = cpu.rho_u()
        if exact:
            assert same_bytes(fg, fc), f"populations differ after chunk {k}: {np.max(np.abs(fg - fc)):.3e}"
            assert same_bytes(rg, rc) and same_bytes(ug, uc)
        else:
            df, dr, du = (float(np.max(np.abs(a - b))) for a, b in ((fg, fc), (rg, rc), (ug, uc)))
            print(f"chunk {k}: max|df|={df:.3e} max|drho|={dr:.3e} max|du|={du:.3e}")
            assert df <= tol and dr <= tol * 4 and du <= tol * 4
    assert gpu.step_count == sum(steps)


@pytest.mark.parametrize(
    "shape,periodic",
    [
        ((7, 6, 5), (True, True, True)),
        ((9, 1, 4), (True, False, True)),
        ((1, 5, 1), (True, False, True)),
        ((1, 1, 1), (True, True, True)),
        ((5, 4, 37), (False, True, False)),
        ((31, 3, 2), (False, False, False)),
    ],
)
def test_f64_walls_and_shapes_bit_exact(shape, periodic):
    wall = {"x-": (0.01, 0.0, 0.02), "x+": (0.0, -0.02, 0.0), "y-": (0.0, 0.0, 0.01),
            "y+": (0.05, 0.0, 0.0), "z-": (0.0, 0.03, 0.0), "z+": (-0.02, 0.0, 0.0)}
    gpu, cpu = pair(shape, 0.63, periodic=periodic, wall_velocity=wall)
    with gpu:
        _advance_and_compare(gpu, cpu, random_state(shape, 11), [1, 1, 5, 13])


def test_f64_cavity_bit_exact():
    gpu, cpu = cavity_case()
    with gpu:
        _advance_and_compare(gpu, cpu, O.feq_field(np.ones(cpu.shape), np.zeros((3, *cpu.shape))), [1, 20, 40])


def test_f64_sphere_channel_bit_exact():
    (gpu, cpu), flags = channel_case()
    assert (flags == 1).sum() > 0
    f0 = O.feq_field(np.ones(cpu.shape), np.tile(np.array([0.04, 0, 0]).reshape(3, 1, 1, 1), (1, *cpu.shape)))
    with gpu:
        _advance_and_compare(gpu, cpu, f0, [1, 30, 30])
        c_gpu, c_cpu = gpu.conservation(), cpu.conservation()
        assert np.allclose(c_gpu, c_cpu, rtol=1e-12, atol=1e-12)


def test_f64_drag_and_force_field_bit_exact():
    gpu, cpu = drag_case()
    with gpu:
        _advance_and_compare(gpu, cpu, random_state(cpu.shape, 12, amp=0.02), [1, 25])
    shape = (6, 5, 7)
    F = 1e-4 * np.random.default_rng(3).standard_normal((3, *shape))
    gpu, cpu = pair(shape, 0.8, periodic=(True, False, True), force_mode="field", force_field=F,
                    wall_velocity={"y+": (0.02, 0.0, 0.0)})
    with gpu:
        _advance_and_compare(gpu, cpu, random_state(shape, 13), [1, 9])
    gpu, cpu = pair(shape, 0.55, force_mode="uniform", body_force=(1e-5, -2e-6, 3e-6))
    with gpu:
        _advance_and_compare(gpu, cpu, random_state(shape, 14), [1, 9])


def test_f64_block_sizes_agree():
    shape = (13, 11, 7)
    f0 = random_state(shape, 21)
    outs = []
    for bs in (32, 96, 256):
        gpu, _ = pair(shape, 0.7, periodic=(False, True, True), block_size=bs)
        with gpu:
            gpu.set_populations(f0)
            gpu.step(10)
            outs.append(gpu.get_populations())
    assert same_bytes(outs[0], outs[1]) and same_bytes(outs[0], outs[2])


def test_set_flags_mid_run_matches_oracle():
    shape = (10, 8, 6)
    gpu, cpu = pair(shape, 0.7)
    f0 = random_state(shape, 22)
    flags = np.zeros(shape, dtype=np.uint8)
    flags[4:6, 3:5, 2:4] = 1
    with gpu:
        gpu.set_populations(f0)
        gpu.step(5)
        cpu.set_populations(f0)
        cpu.step(5)
        gpu.set_flags(flags)
        cpu2 = O.OracleLattice(shape, 0.7, flags=flags)
        cpu2.set_populations(cpu.get_populations())
        gpu.step(7)
        cpu2.step(7)
        assert same_bytes(gpu.get_populations(), cpu2.get_populations())


def test_conservation_f64():
    shape = (16, 12, 10)
    gpu, cpu = pair(shape, 0.6)
    f0 = random_state(shape, 23)
    with gpu:
        gpu.set_populations(f0)
        cpu.set_populations(f0)
        for _ in range(3):
            a, b = gpu.conservation(), cpu.conservation()
            assert np.allclose(a, b, rtol=1e-13, atol=1e-13)
            gpu.step(4)
            cpu.step(4)
        assert gpu.check_health()


FAST_TOL = {"f32": 2e-6, "f16": 2e-4, "bf16": 2e-3}


@pytest.mark.parametrize("storage", ["f32", "f16", "bf16"])
def test_fast_storages_cavity(storage):
    gpu, cpu = cavity_case(storage=storage)
    with gpu:
        _advance_and_compare(gpu, cpu, O.feq_field(np.ones(cpu.shape), np.zeros((3, *cpu.shape))), [1, 20, 40],
                             exact=False, tol=FAST_TOL[storage])


@pytest.mark.parametrize("storage", ["f32", "f16", "bf16"])
def test_fast_storages_channel_and_drag(storage):
    (gpu, cpu), _ = channel_case(storage=storage)
    f0 = O.feq_field(np.ones(cpu.shape), np.tile(np.array([0.04, 0, 0]).reshape(3, 1, 1, 1), (1, *cpu.shape)))
    with gpu:
        _advance_and_compare(gpu, cpu, f0, [1, 30], exact=False, tol=FAST_TOL[storage])
        a, b = gpu.conservation(), cpu.conservation()
        assert abs(a[0] - b[0]) <= 1e-4 * b[0]
    gpu, cpu = drag_case(storage=storage)
    with gpu:
        _advance_and_compare(gpu, cpu, random_state(cpu.shape, 12, amp=0.02), [1, 25], exact=False,
                             tol=FAST_TOL[storage])


@pytest.mark.parametrize("storage", ["f32", "f16", "bf16"])
def test_two_cells_per_thread_matches_one(storage):
    """k_step2 (two z-adjacent cells per thread) against k_step on the sphere
    channel and on a walled box with an odd-sized x/y and even nz."""
    for case in ("channel", "box"):
        outs = []
        for cpt in (1, 2):
            if case == "channel":
                flags, _ = __import__("lattice_boltzmann_d3q19_b200").geometry.sphere_channel(
                    (40, 16, 14), n_spheres=4, radius=(2.0, 4.0), seed=5)
                lat = Lattice((40, 16, 14), 0.56, storage=storage, inflow_u=(0.04, 0.0, 0.0), cells_per_thread=cpt)
                lat.set_flags(flags)
                f0 = random_state((40, 16, 14), 26, amp=0.01)
            else:
                lat = Lattice((7, 5, 10), 0.6, storage=storage, periodic=(False, False, False),
                              wall_velocity={"y+": (0.05, 0.0, 0.0)}, cells_per_thread=cpt)
                f0 = random_state((7, 5, 10), 27, amp=0.01)
            with lat:
                lat.set_populations(f0)
                lat.step(20)
                sums = lat.step_monitor(3)
                outs.append((lat.get_populations(), sums))
        diff = float(np.max(np.abs(outs[0][0] - outs[1][0])))
        print(f"{case} {storage}: max |f(1 cell) - f(2 cells)| = {diff:.3e}")
        assert diff <= FAST_TOL[storage]
        # FP64 sums of per-cell values that each differ by at most ~diff
        cells = outs[0][0][0].size
        assert np.allclose(outs[0][1], outs[1][1], rtol=0.0, atol=4 * cells * FAST_TOL[storage])


TMA_CASES = [
    # shape, tau, periodic, walls, with flags: rows per tile 8 with a partial
    # last tile (ny = 9 / 10), y walls (wrap splits of the row copies), flags
    ((12, 9, 16), 0.6, (True, False, True), {"y+": (0.04, 0.0, 0.0), "y-": (0.0, 0.0, -0.01)}, False),
    ((10, 10, 32), 0.56, (True, True, True), None, True),
    ((6, 3, 8), 0.7, (False, True, False), {"x-": (0.0, 0.02, 0.0), "z+": (0.01, 0.0, 0.0)}, True),
]


@pytest.mark.parametrize("storage", ["f32", "f16", "bf16"])
@pytest.mark.parametrize("case", range(len(TMA_CASES)))
def test_tma_staging_matches_oracle_and_registers(storage, case):
    """The TMA-staged kernel against the CPU oracle (same storage rounding)
    and against the register-staged two-cell kernel."""
    shape, tau, periodic, walls, with_flags = TMA_CASES[case]
    if storage == "f32" and (shape[2] * 4) % 16:
        pytest.skip("row not a multiple of 16 bytes")
    flags = None
    if with_flags:
        flags = np.zeros(shape, dtype=np.uint8)
        flags[0] = 2
        flags[-1] = 3
        flags[shape[0] // 2, 1:3, 2:5] = 1
    f0 = random_state(shape, 40 + case, amp=0.01)
    outs = {}
    for staging in ("tma", "registers"):
        gpu, cpu = pair(shape, tau, storage, periodic=periodic, wall_velocity=walls, flags=flags,
                        inflow_u=(0.03, 0.0, 0.0))
        gpu.close()
        lat = Lattice(shape, tau, storage=storage, periodic=periodic, wall_velocity=walls,
                      inflow_u=(0.03, 0.0, 0.0), staging=staging, cells_per_thread=2)
        with lat:
            if flags is not None:
                lat.set_flags(flags)
            lat.set_populations(f0)
            lat.step(1)
            lat.step(15)
            sums = lat.step_monitor(4)
            outs[staging] = (lat.get_populations(), sums, lat.rho_u())
        cpu.set_populations(f0)
        cpu.step(20)
    fc = cpu.get_populations()
    d_oracle = float(np.max(np.abs(outs["tma"][0] - fc)))
    d_regs = float(np.max(np.abs(outs["tma"][0] - outs["registers"][0])))
    print(f"case {case} {storage}: tma vs oracle {d_oracle:.3e}, tma vs registers {d_regs:.3e}")
    assert d_oracle <= FAST_TOL[storage] and d_regs <= FAST_TOL[storage]
    cells = fc[0].size
    assert np.allclose(outs["tma"][1], outs["registers"][1], rtol=0.0, atol=4 * cells * FAST_TOL[storage])


PIPE_CASES = [
    # shape, tau, periodic, walls, with flags, uniform force
    ((12, 9, 16), 0.6, (True, False, True), {"y+": (0.04, 0.0, 0.0), "y-": (0.0, 0.0, -0.01)}, False, False),
    ((10, 10, 32), 0.56, (True, True, True), None, True, False),
    ((6, 3, 8), 0.7, (False, True, False), {"x-": (0.0, 0.02, 0.0), "z+": (0.01, 0.0, 0.0)}, True, False),
    ((16, 12, 20), 0.8, (True, True, True), None, True, True),
    ((40, 30, 66), 0.55, (True, True, True), None, True, False),
]


@pytest.mark.parametrize("storage", ["f16", "bf16"])
@pytest.mark.parametrize("case", range(len(PIPE_CASES)))
def test_pipelined_staging_bit_identical_to_registers(storage, case):
    """The software-pipelined 16-bit kernel (grid-stride loop, next pair's
    loads issued before this pair's collision) computes exactly what the
    register-staged two-cell kernel computes: same populations, bit for bit."""
    shape, tau, periodic, walls, with_flags, force = PIPE_CASES[case]
    flags = None
    if with_flags:
        flags = np.zeros(shape, dtype=np.uint8)
        flags[0] = 2
        flags[-1] = 3
        flags[shape[0] // 2, 1:3, 2:5] = 1
    f0 = random_state(shape, 70 + case, amp=0.01)
    kw = {"force_mode": "uniform", "body_force": (1e-5, -2e-6, 3e-6)} if force else {}
    outs = {}
    for staging in ("pipelined", "registers"):
        lat = Lattice(shape, tau, storage=storage, periodic=periodic, wall_velocity=walls,
                      inflow_u=(0.03, 0.0, 0.0), staging=staging, cells_per_thread=2, **kw)
        with lat:
            if flags is not None:
                lat.set_flags(flags)
            lat.set_populations(f0)
            lat.step(1)
            lat.step(25)
            outs[staging] = (lat.get_populations(), lat.step_monitor(3), lat.get_populations())
    for k in range(3):
        assert np.array_equal(outs["pipelined"][k], outs["registers"][k]), k


@pytest.mark.parametrize("storage", ["f16", "bf16"])
@pytest.mark.parametrize("force_mode", ["field", "drag"])
def test_pipelined_staging_per_cell_forces_bit_identical(storage, force_mode):
    """Per-cell force inputs (an f32 force field; porosity drag) read as
    (cell, cell + 1) pairs by the pipelined kernel, against the
    register-staged two-cell kernel."""
    from lattice_boltzmann_d3q19_b200 import geometry

    shape = (24, 10, 12)
    flags = np.zeros(shape, dtype=np.uint8)
    flags[0] = 2
    flags[-1] = 3
    flags[12, 3:6, 4:8] = 1
    force = 1e-5 * np.random.default_rng(5).standard_normal((3, *shape))
    alpha = geometry.smooth_porosity(shape, sigma=2.0, seed=9)
    f0 = random_state(shape, 95, amp=0.01)
    outs = {}
    for staging in ("pipelined", "registers"):
        kw = {"drag_k": 0.05, "body_force": (1e-6, 0.0, 0.0)} if force_mode == "drag" else {}
        lat = Lattice(shape, 0.7, storage=storage, force_mode=force_mode, inflow_u=(0.03, 0.0, 0.0),
                      staging=staging, cells_per_thread=2, **kw)
        with lat:
            lat.set_flags(flags)
            if force_mode == "drag":
                lat.set_porosity(alpha)
            else:
                lat.set_force_field(force)
            lat.set_populations(f0)
            lat.step(1)
            lat.step(20)
            outs[staging] = lat.get_populations()
    assert np.array_equal(outs["pipelined"], outs["registers"])


def test_pipelined_staging_covers_many_pairs_per_thread():
    """Several pairs per thread of the resident grid (the prefetch carried
    across loop iterations), against the register-staged kernel."""
    shape = (64, 64, 128)  # 262,144 pairs over at most 148 x 2 x 256 threads
    flags = np.zeros(shape, dtype=np.uint8)
    flags[0] = 2
    flags[-1] = 3
    flags[20:24, 30:34, 60:64] = 1
    f0 = random_state(shape, 91, amp=0.01)
    lat = Lattice(shape, 0.6, storage="f16", inflow_u=(0.03, 0.0, 0.0), staging="pipelined", cells_per_thread=2)
    ref = Lattice(shape, 0.6, storage="f16", inflow_u=(0.03, 0.0, 0.0), staging="registers", cells_per_thread=2)
    with lat, ref:
        for x in (lat, ref):
            x.set_flags(flags)
            x.set_populations(f0)
            x.step(12)
        assert np.array_equal(lat.get_populations(), ref.get_populations())


def test_pipelined_staging_rejected_where_unsupported():
    for storage in ("f32", "f64"):
        with pytest.raises(LbmError) as e:
            Lattice((4, 4, 8), 0.7, storage=storage, staging="pipelined")
        assert e.value.code == N.LBM_ERR_UNSUPPORTED
    with pytest.raises(LbmError) as e:
        Lattice((4, 4, 5), 0.7, storage="f16", staging="pipelined")   # odd nz: one cell per thread
    assert e.value.code == N.LBM_ERR_UNSUPPORTED


@pytest.mark.parametrize("storage", ["f32", "f16"])
def test_step_sums_match_conservation_over_many_pairs_per_thread(storage):
    """The per-step FP64 sums of the grid-stride sums kernel (several pairs
    per thread, one partial row per resident block) against the readback
    sums of the same states."""
    shape = (64, 64, 128)
    flags = np.zeros(shape, dtype=np.uint8)
    flags[0] = 2
    flags[-1] = 3
    flags[20:26, 30:36, 60:66] = 1
    lat = Lattice(shape, 0.6, storage=storage, inflow_u=(0.03, 0.0, 0.0))
    with lat:
        lat.set_flags(flags)
        lat.set_populations(random_state(shape, 93, amp=0.01))
        lat.step(5)
        for _ in range(3):
            c = lat.conservation()
            s = lat.step_monitor(1)[0]
            # per-cell moments in f32 against the readback's own arithmetic:
            # ~1e-9 per cell; a pair left out or counted twice moves the mass
            # sum by ~2
            assert np.allclose(s, c, rtol=0.0, atol=0.2), (s, c)


def test_tma_staging_rejected_where_unsupported():
    with pytest.raises(LbmError) as e:
        Lattice((4, 4, 6), 0.7, storage="f16", staging="tma")   # 12-byte rows
    assert e.value.code == N.LBM_ERR_UNSUPPORTED
    with pytest.raises(LbmError):
        Lattice((4, 4, 8), 0.7, storage="f64", staging="tma")


def test_two_cells_per_thread_rejected_where_unsupported():
    with pytest.raises(LbmError) as e:
        Lattice((4, 4, 5), 0.7, storage="f16", cells_per_thread=2)
    assert e.value.code == N.LBM_ERR_UNSUPPORTED
    with pytest.raises(LbmError):
        Lattice((4, 4, 4), 0.7, storage="f64", cells_per_thread=2)


@pytest.mark.parametrize("storage", ["f32", "f16", "bf16"])
def test_fast_storage_run_to_run_identical(storage):
    (gpu, _), _ = channel_case(storage=storage)
    f0 = random_state(gpu.shape, 24, amp=0.01)
    outs = []
    with gpu:
        for _ in range(2):
            gpu.set_populations(f0)
            gpu.step(17)
            outs.append(gpu.get_populations())
    assert same_bytes(outs[0], outs[1])


def test_error_codes():
    with Lattice((4, 4, 4), 0.7, force_mode="field") as lat:
        with pytest.raises(LbmError) as e:
            lat.step(1)
        assert e.value.code == N.LBM_ERR_STATE
    with Lattice((4, 4, 4), 0.7, force_mode="drag", drag_k=0.1) as lat:
        with pytest.raises(LbmError) as e:
            lat.set_porosity(np.full((4, 4, 4), 1.5, dtype=np.float32))
        assert e.value.code == N.LBM_ERR_INVALID
    with Lattice((4, 4, 4), 0.7) as lat:
        bad = np.zeros((4, 4, 4), dtype=np.uint8)
        bad[1, 1, 1] = 9
        with pytest.raises(LbmError) as e:
            lat.set_flags(bad)
        assert e.value.code == N.LBM_ERR_INVALID
        with pytest.raises(LbmError) as e:
            lat.set_tau(0.5)
        assert e.value.code == N.LBM_ERR_INVALID
        with pytest.raises(LbmError):
            lat.set_force_field(np.zeros((3, 4, 4, 4)))
        assert N.lib().lbm_step(lat.handle, -1) == N.LBM_ERR_INVALID
        assert N.lib().lbm_set_wall_velocity(lat.handle, 7, None) == N.LBM_ERR_INVALID


def test_nonfinite_state_detected():
    with Lattice((4, 4, 4), 0.7) as lat:
        f = random_state((4, 4, 4), 25)
        f[3, 1, 2, 3] = np.nan
        lat.set_populations(f)
        assert not lat.check_health()
        lat.step(2)
        assert not lat.check_health()


def test_many_handles_and_stream():
    lats = [Lattice((8, 8, 8), 0.6 + 0.01 * k, storage=("f64", "f32", "f16", "bf16")[k % 4]) for k in range(8)]
    for lat in lats:
        lat.set_equilibrium(1.0, (0.01, 0.0, 0.0))
        lat.step(3)
    for lat in lats:
        rho, u = lat.rho_u()
        assert np.allclose(u[0], 0.01, atol=1e-3)
        lat.close()
    assert N.lib().lbm_set_stream(C.c_void_p(), None) == N.LBM_ERR_INVALID


def test_rho_u_into_caller_arrays():
    """rho_u(out=...) fills caller-owned arrays with the values rho_u()
    returns, and rejects arrays of the wrong shape, type or layout."""
    shape = (8, 6, 10)
    lat = Lattice(shape, 0.7, storage="f16", inflow_u=(0.03, 0.0, 0.0))
    with lat:
        lat.set_populations(random_state(shape, 97, amp=0.01))
        lat.step(3)
        rho, u = lat.rho_u()
        ro, uo = np.full(shape, np.nan), np.full((3, *shape), np.nan)
        r2, u2 = lat.rho_u(out=(ro, uo))
        assert r2 is ro and u2 is uo
        assert np.array_equal(ro, rho) and np.array_equal(uo, u)
        for bad in ((np.empty(shape, np.float32), uo), (ro, np.empty((3, *shape))[:, ::-1]), (ro, np.empty(shape))):
            with pytest.raises(ValueError):
                lat.rho_u(out=bad)
