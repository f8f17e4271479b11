"""x-slab decomposition on a B200: slabs of real lattices (one process, one
GPU, one stream) exchanging faces through lbm_plane_get / lbm_plane_put step
bit-identically to the unsplit lattice, for every storage, with whole-slab
steps and with the overlapped step (lbm_step_planes / lbm_step_commit)."""

from __future__ import annotations

import numpy as np
import pytest
import torch
from adjoint_cases import case, gpu_lattice

from lattice_boltzmann_d3q19_b200 import Lattice, LbmError
from lattice_boltzmann_d3q19_b200 import _native as N
from lattice_boltzmann_d3q19_b200 import geometry
from lattice_boltzmann_d3q19_b200.slab import GpuEngine, SlabGroup, SlabLattice, exchange_distributed, slab_bounds, \
    step_distributed, with_halos

pytestmark = pytest.mark.gpu


def gpu_slab(c, x0, x1, storage, stream):
    nx = c["shape"][0]
    lat = Lattice((x1 - x0 + 2, *c["shape"][1:]), c["tau"], storage=storage, **c["kw"])
    lat.set_stream(stream.cuda_stream)
    if c["flags"] is not None:
        lat.set_flags(with_halos(c["flags"], x0, x1, nx))
    if c["force"] is not None:
        lat.set_force_field(with_halos(c["force"], x0, x1, nx, axis=1))
    if c["alpha"] is not None:
        lat.set_porosity(with_halos(c["alpha"], x0, x1, nx))
    return SlabLattice(GpuEngine(lat, storage), x0, x1, flags=c["flags"], nx=nx)


def unsplit(c, storage, n_steps):
    lat = gpu_lattice(c, storage)
    lat.set_populations(c["f0"])
    lat.step(n_steps)
    out = (*lat.rho_u(), lat.get_populations(), lat.conservation())
    lat.close()
    return out


@pytest.mark.parametrize("overlap", [False, True], ids=["whole-slab", "overlapped"])
@pytest.mark.parametrize("storage", ["f64", "f32", "f16"])
@pytest.mark.parametrize("name,parts", [("drag_channel", 3), ("field_periodic", 2)])
def test_gpu_slabs_match_unsplit(name, parts, storage, overlap):
    c = case(name)
    n_steps = 12
    rho_ref, u_ref, f_ref, cons_ref = unsplit(c, storage, n_steps)
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        group = SlabGroup([gpu_slab(c, x0, x1, storage, stream) for x0, x1 in slab_bounds(c["shape"][0], parts)],
                          overlap=overlap)
        for s in group.slabs:
            s.set_populations(c["f0"])
        group.step(n_steps)
        rho, u = group.rho_u()
        f = group.get_populations()
        cons = group.conservation()
    assert np.array_equal(rho, rho_ref) and np.array_equal(u, u_ref)
    assert np.array_equal(f, f_ref)
    np.testing.assert_allclose(cons, cons_ref, rtol=1e-12, atol=1e-12)
    for s in group.slabs:
        s.engine.lat.close()


@pytest.mark.parametrize("overlap", [False, True], ids=["whole-slab", "overlapped"])
def test_single_slab_self_exchange_matches_unsplit(overlap):
    """One slab over the whole (x-periodic) lattice exchanging with itself
    through exchange_distributed's / step_distributed's world-1 path."""
    c = case("drag_channel")
    n_steps = 9
    rho_ref, u_ref, _, _ = unsplit(c, "f32", n_steps)
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        s = gpu_slab(c, 0, c["shape"][0], "f32", stream)
        s.set_populations(c["f0"])
        for k in range(n_steps):
            if overlap:
                step_distributed(s, 0, 1, torch.cuda.Stream())
                continue
            if k:
                exchange_distributed(s, 0, 1)
            s.engine.step(1)
        exchange_distributed(s, 0, 1)
        rho, u = s.engine.rho_u()
    assert np.array_equal(s.owned(rho, 0), rho_ref) and np.array_equal(s.owned(u, 1), u_ref)
    s.engine.lat.close()


def test_plane_copy_argument_errors():
    lat = Lattice((4, 3, 2), 0.7, storage="f32")
    buf = torch.empty(5 * 3 * 2 * 4, dtype=torch.uint8, device="cuda")
    for x, mask in ((4, 0x2A82), (-1, 0x2A82), (0, 0), (0, 1 << 19)):
        with pytest.raises(LbmError) as e:
            lat.plane_get_device(x, mask, buf.data_ptr())
        assert e.value.code == N.LBM_ERR_INVALID
    host = np.zeros(30, np.float32)
    with pytest.raises(LbmError):
        lat.plane_put_device(0, 0x2A82, host.ctypes.data)
    with pytest.raises(LbmError):
        lat.conservation_planes(2, 2)
    lat.close()


@pytest.mark.parametrize("storage,cpt", [("f64", 0), ("f32", 0), ("f32", 1), ("f16", 0), ("f16", 2), ("bf16", 0)])
def test_step_planes_match_step(storage, cpt):
    """Plane ranges covering the lattice, advanced in any order and
    committed, equal lbm_step bit for bit (sphere channel with inflow and
    outflow planes: four-cell rule quads fall in every range)."""
    shape = (24, 16, 16)
    flags, _ = geometry.sphere_channel(shape, n_spheres=3, radius=(2.0, 4.0), seed=7)
    lats = []
    for _ in range(2):
        lat = Lattice(shape, 0.56, storage=storage, inflow_u=(0.04, 0.0, 0.0), cells_per_thread=cpt)
        lat.set_flags(flags)
        lat.set_equilibrium(1.0, (0.04, 0.0, 0.0))
        lat.step(1)
        lats.append(lat)
    a, b = lats
    a.step(4)
    for _ in range(4):
        for x0, x1 in ((8, 20), (0, 1), (20, 24), (1, 8)):
            b.step_planes(x0, x1)
        b.step_commit()
    assert a.step_count == b.step_count
    assert np.array_equal(a.get_populations(), b.get_populations())
    for lat in lats:
        lat.close()


def test_step_planes_state_rules():
    lat = Lattice((8, 4, 4), 0.7, storage="f32")
    with pytest.raises(LbmError) as e:  # a state upload is followed by a whole step
        lat.step_planes(0, 8)
    assert e.value.code == N.LBM_ERR_STATE
    lat.step(1)
    for x0, x1 in ((-1, 3), (0, 9), (4, 4)):
        with pytest.raises(LbmError) as e:
            lat.step_planes(x0, x1)
        assert e.value.code == N.LBM_ERR_INVALID
    with pytest.raises(LbmError) as e:
        lat.step_commit()
    assert e.value.code == N.LBM_ERR_STATE
    lat.step_planes(0, 4)
    for call in (lambda: lat.step(1), lambda: lat.set_tau(0.8), lambda: lat.set_equilibrium()):
        with pytest.raises(LbmError) as e:
            call()
        assert e.value.code == N.LBM_ERR_STATE
    lat.rho_u()  # readbacks see the step's source
    lat.step_planes(4, 8)
    lat.step_commit()
    lat.step(1)
    assert lat.check_health()
    lat.close()
