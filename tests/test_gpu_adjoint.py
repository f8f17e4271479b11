"""The adjoint tape against the PyTorch-f64 autograd restatement, central
finite differences of the GPU forward, and itself (checkpoint interval,
storage, the autograd.Function)."""

from __future__ import annotations

import numpy as np
import pytest
import torch
from adjoint_cases import CASES, case, gpu_lattice, loss_fn, torch_lattice

from lattice_boltzmann_d3q19_b200 import LbmError
from lattice_boltzmann_d3q19_b200 import _native as N
from lattice_boltzmann_d3q19_b200 import autograd as AG

pytestmark = pytest.mark.gpu


def box_of(c):
    nx = c["shape"][0]
    return (nx // 2, nx)


def tape_grads(c, n_steps, every, storage="f64"):
    """(loss, dL/dalpha or None, dL/df0) through the CUDA adjoint; torch and
    the lattice share one side stream."""
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        return _tape_grads(c, n_steps, every, storage, stream)


def _tape_grads(c, n_steps, every, storage, stream):
    shape = c["shape"]
    lat = gpu_lattice(c, storage)
    lat.set_stream(stream.cuda_stream)
    lat.set_populations(c["f0"])
    tape = lat.tape(n_steps, every)
    rho = torch.empty(shape, dtype=torch.float64, device="cuda")
    u = torch.empty((3, *shape), dtype=torch.float64, device="cuda")
    lat.rho_u_device(rho.data_ptr(), u.data_ptr())
    r = rho.clone().requires_grad_(True)
    v = u.clone().requires_grad_(True)
    L = loss_fn(r, v, box_of(c))
    L.backward()
    ga = torch.empty(shape, dtype=torch.float64, device="cuda")
    gf = torch.empty((19, *shape), dtype=torch.float64, device="cuda")
    tape.backward(r.grad.data_ptr(), v.grad.data_ptr(), ga.data_ptr(), gf.data_ptr())
    lat.synchronize()
    out = (float(L.detach()), ga.cpu().numpy() if c["alpha"] is not None else None, gf.cpu().numpy())
    tape.close()
    lat.close()
    return out


def torch_grads(c, n_steps):
    tl = torch_lattice(c, device="cuda")
    f0 = torch.tensor(c["f0"], dtype=torch.float64, device="cuda", requires_grad=True)
    a = None
    if c["alpha"] is not None:
        a = torch.tensor(c["alpha"], dtype=torch.float64, device="cuda", requires_grad=True)
    rho, u = tl.run(f0, n_steps, alpha=a, segment=10)
    L = loss_fn(rho, u, box_of(c))
    L.backward()
    return float(L.detach()), None if a is None else a.grad.cpu().numpy(), f0.grad.cpu().numpy()


def rel_err(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


@pytest.mark.parametrize("name", CASES)
def test_adjoint_matches_torch_autograd(name):
    c = case(name)
    L, ga, gf = tape_grads(c, 25, 7)
    Lt, gat, gft = torch_grads(c, 25)
    assert abs(L - Lt) <= 1e-12 * abs(Lt)
    assert rel_err(gf, gft) < 1e-9, rel_err(gf, gft)
    if ga is not None:
        assert np.abs(gat).max() > 0
        assert rel_err(ga, gat) < 1e-9, rel_err(ga, gat)
    # nothing flows into solid cells
    if c["flags"] is not None:
        solid = c["flags"] == 1
        assert not gf[:, solid].any()
        if ga is not None:
            assert not ga[solid].any()


def test_adjoint_32_cube_channel():
    """The porosity-drag channel on a 32^3 lattice, 100 steps, checkpoints
    every 10: CUDA adjoint against PyTorch-f64 autograd."""
    c = case("drag_channel", shape=(32, 32, 32))
    L, ga, gf = tape_grads(c, 100, 10)
    Lt, gat, gft = torch_grads(c, 100)
    assert abs(L - Lt) <= 1e-12 * abs(Lt)
    assert rel_err(ga, gat) < 1e-9, rel_err(ga, gat)
    assert rel_err(gf, gft) < 1e-9, rel_err(gf, gft)


def test_checkpoint_interval_does_not_change_the_gradient():
    c = case("drag_channel")
    ref = tape_grads(c, 13, 13)
    for every in (1, 4, 50):
        got = tape_grads(c, 13, every)
        assert got[0] == ref[0]
        assert np.array_equal(got[1], ref[1])
        assert np.array_equal(got[2], ref[2])


def test_adjoint_central_differences():
    """16 seeded random directions in alpha (and 4 in f0): the directional
    derivative from the adjoint against central differences of the f64 GPU
    forward.  alpha is stored as float32, so each difference uses the
    perturbation as actually stored; the error is measured against
    sum |g_i d_i|, which a cancelling direction does not shrink."""
    c = case("drag_channel")
    n_steps = 60
    _, ga, gf = tape_grads(c, n_steps, 16)
    lat = gpu_lattice(c)
    rng = np.random.default_rng(1234)

    def loss_at(alpha, f0):
        lat.set_porosity(alpha)
        lat.set_populations(f0)
        lat.step(n_steps)
        rho, u = lat.rho_u()
        return float(loss_fn(rho, u, box_of(c)))

    errs, errs_f0 = [], []
    for _ in range(16):
        v = rng.standard_normal(c["alpha"].shape)
        v /= np.linalg.norm(v)
        ap = np.clip(c["alpha"] + 1e-3 * v, 0, 1).astype(np.float32)
        am = np.clip(c["alpha"] - 1e-3 * v, 0, 1).astype(np.float32)
        delta = ap.astype(np.float64) - am.astype(np.float64)
        fd = loss_at(ap, c["f0"]) - loss_at(am, c["f0"])
        errs.append(abs(fd - float((ga * delta).sum())) / float(np.abs(ga * delta).sum()))
    for _ in range(4):
        v = rng.standard_normal(c["f0"].shape)
        v /= np.linalg.norm(v)
        eps = 1e-3
        fd = (loss_at(c["alpha"], c["f0"] + eps * v) - loss_at(c["alpha"], c["f0"] - eps * v)) / (2 * eps)
        errs_f0.append(abs(fd - float((gf * v).sum())) / float(np.abs(gf * v).sum()))
    lat.close()
    assert max(errs) < 1e-6, errs
    assert max(errs_f0) < 1e-6, errs_f0


# Relative max error of the gradient of a low-precision run against the f64
# adjoint of the same case (the forward itself differs by the storage
# rounding; the adjoint runs in f32 arithmetic).  Measured on a B200:
# f32 1.5e-6, f16 1.6e-4, bf16 1.5e-3; the bounds leave a factor 10.
LOW_TOL = {"f32": 2e-5, "f16": 2e-3, "bf16": 2e-2}


@pytest.mark.parametrize("storage", ["f32", "f16", "bf16"])
def test_adjoint_low_precision_storage(storage):
    c = case("drag_channel")
    _, ga64, gf64 = tape_grads(c, 40, 10)
    _, ga, gf = tape_grads(c, 40, 10, storage=storage)
    err = rel_err(ga, ga64)
    print(f"{storage}: grad_alpha rel err {err:.3e}, grad_f0 rel err {rel_err(gf, gf64):.3e}")
    assert err < LOW_TOL[storage]


def test_autograd_function_matches_tape():
    c = case("drag_channel")
    shape = c["shape"]
    n_steps, box = 30, box_of(c)
    lat = gpu_lattice(c)
    alpha = torch.tensor(c["alpha"], device="cuda", requires_grad=True)
    f0 = torch.tensor(c["f0"], dtype=torch.float64, device="cuda", requires_grad=True)
    rho, u = AG.run(lat, alpha, n_steps, f0=f0, checkpoint_every=8)  # default stream: host-ordered
    L = loss_fn(rho, u, box)
    L.backward()
    side = torch.cuda.Stream()
    with torch.cuda.stream(side):  # a side stream: stream-ordered
        a2 = alpha.detach().clone().requires_grad_(True)
        rho2, u2 = AG.run(lat, a2, n_steps, f0=f0.detach(), checkpoint_every=8)
        loss_fn(rho2, u2, box).backward()
    torch.cuda.synchronize()
    assert torch.equal(a2.grad, alpha.grad)
    assert alpha.grad.dtype == torch.float32 and alpha.grad.shape == shape
    Lr, ga, gf = tape_grads(c, n_steps, 8)
    assert float(L.detach()) == pytest.approx(Lr, rel=1e-14)
    np.testing.assert_allclose(alpha.grad.cpu().numpy(), ga.astype(np.float32), rtol=1e-6, atol=0)
    np.testing.assert_allclose(f0.grad.cpu().numpy(), gf, rtol=1e-12, atol=0)
    # the kinetic-energy helper differentiates like any torch loss
    rho, u = AG.run(lat, alpha.detach(), n_steps)
    assert float(AG.box_kinetic_energy(rho, u, box)) > 0
    lat.close()


def test_tape_state_errors():
    c = case("drag_channel")
    lat = gpu_lattice(c)
    lat.set_populations(c["f0"])
    with pytest.raises(LbmError) as e:
        lat.tape(0, 5)
    assert e.value.code == N.LBM_ERR_INVALID
    lat.step(2)
    with pytest.raises(LbmError) as e:
        lat.tape(5, 5)
    assert e.value.code == N.LBM_ERR_STATE
    lat.set_populations(c["f0"])
    tape = lat.tape(6, 4)
    assert tape.nbytes > 0
    lat.set_tau(0.65)
    with pytest.raises(LbmError) as e:
        tape.backward(None, None, None)
    assert e.value.code == N.LBM_ERR_STATE
    tape.close()
    lat.set_populations(c["f0"])
    tape = lat.tape(3, 2)
    host = np.zeros(c["shape"])
    with pytest.raises(LbmError) as e:  # a host pointer is refused, not launched on
        tape.backward(None, None, host.ctypes.data)
    assert e.value.code == N.LBM_ERR_INVALID
    with pytest.raises(LbmError) as e:
        lat.rho_u_device(host.ctypes.data, None)
    assert e.value.code == N.LBM_ERR_INVALID
    lat.close()
    with pytest.raises(LbmError):
        tape.backward(None, None, None)
    tape.close()
