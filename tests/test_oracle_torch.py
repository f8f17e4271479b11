"""The PyTorch-f64 restatement (the adjoint tests' gradient oracle) steps
exactly like the C oracle engine: same readback after N steps on every
adjoint test configuration (flags, walled and moving faces, inflow / outflow
chains, spheres, drag, force fields)."""

from __future__ import annotations

import numpy as np
import pytest
import torch
from adjoint_cases import CASES, case, oracle_lattice, torch_lattice


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("n_steps", [1, 2, 9])
def test_torch_restatement_matches_oracle(name, n_steps):
    c = case(name)
    cpu = oracle_lattice(c)
    cpu.set_populations(c["f0"])
    cpu.step(n_steps)
    rho_o, u_o = cpu.rho_u()
    tl = torch_lattice(c)
    with torch.no_grad():
        rho_t, u_t = tl.run(c["f0"], n_steps, alpha=None if c["alpha"] is None else torch.from_numpy(c["alpha"]))
    np.testing.assert_allclose(rho_t.numpy(), rho_o, rtol=0, atol=1e-14)
    np.testing.assert_allclose(u_t.numpy(), u_o, rtol=0, atol=1e-14)


def test_torch_restatement_gradient_is_finite_difference_consistent():
    """Autograd through the restatement agrees with central differences of
    its own forward (sanity of the checkpointed graph)."""
    c = case("drag_channel", shape=(8, 6, 5))
    c["flags"][3, 2, 2] = 1
    tl = torch_lattice(c)
    alpha = torch.from_numpy(c["alpha"]).to(torch.float64).requires_grad_(True)

    def loss(a):
        rho, u = tl.run(c["f0"], 6, alpha=a, segment=4)
        return 0.5 * (rho[4:] * (u[:, 4:] ** 2).sum(0)).sum()

    L = loss(alpha)
    L.backward()
    g = alpha.grad.numpy()
    rng = np.random.default_rng(2)
    v = torch.from_numpy(rng.standard_normal(alpha.shape))
    eps = 1e-4
    with torch.no_grad():
        fd = (loss(alpha + eps * v) - loss(alpha - eps * v)) / (2 * eps)
    assert abs(float(fd) - float((g * v.numpy()).sum())) <= 1e-7 * abs(float(fd)) + 1e-18
