"""torch.autograd bridge of the adjoint tape.

``run(lattice, alpha, n_steps, f0=None, checkpoint_every=50)`` runs the
lattice for n_steps from f0 (or the rest state) with the porosity field alpha
and returns the final readback (rho, u) as f64 CUDA tensors.  Backward runs
the hand-written adjoint kernels through ``Lattice.tape`` (checkpoints every
``checkpoint_every`` steps, the steps in between recomputed by the forward
kernels) and returns dL/dalpha and dL/df0.  PyTorch is only the autograd and
device-memory plumbing here: every forward and adjoint step is the engine's
CUDA code.
"""

from __future__ import annotations

import torch

from .engine import Lattice


def _bind(lattice: Lattice) -> bool:
    """Run the lattice on torch's current stream when that is a real stream
    (ordered with the torch work around it); on the legacy default stream,
    which cannot carry the lattice's graph captures, the lattice keeps its own
    stream and the caller orders the two by host synchronisation (True)."""
    s = torch.cuda.current_stream()
    if s.cuda_stream:
        lattice.set_stream(s.cuda_stream)
        return False
    s.synchronize()
    return True


class _LatticeRun(torch.autograd.Function):
    @staticmethod
    def forward(ctx, alpha, f0, lattice: Lattice, n_steps: int, checkpoint_every: int):
        shape = lattice.shape
        a32 = None
        if alpha is not None:
            a32 = alpha.detach().to(device="cuda", dtype=torch.float32).contiguous()
            if tuple(a32.shape) != shape:
                raise ValueError(f"alpha must have shape {shape}; got {tuple(a32.shape)}")
        host_sync = _bind(lattice)  # after the torch work the lattice reads
        if a32 is not None:
            lattice.set_porosity_device(a32.data_ptr())
        if f0 is None:
            lattice.set_equilibrium()
        else:
            lattice.set_populations(f0.detach().to("cpu", torch.float64).numpy())
        tape = lattice.tape(n_steps, checkpoint_every)
        rho = torch.empty(shape, dtype=torch.float64, device="cuda")
        u = torch.empty((3, *shape), dtype=torch.float64, device="cuda")
        lattice.rho_u_device(rho.data_ptr(), u.data_ptr())
        if host_sync:
            lattice.synchronize()
        ctx.tape = tape
        ctx.alpha_meta = None if alpha is None else (alpha.dtype, alpha.device)
        ctx.f0_meta = None if f0 is None else (f0.dtype, f0.device)
        return rho, u

    @staticmethod
    def backward(ctx, grad_rho, grad_u):
        tape = ctx.tape
        lattice = tape.lattice
        shape = lattice.shape
        need_alpha = ctx.alpha_meta is not None and ctx.needs_input_grad[0]
        need_f0 = ctx.f0_meta is not None and ctx.needs_input_grad[1]
        gr = None if grad_rho is None else grad_rho.detach().to(torch.float64).contiguous()
        gu = None if grad_u is None else grad_u.detach().to(torch.float64).contiguous()
        ga = torch.empty(shape, dtype=torch.float64, device="cuda") if need_alpha else None
        gf = torch.empty((19, *shape), dtype=torch.float64, device="cuda") if need_f0 else None
        host_sync = _bind(lattice)  # after the seeds are ready
        tape.backward(*(None if t is None else t.data_ptr() for t in (gr, gu, ga, gf)))
        if host_sync:
            lattice.synchronize()
        if ga is not None:
            ga = ga.to(dtype=ctx.alpha_meta[0], device=ctx.alpha_meta[1])
        if gf is not None:
            gf = gf.to(dtype=ctx.f0_meta[0], device=ctx.f0_meta[1])
        return ga, gf, None, None, None


def run(lattice: Lattice, alpha: torch.Tensor | None, n_steps: int, f0: torch.Tensor | None = None,
        checkpoint_every: int = 50) -> tuple[torch.Tensor, torch.Tensor]:
    """Final (rho, u) after n_steps, differentiable w.r.t. alpha (drag model)
    and f0 (initial populations, (19, nx, ny, nz))."""
    return _LatticeRun.apply(alpha, f0, lattice, int(n_steps), int(checkpoint_every))


def box_kinetic_energy(rho: torch.Tensor, u: torch.Tensor, x_range: tuple[int, int]) -> torch.Tensor:
    """Kinetic energy sum 1/2 rho |u|^2 over the cells with x in [x0, x1)."""
    x0, x1 = x_range
    return 0.5 * (rho[x0:x1] * (u[:, x0:x1] ** 2).sum(0)).sum()


__all__ = ["box_kinetic_energy", "run"]
