"""PyTorch-f64 restatement of the engine step, differentiable by autograd --
TEST INFRASTRUCTURE ONLY.

The gradient oracle for the adjoint tape: the same step as the C oracle's
generalised engine (``lbm_oracle.c``: ``orc_engine_collide_local``,
``orc_engine_step``, ``orc_engine_reconstruct``, ``post_stream_state``,
``gather_site``, ``cell_force``, ``readback``, ``collide_exact``), written as
whole-lattice tensor operations so that ``torch.autograd`` differentiates the
final readback (rho, u) with respect to the porosity alpha and the initial
populations.  Its forward is pinned to the C oracle by the tests; the CUDA
adjoint is compared with its gradients.  The reference has no differentiable
LBM (its Warp kernels are not taped), so this restatement stands in for the
"Warp tape gradient".

Only ``tests/`` may import this module.  Storage is f64 (no rounding); the
single-row pairwise wall sum of the reference-exact layer is not restated
(lattices with nx * nz == 1 are rejected).
"""

from __future__ import annotations

import numpy as np
import torch
from torch.utils.checkpoint import checkpoint

# D3Q19 velocity set in the reference's lex order (constants.py:27-48).
CX = np.array([0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0])
CY = np.array([0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1])
CZ = np.array([0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1])
OPP = np.array([0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17])
W = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12)
Q = 19
CELL_FLUID, CELL_SOLID, CELL_INFLOW, CELL_OUTFLOW = 0, 1, 2, 3
# A direction whose source lies beyond several walled faces takes the first
# face in this order (faces: 0 x-, 1 x+, 2 y-, 3 y+, 4 z-, 5 z+).
FACE_PRIORITY = (3, 2, 0, 1, 4, 5)


class TorchLattice:
    """Whole-lattice f64 step with the engine's semantics (flags, walled faces,
    inflow / outflow, force models).  Arrays are (19, nx, ny, nz) /
    (nx, ny, nz) / (3, nx, ny, nz) tensors or arrays."""

    def __init__(self, shape, tau, *, periodic=7, wall_velocity=None, force_mode="none", body_force=(0, 0, 0),
                 drag_k=0.0, inflow_rho=1.0, inflow_u=(0, 0, 0), flags=None, force=None, device="cpu"):
        nx, ny, nz = (int(s) for s in shape)
        if nx * nz == 1:
            raise ValueError("single-cell wall rows (pairwise wall sum) are not restated")
        self.shape = (nx, ny, nz)
        self.n = nx * ny * nz
        self.tau = float(tau)
        self.force_mode = force_mode
        self.device = torch.device(device)
        dev = self.device
        wall = np.zeros((6, 3)) if wall_velocity is None else np.asarray(wall_velocity, dtype=np.float64)
        flags = np.zeros(self.shape, np.uint8) if flags is None else np.asarray(flags, np.uint8) & 3
        n = self.n
        X, Y, Z = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
        X, Y, Z = X.ravel(), Y.ravel(), Z.ravel()
        types = flags.ravel().astype(np.int64)
        src = np.empty((Q, n), np.int64)
        face = np.full((Q, n), -1, np.int64)
        for d in range(Q):
            sx, sy, sz = X - CX[d], Y - CY[d], Z - CZ[d]
            crossed = [np.zeros(n, bool) for _ in range(6)]
            if not periodic & 1:
                crossed[0], crossed[1] = sx < 0, sx >= nx
            if not periodic & 2:
                crossed[2], crossed[3] = sy < 0, sy >= ny
            if not periodic & 4:
                crossed[4], crossed[5] = sz < 0, sz >= nz
            for k in reversed(FACE_PRIORITY):
                face[d][crossed[k]] = k
            src[d] = ((sx % nx) * ny + (sy % ny)) * nz + (sz % nz)
        any_face = (face >= 0).any(axis=0)
        solid_src = (types[src] == CELL_SOLID) & (face < 0)
        # injection per unit wall density: -2 w_d (c_d . u_wall) / c_s^2
        K = np.zeros((Q, n))
        for d in range(Q):
            hit = face[d] >= 0
            uw = wall[face[d][hit]]
            K[d][hit] = -2.0 * W[d] * (CX[d] * uw[:, 0] + CY[d] * uw[:, 1] + CZ[d] * uw[:, 2]) * 3.0
        # gather site of each cell (outflow copies x - 1; an outflow
        # neighbour counts as fluid)
        site = np.arange(n)
        gtype = types.copy()
        out = types == CELL_OUTFLOW
        xm = (X - 1) % nx
        site[out] = (xm[out] * ny + Y[out]) * nz + Z[out]
        gtype[out] = types[site[out]]
        gtype[out & (gtype == CELL_OUTFLOW)] = CELL_FLUID

        def T(a, dtype=torch.float64):
            return torch.as_tensor(a, dtype=dtype, device=dev)

        self.src = T(src, torch.long)
        self.opp = T(OPP, torch.long)
        self.face_hit = T(face >= 0, torch.bool)
        self.any_face = T(any_face, torch.bool)
        self.solid_src = T(solid_src, torch.bool)
        self.K = T(K)
        self.site = T(site, torch.long)
        self.site_inflow = T(gtype == CELL_INFLOW, torch.bool)
        self.site_solid = T(gtype == CELL_SOLID, torch.bool)
        self.solid = T(types == CELL_SOLID, torch.bool)
        self.c = T(np.stack([CX, CY, CZ]))  # (3, 19)
        self.w = T(W)
        self.body = T(np.asarray(body_force, np.float64))
        self.drag_k = float(drag_k)
        self.force = None if force is None else T(np.asarray(force, np.float64).reshape(3, n))
        self.inflow = self._feq(T([float(inflow_rho)]), T(np.asarray(inflow_u, np.float64)).reshape(3, 1))[:, 0]

    # -- pieces of the step ----------------------------------------------------
    def _feq(self, rho, u):
        cu = self.c.T @ u  # (19, n)
        usq = (u * u).sum(0)
        return self.w[:, None] * rho[None, :] * (1.0 + cu * 3.0 + cu * cu * 4.5 - usq[None, :] * 1.5)

    def _force(self, m, alpha):
        n = m.shape[1]
        if self.force_mode == "uniform":
            return self.body[:, None].expand(3, n)
        if self.force_mode == "field":
            return self.force
        if self.force_mode == "drag":
            ka = self.drag_k * alpha
            beta = ka / (1.0 + 0.5 * ka)
            return self.body[:, None] - beta[None, :] * m
        return None

    def _collide(self, f, alpha):
        rho = f.sum(0)
        m = self.c @ f
        F = self._force(m, alpha)
        u = m / rho if F is None else (m + 0.5 * F) / rho
        out = f - (f - self._feq(rho, u)) / self.tau
        if F is not None:
            cu = self.c.T @ u
            t = (self.c[:, :, None] - u[:, None, :]) * 3.0 + cu[None, :, :] * self.c[:, :, None] * 9.0
            out = out + (1.0 - 0.5 / self.tau) * self.w[:, None] * (t * F[:, None, :]).sum(0)
        return out

    def _post_stream(self, P):
        """Pre-collision state of every cell from the stored array P (19, n)."""
        g = torch.gather(P, 1, self.src)
        rho_w = torch.where(self.any_face, g.sum(0), torch.zeros_like(g[0]))
        f_site = torch.where(self.face_hit, g[self.opp] + self.K * rho_w[None, :],
                             torch.where(self.solid_src, P[self.opp], g))
        f = f_site[:, self.site]
        f = torch.where(self.site_inflow[None, :], self.inflow[:, None].expand_as(f), f)
        return torch.where(self.site_solid[None, :], self.w[:, None].expand_as(f), f)

    def _step(self, P, alpha):
        return torch.where(self.solid[None, :], P, self._collide(self._post_stream(P), alpha))

    def _readback(self, f, alpha):
        rho = f.sum(0)
        m = self.c @ f
        F = self._force(m, alpha)
        u = m / rho if F is None else (m + 0.5 * F) / rho
        zero = torch.zeros_like(rho)
        return torch.where(self.solid, zero, rho), torch.where(self.solid[None, :], zero[None, :], u)

    # -- the run ---------------------------------------------------------------
    def run(self, f0, n_steps: int, alpha=None, segment: int = 10):
        """(rho, u) read back after n_steps >= 1 from the PRE state f0; the
        graph is checkpointed every `segment` steps to bound memory."""
        n = self.n
        f0 = torch.as_tensor(f0, dtype=torch.float64, device=self.device).reshape(Q, n)
        a = None if alpha is None else torch.as_tensor(alpha, device=self.device).to(torch.float64).reshape(n)
        P = torch.where(self.solid[None, :], self.w[:, None].expand(Q, n), self._collide(f0, a))

        def seg(P, a, k):
            for _ in range(k):
                P = self._step(P, a)
            return P

        left = n_steps - 1
        while left > 0:
            k = min(segment, left)
            P = checkpoint(seg, P, a, k, use_reentrant=False) if torch.is_grad_enabled() else seg(P, a, k)
            left -= k
        rho, u = self._readback(self._post_stream(P), a)
        return rho.reshape(self.shape), u.reshape(3, *self.shape)
