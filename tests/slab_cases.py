"""Oracle adapter of the slab engine interface and slab builders shared by
the CPU and GPU slab tests."""

from __future__ import annotations

import numpy as np
from adjoint_cases import FORCE

import oracle as O
import torch_lbm
from lattice_boltzmann_d3q19_b200.slab import SlabLattice, with_halos


class OracleEngine:
    """OracleLattice behind the slab engine interface (numpy plane buffers)."""

    def __init__(self, lat: O.OracleLattice, flags):
        self.lat = lat
        self.flags = None if flags is None else np.asarray(flags)

    @staticmethod
    def _dirs(mask):
        return [d for d in range(19) if (mask >> d) & 1]

    def plane_get(self, x, mask, slot=None):
        return np.ascontiguousarray(self.lat._a[self._dirs(mask), x])

    def plane_put(self, x, mask, buf):
        self.lat._a[self._dirs(mask), x] = np.asarray(buf).reshape(self.lat._a[self._dirs(mask), x].shape)

    def step(self, n):
        self.lat.step(n)

    def set_populations(self, f):
        self.lat.set_populations(f)

    def get_populations(self):
        return self.lat.get_populations()

    def rho_u(self):
        return self.lat.rho_u()

    def conservation_planes(self, x0, x1):
        f = self.get_populations()[:, x0:x1]
        keep = np.ones(f.shape[1:], bool) if self.flags is None else (self.flags[x0:x1] & 3) != 1
        c = np.stack([torch_lbm.CX, torch_lbm.CY, torch_lbm.CZ], axis=1).astype(float)
        return np.array([f.sum(0)[keep].sum()] + [np.tensordot(c[:, a], f, 1)[keep].sum() for a in range(3)])


class OracleSplitEngine(OracleEngine):
    """OracleEngine with plane-range steps: step_planes computes the step
    of the whole slab from the current state and keeps the planes asked
    for; planes never advanced before the commit are NaN in the new state,
    so a step that read one would show it."""

    def __init__(self, lat, flags):
        super().__init__(lat, flags)
        self._next = None

    def step_planes(self, x0, x1):
        assert not self.lat._pre, "plane-range steps need a stepped state"
        full = np.empty_like(self.lat._a)
        O.lib().orc_engine_step(self.lat._L, O._ptr(self.lat._a), O._ptr(full), None, None)
        if self._next is None:
            self._next = np.full_like(self.lat._a, np.nan)
        self._next[:, x0:x1] = full[:, x0:x1]

    def step_commit(self):
        self.lat._a, self._next = self._next, None
        self.lat._spare = None


def oracle_slab(c, x0, x1, split=False):
    """SlabLattice of an adjoint_cases case (x periodic) on the oracle."""
    nx = c["shape"][0]
    kw = c["kw"]
    flags = None if c["flags"] is None else with_halos(c["flags"], x0, x1, nx)
    alpha = None if c["alpha"] is None else with_halos(c["alpha"], x0, x1, nx)
    force = None if c["force"] is None else with_halos(c["force"], x0, x1, nx, axis=1)
    lat = O.OracleLattice((x1 - x0 + 2, *c["shape"][1:]), c["tau"], periodic=kw["periodic"],
                          wall_velocity=kw.get("wall_velocity"), flags=flags, force_mode=FORCE[kw["force_mode"]],
                          body_force=kw.get("body_force", (0.0, 0.0, 0.0)), force_field=force, porosity=alpha,
                          drag_k=kw.get("drag_k", 0.0), inflow_u=kw.get("inflow_u", (0, 0, 0)))
    engine = (OracleSplitEngine if split else OracleEngine)(lat, flags)
    return SlabLattice(engine, x0, x1, flags=c["flags"], nx=nx)
