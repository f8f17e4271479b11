"""B200-native D3Q19 BGK lattice-Boltzmann engine.

Drop-in for the Bit-Physics Stack-E ``lattice_boltzmann_d3q19_stack_e``
package's step and state API:

* ``reference``  -- the pure-function surface (bgk_step, stream,
  apply_bounce_back_y_walls, feq_field, density_field, momentum_field,
  macroscopic_velocity, feq, density_moment, momentum_moment, constants)
  running as sm_100a kernels behind the C ABI of ``include/lbm_d3q19.h``;
* ``Lattice``    -- a stateful lattice resident in HBM, stepped by one fused
  pull-stream + bounce-back + collide kernel per step;
* ``Tape``       -- checkpointed forward + hand-written adjoint kernels, and
  ``autograd.run``, its torch.autograd.Function (gradients w.r.t. the
  porosity field and the initial populations);
* ``sim``        -- the canonical Poiseuille / Couette runners;
* ``captures``   -- load / compare captures with the reference's equivalence
  gate and tolerance, and convert them to its HDF5 capture format.
"""

from __future__ import annotations

from . import _native
from ._native import LbmError, device_count
from .constants import C, CS2, OPP, VELOCITIES, WEIGHTS, W
from .engine import Batch, Lattice, Tape

__all__ = ["Batch", "C", "CS2", "Lattice", "LbmError", "OPP", "Tape", "VELOCITIES", "W", "WEIGHTS", "_native",
           "device_count"]
