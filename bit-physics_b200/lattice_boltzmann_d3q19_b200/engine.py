"""Stateful lattice: populations resident on the GPU, stepped by fused kernels.

Stands in for the state the reference's evolve loops carry between calls
(``lattice_boltzmann_d3q19_stack_e/sim.py:119-190``: ``f = bgk_step(f, ...)``
then ``f = apply_bounce_back_y_walls(f, ...)`` then ``density_field`` /
``macroscopic_velocity``).  One ``step()`` is exactly one reference step; with
f64 storage the result is bit-identical to the reference's.

Beyond the reference (project semantics, pinned to the CPU oracle):
* ``periodic``: any axis may be walled; a walled axis applies the
  reference's y-wall rule on its two faces, each with its own velocity;
* ``flags``: uint8 cell types -- fluid, solid (half-way bounce-back),
  inflow (equilibrium at ``inflow_rho``/``inflow_u``), outflow
  (zero-gradient copy of the x-1 neighbour);
* ``force_mode``: none / uniform body force / per-cell field / porosity
  drag F = body_force - beta(alpha) m with beta = k alpha / (1 + k alpha / 2);
* ``storage``: f64 (reference order), f32, or 16-bit deviations (f16 /
  bf16, "shift" storage) with f32 arithmetic; the 16-bit formats hold
  f - feq(1, storage_ref_u), by default the inflow velocity (f - w_i for a
  lattice without inflow), which keeps the stored deviations small: on the
  512x256x256 sphere channel after 5000 steps at tau 0.8 the f16 velocity
  error falls from 5.9e-3 (f - w) to 4.5e-4 (L2-relative to the f64 run);
* ``staging`` / ``cells_per_thread``: which step kernel runs (register-
  staged one, two or -- f16 / bf16 with nz a multiple of 4, the default
  there -- four cells per thread, the software-pipelined two-cell kernel for
  f16 / bf16, or TMA shared-memory staging); they change speed, not
  semantics.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N

_FACE_ORDER = ("x-", "x+", "y-", "y+", "z-", "z+")


def _periodic_mask(periodic) -> int:
    if isinstance(periodic, int):
        return periodic
    px, py, pz = (bool(p) for p in periodic)
    return (1 if px else 0) | (2 if py else 0) | (4 if pz else 0)


class Lattice:
    """A D3Q19 lattice on one GPU.  Arrays in and out are NumPy f64
    (19, nx, ny, nz) / (nx, ny, nz) / (3, nx, ny, nz)."""

    def __init__(
        self,
        shape,
        tau,
        *,
        storage: str = "f64",
        periodic=(True, True, True),
        wall_velocity=None,
        force_mode: str = "none",
        body_force=(0.0, 0.0, 0.0),
        drag_k: float = 0.0,
        inflow_rho: float = 1.0,
        inflow_u=(0.0, 0.0, 0.0),
        device: int = 0,
        block_size: int = 0,
        cells_per_thread: int = 0,
        staging: str = "auto",
        storage_ref_u=None,
    ):
        nx, ny, nz = (int(s) for s in shape)
        if storage not in N.STORAGE:
            raise ValueError(f"storage must be one of {sorted(N.STORAGE)}")
        if force_mode not in N.FORCE:
            raise ValueError(f"force_mode must be one of {sorted(N.FORCE)}")
        self.shape = (nx, ny, nz)
        self.n = nx * ny * nz
        self.storage = storage
        self.force_mode = force_mode
        d = N.LbmDesc()
        N.check(N.lib().lbm_desc_init(C.byref(d)))
        d.nx, d.ny, d.nz = nx, ny, nz
        d.storage = N.STORAGE[storage]
        d.periodic = _periodic_mask(periodic)
        d.force_mode = N.FORCE[force_mode]
        d.tau = float(tau)
        wu = self._wall_array(wall_velocity)
        for k in range(18):
            d.wall_velocity[k] = float(wu[k // 3, k % 3])
        for k in range(3):
            d.body_force[k] = float(body_force[k])
            d.inflow_u[k] = float(inflow_u[k])
        d.drag_k = float(drag_k)
        d.inflow_rho = float(inflow_rho)
        d.device = int(device)
        d.block_size = int(block_size)
        d.cells_per_thread = int(cells_per_thread)
        if staging not in N.STAGING:
            raise ValueError(f"staging must be one of {sorted(N.STAGING)}")
        d.staging = N.STAGING[staging]
        ref = inflow_u if storage_ref_u is None else storage_ref_u
        for k in range(3):
            d.storage_ref_u[k] = float(ref[k])
        self.desc = d
        self._owned = True
        h = C.c_void_p()
        N.check(N.lib().lbm_create(C.byref(d), C.byref(h)))
        self._h = h

    @staticmethod
    def _wall_array(wall_velocity) -> np.ndarray:
        wu = np.zeros((6, 3))
        if wall_velocity is None:
            return wu
        if isinstance(wall_velocity, dict):
            for face, v in wall_velocity.items():
                wu[N.FACES[face] if isinstance(face, str) else int(face)] = v
            return wu
        return N.f64(wall_velocity).reshape(6, 3)

    # -- lifetime -----------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value and getattr(self, "_owned", True):
            N.lib().lbm_destroy(self._h)
        self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    # -- state --------------------------------------------------------------
    def set_populations(self, f) -> None:
        f = N.f64(f)
        if f.shape != (19, *self.shape):
            raise ValueError(f"f must have shape {(19, *self.shape)}; got {f.shape}")
        N.check(N.lib().lbm_set_populations(self._h, N.ptr(f)))

    def get_populations(self) -> np.ndarray:
        out = np.empty((19, *self.shape))
        N.check(N.lib().lbm_get_populations(self._h, N.ptr(out)))
        return out

    def set_equilibrium(self, rho=None, u=None) -> None:
        """f = feq(rho, u) (reciprocal form of equilibrium.py:310-322).  rho: scalar
        or (nx,ny,nz), default 1; u: 3-vector or (3,nx,ny,nz), default 0."""
        r = None if rho is None else N.f64(np.broadcast_to(N.f64(rho), self.shape))
        v = None
        if u is not None:
            ua = N.f64(u)
            if ua.shape == (3,):
                ua = ua.reshape(3, 1, 1, 1)
            v = N.f64(np.broadcast_to(ua, (3, *self.shape)))
        N.check(N.lib().lbm_set_equilibrium(self._h, N.ptr(r), N.ptr(v)))

    def set_flags(self, flags) -> None:
        if flags is None:
            N.check(N.lib().lbm_set_flags(self._h, None))
            return
        fl = np.ascontiguousarray(flags, dtype=np.uint8)
        if fl.shape != self.shape:
            raise ValueError(f"flags must have shape {self.shape}; got {fl.shape}")
        self._flags = fl
        N.check(N.lib().lbm_set_flags(self._h, N.ptr(fl, C.POINTER(C.c_uint8))))

    def set_force_field(self, force) -> None:
        F = N.f64(force)
        if F.shape != (3, *self.shape):
            raise ValueError(f"force must have shape {(3, *self.shape)}; got {F.shape}")
        N.check(N.lib().lbm_set_force_field(self._h, N.ptr(F)))

    def set_porosity(self, alpha) -> None:
        a = np.ascontiguousarray(alpha, dtype=np.float32)
        if a.shape != self.shape:
            raise ValueError(f"porosity must have shape {self.shape}; got {a.shape}")
        N.check(N.lib().lbm_set_porosity(self._h, N.ptr(a, C.POINTER(C.c_float))))

    def set_tau(self, tau: float) -> None:
        N.check(N.lib().lbm_set_tau(self._h, float(tau)))

    def set_wall_velocity(self, face, u3) -> None:
        idx = N.FACES[face] if isinstance(face, str) else int(face)
        N.check(N.lib().lbm_set_wall_velocity(self._h, idx, N.ptr(N.f64(u3))))

    def set_body_force(self, f3) -> None:
        N.check(N.lib().lbm_set_body_force(self._h, N.ptr(N.f64(f3))))

    # -- stepping and readback -----------------------------------------------
    def step(self, n_steps: int = 1) -> None:
        N.check(N.lib().lbm_step(self._h, int(n_steps)))

    def step_planes(self, x_begin: int, x_end: int) -> None:
        """Advance the x-planes [x_begin, x_end) of the current step into the
        next state (enqueued on the lattice's stream); step_commit() ends the
        step.  Until then the current state is the step's source, which
        plane_get_device / plane_put_device read and write; planes not
        advanced hold unspecified values after the commit.  Needs a stepped
        state (the first step after a state upload is a step())."""
        N.check(N.lib().lbm_step_planes(self._h, int(x_begin), int(x_end)))

    def step_commit(self) -> None:
        N.check(N.lib().lbm_step_commit(self._h))

    def set_rule_blocks(self, blocks: int = 0) -> None:
        """Four-cell lattices: the number of leading blocks of each step launch
        that step the quads needing a boundary rule (0: sized from their count)."""
        N.check(N.lib().lbm_set_rule_blocks(self._h, int(blocks)))

    def rule_blocks(self) -> tuple[int, int]:
        """(leading blocks, rule quads) of a four-cell lattice."""
        b, q = C.c_int32(), C.c_int32()
        N.check(N.lib().lbm_get_rule_blocks(self._h, C.byref(b), C.byref(q)))
        return b.value, q.value

    @property
    def step_count(self) -> int:
        return int(N.lib().lbm_step_count(self._h))

    def rho_u(self, out: tuple[np.ndarray, np.ndarray] | None = None) -> tuple[np.ndarray, np.ndarray]:
        """Density (nx, ny, nz) and velocity (3, nx, ny, nz) as f64 host arrays.
        ``out``: caller-owned (rho, u) arrays to fill instead (C-contiguous
        float64 of those shapes), e.g. views of pinned memory, which the
        device-to-host copy then fills at full speed."""
        if out is None:
            rho = N.fresh_host_array(self.shape)
            u = N.fresh_host_array((3, *self.shape))
        else:
            rho, u = out
            for a, shape, name in ((rho, self.shape, "rho"), (u, (3, *self.shape), "u")):
                if not (isinstance(a, np.ndarray) and a.dtype == np.float64 and a.shape == shape
                        and a.flags.c_contiguous and a.flags.writeable):
                    raise ValueError(f"out {name} must be a writeable C-contiguous float64 array of shape {shape}")
        N.check(N.lib().lbm_get_rho_u(self._h, N.ptr(rho), N.ptr(u)))
        return rho, u

    def run_capture(self, n_steps: int, every: int = 1) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
        """Advance n_steps, reading rho/u at step 0, every `every` steps and at
        the end.  Returns (steps, rho_frames, u_frames)."""
        steps = list(range(0, n_steps + 1, every))
        if steps[-1] != n_steps:
            steps.append(n_steps)
        rho = N.fresh_host_array((len(steps), *self.shape))
        u = N.fresh_host_array((len(steps), 3, *self.shape))
        N.check(N.lib().lbm_run_capture(self._h, int(n_steps), int(every), N.ptr(rho), N.ptr(u)))
        return np.array(steps), rho, u

    def step_monitor(self, n_steps: int) -> np.ndarray:
        """Advance n_steps; returns (n_steps, 4) FP64 {sum rho, sum m} of the
        state each step advanced from, reduced on the GPU."""
        out = np.empty((int(n_steps), 4))
        N.check(N.lib().lbm_step_monitor(self._h, int(n_steps), N.ptr(out)))
        return out

    def set_stream(self, cuda_stream: int | None) -> None:
        """Launch on a caller-owned cudaStream_t (an integer handle, e.g.
        torch.cuda.Stream().cuda_stream); None restores the handle's own."""
        N.check(N.lib().lbm_set_stream(self._h, C.c_void_p(cuda_stream) if cuda_stream else None))

    def conservation(self) -> np.ndarray:
        """FP64 {sum rho, sum m_x, sum m_y, sum m_z} over non-solid cells."""
        out = np.empty(4)
        N.check(N.lib().lbm_conservation(self._h, N.ptr(out)))
        return out

    def diagnostics(self, dx_phys: float) -> dict[str, float]:
        """Tier-1 / Tier-2 diagnostics of the current state reduced on the GPU
        (no field readback): the keys and values of sim.health_check and
        sim.vector_field_diagnostics on rho_u()'s arrays."""
        out = np.empty(6)
        N.check(N.lib().lbm_diagnostics(self._h, float(dx_phys), N.ptr(out)))
        keys = ("check_health", "rho_min", "rho_max", "u_max_lat", "check_divergence_free", "check_circulation")
        return {k: float(v) for k, v in zip(keys, out, strict=True)}

    # -- 16-bit moment-encoded state (the reference's frontier format) --------
    def moment16_calibrate(self, n_steps: int, margin: float = 0.05) -> tuple[np.ndarray, np.ndarray]:
        """Step n_steps and return the (lo, hi) ranges of the 19 moments over
        every post-collision state of the run, widened by margin * span."""
        lo, hi = np.empty(19), np.empty(19)
        N.check(N.lib().lbm_moment16_calibrate(self._h, int(n_steps), float(margin), N.ptr(lo), N.ptr(hi)))
        return lo, hi

    def moment16_step(self, lo, hi, n_steps: int) -> None:
        """Advance n_steps (f32 lattice) with the state between steps held as
        16-bit moment codes over the ranges [lo, hi]."""
        N.check(N.lib().lbm_moment16_step(self._h, N.ptr(N.f64(lo)), N.ptr(N.f64(hi)), int(n_steps)))

    def check_health(self) -> bool:
        rc = N.lib().lbm_check_health(self._h)
        if rc == N.LBM_ERR_NONFINITE:
            return False
        N.check(rc)
        return True

    def synchronize(self) -> None:
        N.check(N.lib().lbm_synchronize(self._h))

    # -- x-slab planes ---------------------------------------------------------
    def plane_get_device(self, x: int, dir_mask: int, ptr: int) -> None:
        """Copy plane x of the stored array, directions in dir_mask, to the
        device buffer at ptr (popcount * ny * nz storage elements)."""
        N.check(N.lib().lbm_plane_get(self._h, int(x), int(dir_mask), C.c_void_p(ptr)))

    def plane_put_device(self, x: int, dir_mask: int, ptr: int) -> None:
        """The reverse of plane_get_device."""
        N.check(N.lib().lbm_plane_put(self._h, int(x), int(dir_mask), C.c_void_p(ptr)))

    def conservation_planes(self, x0: int, x1: int) -> np.ndarray:
        """FP64 {sum rho, sum m} over the cells of the x-planes [x0, x1)."""
        out = np.empty(4)
        N.check(N.lib().lbm_conservation_planes(self._h, int(x0), int(x1), N.ptr(out)))
        return out

    # -- device pointers and the adjoint tape ----------------------------------
    def rho_u_device(self, rho_ptr: int | None, u_ptr: int | None) -> None:
        """Write rho (n) and u (3, n) as f64 to device addresses (integers,
        e.g. torch ``tensor.data_ptr()``), enqueued on the lattice's stream."""
        N.check(N.lib().lbm_get_rho_u_dev(self._h, C.c_void_p(rho_ptr) if rho_ptr else None,
                                          C.c_void_p(u_ptr) if u_ptr else None))

    def set_porosity_device(self, alpha_ptr: int) -> None:
        """set_porosity from n float32 values at a device address."""
        N.check(N.lib().lbm_set_porosity_dev(self._h, C.c_void_p(alpha_ptr)))

    def tape(self, n_steps: int, checkpoint_every: int = 50) -> Tape:
        """Run n_steps from the current (just set) populations, keeping the
        checkpoints a backward pass needs; see ``Tape``."""
        t = C.c_void_p()
        N.check(N.lib().lbm_tape_forward(self._h, int(n_steps), int(checkpoint_every), C.byref(t)))
        return Tape(self, t, int(n_steps), int(checkpoint_every))


class Tape:
    """Checkpoints of a forward run (``Lattice.tape``) and the adjoint pass
    back through it.  Pointers are device addresses (integers)."""

    def __init__(self, lattice: Lattice, handle: C.c_void_p, n_steps: int, checkpoint_every: int):
        self.lattice = lattice  # the tape borrows the lattice: keep it alive
        self._t = handle
        self.n_steps = n_steps
        self.checkpoint_every = checkpoint_every

    @property
    def nbytes(self) -> int:
        return int(N.lib().lbm_tape_bytes(self._t))

    def backward(self, grad_rho_ptr: int | None, grad_u_ptr: int | None, grad_alpha_ptr: int | None,
                 grad_f0_ptr: int | None = None) -> None:
        """dL/dalpha (n) and dL/df_0 (19, n), f64, from dL/drho (n) and dL/du
        (3, n) of the final readback; enqueued on the lattice's stream."""
        if not self._t:
            raise N.LbmError(N.LBM_ERR_STATE, "tape is closed")
        if not self.lattice._h.value:
            raise N.LbmError(N.LBM_ERR_STATE, "the tape's lattice is closed")
        vp = [C.c_void_p(p) if p else None for p in (grad_rho_ptr, grad_u_ptr, grad_alpha_ptr, grad_f0_ptr)]
        N.check(N.lib().lbm_tape_backward(self._t, *vp))

    def close(self) -> None:
        if self._t:
            N.lib().lbm_tape_destroy(self._t)
            self._t = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class Batch:
    """Independent lattices advanced together, one kernel launch per step.

    ``specs`` is a list of dicts of ``Lattice`` keyword arguments (``shape``
    and ``tau`` required); all lattices share storage and force model.
    ``batch[i]`` is a ``Lattice`` view of lattice i (state transfer,
    readback, flags) owned by the batch."""

    def __init__(self, specs):
        specs = list(specs)
        if not specs:
            raise ValueError("a batch needs at least one lattice")
        descs = (N.LbmDesc * len(specs))()
        self._views_kw = []
        for k, spec in enumerate(specs):
            kw = dict(spec)
            shape, tau = kw.pop("shape"), kw.pop("tau")
            d = N.LbmDesc()
            N.check(N.lib().lbm_desc_init(C.byref(d)))
            nx, ny, nz = (int(v) for v in shape)
            d.nx, d.ny, d.nz = nx, ny, nz
            d.storage = N.STORAGE[kw.get("storage", "f64")]
            d.periodic = _periodic_mask(kw.get("periodic", (True, True, True)))
            d.force_mode = N.FORCE[kw.get("force_mode", "none")]
            d.tau = float(tau)
            wu = Lattice._wall_array(kw.get("wall_velocity"))
            for j in range(18):
                d.wall_velocity[j] = float(wu[j // 3, j % 3])
            bf = kw.get("body_force", (0.0, 0.0, 0.0))
            iu = kw.get("inflow_u", (0.0, 0.0, 0.0))
            ref = kw.get("storage_ref_u")
            ref = iu if ref is None else ref
            for j in range(3):
                d.body_force[j] = float(bf[j])
                d.inflow_u[j] = float(iu[j])
                d.storage_ref_u[j] = float(ref[j])
            d.drag_k = float(kw.get("drag_k", 0.0))
            d.inflow_rho = float(kw.get("inflow_rho", 1.0))
            d.device = int(kw.get("device", 0))
            descs[k] = d
            self._views_kw.append(((nx, ny, nz), float(tau), kw))
        h = C.c_void_p()
        N.check(N.lib().lbm_batch_create(descs, len(specs), C.byref(h)))
        self._h = h
        self._views = []
        for k, (shape, tau, kw) in enumerate(self._views_kw):
            lh = C.c_void_p()
            N.check(N.lib().lbm_batch_lattice(self._h, k, C.byref(lh)))
            view = Lattice.__new__(Lattice)
            view.shape = shape
            view.n = shape[0] * shape[1] * shape[2]
            view.storage = kw.get("storage", "f64")
            view.force_mode = kw.get("force_mode", "none")
            view.desc = descs[k]
            view._owned = False
            view._h = lh
            self._views.append(view)

    def __len__(self):
        return len(self._views)

    def __getitem__(self, i) -> Lattice:
        return self._views[i]

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            for v in self._views:
                v._h = C.c_void_p()
            N.lib().lbm_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def step(self, n_steps: int = 1) -> None:
        N.check(N.lib().lbm_batch_step(self._h, int(n_steps)))

    def step_unbatched(self, n_steps: int = 1) -> None:
        N.check(N.lib().lbm_batch_step_unbatched(self._h, int(n_steps)))

    def set_schedule(self, schedule: str = "single", block: int = 256, grid: int = 0) -> None:
        N.check(N.lib().lbm_batch_set_schedule(self._h, N.SCHEDULES[schedule], int(block), int(grid)))

    def schedule(self) -> tuple[str, int, int]:
        s, b, g = C.c_int32(), C.c_int32(), C.c_int32()
        N.check(N.lib().lbm_batch_get_schedule(self._h, C.byref(s), C.byref(b), C.byref(g)))
        name = {v: k for k, v in N.SCHEDULES.items()}[s.value]
        return name, b.value, g.value

    def autotune(self, trial_steps: int = 20) -> float:
        """Time every schedule, keep the fastest; returns its ms per step.
        The lattices' states are restored afterwards."""
        ms = C.c_double()
        N.check(N.lib().lbm_batch_autotune(self._h, int(trial_steps), C.byref(ms)))
        return ms.value

    def synchronize(self) -> None:
        N.check(N.lib().lbm_batch_synchronize(self._h))
