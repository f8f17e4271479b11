"""Seeded synthetic geometries for the benchmark lattices.

The reference has only y walls and periodic x/z (bgk.py:145-216); these
builders produce the flag grids and fields of the larger workloads:

* ``lid_driven_cavity`` -- all six faces walled, lid on the top (y+) face;
* ``sphere_channel``    -- inflow plane x = 0, zero-gradient outflow plane
  x = nx-1, periodic y/z, random solid spheres (periodic distance in y/z);
* ``smooth_porosity``   -- Gaussian-filtered (periodic) white noise,
  min-max scaled to [0, 1];
* ``cavity_ensemble``   -- per-lattice sizes / tau / lid speeds of a batch.

All randomness comes from ``numpy.random.default_rng(seed)``.
"""

from __future__ import annotations

import numpy as np

from ._native import CELL_FLUID, CELL_INFLOW, CELL_OUTFLOW, CELL_SOLID


def lid_driven_cavity(lid_speed: float = 0.05):
    """Keyword arguments for ``Lattice``: every axis walled, lid on y+.

    The lid uses the reference's moving-wall sign convention (the injection of
    bgk.py:198-215), under which a lid velocity (+U, 0, 0) drives the fluid
    beneath it towards -x."""
    return {
        "periodic": (False, False, False),
        "wall_velocity": {"y+": (float(lid_speed), 0.0, 0.0)},
    }


def sphere_channel(shape, n_spheres: int = 40, radius=(4.0, 10.0), seed: int = 42, x_band=(0.2, 0.8)):
    """uint8 flag grid and sphere list for a channel past random spheres.

    Centres: x uniform in the middle ``x_band`` of the channel, y/z uniform in
    [0, ny) / [0, nz); radii uniform in ``radius``; a cell is solid when its
    centre lies within a sphere (distances periodic in y and z)."""
    nx, ny, nz = (int(s) for s in shape)
    rng = np.random.default_rng(seed)
    cxs = rng.uniform(x_band[0] * nx, x_band[1] * nx, n_spheres)
    cys = rng.uniform(0.0, ny, n_spheres)
    czs = rng.uniform(0.0, nz, n_spheres)
    rs = rng.uniform(radius[0], radius[1], n_spheres)
    flags = np.full((nx, ny, nz), CELL_FLUID, dtype=np.uint8)
    ys = np.arange(ny, dtype=np.float64)
    zs = np.arange(nz, dtype=np.float64)
    for cx_, cy_, cz_, r in zip(cxs, cys, czs, rs, strict=True):
        x0 = max(0, int(np.floor(cx_ - r)))
        x1 = min(nx - 1, int(np.ceil(cx_ + r)))
        dy = np.abs(ys - cy_)
        dy = np.minimum(dy, ny - dy)
        dz = np.abs(zs - cz_)
        dz = np.minimum(dz, nz - dz)
        d2_yz = dy[:, None] ** 2 + dz[None, :] ** 2
        for x in range(x0, x1 + 1):
            mask = (x - cx_) ** 2 + d2_yz <= r * r
            flags[x][mask] = CELL_SOLID
    flags[0, :, :] = CELL_INFLOW
    flags[nx - 1, :, :] = CELL_OUTFLOW
    spheres = np.stack([cxs, cys, czs, rs], axis=1)
    return flags, spheres


def smooth_porosity(shape, sigma: float = 4.0, seed: int = 42) -> np.ndarray:
    """float32 field in [0, 1]: standard-normal noise filtered by a periodic
    Gaussian of width ``sigma`` cells (in Fourier space), min-max scaled."""
    rng = np.random.default_rng(seed)
    noise = rng.standard_normal(shape)
    spec = np.fft.rfftn(noise, axes=(0, 1, 2))
    k = [np.fft.fftfreq(n) for n in shape[:-1]] + [np.fft.rfftfreq(shape[-1])]
    k2 = sum(np.meshgrid(*[kk * kk for kk in k], indexing="ij"))
    smooth = np.fft.irfftn(spec * np.exp(-2.0 * (np.pi**2) * (sigma**2) * k2), s=shape, axes=(0, 1, 2))
    lo, hi = smooth.min(), smooth.max()
    return ((smooth - lo) / (hi - lo)).astype(np.float32)


def cavity_ensemble(count: int = 64, size_range=(32, 128), tau_range=(0.52, 0.9), lid_range=(0.02, 0.08),
                    seed: int = 42):
    """Per-lattice (shape, tau, lid_speed) of a batch of independent cavities."""
    rng = np.random.default_rng(seed)
    shapes = rng.integers(size_range[0], size_range[1] + 1, size=(count, 3))
    taus = rng.uniform(tau_range[0], tau_range[1], count)
    lids = rng.uniform(lid_range[0], lid_range[1], count)
    return [(tuple(int(v) for v in s), float(t), float(u)) for s, t, u in zip(shapes, taus, lids, strict=True)]


__all__ = ["cavity_ensemble", "lid_driven_cavity", "smooth_porosity", "sphere_channel"]
