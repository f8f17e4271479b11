"""D3Q19 lattice constants and canonical descriptors.

Same values and lex ordering as the reference's
``lattice_boltzmann_d3q19_stack_e/reference/constants.py:27-88`` (velocity
order 0 rest; 1-6 faces; 7-10 xy; 11-14 xz; 15-18 yz; weights 1/3, 1/18,
1/36; c_s^2 = 1/3), which the golden equilibrium table pins.
"""

from __future__ import annotations

from typing import Final

import numpy as np

VELOCITIES: Final[tuple[tuple[int, int, int], ...]] = (
    (0, 0, 0),
    (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1),
    (1, 1, 0), (-1, -1, 0), (1, -1, 0), (-1, 1, 0),
    (1, 0, 1), (-1, 0, -1), (1, 0, -1), (-1, 0, 1),
    (0, 1, 1), (0, -1, -1), (0, 1, -1), (0, -1, 1),
)
WEIGHTS: Final[tuple[float, ...]] = (1.0 / 3.0,) + (1.0 / 18.0,) * 6 + (1.0 / 36.0,) * 12
CS2: Final[float] = 1.0 / 3.0

C: Final[np.ndarray] = np.asarray(VELOCITIES, dtype=np.int64)
W: Final[np.ndarray] = np.asarray(WEIGHTS, dtype=np.float64)
# Opposite direction of each lattice velocity (c[OPP[i]] == -c[i]).
OPP: Final[np.ndarray] = np.array([0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17], dtype=np.int64)

CANONICAL_DESCRIPTOR_POISEUILLE: Final[str] = "poiseuille-64x32-seed42-step1000"
CANONICAL_DESCRIPTOR_COUETTE: Final[str] = "couette-32x16-seed42-step500"
CANONICAL_SEED: Final[int] = 42
CANONICAL_NZ: Final[int] = 3
CANONICAL_POISEUILLE_NX: Final[int] = 64
CANONICAL_POISEUILLE_NY: Final[int] = 32
CANONICAL_POISEUILLE_STEPS: Final[int] = 1000
CANONICAL_COUETTE_NX: Final[int] = 32
CANONICAL_COUETTE_NY: Final[int] = 16
CANONICAL_COUETTE_STEPS: Final[int] = 500
CANONICAL_TAU: Final[float] = 0.7
CANONICAL_POISEUILLE_FORCE_X: Final[float] = 1.0e-5
CANONICAL_COUETTE_WALL_VELOCITY: Final[float] = 0.05

__all__ = [
    "C",
    "CANONICAL_COUETTE_NX",
    "CANONICAL_COUETTE_NY",
    "CANONICAL_COUETTE_STEPS",
    "CANONICAL_COUETTE_WALL_VELOCITY",
    "CANONICAL_DESCRIPTOR_COUETTE",
    "CANONICAL_DESCRIPTOR_POISEUILLE",
    "CANONICAL_NZ",
    "CANONICAL_POISEUILLE_FORCE_X",
    "CANONICAL_POISEUILLE_NX",
    "CANONICAL_POISEUILLE_NY",
    "CANONICAL_POISEUILLE_STEPS",
    "CANONICAL_SEED",
    "CANONICAL_TAU",
    "CS2",
    "OPP",
    "VELOCITIES",
    "W",
    "WEIGHTS",
]
