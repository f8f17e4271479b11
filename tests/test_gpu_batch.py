"""Batched ensembles: one launch per step for many lattices, against the same
lattices stepped one by one and against the CPU oracle."""

from __future__ import annotations

import numpy as np
import pytest
from gpu_cases import random_state
from helpers import same_bytes

import oracle as O
from lattice_boltzmann_d3q19_b200 import Batch, Lattice, LbmError, geometry

pytestmark = pytest.mark.gpu

SHAPES = [(9, 8, 7), (12, 6, 10), (5, 11, 16), (16, 9, 3), (7, 7, 12)]


def _specs(storage, lids=(0.05, 0.03, 0.02, 0.07, 0.04), taus=(0.6, 0.55, 0.8, 0.7, 0.52)):
    cav = geometry.lid_driven_cavity
    return [
        dict(shape=s, tau=t, storage=storage, periodic=cav(u)["periodic"], wall_velocity=cav(u)["wall_velocity"])
        for s, t, u in zip(SHAPES, taus, lids, strict=True)
    ]


def _singles(specs, cells_per_thread):
    """Single lattices of the specs; cells_per_thread "pairs": the two-cell
    kernel where nz is even (the batch's pair schedules share its collision),
    one cell per thread otherwise."""
    out = []
    for sp in specs:
        kw = dict(sp)
        cpt = cells_per_thread
        if cpt == "pairs":
            cpt = 2 if kw["shape"][2] % 2 == 0 else 1
        out.append(Lattice(kw.pop("shape"), kw.pop("tau"), cells_per_thread=cpt, **kw))
    return out


def test_f64_batch_bit_exact_with_oracle():
    specs = _specs("f64")
    with Batch(specs) as b:
        states = [random_state(sp["shape"], 50 + k, amp=0.01) for k, sp in enumerate(specs)]
        for k, f in enumerate(states):
            b[k].set_populations(f)
        b.step(1)
        b.step(12)  # graph path
        b.step(3)   # odd remainder
        for k, sp in enumerate(specs):
            wu = Lattice._wall_array(sp["wall_velocity"])
            cpu = O.OracleLattice(sp["shape"], sp["tau"], periodic=0, wall_velocity=wu)
            cpu.set_populations(states[k])
            cpu.step(16)
            assert same_bytes(b[k].get_populations(), cpu.get_populations()), k
            assert b[k].step_count == 16


@pytest.mark.parametrize("storage", ["f32", "f16", "bf16"])
@pytest.mark.parametrize("schedule", ["single", "pair_scalar", "pair_mixed"])
def test_fast_batch_matches_single_lattices(storage, schedule):
    specs = _specs(storage)
    states = [random_state(sp["shape"], 60 + k, amp=0.01) for k, sp in enumerate(specs)]
    cpt = 1 if schedule == "single" else "pairs"
    singles = _singles(specs, cpt)
    with Batch(specs) as b:
        b.set_schedule(schedule, block=128, grid=37)
        for k, f in enumerate(states):
            b[k].set_populations(f)
            singles[k].set_populations(f)
        b.step(21)
        for k, lat in enumerate(singles):
            lat.step(21)
            fb, fs = b[k].get_populations(), lat.get_populations()
            diff = float(np.max(np.abs(fb - fs)))
            nz_even = specs[k]["shape"][2] % 2 == 0
            if schedule == "single" or (nz_even and schedule in ("pair_scalar", "pair_mixed")):
                # same per-cell arithmetic as the single-lattice kernel
                assert diff == 0.0, (k, diff)
            else:
                tol = {"f32": 2e-6, "f16": 2e-4, "bf16": 2e-3}[storage]
                assert diff <= tol, (k, diff)
            lat.close()


def test_unbatched_equals_batched_and_autotune_restores_state():
    specs = _specs("f16")
    states = [random_state(sp["shape"], 70 + k, amp=0.01) for k, sp in enumerate(specs)]
    with Batch(specs) as a, Batch(specs) as b:
        for k, f in enumerate(states):
            a[k].set_populations(f)
            b[k].set_populations(f)
        a.set_schedule("single", 256, 0)
        b.set_schedule("single", 256, 0)
        a.step(9)
        b.step_unbatched(9)
        for k in range(len(specs)):
            fa, fb = a[k].get_populations(), b[k].get_populations()
            if specs[k]["shape"][2] % 2:
                assert same_bytes(fa, fb)  # both one cell per thread
            else:  # the lattice's own kernel is the two-cell f32x2 one
                assert float(np.max(np.abs(fa - fb))) <= 2e-4
        before = [a[k].get_populations() for k in range(len(specs))]
        counts = [a[k].step_count for k in range(len(specs))]
        ms = a.autotune(4)
        assert ms > 0.0
        sched = a.schedule()
        assert sched[0] in ("single", "pair_scalar", "pair_mixed", "branches")
        for k in range(len(specs)):
            assert same_bytes(a[k].get_populations(), before[k])
            assert a[k].step_count == counts[k]
        a.step(5)  # still steps with the chosen schedule


@pytest.mark.parametrize("storage", ["f64", "f32", "f16"])
def test_branch_schedule_equals_unbatched(storage):
    """LBM_SCHED_BRANCHES runs every lattice's own kernels (four-cell ones
    with their rule quads where nz % 4 == 0): bit-identical to one launch
    per lattice, through graph replays, an odd remainder, a parameter
    change and a lattice stepped on its own (both recapture the graph)."""
    specs = _specs(storage)
    states = [random_state(sp["shape"], 80 + k, amp=0.01) for k, sp in enumerate(specs)]
    with Batch(specs) as a, Batch(specs) as b:
        for k, f in enumerate(states):
            a[k].set_populations(f)
            b[k].set_populations(f)
        a.set_schedule("branches", 128, 3)
        assert a.schedule() == ("branches", 128, 3)
        a.step(8)
        b.step_unbatched(8)
        a[2].set_tau(0.65)
        b[2].set_tau(0.65)
        a.step(5)
        b.step_unbatched(5)
        a[1].step(1)
        b[1].step(1)
        a.step(6)
        b.step_unbatched(6)
        for k in range(len(specs)):
            assert same_bytes(a[k].get_populations(), b[k].get_populations()), k
            assert a[k].step_count == b[k].step_count


def test_batch_rejects_mixed_storage_and_bad_schedule():
    specs = _specs("f16")
    specs[1]["storage"] = "f32"
    with pytest.raises(LbmError):
        Batch(specs)
    with Batch(_specs("f64")) as b:
        with pytest.raises(LbmError):
            b.set_schedule("pair_scalar")
        with pytest.raises(LbmError):
            b.set_schedule("branches", 128, 65)
