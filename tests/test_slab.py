"""x-slab decomposition on the CPU oracle: slabs with halo planes step
bit-identically to the unsplit lattice, in one process and as two gloo ranks
exchanging their faces with torch.distributed."""

from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp
from adjoint_cases import case, oracle_lattice
from slab_cases import oracle_slab

from lattice_boltzmann_d3q19_b200.slab import SlabGroup, conservation_distributed, exchange_distributed, slab_bounds, \
    step_distributed, with_halos


def test_slab_bounds_and_halos():
    assert slab_bounds(10, 3) == [(0, 4), (4, 7), (7, 10)]
    assert slab_bounds(9, 3) == [(0, 3), (3, 6), (6, 9)]
    with pytest.raises(ValueError):
        slab_bounds(8, 3)
    a = np.arange(10)[:, None] * np.ones((1, 2))
    np.testing.assert_array_equal(with_halos(a, 0, 4, 10)[:, 0], [9, 0, 1, 2, 3, 4])
    np.testing.assert_array_equal(with_halos(a, 7, 10, 10)[:, 0], [6, 7, 8, 9, 0])


def test_outflow_on_a_slab_face_is_refused():
    c = case("drag_channel")  # outflow planes x = 18, 19
    with pytest.raises(ValueError):
        oracle_slab(c, 18, 20)


@pytest.mark.parametrize("split", [False, True], ids=["whole-slab", "overlapped"])
@pytest.mark.parametrize("name,parts", [("drag_channel", 3), ("field_periodic", 2)])
def test_slab_group_matches_unsplit(name, parts, split):
    """Whole-slab steps after an exchange, and the overlapped step (interior,
    then imported halos and boundary planes; halo planes never advanced)."""
    c = case(name)
    n_steps = 7
    ref = oracle_lattice(c)
    ref.set_populations(c["f0"])
    ref.step(n_steps)
    rho_ref, u_ref = ref.rho_u()
    group = SlabGroup([oracle_slab(c, x0, x1, split) for x0, x1 in slab_bounds(c["shape"][0], parts)])
    for s in group.slabs:
        s.set_populations(c["f0"])
    group.step(n_steps)
    rho, u = group.rho_u()
    assert np.array_equal(rho, rho_ref) and np.array_equal(u, u_ref)
    assert np.array_equal(group.get_populations(), ref.get_populations())
    np.testing.assert_allclose(group.conservation(), ref.conservation(), rtol=1e-13, atol=1e-13)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, n_steps, out_dir, split):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        c = case("drag_channel")
        x0, x1 = slab_bounds(c["shape"][0], world)[rank]
        s = oracle_slab(c, x0, x1, split)
        s.set_populations(c["f0"])
        to_t = lambda b: torch.from_numpy(np.ascontiguousarray(b))  # noqa: E731
        from_t = lambda t, like: t.numpy().reshape(like.shape)  # noqa: E731
        for k in range(n_steps):
            if split:
                step_distributed(s, rank, world, None, to_t, from_t)
                continue
            if k > 0:
                exchange_distributed(s, rank, world, to_t, from_t)
            s.engine.step(1)
        exchange_distributed(s, rank, world, to_t, from_t)
        rho, u = s.engine.rho_u()
        cons = conservation_distributed(s, rank, world, to_t, from_t)
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), rho=s.owned(rho, 0), u=s.owned(u, 1), cons=cons)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("split", [False, True], ids=["whole-slab", "overlapped"])
def test_two_gloo_ranks_match_unsplit(tmp_path, split):
    """world_size 2 over gloo on the CPU: each rank steps one oracle slab and
    exchanges its faces with exchange_distributed, or takes the overlapped
    step_distributed (the code paths NCCL runs on GPUs); the gathered owned
    planes equal the unsplit oracle's."""
    n_steps, world = 6, 2
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, n_steps, str(tmp_path), split))
             for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    parts = [np.load(tmp_path / f"rank{r}.npz") for r in range(world)]
    rho = np.concatenate([p["rho"] for p in parts], axis=0)
    u = np.concatenate([p["u"] for p in parts], axis=1)
    c = case("drag_channel")
    ref = oracle_lattice(c)
    ref.set_populations(c["f0"])
    ref.step(n_steps)
    rho_ref, u_ref = ref.rho_u()
    assert np.array_equal(rho, rho_ref) and np.array_equal(u, u_ref)
    # the all-reduced FP64 sums: the same on both ranks, those of the whole lattice
    assert np.array_equal(parts[0]["cons"], parts[1]["cons"])
    np.testing.assert_allclose(parts[0]["cons"], ref.conservation(), rtol=1e-13, atol=1e-13)
