"""x-slab decomposition of one lattice over several engines.

x is the slowest axis of the population arrays, so a slab of x-planes is
contiguous per direction.  Slab r owns the global planes [x0, x1) and holds
them in a local lattice of x1 - x0 + 2 planes, periodic in x: local plane 0
and local plane x1 - x0 + 1 are halo planes.  Before every step that pulls
(every step after the first one from a set state), and before a readback,
each slab exchanges one plane per face: the 5 directions with c_x = +1 of its
last owned plane go to the right neighbour's left halo, the 5 with c_x = -1 of
its first owned plane to the left neighbour's right halo -- exactly the
post-collision populations the neighbour's boundary plane pulls.  The halo
planes' own updates are discarded (overwritten by the next exchange); flags,
porosity and force fields carry the neighbours' planes so that bounce-back
masks and forces across a face are those of the global lattice.

Engines with plane-range steps (step_planes / step_commit) take a step in
three parts, so that the exchange overlaps the bulk of the update: the two
boundary planes are exported, the interior planes [2, width) -- which pull
from owned planes only -- are advanced while the faces travel, and the
imported halos are followed by the two boundary planes.  The halo planes
are not advanced at all.

Requirements: x periodic globally (inflow / outflow cells are flags and are
fine), every slab at least 3 planes, and no outflow cell on a slab's first
owned plane (an outflow cell copies the state of x - 1, which a slab holds
only from its second plane on).  No counterpart in the reference (it runs on
one device).
"""

from __future__ import annotations

import numpy as np

PLUS_X = (1, 7, 9, 11, 13)     # c_x = +1: pulled across a slab's left face
MINUS_X = (2, 8, 10, 12, 14)   # c_x = -1: pulled across its right face
MASK_PLUS = sum(1 << d for d in PLUS_X)
MASK_MINUS = sum(1 << d for d in MINUS_X)
CELL_OUTFLOW = 3


def slab_bounds(nx: int, parts: int) -> list[tuple[int, int]]:
    """Contiguous split of [0, nx) into `parts` slabs as even as possible."""
    if parts < 1 or nx < 3 * parts:
        raise ValueError(f"cannot split {nx} x-planes into {parts} slabs of at least 3 planes")
    base, rem = divmod(nx, parts)
    out, x = [], 0
    for r in range(parts):
        w = base + (1 if r < rem else 0)
        out.append((x, x + w))
        x += w
    return out


def with_halos(field, x0: int, x1: int, nx: int, axis: int = 0):
    """Global planes x0 - 1 .. x1 (periodic wrap in x) of a field whose axis
    `axis` is x."""
    idx = np.arange(x0 - 1, x1 + 1) % nx
    return np.take(np.asarray(field), idx, axis=axis)


class SlabLattice:
    """One slab.  `engine` is the local lattice (local shape (x1 - x0 + 2, ny,
    nz), periodic in x) wrapped by an adapter with plane_get(x, mask) ->
    buffer, plane_put(x, mask, buffer), step(n), set_populations(f),
    get_populations(), rho_u(), conservation_planes(x0, x1)."""

    def __init__(self, engine, x0: int, x1: int, flags=None, nx: int | None = None):
        self.engine = engine
        self.x0, self.x1 = int(x0), int(x1)
        self.width = self.x1 - self.x0
        if self.width < 3:
            raise ValueError("a slab needs at least 3 planes")
        if flags is not None and nx is not None:
            first = np.asarray(flags)[self.x0 % nx] & 3
            if np.any(first == CELL_OUTFLOW):
                raise ValueError(f"outflow cells on the first plane (x = {self.x0}) of a slab")
        self.stepped = False

    # faces -------------------------------------------------------------------
    def export_faces(self):
        """(to the left neighbour, to the right neighbour) buffers."""
        return (self.engine.plane_get(1, MASK_MINUS, slot=0), self.engine.plane_get(self.width, MASK_PLUS, slot=1))

    @property
    def split(self) -> bool:
        """The engine takes plane-range steps (the overlapped step)."""
        return hasattr(self.engine, "step_planes")

    def step_interior(self) -> None:
        """Overlapped step, part 1 (after export_faces): the planes that pull
        from owned planes only."""
        self.engine.step_planes(2, self.width)

    def step_boundary(self) -> None:
        """Overlapped step, part 2 (after import_faces): the two boundary
        planes, then the step is committed."""
        self.engine.step_planes(1, 2)
        self.engine.step_planes(self.width, self.width + 1)
        self.engine.step_commit()

    def import_faces(self, from_left, from_right) -> None:
        self.engine.plane_put(0, MASK_PLUS, from_left)
        self.engine.plane_put(self.width + 1, MASK_MINUS, from_right)

    # state ---------------------------------------------------------------------
    def set_populations(self, f_global) -> None:
        """Set from the global populations (19, nx, ny, nz)."""
        f = np.asarray(f_global)
        self.engine.set_populations(with_halos(f, self.x0, self.x1, f.shape[1], axis=1))
        self.stepped = False

    def owned(self, a, axis: int = 0):
        sl = [slice(None)] * np.ndim(a)
        sl[axis] = slice(1, self.width + 1)
        return a[tuple(sl)]


class SlabGroup:
    """Slabs of one lattice in one process (one device or several): the
    exchange is a direct copy between the slabs' engines.  overlap: take the
    overlapped step where every engine has plane-range steps."""

    def __init__(self, slabs: list[SlabLattice], overlap: bool = True):
        self.slabs = slabs
        self.overlap = overlap

    def exchange(self) -> None:
        faces = [s.export_faces() for s in self.slabs]
        k = len(self.slabs)
        for r, s in enumerate(self.slabs):
            s.import_faces(faces[(r - 1) % k][1], faces[(r + 1) % k][0])

    def step(self, n_steps: int = 1) -> None:
        for _ in range(int(n_steps)):
            if self.slabs[0].stepped and self.overlap and all(s.split for s in self.slabs):
                faces = [s.export_faces() for s in self.slabs]
                for s in self.slabs:
                    s.step_interior()
                k = len(self.slabs)
                for r, s in enumerate(self.slabs):
                    s.import_faces(faces[(r - 1) % k][1], faces[(r + 1) % k][0])
                for s in self.slabs:
                    s.step_boundary()
                continue
            if self.slabs[0].stepped:
                self.exchange()
            for s in self.slabs:
                s.engine.step(1)
                s.stepped = True

    def _fresh(self) -> None:
        if self.slabs[0].stepped:
            self.exchange()

    def rho_u(self):
        self._fresh()
        parts = [s.engine.rho_u() for s in self.slabs]
        rho = np.concatenate([s.owned(p[0], 0) for s, p in zip(self.slabs, parts, strict=True)], axis=0)
        u = np.concatenate([s.owned(p[1], 1) for s, p in zip(self.slabs, parts, strict=True)], axis=1)
        return rho, u

    def get_populations(self):
        self._fresh()
        return np.concatenate([s.owned(s.engine.get_populations(), 1) for s in self.slabs], axis=1)

    def conservation(self):
        self._fresh()
        return np.sum([s.engine.conservation_planes(1, s.width + 1) for s in self.slabs], axis=0)


def _recv_buffers(slab: SlabLattice, ls, rs):
    """Receive buffers of the exchange: the engine's own (preallocated) ones
    where it has them."""
    import torch

    bufs = getattr(slab.engine, "recv", None)
    if bufs is not None:
        return bufs
    return torch.empty_like(rs), torch.empty_like(ls)


def _send_recv(rank: int, world: int, ls, rs, lr, rr) -> None:
    """rs to the right neighbour, ls to the left one; lr from the left, rr
    from the right (torch.distributed point-to-point operations)."""
    import torch.distributed as dist

    right, left = (rank + 1) % world, (rank - 1) % world
    ops = [dist.P2POp(dist.isend, rs, right), dist.P2POp(dist.irecv, lr, left),
           dist.P2POp(dist.isend, ls, left), dist.P2POp(dist.irecv, rr, right)]
    for req in dist.batch_isend_irecv(ops):
        req.wait()


def exchange_distributed(slab: SlabLattice, rank: int, world: int, to_tensor=None, from_tensor=None) -> None:
    """The face exchange of one slab per rank with torch.distributed point-to-
    point operations (NCCL for device tensors, gloo for host tensors); world 1
    exchanges with itself (periodic x).  to_tensor / from_tensor convert the
    engine's buffers (identity for torch tensors)."""
    to_t = to_tensor or (lambda b: b)
    from_t = from_tensor or (lambda t, like: t)
    left_send, right_send = slab.export_faces()
    ls, rs = to_t(left_send), to_t(right_send)
    if world == 1:
        slab.import_faces(right_send, left_send)
        return
    lr, rr = _recv_buffers(slab, ls, rs)
    _send_recv(rank, world, ls, rs, lr, rr)
    slab.import_faces(from_t(lr, left_send), from_t(rr, right_send))


def step_distributed(slab: SlabLattice, rank: int, world: int, comm_stream=None, to_tensor=None,
                     from_tensor=None) -> None:
    """One step of one slab per rank.  The first step from a set state is a
    whole-slab step (nothing to pull); after it, an engine with plane-range
    steps takes the overlapped step: export the faces, advance the interior
    while the faces travel, import the halos, advance the boundary planes.
    With device buffers the point-to-point operations run on comm_stream
    (ordered after the export by an event, and the boundary planes after
    them); the interior kernel runs on the engine's (current) stream meanwhile.
    An engine without plane-range steps exchanges, then steps the whole slab."""
    if not slab.stepped:
        slab.engine.step(1)
        slab.stepped = True
        return
    if not slab.split:
        exchange_distributed(slab, rank, world, to_tensor, from_tensor)
        slab.engine.step(1)
        return
    to_t = to_tensor or (lambda b: b)
    from_t = from_tensor or (lambda t, like: t)
    left_send, right_send = slab.export_faces()
    if world == 1:
        slab.step_interior()
        slab.import_faces(right_send, left_send)
        slab.step_boundary()
        return
    ls, rs = to_t(left_send), to_t(right_send)
    lr, rr = _recv_buffers(slab, ls, rs)
    if comm_stream is not None and getattr(ls, "is_cuda", False):
        import torch

        main = torch.cuda.current_stream()
        exported = torch.cuda.Event()
        exported.record(main)
        with torch.cuda.stream(comm_stream):
            comm_stream.wait_event(exported)
            _send_recv(rank, world, ls, rs, lr, rr)
        slab.step_interior()
        main.wait_stream(comm_stream)
    else:
        _send_recv(rank, world, ls, rs, lr, rr)
        slab.step_interior()
    slab.import_faces(from_t(lr, left_send), from_t(rr, right_send))
    slab.step_boundary()


def conservation_distributed(slab: SlabLattice, rank: int, world: int, to_tensor=None,
                             from_tensor=None) -> np.ndarray:
    """FP64 {mass, momentum x, y, z} of the whole lattice: each rank's sums
    over its owned planes (after a face exchange, which the readback of a
    boundary plane pulls from; to_tensor / from_tensor as for
    exchange_distributed), added by an all-reduce of 4 doubles (NCCL on the
    engine's device for a GpuEngine, gloo on the host otherwise)."""
    import torch
    import torch.distributed as dist

    if slab.stepped:
        exchange_distributed(slab, rank, world, to_tensor, from_tensor)
    local = np.asarray(slab.engine.conservation_planes(1, slab.width + 1), dtype=np.float64)
    if world == 1:
        return local
    like = getattr(slab.engine, "send", (None,))[0]
    dev = like.device if like is not None and getattr(like, "is_cuda", False) else torch.device("cpu")
    t = torch.tensor(local, dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return t.cpu().numpy()


class GpuEngine:
    """Adapter of a Lattice (local slab shape) to the SlabLattice engine
    interface: plane buffers are torch device tensors, allocated once (two
    send and two receive buffers of one face each), filled and read on the
    lattice's stream (the caller's current torch stream)."""

    _ELEM = {"f64": 8, "f32": 4, "f16": 2, "bf16": 2}

    def __init__(self, lattice, storage: str):
        import torch

        self.lat = lattice
        self.torch = torch
        nx, ny, nz = lattice.shape
        self.count = 5 * ny * nz * self._ELEM[storage]
        dev = torch.device("cuda", int(lattice.desc.device))
        self.send = tuple(torch.empty(self.count, dtype=torch.uint8, device=dev) for _ in range(2))
        self.recv = tuple(torch.empty(self.count, dtype=torch.uint8, device=dev) for _ in range(2))

    def plane_get(self, x: int, mask: int, slot: int | None = None):
        buf = self.send[slot] if slot is not None else self.torch.empty(self.count, dtype=self.torch.uint8,
                                                                         device=self.send[0].device)
        self.lat.plane_get_device(x, mask, buf.data_ptr())
        return buf

    def plane_put(self, x: int, mask: int, buf) -> None:
        self.lat.plane_put_device(x, mask, buf.data_ptr())

    def step(self, n: int) -> None:
        self.lat.step(n)

    def step_planes(self, x0: int, x1: int) -> None:
        self.lat.step_planes(x0, x1)

    def step_commit(self) -> None:
        self.lat.step_commit()

    def set_populations(self, f) -> None:
        self.lat.set_populations(f)

    def get_populations(self):
        return self.lat.get_populations()

    def rho_u(self):
        return self.lat.rho_u()

    def conservation_planes(self, x0: int, x1: int):
        return self.lat.conservation_planes(x0, x1)


__all__ = ["GpuEngine", "MASK_MINUS", "MASK_PLUS", "MINUS_X", "PLUS_X", "SlabGroup", "SlabLattice",
           "conservation_distributed", "exchange_distributed", "slab_bounds", "step_distributed", "with_halos"]
