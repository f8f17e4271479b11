"""The allocation-free conservation entry point, called through the C ABI.

``lbm_conservation_noalloc`` is for callers that cannot call cudaMalloc at the
point where they want the FP64 mass / momentum sums -- for instance code
running inside another framework whose caching allocator already holds the
GPU's memory, or a monitoring hook in a step loop that must not be stalled by
an allocation.  It keeps its scratch in one fixed device array per GPU.  Its
output must equal ``lbm_conservation`` of a lattice holding the same
populations, call after call (the array keeps the previous call's contents,
so the second call checks that nothing stale leaks into the result).
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest
import torch
from gpu_cases import random_state

from lattice_boltzmann_d3q19_b200 import Lattice
from lattice_boltzmann_d3q19_b200 import _native as N

pytestmark = pytest.mark.gpu


def _noalloc(f_dev, flags_dev, shape, out_dev) -> int:
    flags_ptr = None if flags_dev is None else C.c_void_p(flags_dev.data_ptr())
    return N.lib().lbm_conservation_noalloc(C.c_void_p(f_dev.data_ptr()), flags_ptr, *shape,
                                            C.c_void_p(out_dev.data_ptr()), None)


@pytest.mark.parametrize("with_flags", [False, True])
def test_noalloc_matches_lattice_conservation_on_consecutive_calls(with_flags):
    shapes = [(24, 20, 18), (9, 7, 5)]
    for i, shape in enumerate(shapes):
        f = random_state(shape, 31 + i)
        flags = None
        if with_flags:
            flags = np.zeros(shape, dtype=np.uint8)
            flags[3:7, 2:6, 1:4] = 1
            flags[0] = 2
        with Lattice(shape, 0.7) as lat:
            if flags is not None:
                lat.set_flags(flags)
            lat.set_populations(f)
            expected = lat.conservation()
        f_dev = torch.from_numpy(f).cuda()
        flags_dev = None if flags is None else torch.from_numpy(flags).cuda()
        out = torch.empty(4, dtype=torch.float64, device="cuda")
        for _ in range(2):
            out.fill_(float("nan"))
            assert _noalloc(f_dev, flags_dev, shape, out) == N.LBM_OK, N.lib().lbm_last_error()
            torch.cuda.synchronize()
            got = out.cpu().numpy()
            # same 128-cell blocks and reduction order as a default lattice
            assert got.tobytes() == np.asarray(expected, np.float64).tobytes(), (got, expected)


def test_noalloc_rejects_host_pointers():
    shape = (6, 5, 4)
    f_host = random_state(shape, 3)
    out = torch.empty(4, dtype=torch.float64, device="cuda")
    rc = N.lib().lbm_conservation_noalloc(C.c_void_p(f_host.ctypes.data), None, *shape,
                                          C.c_void_p(out.data_ptr()), None)
    assert rc == N.LBM_ERR_INVALID
    assert b"device memory" in N.lib().lbm_last_error() or b"CUDA pointer" in N.lib().lbm_last_error()


def test_noalloc_rejects_lattices_beyond_its_fixed_scratch():
    f_dev = torch.zeros(19, dtype=torch.float64, device="cuda")
    out = torch.zeros(4, dtype=torch.float64, device="cuda")
    too_big = (256, 256, 257)
    assert np.prod(too_big) > 16777216  # LBM_NOALLOC_MAX_CELLS
    rc = N.lib().lbm_conservation_noalloc(C.c_void_p(f_dev.data_ptr()), None, *too_big,
                                          C.c_void_p(out.data_ptr()), None)
    assert rc == N.LBM_ERR_INVALID
    assert b"limit" in N.lib().lbm_last_error()
    torch.cuda.synchronize()
    assert torch.all(out == 0)
