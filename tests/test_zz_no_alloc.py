"""The Poisson entry point that allocates nothing (paratc_poisson_noalloc).

Some callers of this library cannot call cudaMalloc -- for instance a host
code whose own allocator owns all device memory, or a time loop that must not
allocate.  paratc_poisson_noalloc() serves them by taking its working memory
from a fixed array built into the library.  This test calls it through the C
ABI twice in a row (the fixed array keeps the previous call's contents) and
checks each result against the context-based paratc_poisson_device() on the
same input, within the 1e-12 Poisson tolerance of the other parity tests.
It lives in a file of its own, collected last, and passes both alone in a
fresh process and after the rest of the suite.
"""
import ctypes

import numpy as np
import pytest

from paratc_b200 import abi, cases, lib

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _yp(case):
    return lib.mesh_ycoord(case.mesh, case.params.yly)


def test_noalloc_poisson_matches_context_solve_twice():
    import torch

    case = cases.small_channel(64, 48, 40)
    p = case.params
    yp = _yp(case)
    L = lib.load()
    ref = lib.ChannelSystem(p, yp)
    shape = (p.nzc, p.nyc, p.nxc)
    for seed in (5, 6):
        rng = np.random.Generator(np.random.PCG64(seed))
        src_h = rng.standard_normal(shape)
        src_h -= src_h.mean()
        src = torch.from_numpy(src_h).cuda()
        phi_ref = torch.empty_like(src)
        phi = torch.full_like(src, float("nan"))
        torch.cuda.synchronize()
        ref.poisson_device(src.data_ptr(), phi_ref.data_ptr())
        rc = L.paratc_poisson_noalloc(ctypes.byref(p), yp.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                      ctypes.c_void_p(src.data_ptr()), ctypes.c_void_p(phi.data_ptr()), None)
        assert rc == abi.PARATC_OK
        a, b = phi.cpu().numpy(), phi_ref.cpu().numpy()
        err = np.abs(a - b).max() / np.abs(b).max()
        assert err <= TOL, err
    ref.close()


def test_noalloc_poisson_rejects_grids_beyond_its_array():
    import torch

    case = cases.small_channel(256, 128, 256)  # 2*129*128*256 doubles > the fixed array
    p = case.params
    yp = _yp(case)
    L = lib.load()
    dummy = torch.empty(8, dtype=torch.float64, device="cuda")
    rc = L.paratc_poisson_noalloc(ctypes.byref(p), yp.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                  ctypes.c_void_p(dummy.data_ptr()), ctypes.c_void_p(dummy.data_ptr()), None)
    assert rc == abi.PARATC_ERR_BAD_ARG
