"""The Poisson entry point that allocates nothing (paratc_poisson_noalloc).

Some callers of this library cannot call cudaMalloc -- for instance a host
code whose own allocator owns all device memory, or a time loop that must not
allocate.  paratc_poisson_noalloc() serves them by taking its working memory
from a fixed array built into the library.  These tests call it through the C
ABI twice in a row on each grid (the fixed array keeps the previous call's
contents) and check each result against the context-based
paratc_poisson_device() on the same input, within the 1e-12 Poisson
tolerance of the other parity tests.  The grids reach the limits the entry
point enforces: the largest nyc (256, with the factors 3 and 5 in nxc/2 and
nzc), the largest nxc (1024, the longest stack twiddle tables) and a grid
that nearly fills the fixed array (960 x 40 x 48: 1.85 M of its 2.1 M
doubles).  One odd-radix grid is also checked against the oracle directly.
It lives in a file of its own, collected last, and passes both alone in a
fresh process and after the rest of the suite.
"""
import ctypes

import numpy as np
import pytest

from oracle import oracle_lib as ol
from paratc_b200 import abi, cases, lib

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _yp(case):
    return lib.mesh_ycoord(case.mesh, case.params.yly)


def _noalloc(p, yp, src, phi, stream=None):
    L = lib.load()
    return L.paratc_poisson_noalloc(ctypes.byref(p), yp.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                    ctypes.c_void_p(src.data_ptr()), ctypes.c_void_p(phi.data_ptr()),
                                    None if stream is None else ctypes.c_void_p(stream))


def _source(shape, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    s = rng.standard_normal(shape)
    return s - s.mean()


@pytest.mark.parametrize("dims", [(64, 48, 40), (48, 256, 60), (1024, 8, 32), (960, 40, 48)])
def test_noalloc_poisson_matches_context_solve_twice(dims):
    import torch

    case = cases.small_channel(*dims)
    p = case.params
    yp = _yp(case)
    ref = lib.ChannelSystem(p, yp)
    shape = (p.nzc, p.nyc, p.nxc)
    for seed in (5, 6):
        src = torch.from_numpy(_source(shape, seed)).cuda()
        phi_ref = torch.empty_like(src)
        phi = torch.full_like(src, float("nan"))
        torch.cuda.synchronize()
        ref.poisson_device(src.data_ptr(), phi_ref.data_ptr())
        assert _noalloc(p, yp, src, phi) == abi.PARATC_OK
        a, b = phi.cpu().numpy(), phi_ref.cpu().numpy()
        err = np.abs(a - b).max() / np.abs(b).max()
        assert err <= TOL, (dims, seed, err)
    ref.close()


def test_noalloc_poisson_matches_oracle_odd_radix():
    """nxc/2 = 24 = 2^3 3 and nzc = 60 = 2^2 3 5, against the oracle's solve."""
    import torch

    case = cases.small_channel(48, 36, 60)
    p = case.params
    yp = _yp(case)
    o = ol.Oracle(p, yp)
    shape = (p.nzc, p.nyc, p.nxc)
    for seed in (8, 9):
        src_h = _source(shape, seed)
        src = torch.from_numpy(src_h).cuda()
        phi = torch.full_like(src, float("nan"))
        assert _noalloc(p, yp, src, phi) == abi.PARATC_OK
        ref = o.poisson(src_h)
        err = np.abs(phi.cpu().numpy() - ref).max() / np.abs(ref).max()
        assert err <= TOL, (seed, err)
    o.close()


def test_noalloc_poisson_rejects_grids_beyond_its_array():
    import torch

    case = cases.small_channel(256, 128, 256)  # 2*129*128*256 doubles > the fixed array
    p = case.params
    yp = _yp(case)
    dummy = torch.empty(8, dtype=torch.float64, device="cuda")
    assert _noalloc(p, yp, dummy, dummy) == abi.PARATC_ERR_BAD_ARG


def test_noalloc_poisson_refuses_stream_capture():
    """During stream capture it returns PARATC_ERR_BAD_ARG and enqueues
    nothing, so the capture itself stays valid."""
    import torch

    case = cases.small_channel(32, 24, 16)
    p = case.params
    yp = _yp(case)
    src = torch.from_numpy(_source((p.nzc, p.nyc, p.nxc), 4)).cuda()
    phi = torch.zeros_like(src)
    x = torch.zeros(4, device="cuda")
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    torch.cuda.synchronize()
    with torch.cuda.graph(g, stream=s):
        x.add_(1.0)
        rc = _noalloc(p, yp, src, phi, s.cuda_stream)
    assert rc == abi.PARATC_ERR_BAD_ARG
    g.replay()
    torch.cuda.synchronize()
    assert float(x[0]) == 1.0
    # outside capture the same call works
    assert _noalloc(p, yp, src, phi) == abi.PARATC_OK
