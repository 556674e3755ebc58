"""The z-slab Poisson solve (paratc_slab_*) on the GPU.

G ranks' plans run in one process on one device, their all-to-all
exchanges done by device copies (slabs.LocalExchange); each rank solves its
planes and the assembled phi must match the one-GPU solve
(paratc_poisson_device) of the whole grid and the oracle, within the 1e-12
Poisson tolerance of the other parity tests.  The splits include uneven
ones (nzc or nxc/2+1 not a multiple of G) and G = 1, where the exchanges
are plain copies."""
import numpy as np
import pytest

from oracle import oracle_lib as ol
from paratc_b200 import cases, lib, slabs

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _source(shape, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    s = rng.standard_normal(shape)
    return s - s.mean()


def _slab_solve(p, yp, src, g):
    """phi of the whole grid from G plans on cuda:0 (src: a device tensor
    [nzc][nyc][nxc])."""
    import torch

    plans = [slabs.SlabPoisson(p, yp, r, g, device=0) for r in range(g)]
    srcs, phis, sends, xslabs = [], [], [], []
    for pl in plans:
        srcs.append(src[pl.k0:pl.k0 + pl.nzl].contiguous().reshape(-1))
        phis.append(torch.full_like(srcs[-1], float("nan")))
        b, x = pl.buffers(torch, "cuda")
        sends.append(b)
        xslabs.append(x)
    slabs.LocalExchange.solve(plans, srcs, phis, sends, xslabs)
    torch.cuda.synchronize()
    for pl in plans:
        pl.sync()
    for pl in plans:
        assert (pl.send_counts, pl.recv_counts) == slabs.slab_counts(p.nxc, p.nyc, p.nzc, g, pl.rank)
    phi = torch.cat([f.reshape(pl.nzl, p.nyc, p.nxc) for pl, f in zip(plans, phis)], dim=0)
    for pl in plans:
        pl.close()
    return phi


@pytest.mark.parametrize("dims,g", [((64, 48, 40), 1), ((64, 48, 40), 2), ((64, 48, 40), 3), ((64, 48, 40), 4),
                                    ((128, 96, 128), 2), ((96, 20, 30), 7)])
def test_slab_solve_matches_one_gpu_solve(dims, g):
    import torch

    case = cases.small_channel(*dims)
    p = case.params
    yp = lib.mesh_ycoord(case.mesh, p.yly)
    ref = lib.ChannelSystem(p, yp)
    shape = (p.nzc, p.nyc, p.nxc)
    for seed in (3, 4):  # twice: the plans' buffers keep nothing between solves
        src = torch.from_numpy(_source(shape, seed)).cuda()
        phi_ref = torch.empty_like(src)
        torch.cuda.synchronize()
        ref.poisson_device(src.data_ptr(), phi_ref.data_ptr())
        phi = _slab_solve(p, yp, src, g)
        a, b = phi.cpu().numpy(), phi_ref.cpu().numpy()
        err = np.abs(a - b).max() / np.abs(b).max()
        assert err <= TOL, (dims, g, seed, err)
    ref.close()


def test_slab_solve_matches_oracle_uneven_odd_radix():
    """nxc/2 = 24 = 2^3 3, nzc = 60 = 2^2 3 5; 25 modes and 60 planes over 4
    ranks (7/6/6/6 modes)."""
    import torch

    case = cases.small_channel(48, 36, 60)
    p = case.params
    yp = lib.mesh_ycoord(case.mesh, p.yly)
    o = ol.Oracle(p, yp)
    src_h = _source((p.nzc, p.nyc, p.nxc), 11)
    phi = _slab_solve(p, yp, torch.from_numpy(src_h).cuda(), 4).cpu().numpy()
    ref = o.poisson(src_h)
    err = np.abs(phi - ref).max() / np.abs(ref).max()
    assert err <= TOL, err
    o.close()


def test_slab_create_rejects_bad_splits():
    case = cases.small_channel(16, 12, 8)
    p = case.params
    yp = lib.mesh_ycoord(case.mesh, p.yly)
    with pytest.raises(lib.ParatcError):
        slabs.SlabPoisson(p, yp, 0, 9)   # more ranks than planes (nzc = 8)
    with pytest.raises(lib.ParatcError):
        slabs.SlabPoisson(p, yp, 2, 2)   # rank outside [0, nranks)


_FRESH = r"""
import sys
sys.path.insert(0, %r)
import numpy as np, torch
from oracle import oracle_lib as ol
from paratc_b200 import cases, lib, slabs
case = cases.small_channel(128, 32, 128)
p = case.params
yp = lib.mesh_ycoord(case.mesh, p.yly)
plans = [slabs.SlabPoisson(p, yp, r, 2, device=0) for r in range(2)]  # before any context
rng = np.random.Generator(np.random.PCG64(21))
src = rng.standard_normal((p.nzc, p.nyc, p.nxc)); src -= src.mean()
d = torch.from_numpy(src).cuda()
srcs = [d[pl.k0:pl.k0 + pl.nzl].contiguous().reshape(-1) for pl in plans]
phis = [torch.empty_like(s) for s in srcs]
bufs = [pl.buffers(torch, "cuda") for pl in plans]
slabs.LocalExchange.solve(plans, srcs, phis, [b[0] for b in bufs], [b[1] for b in bufs])
for pl in plans:
    pl.sync()
phi = torch.cat(phis).reshape(p.nzc, p.nyc, p.nxc).cpu().numpy()
o = ol.Oracle(p, yp)
ref = o.poisson(src)
print("ERR", float(np.abs(phi - ref).max() / np.abs(ref).max()))
"""


def test_slab_plan_in_a_fresh_process():
    """A plan made before any context (the compiled-length x and z
    transforms, 128 x 32 x 128 over 2 ranks) in a process of its own."""
    import os
    import subprocess
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, "-c", _FRESH % root], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    err = float(out.stdout.split("ERR")[-1])
    assert err <= TOL, err


@pytest.mark.parametrize("dims,g", [((64, 48, 40), 1), ((64, 48, 40), 3), ((128, 96, 128), 4), ((96, 20, 30), 7)])
def test_slab_peer_form_matches_exchange_form(dims, g):
    """The peer form (scatter into every rank's x-slab, gather back) gives
    bitwise the all-to-all form's potential, and the one-GPU solve's to 1e-12."""
    import torch

    case = cases.small_channel(*dims)
    p = case.params
    yp = lib.mesh_ycoord(case.mesh, p.yly)
    src = torch.from_numpy(_source((p.nzc, p.nyc, p.nxc), 13)).cuda()
    phi_x = _slab_solve(p, yp, src, g).cpu().numpy()
    plans = [slabs.SlabPoisson(p, yp, r, g, device=0) for r in range(g)]
    srcs = [src[pl.k0:pl.k0 + pl.nzl].contiguous().reshape(-1) for pl in plans]
    for rep in range(2):  # twice: x-slabs and spectra are reused
        phis = [torch.full_like(s, float("nan")) for s in srcs]
        slabs.LocalPeers.solve(plans, srcs, phis)
        torch.cuda.synchronize()
        for pl in plans:
            pl.sync()
        phi = torch.cat(phis).reshape(p.nzc, p.nyc, p.nxc).cpu().numpy()
        assert np.array_equal(phi, phi_x), (dims, g, rep)
    ref = lib.ChannelSystem(p, yp)
    phi_ref = torch.empty_like(src)
    ref.poisson_device(src.data_ptr(), phi_ref.data_ptr())
    b = phi_ref.cpu().numpy()
    assert np.abs(phi_x - b).max() / np.abs(b).max() <= TOL
    ref.close()
    for pl in plans:
        pl.close()


def test_ipc_handle_of_a_plan_x_slab():
    """The handle the peer form sends to other processes is produced for the
    plan's own allocation (opening it needs another process)."""
    import ctypes

    case = cases.small_channel(16, 12, 8)
    p = case.params
    pl = slabs.SlabPoisson(p, lib.mesh_ycoord(case.mesh, p.yly), 0, 2, device=0)
    h = (ctypes.c_char * 64)()
    assert lib.load().paratc_ipc_get_handle(ctypes.c_void_p(pl.xslab_ptr), h) == 0
    assert any(bytes(h))
    pl.close()
