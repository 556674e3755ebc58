"""Host side of the z-slab Poisson solve over several GPUs (paratc_slab_*).

The reference's clcPPE_x1 (src/m_Poisson.f90:352-452) solves on 2-D pencils
and moves the array through six MPI_ALLTOALLW transposes per solve
(src/m_Decomp2d.f90:585-1000).  Here rank r of G holds the planes
kc in [k0_r, k0_r + nzl_r) of the source and of phi; the library transforms
them along x and packs the spectrum by destination (paratc_slab_forward), one
all-to-all gives every rank all planes of its modes kx in [kx0_r, kx0_r +
nxl_r) (the x-slab), the library does the z transforms and the y-Thomas solve
there (paratc_slab_middle), a second all-to-all returns the planes, and the
library unpacks them and transforms back (paratc_slab_backward).

The exchanges belong to the caller.  `nccl_exchange` does them with
torch.distributed.all_to_all_single (NCCL between GPUs, gloo on CPU
tensors); `LocalExchange` runs several ranks' plans in one process on one
device and moves the blocks with device copies.  Sizes are in doubles
(complex values as (re, im) pairs).

The peer form needs no collective library: every plan owns its x-slab, the
other ranks map it (CUDA IPC), and the library's scatter kernel stores each
value of the local spectrum straight into its owner's x-slab over NVLink
(the gather loads it back).  `PeerExchange` does the IPC mapping through
torch.distributed and orders the ranks with a stream synchronisation and a
barrier at the three points where one rank's kernels read or overwrite
another's x-slab; `LocalPeers` runs several plans in one process on one
stream, where stream order is enough.
"""
import ctypes

import numpy as np

from .abi import PARATC_OK
from .lib import ParatcError, load


def split(n, g, r):
    """(start, count) of rank r in the balanced split of n items over g ranks;
    the first n % g ranks get one item more (paratc_slab_partition)."""
    base, rem = divmod(n, g)
    return r * base + min(r, rem), base + (1 if r < rem else 0)


def partition_c(n, g, r):
    """paratc_slab_partition through the C ABI (needs no device)."""
    L = load()
    s, c = ctypes.c_int32(), ctypes.c_int32()
    rc = L.paratc_slab_partition(int(n), int(g), int(r), ctypes.byref(s), ctypes.byref(c))
    if rc != PARATC_OK:
        raise ParatcError(rc, "paratc_slab_partition(%d, %d, %d)" % (n, g, r))
    return s.value, c.value


def slab_counts(nx, ny, nz, g, r):
    """Per-peer double counts of rank r's forward exchange: (send, recv).
    The backward exchange sends `recv` and receives `send`."""
    m1 = nx // 2 + 1
    _, nzl = split(nz, g, r)
    _, nxl = split(m1, g, r)
    send = [2 * nzl * ny * split(m1, g, q)[1] for q in range(g)]
    recv = [2 * split(nz, g, q)[1] * ny * nxl for q in range(g)]
    return send, recv


def pack_offsets(nzl, ny, m1, g):
    """Where the forward pack puts each complex value of the local planes'
    spectrum [kl][jc][kx] in the send buffer (complex index), as k_slab_pack
    does: peer q's block [kl][jc][kx - kx0_q] at nzl*ny*kx0_q."""
    kx = np.arange(m1)
    owner = np.empty(m1, dtype=np.int64)
    for q in range(g):
        s, c = split(m1, g, q)
        owner[s:s + c] = q
    kx0 = np.array([split(m1, g, q)[0] for q in owner])
    nxl = np.array([split(m1, g, q)[1] for q in owner])
    row = np.arange(nzl * ny)[:, None]
    return (nzl * ny * kx0[None, :] + row * nxl[None, :] + (kx - kx0)[None, :]).reshape(-1)


def nccl_exchange(group=None):
    """An exchange through torch.distributed.all_to_all_single; send and recv
    are 1-D float64 tensors on this rank's device (or CPU under gloo)."""
    import torch.distributed as dist

    def exchange(send, recv, send_counts, recv_counts):
        dist.all_to_all_single(recv, send, output_split_sizes=[int(c) for c in recv_counts],
                               input_split_sizes=[int(c) for c in send_counts], group=group)
    return exchange


class SlabPoisson:
    """One rank's plan of the z-slab solve (paratc_slab_create)."""

    def __init__(self, params, yp, rank, nranks, device=0):
        self._L = load()
        self.nx, self.ny, self.nz = int(params.nxc), int(params.nyc), int(params.nzc)
        self.rank, self.nranks = int(rank), int(nranks)
        self.m1 = self.nx // 2 + 1
        self.k0, self.nzl = split(self.nz, nranks, rank)
        self.kx0, self.nxl = split(self.m1, nranks, rank)
        yp = np.ascontiguousarray(yp, dtype=np.float64)
        h = ctypes.c_void_p()
        rc = self._L.paratc_slab_create(ctypes.byref(params), yp.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                        int(device), self.rank, self.nranks, ctypes.byref(h))
        if rc != PARATC_OK:
            raise ParatcError(rc, "paratc_slab_create(rank %d of %d)" % (rank, nranks))
        self._h = h
        s = (ctypes.c_int64 * nranks)()
        r = (ctypes.c_int64 * nranks)()
        self._check(self._L.paratc_slab_counts(h, s, r), "paratc_slab_counts")
        self.send_counts = list(s)
        self.recv_counts = list(r)
        self.send_len = 2 * self.nzl * self.ny * self.m1   # doubles of the send / recv buffer
        self.xslab_len = 2 * self.nz * self.ny * self.nxl  # doubles of the x-slab

    def _check(self, rc, what):
        if rc != PARATC_OK:
            raise ParatcError(rc, what)

    @staticmethod
    def _ptr(t):
        return ctypes.c_void_p(t.data_ptr())

    @staticmethod
    def _stream(stream):
        return ctypes.c_void_p(0 if stream is None else int(stream))

    def forward(self, src, send, stream=None):
        self._check(self._L.paratc_slab_forward(self._h, self._ptr(src), self._ptr(send), self._stream(stream)),
                    "paratc_slab_forward")

    def middle(self, xslab, stream=None):
        self._check(self._L.paratc_slab_middle(self._h, self._ptr(xslab), self._stream(stream)), "paratc_slab_middle")

    def backward(self, recv, phi, stream=None):
        self._check(self._L.paratc_slab_backward(self._h, self._ptr(recv), self._ptr(phi), self._stream(stream)),
                    "paratc_slab_backward")

    @property
    def xslab_ptr(self):
        """Device address of the plan's own x-slab (the peer form)."""
        return int(self._L.paratc_slab_xslab(self._h))

    @staticmethod
    def _table(ptrs):
        return (ctypes.c_void_p * len(ptrs))(*[ctypes.c_void_p(int(p)) for p in ptrs])

    def forward_peers(self, src, xslab_ptrs, stream=None):
        self._check(self._L.paratc_slab_forward_peers(self._h, self._ptr(src), self._table(xslab_ptrs),
                                                      self._stream(stream)), "paratc_slab_forward_peers")

    def backward_peers(self, xslab_ptrs, phi, stream=None):
        self._check(self._L.paratc_slab_backward_peers(self._h, self._table(xslab_ptrs), self._ptr(phi),
                                                       self._stream(stream)), "paratc_slab_backward_peers")

    def middle_own(self, stream=None):
        self._check(self._L.paratc_slab_middle(self._h, ctypes.c_void_p(self.xslab_ptr), self._stream(stream)),
                    "paratc_slab_middle")

    def sync(self, stream=None):
        """Waits for the stream; raises if a bounded wait of the plan's
        bulk-copy-fed transforms ran out (PARATC_ERR_TIMEOUT)."""
        self._check(self._L.paratc_slab_sync(self._h, self._stream(stream)), "paratc_slab_sync")

    def buffers(self, torch, device):
        """(send/recv buffer, x-slab) as float64 device tensors."""
        return (torch.empty(self.send_len, dtype=torch.float64, device=device),
                torch.empty(self.xslab_len, dtype=torch.float64, device=device))

    def solve(self, src, phi, exchange, send, xslab, stream=None):
        """phi of this rank's planes from src of its planes (nzl*nyc*nxc
        doubles each, interior layout); `exchange(send, recv, send_counts,
        recv_counts)` moves the blocks between ranks."""
        self.forward(src, send, stream)
        exchange(send, xslab, self.send_counts, self.recv_counts)
        self.middle(xslab, stream)
        exchange(xslab, send, self.recv_counts, self.send_counts)
        self.backward(send, phi, stream)

    def close(self):
        if getattr(self, "_h", None):
            self._L.paratc_slab_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class LocalExchange:
    """All ranks' plans in one process on one device: the all-to-all of
    rank-ordered blocks done with device copies."""

    @staticmethod
    def all_to_all(sends, recvs, send_counts, recv_counts):
        g = len(sends)
        for r in range(g):
            so = np.concatenate([[0], np.cumsum(send_counts[r])])
            for q in range(g):
                ro = np.concatenate([[0], np.cumsum(recv_counts[q])])
                n = int(send_counts[r][q])
                if n != int(recv_counts[q][r]):
                    raise ValueError("block %d -> %d: %d doubles sent, %d expected" % (r, q, n, recv_counts[q][r]))
                recvs[q][int(ro[r]):int(ro[r]) + n].copy_(sends[r][int(so[q]):int(so[q]) + n])

    @staticmethod
    def solve(plans, srcs, phis, sends, xslabs):
        """Every rank's solve, stage by stage, on the current stream."""
        for p, s, b in zip(plans, srcs, sends):
            p.forward(s, b)
        LocalExchange.all_to_all(sends, xslabs, [p.send_counts for p in plans], [p.recv_counts for p in plans])
        for p, x in zip(plans, xslabs):
            p.middle(x)
        LocalExchange.all_to_all(xslabs, sends, [p.recv_counts for p in plans], [p.send_counts for p in plans])
        for p, b, f in zip(plans, sends, phis):
            p.backward(b, f)


class LocalPeers:
    """The peer form with all ranks' plans in one process on one device:
    the x-slab table is the plans' own x-slabs, stream order keeps the
    stages apart."""

    @staticmethod
    def solve(plans, srcs, phis, stream=None):
        ptrs = [p.xslab_ptr for p in plans]
        for p, s in zip(plans, srcs):
            p.forward_peers(s, ptrs, stream)
        for p in plans:
            p.middle_own(stream)
        for p, f in zip(plans, phis):
            p.backward_peers(ptrs, f, stream)


class PeerExchange:
    """The peer form across processes (one rank per GPU): maps every other
    rank's x-slab through CUDA IPC (handles exchanged with
    torch.distributed.all_gather_object) and runs a solve with a stream
    synchronisation and a barrier where the ranks must wait for one another."""

    def __init__(self, plan, dist, stream=None, ipc=None):
        """ipc: (get_handle(ptr) -> bytes, open(bytes) -> ptr, close(ptr)),
        the library's CUDA IPC calls by default."""
        if dist.get_world_size() != plan.nranks or dist.get_rank() != plan.rank:
            raise ValueError("plan of rank %d of %d in a process group of rank %d of %d"
                             % (plan.rank, plan.nranks, dist.get_rank(), dist.get_world_size()))
        self.plan, self.dist, self.stream = plan, dist, stream
        self._ipc = ipc or (ipc_get_handle, ipc_open, ipc_close)
        own = plan.xslab_ptr
        handles = [None] * plan.nranks
        dist.all_gather_object(handles, self._ipc[0](own))
        self.ptrs, self._opened = [], []
        for q, hq in enumerate(handles):
            if q == plan.rank:
                self.ptrs.append(own)
                continue
            ptr = self._ipc[1](hq)
            self.ptrs.append(ptr)
            self._opened.append(ptr)

    def _wait_all(self):
        self.plan.sync(self.stream)
        self.dist.barrier()

    def solve(self, src, phi):
        self.plan.forward_peers(src, self.ptrs, self.stream)
        self._wait_all()       # every rank's values are in every x-slab
        self.plan.middle_own(self.stream)
        self._wait_all()       # every x-slab solved
        self.plan.backward_peers(self.ptrs, phi, self.stream)
        self._wait_all()       # every rank has read its planes back

    def close(self):
        """Unmaps the other ranks' x-slabs, then waits for every rank to do
        the same, so that a plan may free its x-slab once this returns."""
        for p in self._opened:
            self._ipc[2](p)
        self._opened = []
        self.dist.barrier()


def ipc_get_handle(ptr):
    """The CUDA IPC handle (bytes) of the device allocation at ptr."""
    h = (ctypes.c_char * 64)()
    rc = load().paratc_ipc_get_handle(ctypes.c_void_p(int(ptr)), h)
    if rc != PARATC_OK:
        raise ParatcError(rc, "paratc_ipc_get_handle")
    return bytes(h)


def ipc_open(handle):
    """Maps another process's allocation; returns its device address here."""
    buf = (ctypes.c_char * 64).from_buffer_copy(handle)
    p = ctypes.c_void_p()
    rc = load().paratc_ipc_open(buf, ctypes.byref(p))
    if rc != PARATC_OK:
        raise ParatcError(rc, "paratc_ipc_open")
    return int(p.value)


def ipc_close(ptr):
    load().paratc_ipc_close(ctypes.c_void_p(int(ptr)))

