"""The z-slab Poisson decomposition's host logic on the CPU: the balanced
split against the library's paratc_slab_partition, the per-peer counts, the
pack map of the forward exchange, and the two all-to-all exchanges of a
solve run through the same exchange function the GPUs use (gloo ranks here,
NCCL on GPUs) on an index-tagged spectrum: after the first exchange every
rank must hold all planes of its modes, after the second its own planes.
The peer form's host side (IPC handle exchange, pointer table, the waits
between its stages) runs on gloo ranks with a fake plan."""
import json
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

from paratc_b200 import slabs

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_split_matches_library_partition():
    for n, g in [(40, 1), (40, 3), (65, 4), (7, 7), (129, 8), (257, 64)]:
        covered = []
        for r in range(g):
            s, c = slabs.split(n, g, r)
            assert slabs.partition_c(n, g, r) == (s, c)
            assert c in (n // g, n // g + 1)
            covered += list(range(s, s + c))
        assert covered == list(range(n))


def test_partition_rejects_more_ranks_than_items():
    from paratc_b200.lib import ParatcError
    with pytest.raises(ParatcError):
        slabs.partition_c(3, 4, 0)


@pytest.mark.parametrize("dims,g", [((64, 6, 40), 3), ((48, 5, 12), 4), ((16, 3, 8), 2)])
def test_counts_and_pack_map(dims, g):
    nx, ny, nz = dims
    m1 = nx // 2 + 1
    sends, recvs = zip(*(slabs.slab_counts(nx, ny, nz, g, r) for r in range(g)))
    for r in range(g):
        for q in range(g):
            assert sends[r][q] == recvs[q][r]       # what r sends q is what q expects from r
        _, nzl = slabs.split(nz, g, r)
        assert sum(sends[r]) == 2 * nzl * ny * m1   # the send buffer holds the local spectrum once
        _, nxl = slabs.split(m1, g, r)
        assert sum(recvs[r]) == 2 * nz * ny * nxl   # the x-slab holds all planes of the rank's modes
        off = slabs.pack_offsets(nzl, ny, m1, g)
        assert np.array_equal(np.sort(off), np.arange(nzl * ny * m1))  # a permutation
        # peer q's block is contiguous at 2*nzl*ny*kx0_q doubles
        kx = np.tile(np.arange(m1), nzl * ny)
        for q in range(g):
            s, c = slabs.split(m1, g, q)
            blk = off[(kx >= s) & (kx < s + c)]
            assert blk.min() == nzl * ny * s and blk.max() == nzl * ny * (s + c) - 1


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _tagged(nz, ny, m1):
    """A complex spectrum [kc][jc][kx] whose values name their indices."""
    k, j, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(m1), indexing="ij")
    return (k * 1000.0 + j) + 1j * x


def _worker(rank, ws, port, dims, out_dir):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(ws), "LOCAL_RANK": str(rank)})
    sys.path.insert(0, ROOT)
    import torch
    from paratc_b200 import replicas, slabs as sl
    dist = replicas.init("gloo", timeout_s=60)
    nx, ny, nz = dims
    m1 = nx // 2 + 1
    k0, nzl = sl.split(nz, ws, rank)
    kx0, nxl = sl.split(m1, ws, rank)
    send_c, recv_c = sl.slab_counts(nx, ny, nz, ws, rank)
    full = _tagged(nz, ny, m1)
    local = full[k0:k0 + nzl].reshape(-1)
    packed = np.empty_like(local)
    packed[sl.pack_offsets(nzl, ny, m1, ws)] = local
    send = torch.from_numpy(packed.view(np.float64).copy())
    xslab = torch.empty(sum(recv_c), dtype=torch.float64)
    ex = sl.nccl_exchange()
    ex(send, xslab, send_c, recv_c)
    got = xslab.numpy().view(np.complex128).reshape(nz, ny, nxl)
    ok1 = bool(np.array_equal(got, full[:, :, kx0:kx0 + nxl]))
    back = torch.empty_like(send)
    ex(xslab, back, recv_c, send_c)
    unpacked = back.numpy().view(np.complex128)[sl.pack_offsets(nzl, ny, m1, ws)]
    ok2 = bool(np.array_equal(unpacked, local))
    dist.barrier()
    dist.destroy_process_group()
    with open(os.path.join(out_dir, "rank%d.json" % rank), "w") as f:
        json.dump({"xslab": ok1, "planes": ok2}, f)


@pytest.mark.parametrize("ws,dims", [(2, (16, 4, 6)), (3, (20, 3, 7))])
def test_exchanges_over_gloo_ranks(tmp_path, ws, dims):
    mp.start_processes(_worker, args=(ws, _free_port(), dims, str(tmp_path)), nprocs=ws, join=True,
                       start_method="spawn")
    for r in range(ws):
        res = json.load(open(tmp_path / ("rank%d.json" % r)))
        assert res == {"xslab": True, "planes": True}, (r, res)


class _FakePlan:
    """Records the peer form's calls in order (no device)."""

    def __init__(self, rank, nranks, log):
        self.rank, self.nranks, self.log = rank, nranks, log
        self.xslab_ptr = 0x1000 * (rank + 1)

    def forward_peers(self, src, ptrs, stream):
        self.log.append(("forward", list(ptrs)))

    def middle_own(self, stream):
        self.log.append(("middle",))

    def backward_peers(self, ptrs, phi, stream):
        self.log.append(("backward", list(ptrs)))

    def sync(self, stream):
        self.log.append(("sync",))


def _peer_worker(rank, ws, port, out_dir):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(ws), "LOCAL_RANK": str(rank)})
    sys.path.insert(0, ROOT)
    from paratc_b200 import replicas, slabs as sl
    dist = replicas.init("gloo", timeout_s=60)
    log = []
    opened, closed = [], []
    ipc = (lambda ptr: b"H%08x" % ptr,                      # a handle names the owner's address
           lambda h: (opened.append(h), 0x900000 + int(h[1:], 16))[1],  # mapped at another address here
           lambda ptr: closed.append(ptr))
    plan = _FakePlan(rank, ws, log)
    pe = sl.PeerExchange(plan, dist, ipc=ipc)
    orig = dist.barrier
    dist.barrier = lambda *a, **k: (log.append(("barrier",)), orig())[1]
    pe.solve(None, None)
    dist.barrier = orig
    pe.close()
    dist.destroy_process_group()
    with open(os.path.join(out_dir, "peer%d.json" % rank), "w") as f:
        json.dump({"ptrs": pe.ptrs, "log": log, "opened": [h.decode() for h in opened], "closed": closed}, f)


def test_peer_exchange_over_gloo_ranks(tmp_path):
    """The peer form's host side on 3 gloo ranks with a fake plan and fake
    IPC: every rank's table holds its own x-slab at its own index and the
    others' mapped addresses, and each solve is scatter, wait, middle, wait,
    gather, wait (a stream synchronisation and a barrier at each wait)."""
    ws = 3
    mp.start_processes(_peer_worker, args=(ws, _free_port(), str(tmp_path)), nprocs=ws, join=True,
                       start_method="spawn")
    for r in range(ws):
        res = json.load(open(tmp_path / ("peer%d.json" % r)))
        want = [0x1000 * (q + 1) if q == r else 0x900000 + 0x1000 * (q + 1) for q in range(ws)]
        assert res["ptrs"] == want
        assert sorted(res["opened"]) == sorted("H%08x" % (0x1000 * (q + 1)) for q in range(ws) if q != r)
        assert sorted(res["closed"]) == sorted(p for q, p in enumerate(want) if q != r)
        kinds = [e[0] for e in res["log"]]
        assert kinds == ["forward", "sync", "barrier", "middle", "sync", "barrier", "backward", "sync", "barrier"]
        assert res["log"][0][1] == want and res["log"][6][1] == want


def test_local_exchange_moves_rank_ordered_blocks():
    """slabs.LocalExchange.all_to_all (the one-process exchange of the GPU
    tests) on CPU tensors: block r -> q lands at q's offset for r."""
    import torch
    nx, ny, nz, g = 20, 3, 7, 3
    counts = [slabs.slab_counts(nx, ny, nz, g, r) for r in range(g)]
    sends = [torch.arange(sum(c[0]), dtype=torch.float64) + 1000.0 * r for r, c in enumerate(counts)]
    recvs = [torch.full((sum(c[1]),), -1.0, dtype=torch.float64) for c in counts]
    slabs.LocalExchange.all_to_all(sends, recvs, [c[0] for c in counts], [c[1] for c in counts])
    for q in range(g):
        off = 0
        for r in range(g):
            n = counts[q][1][r]
            so = sum(counts[r][0][:q])
            assert torch.equal(recvs[q][off:off + n], sends[r][so:so + n])
            off += n
        assert off == recvs[q].numel()
