"""Host side of domain decomposition: what LAMMPS's Comm does for `fix metad`
when the job runs on several ranks, for callers that are not LAMMPS.

Each rank owns the atoms of one brick of the periodic box and receives, as
ghosts, every periodic image of an atom that lies within the ghost cutoff of
its brick (the reference's ghost atoms nlocal..nlocal+nghost,
src/cvs/CVs_Steinhardt.cu:595).  A rank's context (``Metad.set_domain``) then
treats its owned atoms as the centres of the CV sums and its ghosts as
neighbours only; the totals of all ranks are summed by an allreduce callback
(the reference's MPI_Allreduce, src/cvs/CVs_Steinhardt.cu:836), and the force
rows of ghosts are added back to their owners (LAMMPS reverse communication,
src/core/fix_crystallize.cu:510-520).

``decompose`` builds the per-rank atom sets, ``reverse_sum`` gathers forces
onto owners, ``LocalAllreduce`` sums over ranks that are host threads of one
process (one context per thread), ``TorchAllreduce`` over the processes of a
``torch.distributed`` group (gloo on CPU tensors, NCCL on CUDA tensors), and
``TorchDeviceAllreduce`` enqueues the sum on the library's stream with NCCL,
for ``Metad.set_domain_device`` (no host round trip per step).
``LocalAllgather`` and ``TorchDeviceAllgather`` do the same for walkers
sharded over ranks (``Walkers.set_ranks`` / ``set_ranks_device``).
"""
from __future__ import annotations

import itertools
import threading

import numpy as np


def decompose(x, lo, L, grid, cutoff):
    """Split atoms x (n x 3, inside the periodic box [lo, lo + L)) over a
    px x py x pz grid of bricks.  Returns one dict per rank (rank = (ix * py +
    iy) * pz + iz) with

    * ``owned``: global ids of the owned atoms, ascending;
    * ``ghost``: global ids of the ghost images, and ``shift`` (int, n_g x 3)
      the box periods added to each;
    * ``x``: positions, owned rows first, then ghosts;
    * ``lo``, ``hi``: the brick grown by ``cutoff`` on every side, the box to
      give the rank's context (non-periodic);
    * ``ids``: global id of every row (owned then ghosts).

    The cutoff must be below every box length (images of the nearest periods
    suffice)."""
    x = np.asarray(x, dtype=np.float64)
    lo = np.asarray(lo, dtype=np.float64)
    L = np.asarray(L, dtype=np.float64)
    grid = np.asarray(grid, dtype=np.int64)
    if np.any(cutoff >= L):
        raise ValueError("ghost cutoff must be smaller than the box")
    rel = (x - lo) / L
    rel -= np.floor(rel)
    cell = np.minimum((rel * grid).astype(np.int64), grid - 1)
    owner = (cell[:, 0] * grid[1] + cell[:, 1]) * grid[2] + cell[:, 2]
    xw = lo + rel * L
    shifts = np.array(list(itertools.product((-1, 0, 1), repeat=3)), dtype=np.int64)
    ranks = []
    for r, (ix, iy, iz) in enumerate(itertools.product(range(grid[0]), range(grid[1]), range(grid[2]))):
        blo = lo + L * np.array([ix, iy, iz]) / grid
        bhi = lo + L * np.array([ix + 1, iy + 1, iz + 1]) / grid
        glo, ghi = blo - cutoff, bhi + cutoff
        owned = np.nonzero(owner == r)[0]
        gid, gsh = [], []
        for s in shifts:
            xi = xw + s * L
            inside = np.all((xi >= glo) & (xi < ghi), axis=1)
            if not s.any():
                inside &= owner != r
            idx = np.nonzero(inside)[0]
            gid.append(idx)
            gsh.append(np.repeat(s[None, :], idx.size, axis=0))
        ghost = np.concatenate(gid)
        shift = np.concatenate(gsh).reshape(-1, 3)
        xl = np.concatenate([xw[owned], xw[ghost] + shift * L])
        ranks.append(dict(owned=owned, ghost=ghost, shift=shift, x=np.ascontiguousarray(xl), lo=glo, hi=ghi,
                          ids=np.concatenate([owned, ghost])))
    return ranks


def reverse_sum(n, ranks, rows):
    """Global per-atom array (n x 3) from each rank's rows (owned then ghost,
    as ``decompose`` orders them): every row is added to its owner."""
    out = np.zeros((n, 3))
    for rk, f in zip(ranks, rows):
        np.add.at(out, rk["ids"], np.asarray(f).reshape(-1, 3))
    return out


class LocalAllreduce:
    """Allreduce across ranks that are host threads of one process (one
    context per thread).  ``for_rank(r)`` is the callback of rank r; the sum
    is taken in rank order, so every rank receives the same bits."""

    def __init__(self, nranks, timeout=120.0):
        self.n = nranks
        self._bufs = [None] * nranks
        self._barrier = threading.Barrier(nranks, timeout=timeout)

    def for_rank(self, r):
        def allreduce(buf):
            self._bufs[r] = np.array(buf, copy=True)
            self._barrier.wait()
            tot = self._bufs[0].copy()
            for b in self._bufs[1:]:
                tot += b
            self._barrier.wait()
            buf[:] = tot
        return allreduce

    def abort(self):
        self._barrier.abort()


class TorchAllreduce:
    """Allreduce over a torch.distributed process group (sum, float64).
    device "cpu" for gloo; a CUDA device for NCCL."""

    def __init__(self, group=None, device="cpu"):
        self.group = group
        self.device = device

    def __call__(self, buf):
        import torch
        import torch.distributed as dist

        t = torch.from_numpy(np.array(buf, copy=True)).to(self.device)
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=self.group)
        buf[:] = t.cpu().numpy()


class _DeviceView:
    """A float64 vector at a raw device address, for torch.as_tensor."""

    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (ptr, False), "version": 3,
                                         "strides": None, "stream": None}


class TorchDeviceAllreduce:
    """Device-side allreduce for Metad.set_domain_device: sums the totals in
    place over a torch.distributed NCCL group, enqueued on the library's
    stream (the step goes on without a host synchronisation)."""

    def __init__(self, group=None):
        self.group = group

    def __call__(self, ptr, count, stream):
        import torch
        import torch.distributed as dist

        t = torch.as_tensor(_DeviceView(ptr, count), device="cuda")
        with torch.cuda.stream(torch.cuda.ExternalStream(stream)):
            dist.all_reduce(t, op=dist.ReduceOp.SUM, group=self.group)


class LocalAllgather:
    """Allgather across ranks that are host threads of one process (one
    walkers object per thread); ``for_rank(r)`` is the callback of rank r."""

    def __init__(self, nranks, timeout=120.0):
        self.n = nranks
        self._bufs = [None] * nranks
        self._barrier = threading.Barrier(nranks, timeout=timeout)

    def for_rank(self, r):
        def allgather(send, recv):
            self._bufs[r] = np.array(send, copy=True)
            self._barrier.wait()
            recv[:] = np.concatenate(self._bufs)
            self._barrier.wait()
        return allgather

    def abort(self):
        self._barrier.abort()


class TorchDeviceAllgather:
    """Device-side allgather for Walkers.set_ranks_device over a
    torch.distributed NCCL group, enqueued on the walkers' stream."""

    def __init__(self, nranks, group=None):
        self.n = nranks
        self.group = group

    def __call__(self, send_ptr, count, recv_ptr, stream):
        import torch
        import torch.distributed as dist

        send = torch.as_tensor(_DeviceView(send_ptr, count), device="cuda")
        recv = torch.as_tensor(_DeviceView(recv_ptr, count * self.n), device="cuda")
        with torch.cuda.stream(torch.cuda.ExternalStream(stream)):
            dist.all_gather_into_tensor(recv, send, group=self.group)
