"""Slab decomposition of one problem over ranks (one rank per GPU).

The reference decomposes the mesh with MPI_Dims_create / MPI_Cart_create
(src/MPIContext.cpp:80-170: each rank takes globalN / nProcs cells of an
axis, the first globalN % nProcs ranks one more, nodes sliced from the
global node array), exchanges ghost layers with its Cartesian neighbours
every stage (src/HaloExchange.cpp:387-465) and reduces dt with
MPI_Allreduce(MIN) (src/RKTimeStepping.cpp:148-159).  Here the mesh is cut
along its slowest axis only (y in 2D, z in 3D, x in 1D), so every ghost
layer to exchange is one contiguous block of each field; the faces between
ranks carry SIFV_BC_EXCHANGE, the others keep the global boundary
conditions (a periodic axis that is cut becomes a ring of ranks).

`DistExchange` implements the library's halo-exchange / dt-reduction hooks
(sifv_set_comm) with torch.distributed point-to-point operations and an
all-reduce: NCCL over NVLink for device arrays, gloo for host arrays (the C
oracle in the CPU tests).
"""
from __future__ import annotations

import ctypes
from typing import Dict, Optional, Tuple

import numpy as np

from . import abi


def split(n: int, parts: int, rank: int) -> Tuple[int, int]:
    """(first cell, cell count) of `rank` when n cells are cut into `parts`
    (MPIContext::sliceNodes, src/MPIContext.cpp:60-78)."""
    base, rem = divmod(n, parts)
    start = rank * base + min(rank, rem)
    return start, base + (1 if rank < rem else 0)


def slab_axis(dim: int) -> int:
    return dim - 1


def neighbours(rank: int, world: int, periodic: bool) -> Tuple[Optional[int], Optional[int]]:
    """Ranks below and above along the cut axis (None at a physical face)."""
    lo = rank - 1 if rank > 0 else (world - 1 if periodic and world > 1 else None)
    hi = rank + 1 if rank < world - 1 else (0 if periodic and world > 1 else None)
    return lo, hi


def slab_mesh(mesh: abi.MeshSpec, dim: int, rank: int, world: int) -> Tuple[abi.MeshSpec, int, int]:
    """The rank's part of `mesh` (cut along the slowest axis): its node
    array, its boundary conditions (SIFV_BC_EXCHANGE on faces between
    ranks), and (first cell, cell count) along the cut axis."""
    ax = slab_axis(dim)
    nodes = [mesh.x, mesh.y, mesh.z]
    n = len(nodes[ax]) - 1
    start, count = split(n, world, rank)
    if count < 3:
        raise ValueError(f"rank {rank} would hold {count} cells along the cut axis (at least the ghost depth needed)")
    local = list(nodes)
    local[ax] = nodes[ax][start:start + count + 1].copy()
    bc = list(mesh.bc)
    periodic = bc[2 * ax] == abi.BC_PERIODIC and bc[2 * ax + 1] == abi.BC_PERIODIC
    if world > 1:
        lo, hi = neighbours(rank, world, periodic)
        if lo is not None:
            bc[2 * ax] = abi.BC_EXCHANGE
        if hi is not None:
            bc[2 * ax + 1] = abi.BC_EXCHANGE
    return abi.MeshSpec(local[0], local[1], local[2], bc=bc), start, count


def slab_fields(fields: Dict[int, np.ndarray], cfg, start: int, count: int) -> Dict[int, np.ndarray]:
    """The rank's part of global (k, j, i) field arrays, ghosts included:
    its interior block; its ghost layers start at zero, as in the
    reference's drivers, which set the interior only."""
    ax = slab_axis(cfg.dim)
    g = cfg.nGhost
    out = {}
    for fid, a in fields.items():
        nz, ny, nx = a.shape
        shape = [nz, ny, nx]
        np_ax = 2 - ax                               # numpy axis of the cut axis
        shape[np_ax] = count + 2 * g
        loc = np.zeros(shape, dtype=np.float64)
        src = [slice(None)] * 3
        dst = [slice(None)] * 3
        src[np_ax] = slice(g + start, g + start + count)
        dst[np_ax] = slice(g, g + count)
        loc[tuple(dst)] = a[tuple(src)]
        out[fid] = loc
    return out


def gather_interior(local: np.ndarray, cfg, start: int, count: int, glob: np.ndarray) -> None:
    """Copy the rank's interior block of a (k, j, i) array into the global array."""
    ax = slab_axis(cfg.dim)
    g = cfg.nGhost
    np_ax = 2 - ax
    src = [slice(None)] * 3
    dst = [slice(None)] * 3
    src[np_ax] = slice(g, g + count)
    dst[np_ax] = slice(g + start, g + start + count)
    glob[tuple(dst)] = local[tuple(src)]


class _CudaView:
    """A device array at a raw address, for torch.as_tensor (zero copy)."""

    def __init__(self, ptr: int, n: int):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (ptr, False), "version": 3,
                                         "strides": None}


def _view(ptr: int, n: int, device: bool):
    import torch
    if device:
        return torch.as_tensor(_CudaView(ptr, n), device="cuda")
    buf = (ctypes.c_double * n).from_address(ptr)
    return torch.from_numpy(np.frombuffer(buf, dtype=np.float64))


class DistExchange:
    """sifv_set_comm hooks over torch.distributed for one rank of a slab
    decomposition.  ctx: the rank's context (its extents give the block
    sizes); device: True for a CUDA context (NCCL process group; the
    context must run on torch's current stream so that the collectives
    are ordered with its kernels), False for a host backend (gloo)."""

    TAG_TO_LOW, TAG_TO_HIGH = 0, 1   # message into the receiver's low / high ghost layers

    def __init__(self, ctx, rank: int, world: int, periodic: bool, device: bool):
        self.ctx, self.device = ctx, device
        self.lo, self.hi = neighbours(rank, world, periodic)
        nz, ny, nx = ctx.shape
        dim, g = ctx.cfg.dim, ctx.cfg.nGhost
        plane = {1: 1, 2: nx, 3: nx * ny}[dim]       # cells of one layer across the cut axis
        extent = {1: nx, 2: ny, 3: nz}[dim]           # cut-axis extent, ghosts included
        n_int = extent - 2 * g
        self.n = extent * plane
        self.block = g * plane
        self.low_ghost, self.low_int = 0, g * plane
        self.high_int, self.high_ghost = n_int * plane, (n_int + g) * plane
        # The step asks for the same few field sets (and reduction slots) over
        # and over: the views and operation lists are built once per address
        # set and reused, which keeps the host's work per exchange small.
        self._plans = {}
        self._scalars = {}

    def _plan(self, ptrs):
        import torch.distributed as dist
        key = tuple(ptrs)
        plan = self._plans.get(key)
        if plan is not None:
            return plan
        if len(self._plans) > 64:   # the context re-allocated its arrays: forget old addresses
            self._plans.clear()
        sends, recvs = [], []
        for p in ptrs:
            f = _view(p, self.n, self.device)
            b = self.block
            # send order per peer: into its low ghost first, then into its high ghost;
            # receive order: own low ghost first, then own high ghost (a two-rank ring
            # has the same peer on both sides)
            if self.hi is not None:
                sends.append((f[self.high_int:self.high_int + b], self.hi, self.TAG_TO_LOW))
            if self.lo is not None:
                sends.append((f[self.low_int:self.low_int + b], self.lo, self.TAG_TO_HIGH))
            if self.lo is not None:
                recvs.append((f[self.low_ghost:self.low_ghost + b], self.lo, self.TAG_TO_LOW))
            if self.hi is not None:
                recvs.append((f[self.high_ghost:self.high_ghost + b], self.hi, self.TAG_TO_HIGH))
        ops = None
        if self.device:
            ops = [dist.P2POp(dist.isend, t, peer) for t, peer, _ in sends] + \
                  [dist.P2POp(dist.irecv, t, peer) for t, peer, _ in recvs]
        plan = (sends, recvs, ops)
        self._plans[key] = plan
        return plan

    def _scalar(self, ptr):
        v = self._scalars.get(ptr)
        if v is None:
            if len(self._scalars) > 64:
                self._scalars.clear()
            v = self._scalars[ptr] = _view(ptr, 1, self.device)
        return v

    def exchange(self, ptrs, stream):
        import torch.distributed as dist
        sends, recvs, ops = self._plan(ptrs)
        if self.device:
            if ops:
                for w in dist.batch_isend_irecv(ops):
                    w.wait()
        else:
            works = [dist.isend(t, peer, tag=tag) for t, peer, tag in sends]
            works += [dist.irecv(t, peer, tag=tag) for t, peer, tag in recvs]
            for w in works:
                w.wait()
        return 0

    def allreduce_min(self, ptr, stream):
        import torch.distributed as dist
        dist.all_reduce(self._scalar(ptr), op=dist.ReduceOp.MIN)
        return 0

    def allreduce_max(self, ptr, stream):
        import torch.distributed as dist
        dist.all_reduce(self._scalar(ptr), op=dist.ReduceOp.MAX)
        return 0

    def attach(self):
        self.ctx.set_comm(self.exchange, self.allreduce_min, self.allreduce_max)
        return self
