"""Column sharding of one volume over several ranks (one GPU each).

The cylinder layout stores the volume column by column (`base[col]`), so a
contiguous range of columns is a contiguous range of lines.  Rank r owns the
columns [c_lo, c_hi) of a split balanced by in-mask voxels and holds one halo
column on each side that has a neighbour.  The iteration's stencil reaches one
column in each direction:

  dual step at column c    needs Vbar at c + 1  ->  before it, the right halo
                                                    column's Vbar comes from
                                                    the right neighbour;
  primal step at column c  needs Xi at c - 1    ->  before it, the left halo
                                                    column's Xi comes from the
                                                    left neighbour.

With those two exchanges per iteration every owned voxel goes through exactly
the operations of the single-volume solve, so the owned part of the result has
the same bits.  The halo columns' own updates use missing neighbours and are
overwritten by the next exchange before anything owned reads them.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Callable, Optional

import numpy as np

from .layout import CylinderMapping


def column_voxels(m: CylinderMapping) -> np.ndarray:
    """In-mask voxels of every column."""
    base = np.asarray(m.base, np.int64)
    return (base[1:] - base[:-1]) // m.nstride * m.n_images


def partition_columns(m: CylinderMapping, world: int) -> list[tuple[int, int]]:
    """Contiguous column ranges [c_lo, c_hi) of the active columns, one per rank, with about
    equal in-mask voxels (prefix-sum cuts).  Every range holds at least one column."""
    lo, hi = int(m.col_begin), int(m.col_end)
    if world < 1 or hi - lo < world:
        raise ValueError(f"cannot split {hi - lo} columns over {world} ranks")
    vox = column_voxels(m)[lo:hi].astype(np.float64)
    cum = np.concatenate([[0.0], np.cumsum(vox)])
    cuts = [lo]
    for r in range(1, world):
        target = cum[-1] * r / world
        c = lo + int(np.searchsorted(cum, target, side="left"))
        c = max(c, cuts[-1] + 1)
        c = min(c, hi - (world - r))
        cuts.append(c)
    cuts.append(hi)
    return [(cuts[r], cuts[r + 1]) for r in range(world)]


@dataclass
class ColumnShard:
    rank: int
    world: int
    c_lo: int          # first owned column (global)
    c_hi: int          # one past the last owned column
    first: int         # first local column (c_lo or c_lo - 1 with a left halo)
    last: int          # one past the last local column
    mapping: CylinderMapping   # the local volume: columns [first, last), renumbered from 0
    span_begin: int    # offset of the local volume's first line in the global span

    @property
    def left_halo(self) -> bool:
        return self.first < self.c_lo

    @property
    def right_halo(self) -> bool:
        return self.last > self.c_hi

    def local_col(self, c: int) -> int:
        return c - self.first

    def col_span(self, c: int) -> tuple[int, int]:
        """Span range [b, e) of global column c in the local arrays."""
        lc = self.local_col(c)
        return int(self.mapping.base[lc]), int(self.mapping.base[lc + 1])

    def owned_span(self) -> tuple[int, int]:
        b, _ = self.col_span(self.c_lo)
        _, e = self.col_span(self.c_hi - 1)
        return b, e

    def to_local(self, global_values: np.ndarray) -> np.ndarray:
        """The local part (halo columns included) of an array laid out in the global span."""
        return global_values[..., self.span_begin:self.span_begin + self.mapping.span]


def make_shard(m: CylinderMapping, world: int, rank: int,
               parts: Optional[list[tuple[int, int]]] = None) -> ColumnShard:
    parts = parts or partition_columns(m, world)
    c_lo, c_hi = parts[rank]
    first = c_lo - 1 if rank > 0 else c_lo
    last = c_hi + 1 if rank + 1 < world else c_hi
    base = np.asarray(m.base, np.int64)
    start_row = np.asarray(m.start_row)
    local_base = (base[first:last + 1] - base[first]).astype(np.uint32)
    local = CylinderMapping(n_images=m.n_images, rows=m.rows, cols=last - first, nstride=m.nstride,
                            col_begin=0, col_end=last - first, start_row=start_row[first:last].copy(),
                            base=local_base)
    return ColumnShard(rank, world, c_lo, c_hi, first, last, local, int(base[first]))


@dataclass
class HaloExchange:
    """The two exchanges of an iteration, written against an exchange callable so that the same
    protocol runs over NCCL (CUDA tensors) or gloo (CPU tensors).

    vbar(planes): every rank sends the Vbar planes of its first owned column to rank - 1 and
    receives those of its right halo column from rank + 1.  xi(planes): it sends the Xi planes
    of its last owned column to rank + 1 and receives its left halo column's from rank - 1."""
    shard: ColumnShard
    exchange: Callable[[list, list], None]   # (sends [(peer, array)], recvs [(peer, array)]) -> waits

    def vbar(self, vbar_planes) -> None:
        s = self.shard
        sends, recvs = [], []
        if s.left_halo:   # my first owned column is the left neighbour's right halo
            b, e = s.col_span(s.c_lo)
            sends.append((s.rank - 1, (vbar_planes, b, e)))
        if s.right_halo:
            b, e = s.col_span(s.c_hi)
            recvs.append((s.rank + 1, (vbar_planes, b, e)))
        self.exchange(sends, recvs)

    def xi(self, xi_planes) -> None:
        s = self.shard
        sends, recvs = [], []
        if s.right_halo:  # my last owned column is the right neighbour's left halo
            b, e = s.col_span(s.c_hi - 1)
            sends.append((s.rank + 1, (xi_planes, b, e)))
        if s.left_halo:
            b, e = s.col_span(s.c_lo - 1)
            recvs.append((s.rank - 1, (xi_planes, b, e)))
        self.exchange(sends, recvs)


def torch_exchange(sends, recvs) -> None:
    """send/recv of column planes with torch.distributed (NCCL for CUDA tensors, gloo for CPU
    ones).  Each item is (peer, (planes [C, span] tensor, b, e)): the column's lines are the
    span range [b, e) of every plane."""
    import torch
    import torch.distributed as dist

    ops, fills = [], []
    for peer, (planes, b, e) in sends:
        ops.append(dist.P2POp(dist.isend, planes[:, b:e].contiguous(), peer))
    for peer, (planes, b, e) in recvs:
        buf = torch.empty_like(planes[:, b:e])
        ops.append(dist.P2POp(dist.irecv, buf, peer))
        fills.append((planes, b, e, buf))
    if ops:
        for req in dist.batch_isend_irecv(ops):
            req.wait()
    for planes, b, e, buf in fills:
        planes[:, b:e].copy_(buf)


class _CudaArray:
    """__cuda_array_interface__ over device memory owned by the library (no copy)."""

    def __init__(self, ptr: int, shape, strides):
        self.__cuda_array_interface__ = {"data": (ptr, False), "shape": shape, "strides": strides,
                                         "typestr": "<f4", "version": 2}


def _device_view(ptr: int, planes: int, plane_w: int, span: int, dev):
    import torch

    return torch.as_tensor(_CudaArray(ptr, (planes, span), (4 * plane_w, 4)), device=dev)


class Stepper:
    """One local volume stepped on the GPU (potts_stepper_*).  xi [3(K-1), span], v and vb
    [K-1, span] are torch views of the library's device buffers (valid until close())."""

    def __init__(self, ctx, mapping: CylinderMapping, u_ptr: int, ci, lam: float, tau1: float, tau2: float):
        import ctypes

        import torch

        from . import _native
        from ._native import check

        c = np.ascontiguousarray(np.asarray(ci, np.float32))
        self.K = int(c.size)
        self._lib = _native.host_lib()
        self._check = check
        self._mapping = mapping
        h = ctypes.c_void_p()
        check(self._lib.potts_stepper_create(ctx.handle, ctypes.byref(mapping.as_c()), ctypes.c_void_p(int(u_ptr)),
                                             self.K, c.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), float(lam),
                                             float(tau1), float(tau2), ctypes.byref(h)))
        self._h = h
        ptrs = [ctypes.c_void_p() for _ in range(3)]
        pw = ctypes.c_int64()
        check(self._lib.potts_stepper_state(h, *(ctypes.byref(p) for p in ptrs), ctypes.byref(pw)))
        dev = torch.device("cuda", ctx.device)
        span = mapping.span
        self.xi = _device_view(int(ptrs[0].value), 3 * (self.K - 1), int(pw.value), span, dev)
        self.v = _device_view(int(ptrs[1].value), self.K - 1, int(pw.value), span, dev)
        self.vb = _device_view(int(ptrs[2].value), self.K - 1, int(pw.value), span, dev)

    def dual(self) -> None:
        self._check(self._lib.potts_stepper_dual(self._h))

    def primal(self, it: int) -> None:
        self._check(self._lib.potts_stepper_primal(self._h, int(it)))

    def finish(self, res_ptr: int = 0, labels_ptr: int = 0, V_ptr: int = 0) -> None:
        import ctypes

        self._check(self._lib.potts_stepper_finish(self._h, ctypes.c_void_p(res_ptr), ctypes.c_void_p(labels_ptr),
                                                   ctypes.c_void_p(V_ptr)))

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.potts_stepper_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def exchange_in_process(shards: list[ColumnShard], planes: list, kind: str) -> None:
    """The exchange of one iteration between shards held by one process (device copies): kind
    "vbar" fills every right halo column from the right neighbour's first owned column, "xi"
    every left halo column from the left neighbour's last owned column."""
    for r, s in enumerate(shards):
        if kind == "vbar" and s.right_halo:
            n = shards[r + 1]
            b, e = s.col_span(s.c_hi)
            nb, ne = n.col_span(n.c_lo)
            planes[r][:, b:e].copy_(planes[r + 1][:, nb:ne])
        if kind == "xi" and s.left_halo:
            n = shards[r - 1]
            b, e = s.col_span(s.c_lo - 1)
            nb, ne = n.col_span(n.c_hi - 1)
            planes[r][:, b:e].copy_(planes[r - 1][:, nb:ne])


def solve_sharded(ctx, m: CylinderMapping, u, ci, lam: float, tau1: float, tau2: float, iters: int, rank: int,
                  world: int):
    """This rank's part of a column-sharded solve over torch.distributed (NCCL between GPUs).
    u: the global u on this rank's device (a torch tensor over the mapping's span).  Returns
    the shard and its local (labels uint8 [span], V [K-1, span]) device tensors, exact for the
    owned columns.  The context should run on torch's current stream, which orders the
    exchanges and the steps."""
    import torch

    shard = make_shard(m, world, rank)
    u_loc = u[shard.span_begin:shard.span_begin + shard.mapping.span].contiguous()
    st = Stepper(ctx, shard.mapping, u_loc.data_ptr(), ci, lam, tau1, tau2)
    ex = HaloExchange(shard, torch_exchange)
    for it in range(iters):
        ex.vbar(st.vb)
        st.dual()
        ex.xi(st.xi)
        st.primal(it)
    labels = torch.zeros(shard.mapping.span, dtype=torch.uint8, device=u.device)
    V = torch.zeros((st.K - 1, shard.mapping.span), dtype=torch.float32, device=u.device)
    st.finish(labels_ptr=labels.data_ptr(), V_ptr=V.data_ptr())
    ctx.synchronize()
    st.close()
    return shard, labels, V
