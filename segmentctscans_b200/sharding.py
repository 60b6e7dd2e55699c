"""Column sharding of one volume over several GPUs (potts_shard_* in the native library).

The cylinder layout stores the volume column by column (`base[col]`), so a contiguous range of
columns is a contiguous range of lines.  Shard r owns the columns [c_lo, c_hi) of a split
balanced by in-mask voxels and holds, besides them, the column before c_lo and the two after
c_hi where the volume has them.  Each iteration is one fused launch per shard over the columns
[c_lo, c_hi + 1) followed by one exchange: the Xi planes of a shard's first owned column go to
the left neighbour (its column c_hi), those of its last owned column to the right neighbour (its
column c_lo - 1).  The primal step at c_hi, computed locally, gives V and Vbar there exactly, so
nothing else crosses, and every owned voxel gets the bits of the single-volume fused solve.  The
convergence trace is the max and the FP64 energies the sums over the shards
(potts-model/potts-min-partition.cpp:648-659 is the monitor this reduces).

`partition_columns` / `make_shard` restate the split and the local volumes in Python (the CPU
tests run the same protocol on the oracle over gloo); `solve_local` runs all shards of a volume
in one process on one GPU (halos by device copies), `solve_sharded` one shard per rank over
NCCL (the library's own communicator; the unique id travels over torch.distributed).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

from .layout import CylinderMapping


def column_voxels(m: CylinderMapping) -> np.ndarray:
    """In-mask voxels of every column."""
    base = np.asarray(m.base, np.int64)
    return (base[1:] - base[:-1]) // m.nstride * m.n_images


def partition_columns(m: CylinderMapping, world: int) -> list[tuple[int, int]]:
    """Contiguous column ranges [c_lo, c_hi) of the active columns, one per shard, with about
    equal in-mask voxels (prefix-sum cuts).  Every range holds at least one column."""
    lo, hi = int(m.col_begin), int(m.col_end)
    if world < 1 or hi - lo < world:
        raise ValueError(f"cannot split {hi - lo} columns over {world} shards")
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
    first: int         # first held column: c_lo - 1 with a left neighbour, else c_lo
    last: int          # one past the last held column: c_hi + 2 (at most col_end) with a right neighbour
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

    def to_local(self, global_values):
        """The local part (halo columns included) of an array laid out in the global span."""
        return global_values[..., self.span_begin:self.span_begin + self.mapping.span]


def make_shard(m: CylinderMapping, world: int, rank: int,
               parts: Optional[list[tuple[int, int]]] = None) -> ColumnShard:
    parts = parts or partition_columns(m, world)
    c_lo, c_hi = parts[rank]
    first = c_lo - 1 if rank > 0 else c_lo
    last = min(c_hi + 2, int(m.col_end)) if rank + 1 < world else c_hi
    base = np.asarray(m.base, np.int64)
    start_row = np.asarray(m.start_row)
    local_base = (base[first:last + 1] - base[first]).astype(np.uint32)
    local = CylinderMapping(n_images=m.n_images, rows=m.rows, cols=last - first, nstride=m.nstride,
                            col_begin=0, col_end=last - first, start_row=start_row[first:last].copy(),
                            base=local_base)
    return ColumnShard(rank, world, c_lo, c_hi, first, last, local, int(base[first]))


def native_cuts(m: CylinderMapping, world: int) -> list[int]:
    """The library's split (potts_shard_partition): cuts[0] = col_begin .. cuts[world] = col_end."""
    from . import _native

    cuts = (ctypes.c_uint32 * (world + 1))()
    _native.check(_native.host_lib().potts_shard_partition(ctypes.byref(m.as_c()), int(world), cuts))
    return list(cuts)


def native_bounds(m: CylinderMapping, cuts: Sequence[int], rank: int) -> tuple[tuple[int, ...], tuple[int, int]]:
    """(first, last, own_begin, own_end) and the span range of shard `rank` (potts_shard_bounds)."""
    from . import _native

    world = len(cuts) - 1
    c = (ctypes.c_uint32 * len(cuts))(*cuts)
    cols = (ctypes.c_uint32 * 4)()
    span = (ctypes.c_uint64 * 2)()
    _native.check(_native.host_lib().potts_shard_bounds(ctypes.byref(m.as_c()), c, world, int(rank), cols, span))
    return tuple(int(x) for x in cols), (int(span[0]), int(span[1]))


class Shard:
    """One shard of a volume on the GPU (potts_shard_create).  u_ptr: the device address of the
    shard's u (the global u + 4 * span[0] bytes); it must stay valid while the shard lives."""

    def __init__(self, ctx, m: CylinderMapping, cuts: Sequence[int], rank: int, u_ptr: int, ci, lam: float,
                 tau1: float, tau2: float, **options):
        from . import _native

        self._lib = _native.host_lib()
        self._check = _native.check
        self.world = len(cuts) - 1
        self.rank = int(rank)
        c = np.ascontiguousarray(np.asarray(ci, np.float32))
        self.K = int(c.size)
        self._keep = (m, (ctypes.c_uint32 * len(cuts))(*cuts), c)
        self.cols, self.span = native_bounds(m, cuts, rank)
        opts = _native.default_options(**options)
        self.gap_every = int(opts.gap_every)
        h = ctypes.c_void_p()
        self._check(self._lib.potts_shard_create(ctx.handle, ctypes.byref(m.as_c()), self._keep[1], self.world,
                                                 self.rank, ctypes.c_void_p(int(u_ptr)), self.K,
                                                 c.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), float(lam),
                                                 float(tau1), float(tau2), ctypes.byref(opts), ctypes.byref(h)))
        self._h = h
        self._comm = None

    @property
    def local_span(self) -> int:
        return self.span[1] - self.span[0]

    def link(self, right: "Shard") -> None:
        self._check(self._lib.potts_shard_link(self._h, right._h))

    def use_nccl(self, comm) -> None:
        self._check(self._lib.potts_shard_set_nccl(self._h, comm))
        self._comm = comm

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.potts_shard_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def run_shards(shards: Sequence[Shard], iters: int, res_ptrs=None, label_ptrs=None, V_ptrs=None, stats: bool = True):
    """potts_shard_solve over this process's shards; outputs are device addresses in each shard's
    span layout (0 = none).  Returns SolveStats (dq and energy traces of the whole volume)."""
    from . import _native
    from .potts import _make_stats, _stats_out

    n = len(shards)
    arr = (ctypes.c_void_p * n)(*(s._h.value for s in shards))

    def ptrs(values):
        if values is None:
            return None
        return (ctypes.c_void_p * n)(*(int(v or 0) for v in values))

    st, dq, en = _make_stats(iters, shards[0].gap_every, stats)
    _native.check(_native.host_lib().potts_shard_solve(arr, n, int(iters), ptrs(res_ptrs), ptrs(label_ptrs),
                                                       ptrs(V_ptrs), ctypes.byref(st) if stats else None))
    return _stats_out(st, dq, en) if stats else None


def solve_local(ctx, m: CylinderMapping, u, ci, lam: float, tau1: float, tau2: float, iters: int, world: int,
                **options):
    """Every shard of a `world`-way split in this process, on ctx's device (halos by device copies).
    u: the global u as a torch tensor on that device.  Returns (labels uint8 [span], V [K-1, span],
    SolveStats) in the global layout, filled for every in-mask voxel."""
    import torch

    cuts = native_cuts(m, world)
    K = len(ci)
    shards = []
    try:
        for r in range(world):  # the u of each shard is a range of the global u
            shards.append(Shard(ctx, m, cuts, r, u.data_ptr() + 4 * native_bounds(m, cuts, r)[1][0], ci, lam,
                                tau1, tau2, **options))
        for a, b in zip(shards, shards[1:]):
            a.link(b)
        labels = torch.zeros(m.span, dtype=torch.uint8, device=u.device)
        V = torch.zeros((K - 1, m.span), dtype=torch.float32, device=u.device)
        loc_lab = [torch.zeros(s.local_span, dtype=torch.uint8, device=u.device) for s in shards]
        loc_V = [torch.zeros((K - 1, s.local_span), dtype=torch.float32, device=u.device) for s in shards]
        st = run_shards(shards, iters, label_ptrs=[t.data_ptr() for t in loc_lab], V_ptrs=[t.data_ptr() for t in loc_V])
        for s, lab, v in zip(shards, loc_lab, loc_V):
            first, _, own_b, own_e = s.cols
            b = int(m.base[own_b]) - s.span[0]
            e = int(m.base[own_e]) - s.span[0]
            labels[s.span[0] + b:s.span[0] + e] = lab[b:e]
            V[:, s.span[0] + b:s.span[0] + e] = v[:, b:e]
        return labels, V, st
    finally:
        for s in shards:
            s.close()


def nccl_comm(rank: int, world: int, device: int):
    """The library's NCCL communicator over the ranks of the default torch.distributed group (the
    unique id is made on rank 0 and broadcast through torch.distributed)."""
    import torch.distributed as dist

    from . import _native

    lib = _native.host_lib()
    idbuf = (ctypes.c_uint8 * 128)()
    if rank == 0:
        _native.check(lib.potts_nccl_unique_id(idbuf))
    obj = [bytes(idbuf)]
    dist.broadcast_object_list(obj, src=0)
    idbuf = (ctypes.c_uint8 * 128).from_buffer_copy(obj[0])
    comm = ctypes.c_void_p()
    _native.check(lib.potts_nccl_comm_create(idbuf, int(world), int(rank), int(device), ctypes.byref(comm)))
    return comm


def destroy_comm(comm) -> None:
    from . import _native

    if comm:
        _native.check(_native.host_lib().potts_nccl_comm_destroy(comm))


def solve_sharded(ctx, m: CylinderMapping, u, ci, lam: float, tau1: float, tau2: float, iters: int, rank: int,
                  world: int, comm=None, **options):
    """This rank's shard of a `world`-way split, exchanging with the other ranks over NCCL.
    u: the global u on this rank's device (torch tensor over the mapping's span); comm: a
    communicator from nccl_comm() (made here when None, and then destroyed).  Returns the shard's
    (labels, V, SolveStats): labels [local span] and V [K-1, local span] hold the owned columns,
    the stats the whole volume's dq and energy traces."""
    import torch

    cuts = native_cuts(m, world)
    own_comm = comm is None and world > 1
    if own_comm:
        comm = nccl_comm(rank, world, ctx.device)
    shard = None
    try:
        _, span = native_bounds(m, cuts, rank)
        shard = Shard(ctx, m, cuts, rank, u.data_ptr() + 4 * span[0], ci, lam, tau1, tau2, **options)
        if world > 1:
            shard.use_nccl(comm)
        K = len(ci)
        labels = torch.zeros(shard.local_span, dtype=torch.uint8, device=u.device)
        V = torch.zeros((K - 1, shard.local_span), dtype=torch.float32, device=u.device)
        st = run_shards([shard], iters, label_ptrs=[labels.data_ptr()], V_ptrs=[V.data_ptr()])
        return shard.cols, shard.span, labels, V, st
    finally:
        if shard is not None:
            shard.close()
        if own_comm:
            destroy_comm(comm)
