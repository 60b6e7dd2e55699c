"""Host API mirroring the reference's Potts entry points.

Reference interface (C++):
  make_context()                                   cuda-context/cuda-context.cpp:18-20
  upload(ctx, span) / download(ctx, field, span)   cuda-context/cuda-context.cpp:49-77
  device_memory(ctx)                               cuda-context/cuda-context.cpp:22-42
  potts_min_partition<K>(ctx, g, cpu_map, ci, 𝜆, 𝜏1, 𝜏2, iters)
                                                   potts-model/potts-min-partition.h:8-16

Each call goes through the C ABI of ``libpotts_b200.so``; errors raise
``PottsError`` (the reference throws ``cuda::cuda_error`` and returns an empty
pointer when memory runs out, potts-min-partition.cpp:571-577).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

from . import _native
from ._native import PottsError, check
from .layout import CylinderMapping

MAX_PHASES = _native.MAX_PHASES


def reference_tau() -> float:
    """Step size of the reference CLI: 0.99 * sqrt(1/12) (potts-model/potts-model.cpp:141)."""
    return float(np.float32(0.99) * np.sqrt(np.float32(1.0) / np.float32(12.0)))


class CudaContext:
    """One device and one stream (include/cuda-details/cuda-context-impl.h:35-65)."""

    def __init__(self, device: int = 0, stream: Optional[int] = None):
        lib = _native.host_lib()
        h = ctypes.c_void_p()
        if stream is None:
            check(lib.potts_context_create(int(device), ctypes.byref(h)))
        else:
            check(lib.potts_context_create_on_stream(int(device), ctypes.c_void_p(int(stream)), ctypes.byref(h)))
        self._h = h
        self.device = int(device)

    @property
    def handle(self) -> ctypes.c_void_p:
        if self._h is None:
            raise RuntimeError("context is closed")
        return self._h

    def synchronize(self) -> None:
        check(_native.host_lib().potts_context_synchronize(self.handle))

    def device_memory(self) -> tuple[int, int]:
        a, t = ctypes.c_size_t(), ctypes.c_size_t()
        check(_native.host_lib().potts_device_memory(self.handle, ctypes.byref(a), ctypes.byref(t)))
        return int(a.value), int(t.value)

    def close(self) -> None:
        if self._h is not None:
            _native.host_lib().potts_context_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def make_context(device: int = 0, stream: Optional[int] = None) -> CudaContext:
    """make_context(): a context on `device`; `stream` is an optional cudaStream_t handle to share."""
    return CudaContext(device, stream)


class DeviceField:
    """DeviceField<float> (include/cuda-details/device-field-impl.h:12-54): device voxels + mapping."""

    def __init__(self, ctx: CudaContext, mapping: CylinderMapping, handle: ctypes.c_void_p):
        self.ctx = ctx
        self.mapping = mapping
        self._h = handle

    @property
    def handle(self):
        return self._h

    def data_ptr(self) -> int:
        return int(_native.host_lib().potts_field_data(self._h) or 0)

    @property
    def span(self) -> int:
        return int(_native.host_lib().potts_field_span(self._h))

    def free(self) -> None:
        if self._h is not None:
            _native.host_lib().potts_field_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def upload(ctx: CudaContext, mapping: CylinderMapping, host: np.ndarray) -> DeviceField:
    host = np.ascontiguousarray(host, dtype=np.float32)
    if host.size != mapping.span:
        raise ValueError(f"host array has {host.size} floats, mapping span is {mapping.span}")
    h = ctypes.c_void_p()
    check(_native.host_lib().potts_field_upload(ctx.handle, ctypes.byref(mapping.as_c()),
                                                host.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                                ctypes.byref(h)))
    return DeviceField(ctx, mapping, h)


def download(ctx: CudaContext, fld: DeviceField, out: Optional[np.ndarray] = None) -> np.ndarray:
    span = fld.span
    if out is None:
        out = np.empty(span, dtype=np.float32)
    if out.dtype != np.float32 or not out.flags.c_contiguous:
        raise ValueError("out must be a contiguous float32 array")
    check(_native.host_lib().potts_field_download(ctx.handle, fld.handle,
                                                  out.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                                  ctypes.c_uint64(out.size)))
    return out


def device_memory(ctx: CudaContext) -> tuple[int, int]:
    return ctx.device_memory()


def _ci_array(ci: Sequence[float]) -> np.ndarray:
    c = np.ascontiguousarray(np.asarray(ci, dtype=np.float32))
    if c.ndim != 1 or not (2 <= c.size <= MAX_PHASES):
        raise ValueError(f"need 2..{MAX_PHASES} labels, got {c.size}")
    return c


@dataclass
class SolveStats:
    n_slabs: int
    slab_w: int
    iters: int
    dq_last: float
    solve_ms: float
    loop_ms: float
    loop_launches: int
    total_launches: int
    state_bytes: int
    dq_trace: Optional[np.ndarray] = None       # [iters] max |dV|^2 per iteration (last slab)
    energy_trace: Optional[np.ndarray] = None   # [iters // gap_every, 3] (lagrangian, dual, gap)
    loop_iters: int = 0                         # iterations inside loop_ms


def _make_stats(iters: int, gap_every: int, want_traces: bool):
    st = _native.PottsStats()
    dq = en = None
    if want_traces and iters > 0:
        dq = np.zeros(iters, dtype=np.float32)
        st.dq_trace = dq.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
        if gap_every > 0 and iters // gap_every > 0:
            en = np.zeros((iters // gap_every, 3), dtype=np.float64)
            st.energy_trace = en.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    return st, dq, en


def _stats_out(st, dq, en) -> SolveStats:
    return SolveStats(st.n_slabs, st.slab_w, st.iters, float(st.dq_last), float(st.solve_ms), float(st.loop_ms),
                      int(st.loop_launches), int(st.total_launches), int(st.state_bytes), dq, en,
                      int(st.loop_iters))


def potts_min_partition(ctx: CudaContext, g: DeviceField, cpu_map: CylinderMapping, ci: Sequence[float],
                        lam: float, tau1: float, tau2: float, iters: int, *, stats: bool = False,
                        **options) -> DeviceField | tuple[DeviceField, SolveStats]:
    """potts_min_partition<K> (potts-model/potts-min-partition.h:8-16): a new field holding
    ci[argmax_i V_i] for every in-mask voxel of g."""
    c = _ci_array(ci)
    opts = _native.default_options(**options)
    st, dq, en = _make_stats(iters, opts.gap_every, stats)
    h = ctypes.c_void_p()
    check(_native.host_lib().potts_min_partition(
        ctx.handle, g.handle, ctypes.byref(cpu_map.as_c()), int(c.size),
        c.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), float(lam), float(tau1), float(tau2), int(iters),
        ctypes.byref(opts), ctypes.byref(h), ctypes.byref(st)))
    res = DeviceField(ctx, cpu_map, h)
    return (res, _stats_out(st, dq, en)) if stats else res


def solve_device(ctx: CudaContext, mapping: CylinderMapping, u_ptr: int, ci: Sequence[float], lam: float,
                 tau1: float, tau2: float, iters: int, *, res_ptr: int = 0, labels_ptr: int = 0, V_ptr: int = 0,
                 Xi_ptr: int = 0, stats: bool = True, **options) -> Optional[SolveStats]:
    """Device-pointer solve (potts_solve_device): inputs/outputs are raw device addresses laid out
    with `mapping`; any output address may be 0.  With stats=False nothing waits for the GPU."""
    c = _ci_array(ci)
    opts = _native.default_options(**options)
    st, dq, en = _make_stats(iters, opts.gap_every, stats)
    check(_native.host_lib().potts_solve_device(
        ctx.handle, ctypes.byref(mapping.as_c()), ctypes.c_void_p(int(u_ptr)), int(c.size),
        c.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), float(lam), float(tau1), float(tau2), int(iters),
        ctypes.byref(opts), ctypes.c_void_p(int(res_ptr)), ctypes.c_void_p(int(labels_ptr)),
        ctypes.c_void_p(int(V_ptr)), ctypes.c_void_p(int(Xi_ptr)), ctypes.byref(st) if stats else None))
    return _stats_out(st, dq, en) if stats else None


def solve_device_f64(ctx: CudaContext, mapping: CylinderMapping, u_ptr: int, ci: Sequence[float], lam: float,
                     tau1: float, tau2: float, iters: int, *, res_ptr: int = 0, labels_ptr: int = 0,
                     V_ptr: int = 0, Xi_ptr: int = 0, stats: bool = True, **options) -> Optional[SolveStats]:
    """FP64 solve (potts_solve_device_f64): FP64 state and arithmetic in the split kernel structure;
    V_ptr / Xi_ptr are FP64 planes.  The GPU counterpart of the FP64 oracle for large volumes."""
    c = _ci_array(ci)
    opts = _native.default_options(**options)
    st, dq, en = _make_stats(iters, opts.gap_every, stats)
    check(_native.host_lib().potts_solve_device_f64(
        ctx.handle, ctypes.byref(mapping.as_c()), ctypes.c_void_p(int(u_ptr)), int(c.size),
        c.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), float(lam), float(tau1), float(tau2), int(iters),
        ctypes.byref(opts), ctypes.c_void_p(int(res_ptr)), ctypes.c_void_p(int(labels_ptr)),
        ctypes.c_void_p(int(V_ptr)), ctypes.c_void_p(int(Xi_ptr)), ctypes.byref(st) if stats else None))
    return _stats_out(st, dq, en) if stats else None


def solve_host(ctx: CudaContext, mapping: CylinderMapping, u: np.ndarray, ci: Sequence[float], lam: float,
               tau1: float, tau2: float, iters: int, *, res: Optional[np.ndarray] = None,
               labels: Optional[np.ndarray] = None, stats: bool = False, **options) -> Optional[SolveStats]:
    """Host-buffer solve (potts_solve_host): copies u in, solves, copies res/labels out; blocks."""
    c = _ci_array(ci)
    if u.dtype != np.float32 or not u.flags.c_contiguous or u.size != mapping.span:
        raise ValueError("u must be a contiguous float32 array of mapping.span values")
    for arr, dt in ((res, np.float32), (labels, np.uint8)):
        if arr is not None and (arr.dtype != dt or not arr.flags.c_contiguous or arr.size != mapping.span):
            raise ValueError("outputs must be contiguous arrays of mapping.span values")
    opts = _native.default_options(**options)
    st, dq, en = _make_stats(iters, opts.gap_every, stats)
    check(_native.host_lib().potts_solve_host(
        ctx.handle, ctypes.byref(mapping.as_c()), ctypes.c_void_p(u.ctypes.data), int(c.size),
        c.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), float(lam), float(tau1), float(tau2), int(iters),
        ctypes.byref(opts), ctypes.c_void_p(res.ctypes.data if res is not None else 0),
        ctypes.c_void_p(labels.ctypes.data if labels is not None else 0), ctypes.byref(st) if stats else None))
    return _stats_out(st, dq, en) if stats else None


@dataclass
class PottsResult:
    labels: np.ndarray            # uint8 span: argmax index
    res: np.ndarray               # float32 span: ci[argmax]
    V: Optional[np.ndarray]       # float32 [K-1, span] (float64 for storage="f64")
    Xi: Optional[np.ndarray]      # float32 [3(K-1), span] (float64 for storage="f64")
    stats: SolveStats = field(default=None)


def solve(mapping: CylinderMapping, u: np.ndarray, ci: Sequence[float], lam: float, tau1: float, tau2: float,
          iters: int, *, ctx: Optional[CudaContext] = None, want_state: bool = True, **options) -> PottsResult:
    """Convenience: solve a host volume on the GPU (through torch device buffers) and return host arrays."""
    import torch

    c = _ci_array(ci)
    K = c.size
    own = ctx is None
    if own:
        ctx = make_context(0, stream=torch.cuda.current_stream().cuda_stream)
    try:
        dev = torch.device("cuda", ctx.device)
        span = mapping.span
        du = torch.from_numpy(np.ascontiguousarray(u, dtype=np.float32)).to(dev)
        dres = torch.zeros(span, dtype=torch.float32, device=dev)
        dlab = torch.zeros(span, dtype=torch.uint8, device=dev)
        f64 = options.get("storage") in ("f64", _native.STORE_F64)
        sdt = torch.float64 if f64 else torch.float32
        dV = torch.zeros((K - 1, span), dtype=sdt, device=dev) if want_state else None
        dX = torch.zeros((3 * (K - 1), span), dtype=sdt, device=dev) if want_state else None
        st = (solve_device_f64 if f64 else solve_device)(
            ctx, mapping, du.data_ptr(), c, lam, tau1, tau2, iters, res_ptr=dres.data_ptr(),
            labels_ptr=dlab.data_ptr(), V_ptr=dV.data_ptr() if dV is not None else 0,
            Xi_ptr=dX.data_ptr() if dX is not None else 0, stats=True, **options)
        torch.cuda.synchronize(dev)
        return PottsResult(dlab.cpu().numpy(), dres.cpu().numpy(),
                           dV.cpu().numpy() if dV is not None else None,
                           dX.cpu().numpy() if dX is not None else None, st)
    finally:
        if own:
            ctx.close()


# --------------------------------------------------------------------------- batches
@dataclass
class BatchVolume:
    """One volume of a batch: its mapping, device u and outputs (raw device addresses, 0 = none)."""
    mapping: CylinderMapping
    u_ptr: int
    ci: Sequence[float]
    lam: float
    res_ptr: int = 0
    labels_ptr: int = 0
    V_ptr: int = 0


@dataclass
class BatchInfo:
    n_volumes: int
    n_work: int
    tile: tuple
    voxels: int
    state_bytes: int
    graph_launches: int
    autotune_ms: float
    persistent: int = 0          # 1: the iterations run as one persistent launch


class Batch:
    """A planned batch of independent volumes run as one captured CUDA graph (potts_batch_create).
    The device buffers named by the volumes must outlive the batch."""

    def __init__(self, ctx: CudaContext, volumes: Sequence[BatchVolume], tau1: float, tau2: float, iters: int,
                 **options):
        if not volumes:
            raise ValueError("a batch needs at least one volume")
        K = len(volumes[0].ci)
        self.ctx = ctx
        self.iters = int(iters)
        self._keep = []
        arr = (_native.PottsBatchVolume * len(volumes))()
        for i, v in enumerate(volumes):
            c = _ci_array(v.ci)
            if c.size != K:
                raise ValueError("every volume of a batch needs the same number of labels")
            self._keep.append((v.mapping, c))
            arr[i].map = v.mapping.as_c()
            arr[i].d_u = ctypes.c_void_p(int(v.u_ptr))
            arr[i].ci = c.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
            arr[i].lambda_ = float(v.lam)
            arr[i].d_res = ctypes.c_void_p(int(v.res_ptr))
            arr[i].d_labels = ctypes.c_void_p(int(v.labels_ptr))
            arr[i].d_V = ctypes.c_void_p(int(v.V_ptr))
        opts = _native.default_options(**options)
        self.track_dq = bool(opts.track_dq)
        h = ctypes.c_void_p()
        check(_native.host_lib().potts_batch_create(ctx.handle, len(volumes), arr, K, float(tau1), float(tau2),
                                                    int(iters), ctypes.byref(opts), ctypes.byref(h)))
        self._h = h
        self.n_volumes = len(volumes)

    def run(self, stats: bool = True) -> Optional[SolveStats]:
        """Replay the graph; with stats, wait and report (dq_trace: max over the volumes)."""
        st, dq, en = _make_stats(self.iters, 0, stats)
        check(_native.host_lib().potts_batch_run(self._h, ctypes.byref(st) if stats else None))
        return _stats_out(st, dq, en) if stats else None

    def info(self) -> BatchInfo:
        i = _native.PottsBatchInfo()
        check(_native.host_lib().potts_batch_get_info(self._h, ctypes.byref(i)))
        return BatchInfo(i.n_volumes, i.n_work, (i.tile_rows, i.tile_slices, i.tile_vpt, i.segment_cols),
                         int(i.voxels), int(i.state_bytes), i.graph_launches, float(i.autotune_ms),
                         int(i.persistent))

    def dq(self) -> np.ndarray:
        """[n_volumes, iters] max |dV|^2 of every volume and iteration of the last run."""
        out = np.zeros((self.n_volumes, self.iters), np.float32)
        check(_native.host_lib().potts_batch_read_dq(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
        return out

    def close(self) -> None:
        if getattr(self, "_h", None):
            _native.host_lib().potts_batch_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# --------------------------------------------------------------------------- differentiable solve
class Tape:
    """Forward pass with checkpoints of a differentiable solve (potts_forward_ckpt); `loss` is
    -1/|mask| sum log(V_t + eps).  The device buffers u and truth must stay valid until backward()."""

    def __init__(self, ctx: CudaContext, mapping: CylinderMapping, u_ptr: int, truth_ptr: int, ci: Sequence[float],
                 lam: float, tau1: float, tau2: float, iters: int, ckpt_every: int = 20, eps: float = 1e-3,
                 V_ptr: int = 0):
        c = _ci_array(ci)
        self.K = int(c.size)
        self._mapping = mapping
        loss = ctypes.c_double()
        h = ctypes.c_void_p()
        check(_native.host_lib().potts_forward_ckpt(
            ctx.handle, ctypes.byref(mapping.as_c()), ctypes.c_void_p(int(u_ptr)), ctypes.c_void_p(int(truth_ptr)),
            self.K, c.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), float(lam), float(tau1), float(tau2),
            int(iters), int(ckpt_every), float(eps), ctypes.c_void_p(int(V_ptr)), ctypes.byref(loss),
            ctypes.byref(h)))
        self._h = h
        self.loss = float(loss.value)

    def backward(self, grad_u_ptr: int) -> tuple[np.ndarray, float]:
        """dL/du into the device buffer at grad_u_ptr (the mapping's span); returns (dL/dc, dL/dlambda)."""
        gc = np.zeros(self.K, np.float64)
        gl = ctypes.c_double()
        check(_native.host_lib().potts_backward(self._h, ctypes.c_void_p(int(grad_u_ptr)),
                                                gc.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                                ctypes.byref(gl)))
        return gc, float(gl.value)

    def close(self) -> None:
        if getattr(self, "_h", None):
            _native.host_lib().potts_tape_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def loss_and_grad(mapping: CylinderMapping, u: np.ndarray, truth: np.ndarray, ci: Sequence[float], lam: float,
                  tau1: float, tau2: float, iters: int, *, ckpt_every: int = 20, eps: float = 1e-3,
                  ctx: Optional[CudaContext] = None):
    """Loss, dL/du (host, span), dL/dc and dL/dlambda of the unrolled solve on host arrays."""
    import torch

    own = ctx is None
    ctx = ctx or make_context(0)
    try:
        dev = torch.device("cuda", ctx.device)
        du = torch.from_numpy(np.ascontiguousarray(u, np.float32)).to(dev)
        dt = torch.from_numpy(np.ascontiguousarray(truth, np.uint8)).to(dev)
        gu = torch.zeros(mapping.span, dtype=torch.float32, device=dev)
        torch.cuda.synchronize(dev)
        with Tape(ctx, mapping, du.data_ptr(), dt.data_ptr(), ci, lam, tau1, tau2, iters, ckpt_every, eps) as t:
            gc, gl = t.backward(gu.data_ptr())
            loss = t.loss
        ctx.synchronize()
        return loss, gu.cpu().numpy(), gc, gl
    finally:
        if own:
            ctx.close()


# --------------------------------------------------------------------------- TV-L2 denoising
def tv_denoise(ctx: CudaContext, mapping: CylinderMapping, g_ptr: int, lam: float, tau: float, iters: int, *,
               variant: int = 0, stats: bool = True) -> Optional[SolveStats]:
    """chambolle() (totalvarmin/chambolle.cpp:220-276): TV-L2 denoising of the device field at g_ptr
    (the mapping's span, float32) in place; variant 0 = fused, 1 = the reference's two launches."""
    st, dq, en = _make_stats(iters, 0, stats)
    check(_native.host_lib().potts_tv_denoise(ctx.handle, ctypes.byref(mapping.as_c()), ctypes.c_void_p(int(g_ptr)),
                                              float(lam), float(tau), int(iters), int(variant),
                                              ctypes.byref(st) if stats else None))
    return _stats_out(st, dq, en) if stats else None


def tv_denoise_host(mapping: CylinderMapping, g: np.ndarray, lam: float, tau: float, iters: int, *,
                    variant: int = 0, ctx: Optional[CudaContext] = None) -> tuple[np.ndarray, SolveStats]:
    """TV-L2 denoising of a host field (float32, the mapping's span); returns (result, stats)."""
    own = ctx is None
    ctx = ctx or make_context(0)
    try:
        fld = upload(ctx, mapping, np.ascontiguousarray(g, np.float32))
        st = tv_denoise(ctx, mapping, fld.data_ptr(), lam, tau, iters, variant=variant)
        out = download(ctx, fld)
        fld.free()
        return out, st
    finally:
        if own:
            ctx.close()


# ---- label-finding inputs -----------------------------------------------------

def min_max(ctx: CudaContext, mapping: CylinderMapping, f_ptr: int, *, positive: bool = False) -> tuple[float, float]:
    """min_max() (min_max/min_max.cpp:56-81) of the device field at f_ptr over the in-mask voxels;
    positive=True: over its strictly positive values (uv-hist-kernel.cpp:70-92)."""
    lo, hi = ctypes.c_float(), ctypes.c_float()
    fn = _native.host_lib().potts_min_max_positive if positive else _native.host_lib().potts_min_max
    check(fn(ctx.handle, ctypes.byref(mapping.as_c()), ctypes.c_void_p(int(f_ptr)), ctypes.byref(lo),
             ctypes.byref(hi)))
    return lo.value, hi.value


def grad_magn(ctx: CudaContext, mapping: CylinderMapping, u_ptr: int, v_ptr: int) -> None:
    """grad_magn() (grad-magn/grad_magn.cpp:17-79): v = 0.5 |central-difference gradient of u|, -1 at
    the mask boundary; enqueued on the context's stream."""
    check(_native.host_lib().potts_grad_magn(ctx.handle, ctypes.byref(mapping.as_c()), ctypes.c_void_p(int(u_ptr)),
                                             ctypes.c_void_p(int(v_ptr))))


def calc_hist(ctx: CudaContext, mapping: CylinderMapping, f_ptr: int, range_start: float, range_end: float,
              nbins: int, *, jitter: float = 0.0, seed: int = 0) -> tuple[np.ndarray, np.ndarray]:
    """calc_hist(ctx, in, range_start, range_end, nbins, delta) (calc_hist/calc_hist.cpp:93-138):
    (counts uint32, density float64 = counts / (in-mask voxels x bin width))."""
    counts = np.zeros(int(nbins), np.uint32)
    dens = np.zeros(int(nbins), np.float64)
    check(_native.host_lib().potts_calc_hist(ctx.handle, ctypes.byref(mapping.as_c()), ctypes.c_void_p(int(f_ptr)),
                                             float(range_start), float(range_end), int(nbins), float(jitter),
                                             int(seed) & (2**64 - 1), counts.ctypes.data, dens.ctypes.data))
    return counts, dens


def calc_hist_auto(ctx: CudaContext, mapping: CylinderMapping, f_ptr: int, nbins: int, *, jitter: float = 0.0,
                   seed: int = 0) -> tuple[np.ndarray, np.ndarray, float, float]:
    """calc_hist(ctx, in, nbins, delta) (calc_hist.cpp:82-91): the histogram over [min, max] of the
    field; returns (counts, density, min, max)."""
    counts = np.zeros(int(nbins), np.uint32)
    dens = np.zeros(int(nbins), np.float64)
    lo, hi = ctypes.c_float(), ctypes.c_float()
    check(_native.host_lib().potts_calc_hist_auto(ctx.handle, ctypes.byref(mapping.as_c()),
                                                  ctypes.c_void_p(int(f_ptr)), int(nbins), float(jitter),
                                                  int(seed) & (2**64 - 1), counts.ctypes.data, dens.ctypes.data,
                                                  ctypes.byref(lo), ctypes.byref(hi)))
    return counts, dens, lo.value, hi.value


def uv_hist_matrix(hist: np.ndarray, nbins: int) -> np.ndarray:
    """The nbins x nbins view (row ybin, column xbin) of a 2-D histogram's span."""
    stride = int(_native.host_lib().potts_uv_hist_stride(int(nbins)))
    return np.lib.stride_tricks.as_strided(hist, shape=(nbins, nbins), strides=(4 * stride, 4), writeable=False)


def uv_hist(ctx: CudaContext, mapping: CylinderMapping, u_ptr: int, v_ptr: int, u_start: float, u_end: float,
            v_start: float, v_end: float, nbins: int) -> np.ndarray:
    """uv_hist(ctx, u, v, u_start, u_end, v_start, v_end, nbins) (uv-hist-kernel.cpp:100-197): the
    counts span ((nbins - 1) * stride + nbins, row ybin of v, column xbin of u)."""
    hist = np.zeros(int(_native.host_lib().potts_uv_hist_span(int(nbins))), np.uint32)
    check(_native.host_lib().potts_uv_hist(ctx.handle, ctypes.byref(mapping.as_c()), ctypes.c_void_p(int(u_ptr)),
                                           ctypes.c_void_p(int(v_ptr)), float(u_start), float(u_end), float(v_start),
                                           float(v_end), int(nbins), hist.ctypes.data))
    return hist


def uv_hist_auto(ctx: CudaContext, mapping: CylinderMapping, u_ptr: int, v_ptr: int,
                 nbins: int) -> tuple[np.ndarray, tuple[float, float, float, float]]:
    """uv_hist(ctx, u, v, nbins) (uv-hist-kernel.cpp:70-98): ranges from u's min/max and the min/max of
    v's strictly positive values; returns (counts span, (u_start, u_end, v_start, v_end))."""
    hist = np.zeros(int(_native.host_lib().potts_uv_hist_span(int(nbins))), np.uint32)
    rng = np.zeros(4, np.float32)
    check(_native.host_lib().potts_uv_hist_auto(ctx.handle, ctypes.byref(mapping.as_c()), ctypes.c_void_p(int(u_ptr)),
                                                ctypes.c_void_p(int(v_ptr)), int(nbins), hist.ctypes.data,
                                                rng.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
    return hist, tuple(float(x) for x in rng)


# ---- field archive (.bin), convert_to_fp, find_intensity_range, output writers ------------

def _elem(elem: str) -> int:
    if elem not in _native.ELEMENTS:
        raise ValueError(f"unknown element type {elem!r}; one of {sorted(_native.ELEMENTS)}")
    return _native.ELEMENTS[elem]


def _bytes_ptr(data) -> tuple[np.ndarray, int]:
    buf = np.frombuffer(data, np.uint8) if isinstance(data, (bytes, bytearray, memoryview)) else np.asarray(data)
    if buf.dtype != np.uint8 or not buf.flags.c_contiguous:
        buf = np.ascontiguousarray(buf).view(np.uint8)
    return buf, buf.ctypes.data


@dataclass
class ArchiveInfo:
    mapping: CylinderMapping
    lo: float
    hi: float
    header_bits: int
    voxels: int
    total_bytes: int


def archive_read_header(data, elem: str = "f32") -> ArchiveInfo:
    """mapping_storage::load + Field<float>::load's lo/hi (include/layout_cylinder.h:259-312,
    include/field.h:121-131): the mapping and sizes of a .bin archive (host only)."""
    buf, ptr = _bytes_ptr(data)
    lib = _native.host_lib()
    info = _native.PottsArchiveInfo()
    check(lib.potts_archive_read_header(ptr, buf.size, _elem(elem), ctypes.byref(info), None, None))
    sr = np.zeros(info.cols, np.uint32)
    bs = np.zeros(info.cols + 1, np.uint32)
    check(lib.potts_archive_read_header(ptr, buf.size, _elem(elem), ctypes.byref(info), sr.ctypes.data,
                                        bs.ctypes.data))
    m = CylinderMapping(info.n_images, info.rows, info.cols, info.nstride, info.col_begin, info.col_end, sr, bs)
    return ArchiveInfo(m, info.lo, info.hi, info.header_bits, info.voxels, info.total_bytes)


def archive_size(mapping: CylinderMapping, elem: str = "f32") -> tuple[int, int]:
    """(archive bytes, header bits) of a field with this mapping (host only)."""
    tb, hb = ctypes.c_uint64(), ctypes.c_uint64()
    check(_native.host_lib().potts_archive_size(ctypes.byref(mapping.as_c()), _elem(elem), ctypes.byref(tb),
                                                ctypes.byref(hb)))
    return int(tb.value), int(hb.value)


def archive_load(ctx: CudaContext, data, elem: str, d_ptr: int, capacity: int) -> tuple[ArchiveInfo, float]:
    """Field<T>::load (include/field.h:121-147) of host archive bytes into the device field at d_ptr
    (float32 or uint16 elements, `capacity` of them); returns (header, unpack kernel ms)."""
    buf, ptr = _bytes_ptr(data)
    info = _native.PottsArchiveInfo()
    st = _native.PottsIoStats()
    check(_native.host_lib().potts_archive_load(ctx.handle, ptr, buf.size, _elem(elem), ctypes.c_void_p(int(d_ptr)),
                                                int(capacity), ctypes.byref(info), ctypes.byref(st)))
    hdr = archive_read_header(buf, elem)
    return hdr, st.kernel_ms


def archive_save(ctx: CudaContext, mapping: CylinderMapping, elem: str, d_ptr: int, lo: float = 0.0, hi: float = 0.0,
                 out: Optional[np.ndarray] = None) -> tuple[np.ndarray, float]:
    """Field<T>::save (include/field.h:92-119) of the device field at d_ptr: (archive bytes as uint8 array,
    pack kernel ms).  `out` (uint8, e.g. pinned) receives the bytes when given."""
    lib = _native.host_lib()
    n = ctypes.c_uint64()
    mc = mapping.as_c()
    check(lib.potts_archive_save(ctx.handle, ctypes.byref(mc), _elem(elem), None, 0.0, 0.0, None, 0, ctypes.byref(n),
                                 None))
    if out is None:
        out = np.zeros(int(n.value), np.uint8)
    st = _native.PottsIoStats()
    check(lib.potts_archive_save(ctx.handle, ctypes.byref(mc), _elem(elem), ctypes.c_void_p(int(d_ptr)), float(lo),
                                 float(hi), out.ctypes.data, out.size, ctypes.byref(n), ctypes.byref(st)))
    return out[: int(n.value)], st.kernel_ms


def convert_to_fp(ctx: CudaContext, mapping: CylinderMapping, elem: str, in_ptr: int, lo: float, hi: float,
                  out_ptr: int) -> None:
    """convert_to_fp(ctx, in, lo, hi) (transpose/convert_to_fp.cpp:11-79) into the float32 field at
    out_ptr; enqueued on the context's stream."""
    check(_native.host_lib().potts_convert_to_fp(ctx.handle, ctypes.byref(mapping.as_c()), _elem(elem),
                                                 ctypes.c_void_p(int(in_ptr)), float(lo), float(hi),
                                                 ctypes.c_void_p(int(out_ptr))))


def find_intensity_range(ctx: CudaContext, mapping: CylinderMapping, u16_ptr: int,
                         tail_thr: float) -> tuple[int, int, np.ndarray]:
    """find_intensity_range(ctx, field, tail_thr) (transpose/find_intensity_range.cpp:64-110) of a
    uint16 device field: (lo, hi, the 65536 counts)."""
    lo, hi = ctypes.c_uint16(), ctypes.c_uint16()
    hist = np.zeros(65536, np.uint64)
    check(_native.host_lib().potts_find_intensity_range(ctx.handle, ctypes.byref(mapping.as_c()),
                                                        ctypes.c_void_p(int(u16_ptr)), float(tail_thr),
                                                        ctypes.byref(lo), ctypes.byref(hi), hist.ctypes.data))
    return int(lo.value), int(hi.value), hist


def raw_labels_dims(mapping: CylinderMapping) -> tuple[int, int, int, int]:
    """(slices, rows, cols, row_begin) of the raw label box (potts-model.cpp:186-202); host only."""
    v = [ctypes.c_uint32() for _ in range(4)]
    check(_native.host_lib().potts_raw_labels_dims(ctypes.byref(mapping.as_c()), *[ctypes.byref(x) for x in v]))
    return tuple(int(x.value) for x in v)


def raw_labels(ctx: CudaContext, mapping: CylinderMapping, f_ptr: int, box_ptr: int) -> None:
    """The raw label box (potts-model.cpp:203-217) into device bytes at box_ptr (cols x rows x slices)."""
    check(_native.host_lib().potts_raw_labels(ctx.handle, ctypes.byref(mapping.as_c()), ctypes.c_void_p(int(f_ptr)),
                                              ctypes.c_void_p(int(box_ptr))))


def vtk_labels(ctx: CudaContext, mapping: CylinderMapping, f_ptr: int,
               out: Optional[np.ndarray] = None) -> tuple[np.ndarray, float]:
    """The --rawout VTK file (potts-model.cpp:184-243) of the device field at f_ptr: (file bytes, box
    kernel ms)."""
    lib = _native.host_lib()
    n = ctypes.c_uint64()
    mc = mapping.as_c()
    check(lib.potts_vtk_labels(ctx.handle, ctypes.byref(mc), ctypes.c_void_p(int(f_ptr)), None, 0, ctypes.byref(n),
                               None))
    if out is None:
        out = np.zeros(int(n.value), np.uint8)
    st = _native.PottsIoStats()
    check(lib.potts_vtk_labels(ctx.handle, ctypes.byref(mc), ctypes.c_void_p(int(f_ptr)), out.ctypes.data, out.size,
                               ctypes.byref(n), ctypes.byref(st)))
    return out[: int(n.value)], st.kernel_ms


def write_vtk_labels(ctx: CudaContext, mapping: CylinderMapping, f_ptr: int, path) -> None:
    """Writes the --rawout file of potts-model (potts-model.cpp:184-243) to `path`."""
    data, _ = vtk_labels(ctx, mapping, f_ptr)
    with open(path, "wb") as fh:
        fh.write(data.tobytes())


def png_slice(ctx: CudaContext, mapping: CylinderMapping, f_ptr: int, col: int) -> bytes:
    """write_png's image of column `col` (potts-model.cpp:34-49) as PNG bytes."""
    lib = _native.host_lib()
    n = ctypes.c_uint64()
    mc = mapping.as_c()
    check(lib.potts_png_slice(ctx.handle, ctypes.byref(mc), ctypes.c_void_p(int(f_ptr)), int(col), None, 0,
                              ctypes.byref(n)))
    out = np.zeros(int(n.value), np.uint8)
    check(lib.potts_png_slice(ctx.handle, ctypes.byref(mc), ctypes.c_void_p(int(f_ptr)), int(col), out.ctypes.data,
                              out.size, ctypes.byref(n)))
    return out.tobytes()


def png_slice_name(col: int, lam: float) -> str:
    """The file name write_png uses (potts-model.cpp:48): "slice-{col} (𝜆 = {lam:07.3f}).png"."""
    return f"slice-{int(col)} (\U0001d706 = {float(lam):07.3f}).png"


def write_png(ctx: CudaContext, mapping: CylinderMapping, f_ptr: int, col: int, lam: float, directory=".") -> str:
    """write_png(img, col, lambda) (potts-model.cpp:34-49): writes the slice PNG under the reference's
    file name in `directory`; returns the path."""
    import os

    path = os.path.join(str(directory), png_slice_name(col, lam))
    with open(path, "wb") as fh:
        fh.write(png_slice(ctx, mapping, f_ptr, col))
    return path
