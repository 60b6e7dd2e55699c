"""ctypes wrapper of the CPU oracle (test infrastructure only).

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of bench.py
use this module, as the checker.  The restated algorithm lives in
``potts_oracle.c`` (FP64 and FP32 builds), ``cylinder_oracle.c``, ``label_oracle.c`` and
``fieldio_oracle.c``; see their
headers for the reference lines each function follows.  Parity unpinned: the
reference has no tests or golden vectors for this path and cannot be built
here.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Optional

import numpy as np

from .build import LIB_PATH, build_oracle


class OCyl(ctypes.Structure):
    _fields_ = [
        ("n_images", ctypes.c_uint32), ("rows", ctypes.c_uint32), ("cols", ctypes.c_uint32),
        ("nstride", ctypes.c_uint32), ("col_begin", ctypes.c_uint32), ("col_end", ctypes.c_uint32),
        ("start_row", ctypes.POINTER(ctypes.c_uint32)), ("base", ctypes.POINTER(ctypes.c_uint32)),
    ]


_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build_oracle()
        _lib = ctypes.CDLL(str(LIB_PATH))
    return _lib


def _ptr(a, ct):
    return a.ctypes.data_as(ctypes.POINTER(ct)) if a is not None else None


def _real(precision: str):
    if precision == "f64":
        return np.float64, ctypes.c_double
    if precision == "f32":
        return np.float32, ctypes.c_float
    raise ValueError(precision)


def set_threads(n: int) -> None:
    lib().oracle_set_threads(int(n))


def max_threads() -> int:
    return int(lib().oracle_max_threads())


def ocyl(m) -> OCyl:
    sr = np.ascontiguousarray(m.start_row, dtype=np.uint32)
    bs = np.ascontiguousarray(m.base, dtype=np.uint32)
    c = OCyl(m.n_images, m.rows, m.cols, m.nstride, m.col_begin, m.col_end, _ptr(sr, ctypes.c_uint32),
             _ptr(bs, ctypes.c_uint32))
    c._keep = (sr, bs)
    return c


def cylinder_mask(rows: int, cols: int, xc: float, yc: float, r: float, nstride: int):
    """(start_row, base, col_begin, col_end, span) per include/layout_cylinder.h:152-195."""
    sr = np.zeros(cols, np.uint32)
    bs = np.zeros(cols + 1, np.uint32)
    cb, ce = ctypes.c_uint32(), ctypes.c_uint32()
    f = lib().oracle_cylinder_mask
    f.restype = ctypes.c_uint64
    f.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                  ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint32),
                  ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint32)]
    span = f(rows, cols, xc, yc, r, nstride, _ptr(sr, ctypes.c_uint32), _ptr(bs, ctypes.c_uint32),
             ctypes.byref(cb), ctypes.byref(ce))
    return sr, bs, int(cb.value), int(ce.value), int(span)


def project_simplex(q: np.ndarray, precision: str = "f64") -> np.ndarray:
    dt, ct = _real(precision)
    out = np.ascontiguousarray(np.array(q, dtype=dt))
    f = getattr(lib(), f"oracle_project_simplex_{precision}")
    f.argtypes = [ctypes.POINTER(ct), ctypes.c_int]
    f(_ptr(out, ct), int(out.size))
    return out


def project_K(q: np.ndarray, precision: str = "f64") -> tuple[np.ndarray, int]:
    """q: [K, 3] -> (projected [K, 3], sweeps)."""
    dt, ct = _real(precision)
    out = np.ascontiguousarray(np.array(q, dtype=dt).reshape(-1, 3))
    f = getattr(lib(), f"oracle_project_K_{precision}")
    f.argtypes = [ctypes.POINTER(ct), ctypes.c_int]
    f.restype = ctypes.c_int
    sw = f(_ptr(out, ct), int(out.shape[0]))
    return out, int(sw)


@dataclass
class OracleResult:
    res: np.ndarray
    labels: np.ndarray
    V: Optional[np.ndarray]
    Xi: Optional[np.ndarray]
    dq_trace: np.ndarray
    energy_trace: Optional[np.ndarray]
    sweep_hist: np.ndarray


STORE = {"f32": 0, "native": 0, "bf16": 1, "f16": 2}


def solve(m, u: np.ndarray, ci, lam: float, tau1: float, tau2: float, iters: int, *, precision: str = "f64",
          slab_w: int = 0, want_state: bool = True, gap_every: int = 0, store: str = "native") -> OracleResult:
    """The whole solve (potts-model/potts-min-partition.cpp:540-679) on the CPU.

    `store` models reduced-precision storage of the state: "bf16" or "f16" round every stored value
    of Xi, V and Vbar to that format (to nearest, ties to even), except the stored V of "bf16", which
    is rounded stochastically with bits from a counter hash of (line, n, iteration, component pair)."""
    dt, ct = _real(precision)
    K = len(ci)
    span = int(m.base[m.cols])
    c = np.ascontiguousarray(np.asarray(ci, np.float32))
    u = np.ascontiguousarray(u, dtype=np.float32)
    if u.size != span:
        raise ValueError("u size != span")
    res = np.zeros(span, np.float32)
    labels = np.zeros(span, np.uint8)
    V = np.zeros((K - 1, span), dt) if want_state else None
    Xi = np.zeros((3 * (K - 1), span), dt) if want_state else None
    dq = np.zeros(max(iters, 1), np.float32)
    ne = iters // gap_every if gap_every > 0 else 0
    en = np.zeros((max(ne, 1), 3), np.float64) if ne > 0 else None
    hist = np.zeros(21, np.int32)
    f = getattr(lib(), f"oracle_solve_store_{precision}")
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.POINTER(OCyl), ctypes.POINTER(ctypes.c_float), ctypes.c_int, ctypes.POINTER(ctypes.c_float),
                  ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_int, ctypes.c_int,
                  ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_uint8), ctypes.POINTER(ct),
                  ctypes.POINTER(ct), ctypes.POINTER(ctypes.c_float), ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                  ctypes.POINTER(ctypes.c_int), ctypes.c_int]
    oc = ocyl(m)
    rc = f(ctypes.byref(oc), _ptr(u, ctypes.c_float), K, _ptr(c, ctypes.c_float), float(lam), float(tau1),
           float(tau2), int(iters), int(slab_w), _ptr(res, ctypes.c_float), _ptr(labels, ctypes.c_uint8),
           _ptr(V, ct), _ptr(Xi, ct), _ptr(dq, ctypes.c_float), int(gap_every), _ptr(en, ctypes.c_double),
           _ptr(hist, ctypes.c_int), STORE[store])
    if rc != 0:
        raise RuntimeError("oracle_solve failed (bad arguments or slab planner)")
    return OracleResult(res, labels, V, Xi, dq[:iters], en, hist)


def grad_step(m, K: int, xi: np.ndarray, Vb: np.ndarray, tau2: float, precision: str = "f64") -> np.ndarray:
    dt, ct = _real(precision)
    xi = np.ascontiguousarray(xi, dtype=dt).copy()
    Vb = np.ascontiguousarray(Vb, dtype=dt)
    f = getattr(lib(), f"oracle_grad_step_{precision}")
    f.argtypes = [ctypes.POINTER(OCyl), ctypes.c_int, ctypes.POINTER(ct), ctypes.POINTER(ct), ctypes.c_float]
    oc = ocyl(m)
    f(ctypes.byref(oc), K, _ptr(xi, ct), _ptr(Vb, ct), float(tau2))
    return xi


def div_step(m, K: int, xi, V, u, ci, lam, tau1, precision: str = "f64"):
    """One primal step: returns (V_new, Vbar_new, max |dV|^2)."""
    dt, ct = _real(precision)
    xi = np.ascontiguousarray(xi, dtype=dt)
    V = np.ascontiguousarray(V, dtype=dt).copy()
    Vb = np.zeros_like(V)
    u = np.ascontiguousarray(u, dtype=np.float32)
    c = np.ascontiguousarray(np.asarray(ci, np.float32))
    f = getattr(lib(), f"oracle_div_step_{precision}")
    f.restype = ct
    f.argtypes = [ctypes.POINTER(OCyl), ctypes.c_int, ctypes.POINTER(ct), ctypes.POINTER(ct), ctypes.POINTER(ct),
                  ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float), ctypes.c_float, ctypes.c_float]
    oc = ocyl(m)
    dq = f(ctypes.byref(oc), K, _ptr(xi, ct), _ptr(V, ct), _ptr(Vb, ct), _ptr(u, ctypes.c_float),
           _ptr(c, ctypes.c_float), float(lam), float(tau1))
    return V, Vb, float(dq)


def div_step_cols(m, K: int, xi, V, u, ci, lam, tau1, col_lo: int, col_hi: int, precision: str = "f64"):
    """One primal step over every column; the returned max |dV|^2 covers the columns [col_lo, col_hi)
    only (the owned columns of a shard)."""
    dt, ct = _real(precision)
    xi = np.ascontiguousarray(xi, dtype=dt)
    V = np.ascontiguousarray(V, dtype=dt).copy()
    Vb = np.zeros_like(V)
    u = np.ascontiguousarray(u, dtype=np.float32)
    c = np.ascontiguousarray(np.asarray(ci, np.float32))
    f = getattr(lib(), f"oracle_div_step_cols_{precision}")
    f.restype = ct
    f.argtypes = [ctypes.POINTER(OCyl), ctypes.c_int, ctypes.POINTER(ct), ctypes.POINTER(ct), ctypes.POINTER(ct),
                  ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float), ctypes.c_float, ctypes.c_float,
                  ctypes.c_int64, ctypes.c_int64]
    oc = ocyl(m)
    dq = f(ctypes.byref(oc), K, _ptr(xi, ct), _ptr(V, ct), _ptr(Vb, ct), _ptr(u, ctypes.c_float),
           _ptr(c, ctypes.c_float), float(lam), float(tau1), int(col_lo), int(col_hi))
    return V, Vb, float(dq)


def energies_cols(m, K: int, xi, V, u, ci, lam, col_lo: int, col_hi: int, precision: str = "f64") -> np.ndarray:
    """(lagrangian, dual, gap) in FP64 over the voxels of the columns [col_lo, col_hi)."""
    dt, ct = _real(precision)
    xi = np.ascontiguousarray(xi, dtype=dt)
    V = np.ascontiguousarray(V, dtype=dt)
    u = np.ascontiguousarray(u, dtype=np.float32)
    c = np.ascontiguousarray(np.asarray(ci, np.float32))
    out = np.zeros(3, np.float64)
    f = getattr(lib(), f"oracle_energies_cols_{precision}")
    f.argtypes = [ctypes.POINTER(OCyl), ctypes.c_int, ctypes.POINTER(ct), ctypes.POINTER(ct),
                  ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float), ctypes.c_float, ctypes.c_int64,
                  ctypes.c_int64, ctypes.POINTER(ctypes.c_double)]
    oc = ocyl(m)
    f(ctypes.byref(oc), K, _ptr(xi, ct), _ptr(V, ct), _ptr(u, ctypes.c_float), _ptr(c, ctypes.c_float), float(lam),
      int(col_lo), int(col_hi), _ptr(out, ctypes.c_double))
    return out


def energies(m, K: int, xi, V, u, ci, lam, precision: str = "f64") -> np.ndarray:
    """(lagrangian, dual, gap) in FP64."""
    dt, ct = _real(precision)
    xi = np.ascontiguousarray(xi, dtype=dt)
    V = np.ascontiguousarray(V, dtype=dt)
    u = np.ascontiguousarray(u, dtype=np.float32)
    c = np.ascontiguousarray(np.asarray(ci, np.float32))
    out = np.zeros(3, np.float64)
    f = getattr(lib(), f"oracle_energies_{precision}")
    f.argtypes = [ctypes.POINTER(OCyl), ctypes.c_int, ctypes.POINTER(ct), ctypes.POINTER(ct),
                  ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float), ctypes.c_float,
                  ctypes.POINTER(ctypes.c_double)]
    oc = ocyl(m)
    f(ctypes.byref(oc), K, _ptr(xi, ct), _ptr(V, ct), _ptr(u, ctypes.c_float), _ptr(c, ctypes.c_float), float(lam),
      _ptr(out, ctypes.c_double))
    return out


def tv(m, g: np.ndarray, lam: float, tau: float, iters: int, precision: str = "f64"):
    """TV-L2 denoising by Chambolle's projection algorithm (totalvarmin/chambolle.cpp:220-276) on the
    CPU: returns (the denoised field, float32 over the span; the per-iteration max |dxi|^2)."""
    _, ct = _real(precision)
    out = np.ascontiguousarray(g, dtype=np.float32).copy()
    dq = np.zeros(max(iters, 1), np.float32)
    f = getattr(lib(), f"oracle_tv_{precision}")
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.POINTER(OCyl), ctypes.POINTER(ctypes.c_float), ctypes.c_float, ctypes.c_float,
                  ctypes.c_int, ctypes.POINTER(ctypes.c_float)]
    oc = ocyl(m)
    if f(ctypes.byref(oc), _ptr(out, ctypes.c_float), float(lam), float(tau), int(iters),
         _ptr(dq, ctypes.c_float)) != 0:
        raise RuntimeError("oracle_tv failed")
    return out, dq[:iters]


# ---- label-finding inputs (label_oracle.c) ----------------------------------

def _fptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def _uptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))


def min_max(m, f: np.ndarray, positive: bool = False):
    """min_max (min_max/min_max.cpp:18-54) or, positive, the min/max of the strictly positive values
    (uv-hist-kernel.cpp:29-68) over the in-mask voxels."""
    f = np.ascontiguousarray(f, dtype=np.float32)
    out = np.zeros(2, np.float32)
    fn = lib().oracle_min_max
    fn.argtypes = [ctypes.POINTER(OCyl), ctypes.POINTER(ctypes.c_float), ctypes.c_int, ctypes.POINTER(ctypes.c_float)]
    oc = ocyl(m)
    fn(ctypes.byref(oc), _fptr(f), int(bool(positive)), _fptr(out))
    return float(out[0]), float(out[1])


def grad_magn(m, u: np.ndarray) -> np.ndarray:
    """grad_magn (grad-magn/grad_magn.cpp:17-58): the span, in-mask voxels written, others 0."""
    u = np.ascontiguousarray(u, dtype=np.float32)
    v = np.zeros_like(u)
    fn = lib().oracle_grad_magn
    fn.argtypes = [ctypes.POINTER(OCyl), ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float)]
    oc = ocyl(m)
    fn(ctypes.byref(oc), _fptr(u), _fptr(v))
    return v


def calc_hist(m, f: np.ndarray, range_start: float, range_end: float, nbins: int, jitter: float = 0.0,
              seed: int = 0) -> np.ndarray:
    """calc_hist counts (calc_hist/calc_hist.cpp:23-80), jitter from (seed, voxel)."""
    f = np.ascontiguousarray(f, dtype=np.float32)
    counts = np.zeros(nbins, np.uint32)
    fn = lib().oracle_calc_hist
    fn.argtypes = [ctypes.POINTER(OCyl), ctypes.POINTER(ctypes.c_float), ctypes.c_float, ctypes.c_float,
                   ctypes.c_uint32, ctypes.c_float, ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint32)]
    oc = ocyl(m)
    fn(ctypes.byref(oc), _fptr(f), float(range_start), float(range_end), int(nbins), float(jitter),
       int(seed) & (2**64 - 1), _uptr(counts))
    return counts


def uv_stride(nbins: int) -> int:
    return (nbins + 31) // 32 * 32


def uv_hist(m, u: np.ndarray, v: np.ndarray, u_start: float, u_end: float, v_start: float, v_end: float,
            nbins: int) -> np.ndarray:
    """uv_hist counts (uv-hist/uv-hist-kernel.cpp:100-197): (nbins - 1) * stride + nbins values,
    row ybin (v), column xbin (u)."""
    u = np.ascontiguousarray(u, dtype=np.float32)
    v = np.ascontiguousarray(v, dtype=np.float32)
    stride = uv_stride(nbins)
    hist = np.zeros((nbins - 1) * stride + nbins, np.uint32)
    fn = lib().oracle_uv_hist
    fn.argtypes = [ctypes.POINTER(OCyl), ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float),
                   ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_uint32, ctypes.c_uint32,
                   ctypes.POINTER(ctypes.c_uint32)]
    oc = ocyl(m)
    fn(ctypes.byref(oc), _fptr(u), _fptr(v), float(u_start), float(u_end), float(v_start), float(v_end), int(nbins),
       stride, _uptr(hist))
    return hist


# ---- field archive, convert_to_fp, intensity range, writers (fieldio_oracle.c) ----------

ELEM_BITS = {"f32": 32, "u16": 16}


def archive_encode(m, field: np.ndarray, elem: str = "f32", lo: float = 0.0, hi: float = 0.0) -> tuple[bytes, int]:
    """Field<T>::save (include/field.h:92-119): (archive bytes, header bits).  `field` is the span
    (float32 or uint16)."""
    bits = ELEM_BITS[elem]
    raw = np.ascontiguousarray(field, dtype=np.float32 if bits == 32 else np.uint16)
    fn = lib().oracle_archive_encode
    fn.restype = ctypes.c_uint64
    fn.argtypes = [ctypes.POINTER(OCyl), ctypes.c_int, ctypes.c_void_p, ctypes.c_float, ctypes.c_float,
                   ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint64)]
    oc = ocyl(m)
    hb = ctypes.c_uint64()
    n = fn(ctypes.byref(oc), bits, raw.ctypes.data, float(lo), float(hi), None, ctypes.byref(hb))
    out = np.zeros(int(n), np.uint8)
    fn(ctypes.byref(oc), bits, raw.ctypes.data, float(lo), float(hi), out.ctypes.data, ctypes.byref(hb))
    return out.tobytes(), int(hb.value)


@dataclass
class ArchiveContents:
    mapping: object
    lo: float
    hi: float
    header_bits: int
    field: np.ndarray  # the span, float32 or uint16; padding slices 0


def archive_decode(data: bytes, elem: str = "f32") -> ArchiveContents:
    """Field<T>::load (include/field.h:121-147, include/layout_cylinder.h:259-312)."""
    from segmentctscans_b200.layout import CylinderMapping

    bits = ELEM_BITS[elem]
    buf = np.frombuffer(data, np.uint8)
    fn = lib().oracle_archive_decode
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int, ctypes.POINTER(ctypes.c_uint32),
                   ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_float),
                   ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint64)]
    hdr = np.zeros(6, np.uint32)
    hb = ctypes.c_uint64()
    if fn(buf.ctypes.data, buf.size, bits, _uptr(hdr), None, None, None, None, ctypes.byref(hb)) != 0:
        raise ValueError("archive header is malformed or truncated")
    cols = int(hdr[2])
    sr = np.zeros(cols, np.uint32)
    bs = np.zeros(cols + 1, np.uint32)
    lohi = np.zeros(2, np.float32)
    if fn(buf.ctypes.data, buf.size, bits, _uptr(hdr), _uptr(sr), _uptr(bs), _fptr(lohi), None, None) != 0:
        raise ValueError("archive header is malformed or truncated")
    m = CylinderMapping(int(hdr[0]), int(hdr[1]), cols, int(hdr[3]), int(hdr[4]), int(hdr[5]), sr, bs)
    field = np.zeros(m.span, np.float32 if bits == 32 else np.uint16)
    if fn(buf.ctypes.data, buf.size, bits, _uptr(hdr), _uptr(sr), _uptr(bs), _fptr(lohi), field.ctypes.data,
          ctypes.byref(hb)) != 0:
        raise ValueError("archive ends inside the voxel payload")
    return ArchiveContents(m, float(lohi[0]), float(lohi[1]), int(hb.value), field)


def convert_to_fp(m, field: np.ndarray, lo: float, hi: float) -> np.ndarray:
    """convert_to_fp_kernel (transpose/convert_to_fp.cpp:11-47) of a float32 or uint16 span; other
    entries 0."""
    bits = 16 if field.dtype == np.uint16 else 32
    raw = np.ascontiguousarray(field, dtype=np.uint16 if bits == 16 else np.float32)
    out = np.zeros(raw.size, np.float32)
    fn = lib().oracle_convert_to_fp
    fn.argtypes = [ctypes.POINTER(OCyl), ctypes.c_int, ctypes.c_void_p, ctypes.c_float, ctypes.c_float,
                   ctypes.POINTER(ctypes.c_float)]
    oc = ocyl(m)
    fn(ctypes.byref(oc), bits, raw.ctypes.data, float(lo), float(hi), _fptr(out))
    return out


def intensity_range(m, field: np.ndarray, tail: float) -> tuple[int, int, np.ndarray]:
    """find_intensity_range (transpose/find_intensity_range.cpp:22-110): (lo, hi, 65536 counts)."""
    raw = np.ascontiguousarray(field, dtype=np.uint16)
    hist = np.zeros(65536, np.uint64)
    fh = lib().oracle_u16_hist
    fh.argtypes = [ctypes.POINTER(OCyl), ctypes.c_void_p, ctypes.c_void_p]
    oc = ocyl(m)
    fh(ctypes.byref(oc), raw.ctypes.data, hist.ctypes.data)
    lo, hi = ctypes.c_uint16(), ctypes.c_uint16()
    fr = lib().oracle_intensity_range
    fr.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.POINTER(ctypes.c_uint16), ctypes.POINTER(ctypes.c_uint16)]
    fr(hist.ctypes.data, float(tail), ctypes.byref(lo), ctypes.byref(hi))
    return int(lo.value), int(hi.value), hist


def raw_box(m, field: np.ndarray) -> tuple[np.ndarray, tuple[int, int, int, int]]:
    """The --rawout label box (potts-model/potts-model.cpp:184-217): (bytes [cols, rows, slices],
    (slices, rows, cols, row_begin))."""
    f = np.ascontiguousarray(field, dtype=np.float32)
    dims = np.zeros(4, np.uint32)
    fn = lib().oracle_raw_box
    fn.argtypes = [ctypes.POINTER(OCyl), ctypes.POINTER(ctypes.c_float), ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint32)]
    oc = ocyl(m)
    fn(ctypes.byref(oc), _fptr(f), None, _uptr(dims))
    out = np.zeros(int(dims[0]) * int(dims[1]) * int(dims[2]), np.uint8)
    fn(ctypes.byref(oc), _fptr(f), out.ctypes.data, _uptr(dims))
    return out.reshape(int(dims[2]), int(dims[1]), int(dims[0])), tuple(int(x) for x in dims)


def vtk_file(m, field: np.ndarray) -> bytes:
    """The whole --rawout file (potts-model.cpp:218-241) around the oracle's raw box."""
    box, (s, r, c, _) = raw_box(m, field)
    head = ("<?xml version=\"1.0\"?>\n"
            "<VTKFile type=\"ImageData\" byte_order=\"LittleEndian\">\n"
            f"  <ImageData WholeExtent=\"0 {s - 1} 0 {r - 1} 0 {c - 1}\">\n"
            f"    <Piece Extent=\"0 {s - 1} 0 {r - 1} 0 {c - 1}\">\n"
            "      <PointData Scalars=\"labels\">\n"
            "        <DataArray type=\"UInt8\" Name=\"labels\" format=\"appended\" offset=\"0\"/>\n"
            "      </PointData>\n"
            "    </Piece>\n"
            "  </ImageData>\n"
            "  <AppendedData encoding=\"raw\">\n_")
    return (head.encode() + np.uint32(box.size & 0xffffffff).tobytes() + box.tobytes()
            + b"\n  </AppendedData>\n</VTKFile>\n")


def png_gray(m, field: np.ndarray, col: int) -> np.ndarray:
    """write_png's grey levels (potts-model/potts-model.cpp:34-49) of column col: [rows, n_images]."""
    f = np.ascontiguousarray(field, dtype=np.float32)
    rows = m.row_end(col) - m.row_begin(col)
    pix = np.zeros((rows, m.n_images), np.uint8)
    fn = lib().oracle_png_gray
    fn.argtypes = [ctypes.POINTER(OCyl), ctypes.POINTER(ctypes.c_float), ctypes.c_uint32, ctypes.c_void_p]
    oc = ocyl(m)
    fn(ctypes.byref(oc), _fptr(f), int(col), pix.ctypes.data)
    return pix
