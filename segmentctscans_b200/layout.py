"""Cylindrical-core volume layout (host side).

Mirrors ``layout_cylinder::mapping`` / ``mapping_storage`` of the reference
(include/layout_cylinder.h:22-322) and ``Field<float>`` strides
(include/field.h:37-45): voxel (n, row, col) lives at
``base[col] + (row - start_row[col]) * nstride + n``; only rows strictly inside
the circle (col - xc)^2 + (row - yc)^2 < r^2 are stored.  The mask tables are
built by the native library (``potts_cylinder_mapping``), so the host code and
the kernels share one definition.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import _native


def get_stride(n: int) -> int:
    """Field<float>::get_stride (include/field.h:37-40): n rounded up to 128 bytes of floats."""
    return ((int(n) + 31) // 32) * 32


def prev_stride(n: int) -> int:
    """Field<float>::prev_stride (include/field.h:42-45)."""
    return (int(n) // 32) * 32


@dataclass
class CylinderMapping:
    n_images: int
    rows: int
    cols: int
    nstride: int
    col_begin: int
    col_end: int
    start_row: np.ndarray  # uint32 [cols]
    base: np.ndarray       # uint32 [cols + 1]
    _c: object = field(default=None, repr=False, compare=False)

    @classmethod
    def cylinder(cls, n_images: int, rows: int, cols: int, r: float, xc: float | None = None,
                 yc: float | None = None, nstride: int | None = None) -> "CylinderMapping":
        """Mask constructor (include/layout_cylinder.h:152-195).  The centre
        defaults to ((cols-1)/2, (rows-1)/2); nstride to get_stride(n_images)."""
        xc = (cols - 1) / 2.0 if xc is None else float(xc)
        yc = (rows - 1) / 2.0 if yc is None else float(yc)
        nstride = get_stride(n_images) if nstride is None else int(nstride)
        start_row = np.zeros(cols, dtype=np.uint32)
        base = np.zeros(cols + 1, dtype=np.uint32)
        cb = ctypes.c_uint32()
        ce = ctypes.c_uint32()
        lib = _native.host_lib()
        lib.potts_cylinder_mapping(rows, cols, xc, yc, float(r), nstride,
                                   start_row.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)),
                                   base.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)),
                                   ctypes.byref(cb), ctypes.byref(ce))
        return cls(int(n_images), int(rows), int(cols), nstride, int(cb.value), int(ce.value), start_row, base)

    # -- layout_cylinder::mapping accessors (include/layout_cylinder.h:86-101)
    @property
    def span(self) -> int:
        """required_span_size(): floats of storage."""
        return int(self.base[self.cols])

    @property
    def n_lines(self) -> int:
        return self.span // self.nstride

    def row_begin(self, col: int) -> int:
        return int(self.start_row[col])

    def row_end(self, col: int) -> int:
        return int(self.start_row[col]) + int(self.base[col + 1] - self.base[col]) // self.nstride

    @property
    def data_size(self) -> int:
        """In-mask voxels: stored lines x n_images."""
        return self.n_lines * self.n_images

    def offset(self, n, row, col):
        return self.base[col].astype(np.int64) + (np.asarray(row, np.int64) - self.start_row[col]) * self.nstride + n

    def lines(self) -> tuple[np.ndarray, np.ndarray]:
        """(row, col) of every stored line, in storage order."""
        rows, cols = [], []
        for col in range(self.col_begin, self.col_end):
            rb, re = self.row_begin(col), self.row_end(col)
            rows.append(np.arange(rb, re, dtype=np.int64))
            cols.append(np.full(re - rb, col, dtype=np.int64))
        if not rows:
            return np.zeros(0, np.int64), np.zeros(0, np.int64)
        return np.concatenate(rows), np.concatenate(cols)

    def with_slab_width(self, slab_w: int, nstride: int | None = None) -> "CylinderMapping":
        """mapping_storage(other, slab_w, nstride) (include/layout_cylinder.h:137-149)."""
        nstride = get_stride(slab_w) if nstride is None else int(nstride)
        base = ((self.base // self.nstride) * nstride).astype(np.uint32)
        return CylinderMapping(int(slab_w), self.rows, self.cols, nstride, self.col_begin, self.col_end,
                               self.start_row.copy(), base)

    # -- conversions between the cylinder layout and a dense (col, row, n) box
    def gather(self, box: np.ndarray) -> np.ndarray:
        """Dense box[col, row, n] (n_images along the last axis) -> span array."""
        out = np.zeros(self.span, dtype=box.dtype)
        rows, cols = self.lines()
        lines = box[cols, rows, :]  # [n_lines, n_images]
        out.reshape(self.n_lines, self.nstride)[:, : self.n_images] = lines
        return out

    def scatter(self, values: np.ndarray, fill=0) -> np.ndarray:
        """Span array -> dense box[col, row, n]; voxels outside the mask get `fill`."""
        box = np.full((self.cols, self.rows, self.n_images), fill, dtype=values.dtype)
        rows, cols = self.lines()
        box[cols, rows, :] = values.reshape(self.n_lines, self.nstride)[:, : self.n_images]
        return box

    def mask_values(self, values: np.ndarray) -> np.ndarray:
        """In-mask voxels of span arrays (padding n >= n_images dropped): [..., n_lines, n_images]."""
        v = np.asarray(values)
        return v.reshape(*v.shape[:-1], self.n_lines, self.nstride)[..., : self.n_images]

    def as_c(self) -> "_native.PottsMapping":
        """A potts_mapping struct pointing into this object's tables (kept alive here)."""
        self.start_row = np.ascontiguousarray(self.start_row, dtype=np.uint32)
        self.base = np.ascontiguousarray(self.base, dtype=np.uint32)
        m = _native.PottsMapping()
        m.n_images, m.rows, m.cols = self.n_images, self.rows, self.cols
        m.nstride, m.col_begin, m.col_end = self.nstride, self.col_begin, self.col_end
        m.start_row = self.start_row.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))
        m.base = self.base.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))
        self._c = m
        return m
