"""CPU checks of the native library: it loads, exports the C ABI, and its host-side
layout code agrees with the oracle.  No GPU work here."""
import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

from segmentctscans_b200 import _native
from segmentctscans_b200.layout import CylinderMapping, get_stride

HEADER = Path(__file__).resolve().parents[1] / "include" / "potts_b200.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(potts_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(native_lib):
    names = declared_functions()
    assert len(names) >= 19
    for name in names:
        assert hasattr(native_lib, name), name
    assert set(names) == set(_native.SIGNATURES), "binding table and header disagree"


def test_library_is_built_for_sm100a_only():
    from segmentctscans_b200.build import COMPILE_FLAGS, LINK_FLAGS

    assert "arch=compute_100a,code=sm_100a" in COMPILE_FLAGS
    assert "arch=compute_100a,code=sm_100a" in LINK_FLAGS
    assert "-fmad=false" in COMPILE_FLAGS


def test_status_strings(native_lib):
    assert native_lib.potts_status_string(0) == b"ok"
    assert b"memory" in native_lib.potts_status_string(2)
    assert native_lib.potts_get_stride(1) == 32 and native_lib.potts_get_stride(33) == 64
    assert native_lib.potts_context_launches(None) == 0


def test_default_options(native_lib):
    o = _native.default_options()
    assert (o.variant, o.storage, o.gap_every, o.slab_w, o.track_dq, o.sync_monitor) == (0, 0, 0, 0, 1, 0)
    with pytest.raises(TypeError):
        _native.default_options(nope=1)


@pytest.mark.parametrize("geom", [
    (64, 64, 31.5, None, None), (128, 128, 60.0, None, None), (768, 768, 370.0, None, None),
    (20, 30, 10.0, 14.0, 9.0),     # rows exactly on the circle are dropped
    (17, 13, 40.0, None, None),    # circle larger than the image
    (10, 10, 0.5, 4.5, 4.5),       # tiny radius
    (9, 12, 3.0, -1.0, 4.0),       # centre outside the image
])
def test_mask_matches_oracle(native_lib, oracle_mod, geom):
    rows, cols, r, xc, yc = geom
    xc = (cols - 1) / 2 if xc is None else xc
    yc = (rows - 1) / 2 if yc is None else yc
    m = CylinderMapping.cylinder(40, rows, cols, r, xc=xc, yc=yc)
    sr, bs, cb, ce, span = oracle_mod.cylinder_mask(rows, cols, xc, yc, r, get_stride(40))
    assert np.array_equal(m.base, bs) and m.span == span
    live = np.diff(bs) > 0
    assert np.array_equal(m.start_row[live], sr[live])
    if live.any():
        assert (m.col_begin, m.col_end) == (cb, ce)


def test_mask_counts_of_the_benchmark_geometries(native_lib):
    m0 = CylinderMapping.cylinder(128, 128, 128, 60.0)
    assert (m0.n_lines, m0.data_size) == (11304, 1446912)
    m1 = CylinderMapping.cylinder(1024, 768, 768, 370.0)
    assert (m1.n_lines, m1.data_size) == (430112, 440434688)


def test_mask_excludes_boundary_rows(native_lib):
    """(col - xc)^2 + (row - yc)^2 < r^2 strictly (include/layout_cylinder.h:166-169)."""
    m = CylinderMapping.cylinder(4, 11, 11, 5.0)
    rows, cols = m.lines()
    d2 = (cols - 5.0) ** 2 + (rows - 5.0) ** 2
    assert np.all(d2 < 25.0)
    rr, cc = np.meshgrid(np.arange(11), np.arange(11), indexing="ij")
    assert len(rows) == int(((cc - 5.0) ** 2 + (rr - 5.0) ** 2 < 25.0).sum())


def test_gather_scatter_roundtrip(native_lib):
    m = CylinderMapping.cylinder(7, 9, 8, 3.9)
    box = np.random.default_rng(0).normal(size=(8, 9, 7)).astype(np.float32)
    span = m.gather(box)
    back = m.scatter(span, fill=np.nan)
    rows, cols = m.lines()
    np.testing.assert_array_equal(back[cols, rows, :], box[cols, rows, :])
    assert np.isnan(back).sum() == box.size - len(rows) * 7


def test_slab_mapping(native_lib):
    m = CylinderMapping.cylinder(100, 20, 20, 8.0)
    s = m.with_slab_width(40)
    assert s.nstride == 64 and s.n_lines == m.n_lines and s.span == m.n_lines * 64


def test_context_without_gpu_fails_loudly(native_lib):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = ctypes.c_void_p()
    st = native_lib.potts_context_create(0, ctypes.byref(h))
    assert st == _native.POTTS_ENODEV and not h.value
    assert b"device" in native_lib.potts_last_error()


def test_uv_hist_layout(native_lib):
    """uv-hist-kernel.cpp:112-118: rows padded to 32 counts (128 bytes), span (nbins-1) stride + nbins."""
    assert native_lib.potts_uv_hist_stride(512) == 512 and native_lib.potts_uv_hist_stride(7) == 32
    assert native_lib.potts_uv_hist_span(512) == 511 * 512 + 512
    assert native_lib.potts_uv_hist_span(7) == 6 * 32 + 7 and native_lib.potts_uv_hist_span(1) == 1


@pytest.mark.parametrize("flaw", ["decreasing_base", "unaligned_base", "rows_beyond_extent", "no_slices"])
def test_static_energies_reject_bad_mappings_on_the_host(native_lib, flaw):
    """potts_energies_static runs the solver's mapping checks before it touches the GPU: a
    decreasing base[] would otherwise turn into ~2^32 rows and reads far outside u, V and Xi."""
    import numpy as np

    m = CylinderMapping.cylinder(8, 12, 12, 5.0)
    base, start_row, n_images = m.base.copy(), m.start_row.copy(), m.n_images
    c = m.col_begin + 2
    if flaw == "decreasing_base":
        base[c + 1] = base[c] - m.nstride
    elif flaw == "unaligned_base":
        base[c] += 1
    elif flaw == "rows_beyond_extent":
        start_row[c] = m.rows
    else:
        n_images = 0
    bad = _native.PottsMapping(n_images, m.rows, m.cols, m.nstride, m.col_begin, m.col_end,
                               start_row.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)),
                               base.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)))
    ci = np.array([0.2, 0.5, 0.8], np.float32)
    out = (ctypes.c_double * 3)()
    fake = ctypes.c_void_p(0x1000)  # never dereferenced: the call is rejected on the host
    st = native_lib.potts_energies_static(ctypes.byref(bad), fake, 3, ci.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                          30.0, fake, fake, None, out)
    assert st == _native.POTTS_EINVAL, native_lib.potts_last_error()
