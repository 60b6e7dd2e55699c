"""Field archive (.bin), convert_to_fp, find_intensity_range and the output writers: the CPU oracle
(oracle/fieldio_oracle.c) against known answers and an independent bit-by-bit Python coder, and the
library's host-only entry points (header parsing, sizes, box extent) against the oracle."""
import numpy as np
import pytest

from segmentctscans_b200 import potts
from segmentctscans_b200._native import POTTS_EINVAL, PottsError
from segmentctscans_b200.layout import CylinderMapping
from tests._cases import random_volume


# -- an independent restatement for small cases: a string of '0'/'1' characters -------------------
def ue_bits(v: int) -> str:
    """Exp-Golomb code of include/io/writeprimitives.h:55-60."""
    m = bin(v + 1)[2:]
    return "0" * (len(m) - 1) + m


def se_bits(v: int) -> str:
    """writeprimitives.h:62-66: v > 0 -> 2v - 1, v <= 0 -> -2v."""
    return ue_bits(2 * v - 1 if v > 0 else -2 * v)


def header_bits(m: CylinderMapping, elem: str, lo=0.0, hi=0.0) -> str:
    s = "".join(ue_bits(int(x)) for x in (m.n_images, m.rows, m.cols, m.nstride, m.col_begin, m.col_end))
    sr = [int(x) for x in m.start_row]
    bs = [int(x) for x in m.base]
    s += ue_bits(len(sr)) + ue_bits(sr[0]) + "".join(se_bits(sr[i] - sr[i - 1]) for i in range(1, len(sr)))
    s += ue_bits(len(bs)) + ue_bits(bs[0]) + "".join(se_bits(bs[i] - bs[i - 1]) for i in range(1, len(bs)))
    if elem == "f32":
        s += format(int(np.float32(lo).view(np.uint32)), "032b") + format(int(np.float32(hi).view(np.uint32)), "032b")
    return s


def archive_bits(m: CylinderMapping, field: np.ndarray, elem: str, lo=0.0, hi=0.0) -> bytes:
    s = header_bits(m, elem, lo, hi)
    vals = m.mask_values(field.view(np.uint32) if elem == "f32" else field).reshape(-1)
    width = 32 if elem == "f32" else 16
    s += "".join(format(int(v), f"0{width}b") for v in vals)
    s += "0" * (-len(s) % 8)
    return bytes(int(s[i:i + 8], 2) for i in range(0, len(s), 8))


def test_exp_golomb_known_answers():
    # the codes of the first values (H.264-style ue(v)) and the signed mapping
    assert [ue_bits(v) for v in range(5)] == ["1", "010", "011", "00100", "00101"]
    assert [se_bits(v) for v in (0, 1, -1, 2, -2)] == ["1", "010", "011", "00100", "00101"]


def _tiny_mapping():
    return CylinderMapping.cylinder(5, 6, 7, 2.6)


def test_oracle_header_known_answer(oracle_mod):
    m = _tiny_mapping()
    f = np.zeros(m.span, np.float32)
    data, hb = oracle_mod.archive_encode(m, f, "f32", lo=0.25, hi=3.0)
    assert hb == len(header_bits(m, "f32", 0.25, 3.0))
    assert data == archive_bits(m, f, "f32", 0.25, 3.0)


@pytest.mark.parametrize("elem", ["f32", "u16"])
@pytest.mark.parametrize("geom", [(5, 6, 7, 2.6), (3, 9, 9, 4.0), (33, 12, 10, 5.2), (1, 5, 40, 1.3)])
def test_oracle_archive_matches_bitwise_coder(oracle_mod, elem, geom):
    n, rows, cols, r = geom
    m = CylinderMapping.cylinder(n, rows, cols, r)
    rng = np.random.default_rng(n * 100 + cols)
    if elem == "f32":
        f = rng.normal(0, 1, m.span).astype(np.float32)
        lo, hi = 0.125, 7.5
    else:
        f = rng.integers(0, 65536, m.span).astype(np.uint16)
        lo = hi = 0.0
    data, _ = oracle_mod.archive_encode(m, f, elem, lo, hi)
    assert data == archive_bits(m, f, elem, lo, hi)
    back = oracle_mod.archive_decode(data, elem)
    assert back.mapping.n_images == m.n_images and back.mapping.nstride == m.nstride
    assert np.array_equal(back.mapping.start_row, m.start_row) and np.array_equal(back.mapping.base, m.base)
    assert (back.lo, back.hi) == (np.float32(lo), np.float32(hi))
    mv = m.mask_values
    assert np.array_equal(mv(back.field).view(np.uint8), mv(f).view(np.uint8))


def test_oracle_empty_columns_keep_all_ones_start_row(oracle_mod):
    """Columns outside the circle hold start_row = ~0 (include/layout_cylinder.h:186); the header codes
    the jump as a signed difference beyond 32 bits."""
    m = CylinderMapping.cylinder(4, 20, 20, 3.1)
    assert m.start_row[0] == 0xFFFFFFFF
    f = np.ones(m.span, np.float32)
    data, _ = oracle_mod.archive_encode(m, f, "f32")
    assert data == archive_bits(m, f, "f32")
    assert np.array_equal(oracle_mod.archive_decode(data, "f32").mapping.start_row, m.start_row)


@pytest.mark.parametrize("elem", ["f32", "u16"])
def test_library_header_matches_oracle(native_lib, oracle_mod, elem):
    for geom in [(5, 6, 7, 2.6), (33, 12, 10, 5.2), (64, 40, 41, 19.7), (1, 5, 40, 1.3)]:
        m = CylinderMapping.cylinder(*geom)
        f = np.arange(m.span, dtype=np.float32) if elem == "f32" else (np.arange(m.span) % 65536).astype(np.uint16)
        data, hb = oracle_mod.archive_encode(m, f, elem, 0.5, 2.0)
        info = potts.archive_read_header(data, elem)
        assert info.header_bits == hb and info.total_bytes == len(data)
        assert info.voxels == m.data_size
        got = info.mapping
        assert (got.n_images, got.rows, got.cols, got.nstride, got.col_begin, got.col_end) == (
            m.n_images, m.rows, m.cols, m.nstride, m.col_begin, m.col_end)
        assert np.array_equal(got.start_row, m.start_row) and np.array_equal(got.base, m.base)
        if elem == "f32":
            assert (info.lo, info.hi) == (0.5, 2.0)
        assert potts.archive_size(m, elem) == (len(data), hb)


def test_library_header_errors(native_lib, oracle_mod):
    m = _tiny_mapping()
    data, hb = oracle_mod.archive_encode(m, np.zeros(m.span, np.float32), "f32")
    for cut in (0, 1, hb // 8 - 1):
        with pytest.raises(PottsError) as e:
            potts.archive_read_header(data[:cut], "f32")
        assert e.value.status == POTTS_EINVAL
    with pytest.raises(ValueError):
        potts.archive_read_header(data, "f64")
    # a header that claims a start_row table of the wrong length
    bad = "".join(ue_bits(int(x)) for x in (m.n_images, m.rows, m.cols, m.nstride, m.col_begin, m.col_end))
    bad += ue_bits(m.cols + 1) + "1" * 64
    bad += "0" * (-len(bad) % 8)
    with pytest.raises(PottsError):
        potts.archive_read_header(bytes(int(bad[i:i + 8], 2) for i in range(0, len(bad), 8)), "f32")


def test_oracle_convert_to_fp(oracle_mod):
    m, u, _ = random_volume(9, 10, 11, 4.4, 3, seed=3)
    f = (u * 3.0 - 1.0).astype(np.float32)
    out = oracle_mod.convert_to_fp(m, f, -0.5, 1.25)
    x = m.mask_values(f)
    ref = np.where(x <= np.float32(-0.5), np.float32(0),
                   np.where(x >= np.float32(1.25), np.float32(1),
                            (x - np.float32(-0.5)) / (np.float32(1.25) - np.float32(-0.5)))).astype(np.float32)
    assert np.array_equal(m.mask_values(out), ref)
    w = (np.arange(m.span) * 37 % 65536).astype(np.uint16)
    out16 = oracle_mod.convert_to_fp(m, w, 1000.0, 50000.0)
    xw = m.mask_values(w).astype(np.float32)
    ref16 = np.where(xw <= 1000, 0, np.where(xw >= 50000, 1, (xw - np.float32(1000)) / np.float32(49000)))
    assert np.array_equal(m.mask_values(out16), ref16.astype(np.float32))


def test_oracle_intensity_range(oracle_mod):
    m, _, _ = random_volume(16, 20, 20, 8.3, 3, seed=4)
    rng = np.random.default_rng(0)
    w = np.clip(rng.normal(20000, 3000, m.span), 0, 65535).astype(np.uint16)
    for tail in (0.0, 1e-3, 0.05, 0.5):
        lo, hi, hist = oracle_mod.intensity_range(m, w, tail)
        vals = m.mask_values(w).reshape(-1)
        assert np.array_equal(hist, np.bincount(vals, minlength=65536).astype(np.uint64))
        cum = np.cumsum(hist)
        # find_intensity_range.cpp:99-106: the last bin with cum <= tail * total, the first with cum >= (1 - tail) * total
        below = np.nonzero(tail * cum[-1] >= cum)[0]
        first_hi = int(np.nonzero((1 - tail) * cum[-1] <= cum)[0][0])
        exp_lo = int(below[below <= first_hi][-1]) if below.size and below[0] <= first_hi else 0
        assert (lo, hi) == (exp_lo, first_hi)


def test_oracle_raw_box_and_dims(native_lib, oracle_mod):
    m, u, _ = random_volume(7, 15, 13, 6.2, 3, seed=6)
    v = (u * 1.2 - 0.1).astype(np.float32)
    box, dims = oracle_mod.raw_box(m, v)
    assert potts.raw_labels_dims(m) == dims
    s, rows, cols, rb = dims
    dense = m.scatter(v, fill=np.float32(np.nan))[m.col_begin:m.col_end, rb:rb + rows, :]
    t = (np.float32(255) * dense).astype(np.float64)  # the product in FP32, rounded half away from zero
    exp = np.where(np.isnan(dense), 255, np.clip(np.floor(np.abs(t) + 0.5) * np.sign(t), 0, 255)).astype(np.uint8)
    assert np.array_equal(box, exp)
    f = oracle_mod.vtk_file(m, v)
    assert f.startswith(b"<?xml version=\"1.0\"?>\n<VTKFile type=\"ImageData\"")
    assert f.endswith(b"\n  </AppendedData>\n</VTKFile>\n")


def test_header_length_is_odd(native_lib):
    """Every code of the header has odd length and there are 2 cols + 9 of them (64 more bits for FP32
    fields): the voxel payload always starts at an odd bit offset within a byte."""
    for geom in [(5, 6, 7, 2.6), (33, 12, 10, 5.2), (64, 40, 41, 19.7), (1, 5, 40, 1.3), (1024, 768, 768, 370.0)]:
        m = CylinderMapping.cylinder(*geom)
        for elem in ("f32", "u16"):
            _, hb = potts.archive_size(m, elem)
            assert hb % 2 == 1 and hb == len(header_bits(m, elem))


def test_empty_mask_header(native_lib, oracle_mod):
    """A radius that keeps no row: col_begin stays ~0 and every table entry is ~0 or 0; the archive is
    the header alone and parses back."""
    m = CylinderMapping.cylinder(4, 10, 10, 0.3)
    assert m.span == 0 and m.col_begin == 0xFFFFFFFF and m.col_end == 0
    for elem in ("f32", "u16"):
        data, hb = oracle_mod.archive_encode(m, np.zeros(0, np.float32 if elem == "f32" else np.uint16), elem)
        assert data == archive_bits(m, np.zeros(0, np.float32 if elem == "f32" else np.uint16), elem)
        info = potts.archive_read_header(data, elem)
        assert info.voxels == 0 and info.total_bytes == len(data) == (hb + 7) // 8
        assert info.mapping.col_begin == 0xFFFFFFFF and np.array_equal(info.mapping.start_row, m.start_row)
        assert potts.archive_size(m, elem) == (len(data), hb)
    with pytest.raises(PottsError):
        potts.raw_labels_dims(m)


def test_header_value_beyond_32_bits_is_rejected(native_lib):
    bits = ue_bits(2**32) + "".join(ue_bits(v) for v in (4, 4, 32, 0, 4, 4)) + "1" * 200
    bits += "0" * (-len(bits) % 8)
    with pytest.raises(PottsError) as e:
        potts.archive_read_header(bytes(int(bits[i:i + 8], 2) for i in range(0, len(bits), 8)), "u16")
    assert e.value.status == POTTS_EINVAL
