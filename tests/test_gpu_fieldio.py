"""Field archive (.bin), convert_to_fp, find_intensity_range and the output writers on the GPU,
through the C ABI: bit- and byte-identical to the CPU oracle (oracle/fieldio_oracle.c)."""
import io

import numpy as np
import pytest

from segmentctscans_b200 import potts
from segmentctscans_b200._native import PottsError
from segmentctscans_b200.layout import CylinderMapping
from tests._cases import phantom_volume, random_volume

pytestmark = pytest.mark.gpu

# (n_images, rows, cols, r): the header lengths of these mappings put the payload at each of the
# bit offsets 1, 3, 5, 7 within a byte (a header is 2 cols + 9 Exp-Golomb codes of odd length, plus
# 64 bits for FP32 fields, so its length is always odd); n_images 64 and 300 take the vectorised
# kernels, the others the per-voxel ones
GEOMS = [(5, 6, 7, 2.6), (33, 12, 10, 5.2), (1, 9, 9, 4.0), (3, 5, 40, 1.3), (300, 14, 13, 6.1), (64, 40, 41, 19.7),
         (17, 23, 19, 10.4), (2, 31, 30, 14.2), (129, 11, 12, 5.3), (7, 50, 48, 22.9)]


def _torch():
    import torch

    return torch


def _device_u16(values: np.ndarray):
    torch = _torch()
    return torch.from_numpy(np.ascontiguousarray(values, np.uint16).view(np.int16)).cuda()


def _device_f32(values: np.ndarray):
    torch = _torch()
    return torch.from_numpy(np.ascontiguousarray(values, np.float32)).cuda()


def _field(m, elem, seed):
    rng = np.random.default_rng(seed)
    if elem == "f32":
        f = rng.normal(0, 1, m.span).astype(np.float32)
        f[::7] = -0.0
        return f
    return rng.integers(0, 65536, m.span).astype(np.uint16)


@pytest.mark.parametrize("elem", ["f32", "u16"])
def test_archive_load_bitwise(cuda_device, oracle_mod, elem):
    shifts = set()
    torch = _torch()
    with potts.make_context(0) as ctx:
        for k, geom in enumerate(GEOMS):
            m = CylinderMapping.cylinder(*geom)
            f = _field(m, elem, k)
            data, hb = oracle_mod.archive_encode(m, f, elem, 0.75, 1.5)
            shifts.add(hb % 8)
            # padding slices keep what was there: fill the device field with a sentinel
            sentinel = np.full(m.span, 0xABCD if elem == "u16" else np.float32(9.5),
                               np.uint16 if elem == "u16" else np.float32)
            d = _device_u16(sentinel) if elem == "u16" else _device_f32(sentinel)
            info, _ = potts.archive_load(ctx, data, elem, d.data_ptr(), m.span)
            torch.cuda.synchronize()
            got = d.cpu().numpy().view(np.uint16 if elem == "u16" else np.float32)
            ref = oracle_mod.archive_decode(data, elem)
            assert info.header_bits == hb and info.total_bytes == len(data)
            if elem == "f32":
                assert (info.lo, info.hi) == (0.75, 1.5)
            mv = m.mask_values
            assert np.array_equal(mv(got).view(np.uint8), mv(ref.field).view(np.uint8))
            pad = got.reshape(m.n_lines, m.nstride)[:, m.n_images:]
            assert np.array_equal(pad.view(np.uint8), sentinel.reshape(m.n_lines, m.nstride)[:, m.n_images:].view(np.uint8))
    assert shifts == {1, 3, 5, 7}, shifts


@pytest.mark.parametrize("elem", ["f32", "u16"])
def test_archive_load_unaligned_field(cuda_device, oracle_mod, elem):
    """A field pointer off a 16-byte boundary takes the per-voxel kernel: the same values."""
    torch = _torch()
    m = CylinderMapping.cylinder(64, 40, 41, 19.7)
    f = _field(m, elem, 7)
    data, _ = oracle_mod.archive_encode(m, f, elem)
    with potts.make_context(0) as ctx:
        buf = torch.zeros(m.span + 8, dtype=torch.int16 if elem == "u16" else torch.float32, device="cuda")
        potts.archive_load(ctx, data, elem, buf[1:].data_ptr(), m.span)
        torch.cuda.synchronize()
    got = buf[1:1 + m.span].cpu().numpy().view(np.uint16 if elem == "u16" else np.float32)
    mv = m.mask_values
    assert np.array_equal(mv(got).view(np.uint8), mv(f).view(np.uint8))


@pytest.mark.parametrize("elem", ["f32", "u16"])
def test_archive_save_bytewise(cuda_device, oracle_mod, elem):
    with potts.make_context(0) as ctx:
        for k, geom in enumerate(GEOMS):
            m = CylinderMapping.cylinder(*geom)
            f = _field(m, elem, 100 + k)
            d = _device_u16(f) if elem == "u16" else _device_f32(f)
            got, _ = potts.archive_save(ctx, m, elem, d.data_ptr(), 0.25, 4.0)
            ref, _ = oracle_mod.archive_encode(m, f, elem, 0.25, 4.0)
            assert got.tobytes() == ref, geom


def test_archive_round_trip_and_errors(cuda_device, oracle_mod):
    m, u, _, _ = phantom_volume(48, 21.0, seed=3)
    torch = _torch()
    with potts.make_context(0) as ctx:
        d = _device_f32(u)
        data, _ = potts.archive_save(ctx, m, "f32", d.data_ptr(), 0.1, 0.9)
        back = torch.zeros(m.span, dtype=torch.float32, device="cuda")
        info, _ = potts.archive_load(ctx, data, "f32", back.data_ptr(), m.span)
        torch.cuda.synchronize()
        assert np.array_equal(m.mask_values(back.cpu().numpy()), m.mask_values(u))
        assert (info.lo, info.hi) == (np.float32(0.1), np.float32(0.9))
        with pytest.raises(PottsError):  # the payload is cut short
            potts.archive_load(ctx, data[:-1], "f32", back.data_ptr(), m.span)
        with pytest.raises(PottsError):  # the device field is too small
            potts.archive_load(ctx, data, "f32", back.data_ptr(), m.span - 1)
        with pytest.raises(PottsError):
            potts.archive_save(ctx, m, "f32", d.data_ptr(), out=np.zeros(len(data) - 1, np.uint8))


@pytest.mark.parametrize("n", [70, 68, 64], ids=["per-voxel", "vector-68", "vector-64"])
@pytest.mark.parametrize("elem", ["f32", "u16"])
def test_convert_to_fp_bitwise(cuda_device, oracle_mod, elem, n):
    torch = _torch()
    m, u, _ = random_volume(n, 22, 21, 10.3, 3, seed=9)
    if elem == "f32":
        f = (u * 2.0 - 0.5).astype(np.float32)
        lo, hi = -0.25, 1.1
        d = _device_f32(f)
    else:
        f = (u * 60000.0).astype(np.uint16)
        lo, hi = 3000.0, 51234.0
        d = _device_u16(f)
    out = torch.zeros(m.span, dtype=torch.float32, device="cuda")
    with potts.make_context(0) as ctx:
        potts.convert_to_fp(ctx, m, elem, d.data_ptr(), lo, hi, out.data_ptr())
        ctx.synchronize()
    ref = oracle_mod.convert_to_fp(m, f, lo, hi)
    assert np.array_equal(m.mask_values(out.cpu().numpy()), m.mask_values(ref))


@pytest.mark.parametrize("n,tail", [(96, 0.0), (96, 1e-3), (96, 0.02), (97, 0.5), (97, 1e-3)])
def test_find_intensity_range(cuda_device, oracle_mod, n, tail):
    m, u, _ = random_volume(n, 40, 41, 19.2, 3, seed=11)
    rng = np.random.default_rng(5)
    w = np.clip(u * 40000 + rng.normal(8000, 2500, m.span), 0, 65535).astype(np.uint16)
    w[: m.nstride] = 65535  # the top bin is used
    d = _device_u16(w)
    with potts.make_context(0) as ctx:
        lo, hi, hist = potts.find_intensity_range(ctx, m, d.data_ptr(), tail)
    rlo, rhi, rhist = oracle_mod.intensity_range(m, w, tail)
    assert np.array_equal(hist, rhist)
    assert (lo, hi) == (rlo, rhi)
    assert int(hist.sum()) == m.data_size


def test_raw_labels_and_vtk_file(cuda_device, oracle_mod):
    torch = _torch()
    for k, geom in enumerate([(33, 12, 10, 5.2), (64, 40, 41, 19.7), (1, 9, 9, 4.0)]):
        m = CylinderMapping.cylinder(*geom)
        rng = np.random.default_rng(k)
        v = rng.uniform(-0.2, 1.2, m.span).astype(np.float32)
        v[::5] = np.float32(0.5) / np.float32(255) * np.float32(2 * (k + 1) + 1)  # near-halves
        d = _device_f32(v)
        s, rows, cols, rb = potts.raw_labels_dims(m)
        box = torch.zeros(s * rows * cols, dtype=torch.uint8, device="cuda")
        with potts.make_context(0) as ctx:
            potts.raw_labels(ctx, m, d.data_ptr(), box.data_ptr())
            ctx.synchronize()
            vtk, _ = potts.vtk_labels(ctx, m, d.data_ptr())
        ref_box, dims = oracle_mod.raw_box(m, v)
        assert dims == (s, rows, cols, rb)
        assert np.array_equal(box.cpu().numpy().reshape(cols, rows, s), ref_box)
        assert vtk.tobytes() == oracle_mod.vtk_file(m, v)


def test_png_slice(cuda_device, oracle_mod, tmp_path):
    from PIL import Image

    m, u, _, _ = phantom_volume(48, 21.0, seed=2)
    v = u.copy()
    v[::11] = -v[::11]  # cv::pow raises |x|
    d = _device_f32(v)
    col = (m.col_begin + m.col_end) // 2
    with potts.make_context(0) as ctx:
        png = potts.png_slice(ctx, m, d.data_ptr(), col)
        path = potts.write_png(ctx, m, d.data_ptr(), col, 30.0, tmp_path)
        with pytest.raises(PottsError):
            potts.png_slice(ctx, m, d.data_ptr(), m.col_end)
    img = np.asarray(Image.open(io.BytesIO(png)))
    assert img.dtype == np.uint8 and img.shape == (m.row_end(col) - m.row_begin(col), m.n_images)
    assert np.array_equal(img, oracle_mod.png_gray(m, v, col))
    assert path.endswith(f"slice-{col} (\U0001d706 = 030.000).png")
    with open(path, "rb") as fh:
        assert fh.read() == png


def test_empty_mask_and_single_slice_archives(cuda_device, oracle_mod):
    """Edge cases of the payload: no voxel at all (the archive is the header) and one slice per line."""
    torch = _torch()
    with potts.make_context(0) as ctx:
        empty = CylinderMapping.cylinder(4, 10, 10, 0.3)
        dummy = torch.zeros(16, dtype=torch.float32, device="cuda")
        data, _ = potts.archive_save(ctx, empty, "f32", dummy.data_ptr(), 1.0, 2.0)
        ref, _ = oracle_mod.archive_encode(empty, np.zeros(0, np.float32), "f32", 1.0, 2.0)
        assert data.tobytes() == ref
        info, _ = potts.archive_load(ctx, ref, "f32", dummy.data_ptr(), 0)
        assert info.voxels == 0 and (info.lo, info.hi) == (1.0, 2.0)
        for elem in ("f32", "u16"):
            m = CylinderMapping.cylinder(1, 33, 31, 15.2)
            f = _field(m, elem, 3)
            d = _device_u16(f) if elem == "u16" else _device_f32(f)
            got, _ = potts.archive_save(ctx, m, elem, d.data_ptr())
            ref, _ = oracle_mod.archive_encode(m, f, elem)
            assert got.tobytes() == ref
            back = torch.zeros_like(d)
            potts.archive_load(ctx, ref, elem, back.data_ptr(), m.span)
            torch.cuda.synchronize()
            b = back.cpu().numpy().view(np.uint16 if elem == "u16" else np.float32)
            assert np.array_equal(m.mask_values(b).view(np.uint8), m.mask_values(f).view(np.uint8))


def test_archive_to_solve_to_vtk_pipeline(cuda_device, oracle_mod):
    """potts-model's path on one context: read the .bin archive (Field<float>, lo/hi), solve with the
    labels normalised by lo/hi (potts-model.cpp:145-148), write the --rawout file.  The staging
    buffers of the archive call are released when the solve plans its slabs."""
    torch = _torch()
    m, u, ci, _ = phantom_volume(32, 14.0, seed=4)
    lo, hi = 0.0125, 0.0625
    raw_labels = [lo + c * (hi - lo) for c in ci]
    data, _ = oracle_mod.archive_encode(m, u, "f32", lo, hi)
    tau = potts.reference_tau()
    with potts.make_context(0, stream=torch.cuda.current_stream().cuda_stream) as ctx:
        du = torch.zeros(m.span, dtype=torch.float32, device="cuda")
        info, _ = potts.archive_load(ctx, data, "f32", du.data_ptr(), m.span)
        cn = [(np.float32(x) - np.float32(info.lo)) / (np.float32(info.hi) - np.float32(info.lo)) for x in raw_labels]
        res = torch.zeros(m.span, dtype=torch.float32, device="cuda")
        potts.solve_device(ctx, info.mapping, du.data_ptr(), cn, 30.0, tau, tau, 30, res_ptr=res.data_ptr())
        vtk, _ = potts.vtk_labels(ctx, info.mapping, res.data_ptr())
        torch.cuda.synchronize()
    ref = oracle_mod.solve(m, u, [float(c) for c in cn], 30.0, tau, tau, 30, precision="f32")
    got = res.cpu().numpy()
    assert np.array_equal(m.mask_values(got), m.mask_values(ref.res.astype(np.float32)))
    assert vtk.tobytes() == oracle_mod.vtk_file(m, got)
