"""Label-finding inputs on the GPU (potts_min_max, potts_grad_magn, potts_calc_hist, potts_uv_hist):
bit-identical to the CPU oracle (oracle/label_oracle.c), through the C ABI."""
import numpy as np
import pytest

from segmentctscans_b200 import potts
from segmentctscans_b200._native import PottsError
from tests._cases import phantom_volume, random_volume

pytestmark = pytest.mark.gpu

GEOMS = [
    (20, 18, 17, 7.9),
    (33, 21, 19, 9.3),
    (1, 9, 9, 4.0),     # a single slice: every gradient is -1
    (5, 3, 40, 1.2),    # columns of one row
    (300, 12, 12, 5.1),  # lines longer than a block
]


def _dev(ctx, m, a):
    return potts.upload(ctx, m, np.ascontiguousarray(a, np.float32))


@pytest.mark.parametrize("geom", GEOMS)
def test_min_max_and_grad_magn_bitwise(cuda_device, oracle_mod, geom):
    n, rows, cols, r = geom
    m, u, _ = random_volume(n, rows, cols, r, 3, seed=n + rows)
    u = u - np.float32(0.2)
    with potts.make_context(0) as ctx:
        du = _dev(ctx, m, u)
        assert potts.min_max(ctx, m, du.data_ptr()) == oracle_mod.min_max(m, u)
        assert potts.min_max(ctx, m, du.data_ptr(), positive=True) == oracle_mod.min_max(m, u, positive=True)
        dv = _dev(ctx, m, np.zeros_like(u))
        potts.grad_magn(ctx, m, du.data_ptr(), dv.data_ptr())
        v = potts.download(ctx, dv)
        for f in (du, dv):
            f.free()
    ref = oracle_mod.grad_magn(m, u)
    assert np.array_equal(m.mask_values(v), m.mask_values(ref))


@pytest.mark.parametrize("geom", [(260, 150, 150, 70.0, None), (132, 37, 70, 16.5, 136), (8, 90, 20, 9.5, None)],
                         ids=["segments", "padded-stride", "short-lines"])
def test_grad_magn_column_march(cuda_device, oracle_mod, geom):
    """Fields of 16-byte lines march along the columns in 16 x 128 tiles: several row tiles, slice
    tiles and 64-column segments, a line stride above the slice count, lines shorter than a tile."""
    n, rows, cols, r, nstride = geom
    m, u, _ = random_volume(n, rows, cols, r, 3, seed=n + cols, nstride=nstride)
    with potts.make_context(0) as ctx:
        du = _dev(ctx, m, u)
        dv = _dev(ctx, m, np.zeros_like(u))
        potts.grad_magn(ctx, m, du.data_ptr(), dv.data_ptr())
        v = potts.download(ctx, dv)
        for f in (du, dv):
            f.free()
    ref = oracle_mod.grad_magn(m, u)
    assert np.array_equal(m.mask_values(v), m.mask_values(ref))
    assert (m.mask_values(ref) >= 0).any() and (m.mask_values(ref) == -1).any()


@pytest.mark.parametrize("nb,jitter", [(1024, 0.0), (1, 0.0), (37, 0.0), (500, 0.004), (60000, 0.0)],
                         ids=["1024", "1", "37", "500-jitter", "60000-global"])
def test_calc_hist_bitwise(cuda_device, oracle_mod, nb, jitter):
    m, u, _ = random_volume(40, 26, 25, 11.7, 3, seed=nb)
    with potts.make_context(0) as ctx:
        du = _dev(ctx, m, u)
        counts, dens, lo, hi = potts.calc_hist_auto(ctx, m, du.data_ptr(), nb, jitter=jitter, seed=77)
        c2, _ = potts.calc_hist(ctx, m, du.data_ptr(), 0.25, 0.75, nb, jitter=jitter, seed=78)
        du.free()
    assert (lo, hi) == oracle_mod.min_max(m, u)
    assert np.array_equal(counts, oracle_mod.calc_hist(m, u, lo, hi, nb, jitter=jitter, seed=77))
    assert np.array_equal(c2, oracle_mod.calc_hist(m, u, 0.25, 0.75, nb, jitter=jitter, seed=78))
    # calc_hist.cpp:129-135: density = counts / (in-mask voxels x bin width)
    bw = (np.float64(hi) - np.float64(lo)) / nb
    np.testing.assert_allclose(dens, counts / (m.data_size * bw), rtol=1e-15)


@pytest.mark.parametrize("nb", [512, 7, 1, 600])
def test_uv_hist_bitwise(cuda_device, oracle_mod, nb):
    m, u, _, _ = phantom_volume(48, 21.0, seed=5, radius_range=(3.0, 8.0))
    with potts.make_context(0) as ctx:
        du = _dev(ctx, m, u)
        dv = _dev(ctx, m, np.zeros_like(u))
        potts.grad_magn(ctx, m, du.data_ptr(), dv.data_ptr())
        h, rng = potts.uv_hist_auto(ctx, m, du.data_ptr(), dv.data_ptr(), nb)
        v = potts.download(ctx, dv)
        h2 = potts.uv_hist(ctx, m, du.data_ptr(), dv.data_ptr(), 0.2, 0.8, 0.0, 0.05, nb)
        for f in (du, dv):
            f.free()
    us, ue = oracle_mod.min_max(m, u)
    vs, ve = oracle_mod.min_max(m, v, positive=True)
    assert rng == (us, ue, vs, ve)
    ref = oracle_mod.uv_hist(m, u, v, us, ue, vs, ve, nb)
    assert h.shape == ref.shape and np.array_equal(h, ref)
    assert int(h.sum()) > 0
    assert np.array_equal(h2, oracle_mod.uv_hist(m, u, v, 0.2, 0.8, 0.0, 0.05, nb))
    mat = potts.uv_hist_matrix(h, nb)
    assert mat.shape == (nb, nb) and int(mat.sum()) == int(h.sum())


@pytest.mark.parametrize("nb", [512, 129, 1000, 64])
def test_uv_hist_spread_values(cuda_device, oracle_mod, nb):
    """Uniform values spread the counts over every coarse cell, so the cells held in shared memory
    take only part of them and the rest go to global counters; nb = 129 and 1000 leave the last
    coarse cells partly outside the histogram."""
    m, _, _ = random_volume(70, 40, 38, 18.1, 3, seed=9)
    rng = np.random.default_rng(nb)
    u = rng.uniform(0.0, 1.0, m.span).astype(np.float32)
    v = rng.uniform(0.0, 1.0, m.span).astype(np.float32)
    with potts.make_context(0) as ctx:
        du, dv = _dev(ctx, m, u), _dev(ctx, m, v)
        h = potts.uv_hist(ctx, m, du.data_ptr(), dv.data_ptr(), 0.05, 0.95, 0.1, 0.9, nb)
        for f in (du, dv):
            f.free()
    ref = oracle_mod.uv_hist(m, u, v, 0.05, 0.95, 0.1, 0.9, nb)
    assert np.array_equal(h, ref) and int(h.sum()) > 0


@pytest.mark.parametrize("nb", [1024, 1, 2, 333])
def test_histograms_of_saturated_fields(cuda_device, oracle_mod, nb):
    """A field clamped to its range: about a quarter of the values sit exactly at each end, where the
    bin formula lands on the half-integers -1/2 and nb - 1/2 (the first and the last bin take them
    without the division).  Also with jitter, and in the 2-D histogram."""
    m, u, _ = random_volume(40, 26, 25, 11.7, 3, seed=nb + 3)
    q1, q3 = np.quantile(m.mask_values(u), [0.25, 0.75])
    s = np.clip((u - np.float32(q1)) / np.float32(q3 - q1), 0.0, 1.0).astype(np.float32)
    with potts.make_context(0) as ctx:
        ds = _dev(ctx, m, s)
        counts, _, lo, hi = potts.calc_hist_auto(ctx, m, ds.data_ptr(), nb)
        cj, _ = potts.calc_hist(ctx, m, ds.data_ptr(), 0.0, 1.0, nb, jitter=0.01, seed=5)
        dv = _dev(ctx, m, np.zeros_like(s))
        potts.grad_magn(ctx, m, ds.data_ptr(), dv.data_ptr())
        v = potts.download(ctx, dv)
        h, rng = potts.uv_hist_auto(ctx, m, ds.data_ptr(), dv.data_ptr(), max(nb // 2, 1))
        for f in (ds, dv):
            f.free()
    assert (lo, hi) == (0.0, 1.0)
    assert np.array_equal(counts, oracle_mod.calc_hist(m, s, 0.0, 1.0, nb))
    assert counts[0] >= m.data_size // 5 and counts[-1] >= m.data_size // 5
    assert np.array_equal(cj, oracle_mod.calc_hist(m, s, 0.0, 1.0, nb, jitter=0.01, seed=5))
    assert np.array_equal(h, oracle_mod.uv_hist(m, s, v, *rng, max(nb // 2, 1)))


def test_empty_range_and_constant_field(cuda_device, oracle_mod):
    """start == end: every in-range value goes to bin 0 (the quotient is NaN), as on the reference's GPU."""
    m, u, _ = random_volume(9, 11, 11, 4.6, 3, seed=2)
    c = np.full_like(u, 0.5)
    with potts.make_context(0) as ctx:
        dc = _dev(ctx, m, c)
        counts, _, lo, hi = potts.calc_hist_auto(ctx, m, dc.data_ptr(), 16)
        dv = _dev(ctx, m, np.zeros_like(u))
        potts.grad_magn(ctx, m, dc.data_ptr(), dv.data_ptr())
        h, rng = potts.uv_hist_auto(ctx, m, dc.data_ptr(), dv.data_ptr(), 8)
        for f in (dc, dv):
            f.free()
    assert lo == hi == 0.5
    assert counts[0] == m.data_size and counts[1:].sum() == 0
    assert np.array_equal(counts, oracle_mod.calc_hist(m, c, 0.5, 0.5, 16))
    # a constant field has no strictly positive gradient: the v range is empty and nothing is counted
    assert rng[2] > rng[3] and int(h.sum()) == 0


def test_label_input_errors(cuda_device):
    m, u, _ = random_volume(8, 8, 8, 3.5, 3, seed=2)
    with potts.make_context(0) as ctx:
        du = _dev(ctx, m, u)
        for nb in (0, 65536):
            with pytest.raises(PottsError):
                potts.calc_hist(ctx, m, du.data_ptr(), 0.0, 1.0, nb)
            with pytest.raises(PottsError):
                potts.uv_hist(ctx, m, du.data_ptr(), du.data_ptr(), 0.0, 1.0, 0.0, 1.0, nb)
        with pytest.raises(PottsError):
            potts.calc_hist(ctx, m, du.data_ptr(), 0.0, 1.0, 8, jitter=-1.0)
        with pytest.raises(PottsError):
            potts.grad_magn(ctx, m, du.data_ptr(), du.data_ptr())
        potts.calc_hist(ctx, m, du.data_ptr(), 0.0, 1.0, 8)
        du.free()
