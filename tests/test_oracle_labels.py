"""CPU oracle of the label-finding inputs (oracle/label_oracle.c): min/max, gradient magnitude,
1-D and 2-D histograms checked against hand-derived answers and independent numpy restatements."""
import numpy as np
import pytest

from segmentctscans_b200.layout import CylinderMapping
from tests._cases import random_volume


def _linear_field(m, a, b, c):
    """u = a n + b row + c col at every in-mask voxel (small integers: exact in float32)."""
    n = np.arange(m.n_images)
    box = (a * n[None, None, :] + b * np.arange(m.rows)[None, :, None] + c * np.arange(m.cols)[:, None, None])
    return m.gather(box.astype(np.float32))


def _interior(m):
    """In-mask voxels whose six neighbours are all in the mask (grad_magn.cpp:36-43), [n_lines, n]."""
    rows, cols = m.lines()
    def stored(r, c):
        ok = np.zeros(r.shape, bool)
        for i, (rr, cc) in enumerate(zip(r, c)):
            ok[i] = m.col_begin <= cc < m.col_end and m.row_begin(cc) <= rr < m.row_end(cc)
        return ok
    line_ok = stored(rows + 1, cols) & stored(rows - 1, cols) & stored(rows, cols + 1) & stored(rows, cols - 1)
    n = np.arange(m.n_images)
    n_ok = (n > 0) & (n + 1 < m.n_images)
    return line_ok[:, None] & n_ok[None, :]


def test_grad_magn_of_a_linear_field(oracle_mod):
    m = CylinderMapping.cylinder(12, 15, 14, 6.3)
    u = _linear_field(m, 1, 2, 3)
    v = m.mask_values(oracle_mod.grad_magn(m, u))
    inner = _interior(m)
    assert inner.any() and (~inner).any()
    # central differences 2a, 2b, 2c: 0.5 sqrt(4 + 16 + 36), squares contracted as 4 + fma(4, 4, ...)
    s = np.float32(2.0) * np.float32(2.0)
    expect = np.float32(0.5) * np.sqrt(np.float32(np.float64(s) + 16.0 + 36.0))
    assert np.all(v[inner] == expect)
    assert np.all(v[~inner] == -1.0)


def test_grad_magn_single_slice_is_boundary(oracle_mod):
    m, u, _ = random_volume(1, 9, 9, 4.0, 3, seed=1)
    assert np.all(m.mask_values(oracle_mod.grad_magn(m, u)) == -1.0)


def test_min_max(oracle_mod):
    m, u, _ = random_volume(17, 20, 19, 8.2, 3, seed=3)
    u = u - np.float32(0.3)
    mv = m.mask_values(u)
    assert oracle_mod.min_max(m, u) == (float(mv.min()), float(mv.max()))
    pos = mv[mv > 0]
    assert oracle_mod.min_max(m, u, positive=True) == (float(pos.min()), float(pos.max()))
    assert oracle_mod.min_max(m, np.full_like(u, -1.0), positive=True) == (
        float(np.finfo(np.float32).max), float(-np.finfo(np.float32).max))


def test_hist_known_bins(oracle_mod):
    """Bin centres of [0, 1] in 4 bins land in their bins; the range ends go to the end bins."""
    m = CylinderMapping.cylinder(8, 3, 3, 0.6)  # one line (the centre), 8 slices
    assert m.n_lines == 1
    vals = np.array([0.0, 0.125, 0.375, 0.625, 0.875, 1.0, -0.01, 1.01], np.float32)
    u = np.zeros(m.span, np.float32)
    u[:8] = vals
    c = oracle_mod.calc_hist(m, u, 0.0, 1.0, 4)
    assert c.tolist() == [2, 1, 1, 2]  # 0 and 0.125 -> 0; 0.875 and 1.0 -> 3; outside values dropped
    # jitter narrows the accepted range by jitter/2 at both ends
    cj = oracle_mod.calc_hist(m, u, 0.0, 1.0, 4, jitter=0.1, seed=5)
    assert cj.sum() <= 6 and cj.sum() >= 4


def _np_bins(x, start, end, nb):
    """numpy restatement of the bin rule in float64 (equal to the float32 rule away from ties)."""
    t = (x.astype(np.float64) - start) / (end - start)
    return np.clip(np.floor(nb * t), 0, nb - 1).astype(np.int64)


def test_hist_against_numpy(oracle_mod):
    m, u, _ = random_volume(23, 24, 22, 10.5, 3, seed=7)
    mv = m.mask_values(u).ravel()
    lo, hi = float(mv.min()), float(mv.max())
    nb = 37
    c = oracle_mod.calc_hist(m, u, lo, hi, nb)
    assert int(c.sum()) == mv.size
    ref = np.bincount(_np_bins(mv, lo, hi, nb), minlength=nb)
    # the float32 rule and the float64 floor agree except for values within rounding of a bin edge
    assert np.abs(c.astype(np.int64) - ref).sum() <= 2 * max(1, mv.size // 20000)


def test_hist_jitter_reproducible(oracle_mod):
    m, u, _ = random_volume(16, 18, 18, 7.5, 3, seed=9)
    a = oracle_mod.calc_hist(m, u, 0.0, 1.0, 64, jitter=0.05, seed=11)
    b = oracle_mod.calc_hist(m, u, 0.0, 1.0, 64, jitter=0.05, seed=11)
    c = oracle_mod.calc_hist(m, u, 0.0, 1.0, 64, jitter=0.05, seed=12)
    assert np.array_equal(a, b) and not np.array_equal(a, c)
    plain = oracle_mod.calc_hist(m, u, 0.0, 1.0, 64)
    assert abs(int(a.sum()) - int(plain.sum())) <= int(0.1 * plain.sum())


@pytest.mark.parametrize("nb", [1, 7, 40])
def test_uv_hist_marginals(oracle_mod, nb):
    """Row sums are the 1-D histogram of v over the pairs inside both ranges, column sums that of u
    (calc_hist's bin rule with the same range)."""
    m, u, _ = random_volume(19, 21, 20, 9.1, 3, seed=13)
    v = oracle_mod.grad_magn(m, u)
    us, ue = oracle_mod.min_max(m, u)
    vs, ve = oracle_mod.min_max(m, v, positive=True)
    h = oracle_mod.uv_hist(m, u, v, us, ue, vs, ve, nb)
    stride = oracle_mod.uv_stride(nb)
    assert h.size == (nb - 1) * stride + nb
    mat = np.lib.stride_tricks.as_strided(h, shape=(nb, nb), strides=(4 * stride, 4))
    both = (u >= us) & (u <= ue) & (v >= vs) & (v <= ve)
    nan = np.float32(np.nan)
    assert np.array_equal(mat.sum(axis=0), oracle_mod.calc_hist(m, np.where(both, u, nan), us, ue, nb))
    assert np.array_equal(mat.sum(axis=1), oracle_mod.calc_hist(m, np.where(both, v, nan), vs, ve, nb))
    assert int(h.sum()) == int(m.mask_values(both).sum())
