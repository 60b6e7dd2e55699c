"""GPU parity: the sm_100a kernels, called through the C ABI, against the CPU oracle.

FP32 forms (split and fused) must equal the FP32 oracle exactly (same IEEE
operations in the same order; +0 and -0 compare equal).  Against the FP64
oracle the FP32 solve must be within 1e-5 relative L2 on V, with identical
argmax labels except where the FP64 maximum is tied.
"""
import numpy as np
import pytest

from segmentctscans_b200 import potts
from segmentctscans_b200._native import PottsError
from tests._cases import TAU, TAU_BASELINE, phantom_volume, random_volume

pytestmark = pytest.mark.gpu

V_REL_TOL_FP64 = 1e-5   # relative L2 of V against the FP64 oracle
ENERGY_REL_TOL = 1e-9   # FP64 energies: same per-voxel terms, different summation order


def gpu_solve(m, u, ci, lam, tau1, tau2, iters, **opts):
    return potts.solve(m, u, ci, lam, tau1, tau2, iters, **opts)


def assert_same(m, gpu, orc, what=("V", "Xi", "labels", "res")):
    mv = m.mask_values
    for name in what:
        a = getattr(gpu, name)
        b = getattr(orc, name)
        assert np.array_equal(mv(a), mv(b.astype(a.dtype))), f"{name} differs in {np.sum(mv(a) != mv(b))} voxels"


CASES = [
    # n, rows, cols, r, K, iters
    (20, 18, 17, 7.9, 2, 25),
    (33, 21, 19, 9.3, 3, 30),
    (16, 24, 24, 11.2, 4, 20),
    (40, 15, 13, 6.4, 5, 15),
    (9, 17, 20, 8.1, 6, 20),
]


@pytest.mark.parametrize("case", CASES, ids=[f"K{c[4]}" for c in CASES])
@pytest.mark.parametrize("variant", [1, 0], ids=["plain", "fused"])
def test_fp32_bitwise_equal_to_oracle(cuda_device, oracle_mod, case, variant):
    n, rows, cols, r, K, iters = case
    m, u, ci = random_volume(n, rows, cols, r, K, seed=K)
    g = gpu_solve(m, u, ci, 30.0, TAU, TAU, iters, variant=variant)
    o = oracle_mod.solve(m, u, ci, 30.0, TAU, TAU, iters, precision="f32")
    assert_same(m, g, o)
    np.testing.assert_array_equal(g.stats.dq_trace, o.dq_trace)


def test_fused_equals_split_on_phantom(cuda_device):
    m, u, ci, _ = phantom_volume(48, 21.0, seed=3, radius_range=(3.0, 8.0))
    a = gpu_solve(m, u, ci, 30.0, TAU_BASELINE, TAU_BASELINE, 120, variant=0)
    b = gpu_solve(m, u, ci, 30.0, TAU_BASELINE, TAU_BASELINE, 120, variant=1)
    mv = m.mask_values
    for name in ("V", "Xi", "labels", "res"):
        assert np.array_equal(mv(getattr(a, name)), mv(getattr(b, name))), name
    np.testing.assert_array_equal(a.stats.dq_trace, b.stats.dq_trace)


def _tie_mask(V64):
    """Voxels whose two largest V (all K labels) are exactly equal in the FP64 oracle."""
    full = np.concatenate([V64, 1.0 - V64.sum(0, keepdims=True)])
    s = np.sort(full, axis=0)
    return s[-1] == s[-2]


def test_config0_against_fp64_oracle(cuda_device, oracle_mod):
    """128^3, r = 60, K = 3, lam = 30, tau = tau' = 1/sqrt(12), 500 iterations (the plain-form parity case)."""
    from segmentctscans_b200.phantom import config0_phantom

    ph = config0_phantom(seed=0, device="cpu")
    m, u, ci = ph.mapping, ph.u.numpy().copy(), ph.ci
    iters = 500
    o = oracle_mod.solve(m, u, ci, 30.0, TAU_BASELINE, TAU_BASELINE, iters, precision="f64")
    mv = m.mask_values
    ties = _tie_mask(mv(o.V))
    for variant in (1, 0):
        g = gpu_solve(m, u, ci, 30.0, TAU_BASELINE, TAU_BASELINE, iters, variant=variant)
        rel = np.linalg.norm(mv(g.V) - mv(o.V)) / np.linalg.norm(mv(o.V))
        assert rel <= V_REL_TOL_FP64, f"variant {variant}: V rel err {rel:.3e}"
        diff = mv(g.labels) != mv(o.labels)
        assert not np.any(diff & ~ties), f"variant {variant}: {int(np.sum(diff & ~ties))} label flips off ties"


def test_energy_trace_matches_oracle(cuda_device, oracle_mod):
    m, u, ci = random_volume(24, 20, 20, 9.1, 3, seed=11)
    for variant in (1, 0):
        g = gpu_solve(m, u, ci, 30.0, TAU, TAU, 40, variant=variant, gap_every=10, want_state=False)
        o = oracle_mod.solve(m, u, ci, 30.0, TAU, TAU, 40, precision="f32", gap_every=10, want_state=False)
        assert g.stats.energy_trace.shape == (4, 3)
        np.testing.assert_allclose(g.stats.energy_trace[:, :2], o.energy_trace[:, :2], rtol=ENERGY_REL_TOL)
        np.testing.assert_allclose(g.stats.energy_trace[:, 2], o.energy_trace[:, 2], rtol=1e-6, atol=1e-9)


@pytest.mark.parametrize("variant", [1, 0], ids=["plain", "fused"])
def test_forced_slabs_match_oracle_slabs(cuda_device, oracle_mod, variant):
    m, u, ci = random_volume(90, 14, 15, 6.6, 3, seed=12)
    iters = 8
    g = gpu_solve(m, u, ci, 30.0, TAU, TAU, iters, variant=variant, slab_w=40, want_state=False)
    o = oracle_mod.solve(m, u, ci, 30.0, TAU, TAU, iters, precision="f32", slab_w=40, want_state=False)
    assert g.stats.n_slabs == 1 + (90 - 40 + 24 - 1) // 24
    assert_same(m, g, o, what=("labels", "res"))
    whole = oracle_mod.solve(m, u, ci, 30.0, TAU, TAU, iters, precision="f32", want_state=False)
    assert_same(m, g, whole, what=("labels", "res"))


@pytest.mark.parametrize("geom", [
    (1, 9, 9, 4.0, 3, 5),       # a single slice
    (33, 6, 6, 2.6, 3, 12),     # n not a multiple of 32, short columns
    (5, 3, 40, 1.2, 2, 7),      # columns of one row
    (12, 10, 10, 4.3, 3, 0),    # zero iterations: nearest label
    (12, 10, 10, 4.3, 4, 1),    # one iteration
])
@pytest.mark.parametrize("variant", [1, 0], ids=["plain", "fused"])
def test_edge_geometries(cuda_device, oracle_mod, geom, variant):
    n, rows, cols, r, K, iters = geom
    m, u, ci = random_volume(n, rows, cols, r, K, seed=n + rows)
    g = gpu_solve(m, u, ci, 30.0, TAU, TAU, iters, variant=variant)
    o = oracle_mod.solve(m, u, ci, 30.0, TAU, TAU, iters, precision="f32")
    assert_same(m, g, o)


def test_padded_stride(cuda_device, oracle_mod):
    m, u, ci = random_volume(20, 12, 12, 5.5, 3, seed=13, nstride=96)
    g = gpu_solve(m, u, ci, 30.0, TAU, TAU, 15)
    o = oracle_mod.solve(m, u, ci, 30.0, TAU, TAU, 15, precision="f32")
    assert_same(m, g, o)


def test_field_api_roundtrip(cuda_device, oracle_mod):
    """make_context / upload / potts_min_partition / download, as potts-model.cpp:139-179 uses them."""
    m, u, ci = random_volume(24, 16, 16, 7.2, 3, seed=14)
    with potts.make_context(0) as ctx:
        g = potts.upload(ctx, m, u)
        np.testing.assert_array_equal(potts.download(ctx, g), u)
        res, st = potts.potts_min_partition(ctx, g, m, ci, 30.0, TAU, TAU, 20, stats=True)
        out = potts.download(ctx, res)
        assert st.n_slabs == 1 and st.iters == 20 and st.solve_ms > 0
        avail, total = potts.device_memory(ctx)
        assert 0 < avail <= total
    o = oracle_mod.solve(m, u, ci, 30.0, TAU, TAU, 20, precision="f32")
    mv = m.mask_values
    assert np.array_equal(mv(out), mv(o.res))


def test_host_form_matches_device_form(cuda_device):
    m, u, ci = random_volume(30, 18, 18, 8.3, 4, seed=15)
    d = gpu_solve(m, u, ci, 30.0, TAU, TAU, 25)
    with potts.make_context(0) as ctx:
        res = np.zeros(m.span, np.float32)
        lab = np.zeros(m.span, np.uint8)
        potts.solve_host(ctx, m, u, ci, 30.0, TAU, TAU, 25, res=res, labels=lab)
        mv = m.mask_values
        assert np.array_equal(mv(lab), mv(d.labels)) and np.array_equal(mv(res), mv(d.res))
        # reference behaviour: read the monitor back after every iteration; same result
        res2 = np.zeros(m.span, np.float32)
        st = potts.solve_host(ctx, m, u, ci, 30.0, TAU, TAU, 25, res=res2, stats=True, sync_monitor=1)
        assert np.array_equal(mv(res2), mv(res)) and st.dq_last > 0


def test_errors_are_reported(cuda_device):
    m, u, ci = random_volume(16, 10, 10, 4.4, 3, seed=16)
    with potts.make_context(0) as ctx:
        g = potts.upload(ctx, m, u)
        with pytest.raises(ValueError):
            potts.potts_min_partition(ctx, g, m, [0.1] * 7, 30.0, TAU, TAU, 5)
        with pytest.raises(PottsError) as e:
            potts.potts_min_partition(ctx, g, m, ci, float("nan"), TAU, TAU, 5)
        assert e.value.status == 1
        with pytest.raises(PottsError) as e:
            potts.potts_min_partition(ctx, g, m, ci, 30.0, TAU, TAU, -1)
        assert e.value.status == 1
        # a slab narrower than 2 * iters + 1: the reference's "Not enough memory" path
        with pytest.raises(PottsError) as e:
            potts.potts_min_partition(ctx, g, m, ci, 30.0, TAU, TAU, 8, slab_w=10)
        assert e.value.status == 2 and "Not enough memory" in str(e.value)
        # the context stays usable after errors
        res = potts.potts_min_partition(ctx, g, m, ci, 30.0, TAU, TAU, 3)
        assert res.span == m.span


TILE_SHAPES = {2: [(8, 128, 2), (8, 64, 4)], 3: [(8, 128, 2), (16, 64, 2), (8, 64, 2), (8, 128, 4)],
               4: [(8, 64, 2), (8, 64, 4), (4, 128, 4)], 5: [(4, 64, 4), (8, 64, 2)], 6: [(4, 64, 4)]}


@pytest.mark.parametrize("K", [2, 3, 4, 5, 6])
def test_every_tile_shape_and_segment_length(cuda_device, oracle_mod, K):
    """Partial n-tiles (n = 150), the n/row halos, segment starts and ends (1, 3 and 32 columns)."""
    m, u, ci = random_volume(150, 37, 35, 16.3, K, seed=20 + K)
    o = oracle_mod.solve(m, u, ci, 30.0, TAU, TAU, 9, precision="f32")
    for rows, slices, vpt in TILE_SHAPES[K]:
        for seg in (1, 3, 32, 64):
            g = gpu_solve(m, u, ci, 30.0, TAU, TAU, 9, variant=0, tile_rows=rows, tile_slices=slices,
                          tile_vpt=vpt, segment_cols=seg)
            assert_same(m, g, o)


def test_unaligned_slab_starts_stage_u(cuda_device, oracle_mod):
    """iters = 7, slab_w = 40: slabs start at 0, 26, 52, 78 (u staged when not 16-byte aligned)."""
    m, u, ci = random_volume(100, 16, 16, 7.1, 3, seed=30)
    g = gpu_solve(m, u, ci, 30.0, TAU, TAU, 7, variant=0, slab_w=40, want_state=False)
    o = oracle_mod.solve(m, u, ci, 30.0, TAU, TAU, 7, precision="f32", slab_w=40, want_state=False)
    assert g.stats.n_slabs == 4
    assert_same(m, g, o, what=("labels", "res"))


def test_unknown_tile_shape_is_rejected(cuda_device):
    m, u, ci = random_volume(16, 10, 10, 4.4, 3, seed=31)
    with pytest.raises(PottsError) as e:
        gpu_solve(m, u, ci, 30.0, TAU, TAU, 5, variant=0, tile_rows=5, tile_slices=40)
    assert e.value.status == 1
    with pytest.raises(PottsError):
        gpu_solve(m, u, ci, 30.0, TAU, TAU, 5, variant=0, segment_cols=65)
