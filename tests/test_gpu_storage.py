"""GPU parity of the 16-bit storage formats (Xi, V, Vbar in bfloat16 or binary16, FP32 arithmetic).

Both kernel forms must equal the FP32 oracle run with the same storage rounding
bit for bit (same operations, same rounding of every stored value, the same
counter-hash bits for the stochastically rounded bfloat16 V).  Against the FP64
oracle the 128^3 phantom solve (500 iterations) must flip at most 1e-4 of the
in-mask labels, with the relative L2 error of V stated in the bound below.
"""
import numpy as np
import pytest

from segmentctscans_b200 import potts
from segmentctscans_b200._native import PottsError
from tests._cases import TAU, TAU_BASELINE, phantom_volume, random_volume
from tests.test_gpu_parity import CASES, assert_same

pytestmark = pytest.mark.gpu

STORES = ["bf16", "f16"]
FLIP_RATE_MAX = 1e-4                      # label flips / in-mask voxels against the FP64 oracle
V_REL_MAX = {"bf16": 3e-3, "f16": 1.5e-3}  # relative L2 of V against the FP64 oracle


@pytest.mark.parametrize("store", STORES)
@pytest.mark.parametrize("case", CASES, ids=[f"K{c[4]}" for c in CASES])
@pytest.mark.parametrize("variant", [1, 0], ids=["plain", "fused"])
def test_store_bitwise_equal_to_oracle(cuda_device, oracle_mod, case, variant, store):
    n, rows, cols, r, K, iters = case
    m, u, ci = random_volume(n, rows, cols, r, K, seed=K)
    g = potts.solve(m, u, ci, 30.0, TAU, TAU, iters, variant=variant, storage=store)
    o = oracle_mod.solve(m, u, ci, 30.0, TAU, TAU, iters, precision="f32", store=store)
    assert_same(m, g, o)
    np.testing.assert_array_equal(g.stats.dq_trace, o.dq_trace)


@pytest.mark.parametrize("store", STORES)
def test_store_fused_equals_split_on_phantom(cuda_device, store):
    m, u, ci, _ = phantom_volume(48, 21.0, seed=3, radius_range=(3.0, 8.0))
    a = potts.solve(m, u, ci, 30.0, TAU_BASELINE, TAU_BASELINE, 120, variant=0, storage=store)
    b = potts.solve(m, u, ci, 30.0, TAU_BASELINE, TAU_BASELINE, 120, variant=1, storage=store)
    mv = m.mask_values
    for name in ("V", "Xi", "labels", "res"):
        assert np.array_equal(mv(getattr(a, name)), mv(getattr(b, name))), name
    np.testing.assert_array_equal(a.stats.dq_trace, b.stats.dq_trace)
    # the state takes half the bytes of FP32
    f = potts.solve(m, u, ci, 30.0, TAU_BASELINE, TAU_BASELINE, 2, variant=0, want_state=False)
    assert 2 * a.stats.state_bytes == f.stats.state_bytes


@pytest.mark.parametrize("store", STORES)
@pytest.mark.parametrize("variant", [1, 0], ids=["plain", "fused"])
def test_store_slabs_and_unaligned_starts(cuda_device, oracle_mod, store, variant):
    """Slabs start at 0, 26, 52, 78: the hash keys use the global slice, u is staged."""
    m, u, ci = random_volume(100, 16, 16, 7.1, 3, seed=30)
    g = potts.solve(m, u, ci, 30.0, TAU, TAU, 7, variant=variant, slab_w=40, want_state=False, storage=store)
    o = oracle_mod.solve(m, u, ci, 30.0, TAU, TAU, 7, precision="f32", slab_w=40, want_state=False, store=store)
    assert g.stats.n_slabs == 4
    assert_same(m, g, o, what=("labels", "res"))


@pytest.mark.parametrize("store", STORES)
def test_store_energy_trace_matches_oracle(cuda_device, oracle_mod, store):
    m, u, ci = random_volume(24, 20, 20, 9.1, 3, seed=11)
    g = potts.solve(m, u, ci, 30.0, TAU, TAU, 40, variant=0, gap_every=10, want_state=False, storage=store)
    o = oracle_mod.solve(m, u, ci, 30.0, TAU, TAU, 40, precision="f32", gap_every=10, want_state=False, store=store)
    np.testing.assert_allclose(g.stats.energy_trace[:, :2], o.energy_trace[:, :2], rtol=1e-9)
    np.testing.assert_allclose(g.stats.energy_trace[:, 2], o.energy_trace[:, 2], rtol=1e-6, atol=1e-9)


STORE_TILE_SHAPES = {2: [(8, 128, 2), (8, 64, 4)], 3: [(16, 64, 2), (8, 128, 2)], 4: [(8, 64, 2)],
                     5: [(4, 64, 4), (8, 64, 2)], 6: [(4, 64, 4), (8, 64, 2)]}


@pytest.mark.parametrize("store", STORES)
def test_store_every_tile_shape_and_segment_length(cuda_device, oracle_mod, store):
    """Partial n-tiles (n = 150), halos, 1/3/64-column segments, K = 2 .. 6, every compiled tile."""
    for K in (2, 3, 4, 5, 6):
        m, u, ci = random_volume(150, 37, 35, 16.3, K, seed=20 + K)
        o = oracle_mod.solve(m, u, ci, 30.0, TAU, TAU, 9, precision="f32", store=store)
        for rows, slices, vpt in STORE_TILE_SHAPES[K]:
            for seg in (1, 3, 64):
                g = potts.solve(m, u, ci, 30.0, TAU, TAU, 9, variant=0, segment_cols=seg, storage=store,
                                tile_rows=rows, tile_slices=slices, tile_vpt=vpt)
                assert_same(m, g, o)


def test_store_rejects_uncompiled_tile_shape(cuda_device):
    m, u, ci = random_volume(16, 10, 10, 4.4, 3, seed=31)
    with pytest.raises(PottsError) as e:
        potts.solve(m, u, ci, 30.0, TAU, TAU, 5, variant=0, tile_rows=8, tile_slices=64, tile_vpt=2,
                    storage="bf16")
    assert e.value.status == 1
    with pytest.raises(PottsError) as e:
        potts.solve(m, u, ci, 30.0, TAU, TAU, 5, storage=7)
    assert e.value.status == 1


@pytest.fixture(scope="module")
def config0_fp64(oracle_mod):
    from segmentctscans_b200.phantom import config0_phantom

    ph = config0_phantom(seed=0, device="cpu")
    m, u, ci = ph.mapping, ph.u.numpy().copy(), ph.ci
    o = oracle_mod.solve(m, u, ci, 30.0, TAU_BASELINE, TAU_BASELINE, 500, precision="f64")
    return m, u, ci, o


@pytest.mark.parametrize("store", STORES)
def test_store_quality_against_fp64_oracle(cuda_device, config0_fp64, store):
    """128^3, r = 60, K = 3, lam = 30, tau = tau' = 1/sqrt(12), 500 iterations."""
    m, u, ci, o = config0_fp64
    g = potts.solve(m, u, ci, 30.0, TAU_BASELINE, TAU_BASELINE, 500, variant=0, storage=store)
    mv = m.mask_values
    flips = int(np.sum(mv(g.labels) != mv(o.labels)))
    rate = flips / mv(o.labels).size
    rel = float(np.linalg.norm(mv(g.V) - mv(o.V)) / np.linalg.norm(mv(o.V)))
    print(f"{store}: label flips {flips} ({rate:.2e}), V rel L2 {rel:.2e}")
    assert rate <= FLIP_RATE_MAX
    assert rel <= V_REL_MAX[store]
