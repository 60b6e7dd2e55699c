"""The fast FP32 arithmetic (arith="fast") through the C ABI.

The fast form computes the reference iteration with fewer operations, so it is not bit-identical
to the FP32 oracle; it is held to the FP64 oracle with the plain form's bar (relative L2 of V within
1e-5 after 500 iterations of the 128^3 case, argmax labels equal except where the FP64 maximum is
tied).  Its split and fused kernels run the same operations per voxel, so they must agree bit for
bit on every geometry, tile shape, segment length, slab cut and storage format; that is what
catches an indexing error in the tiled kernel's fast path.
"""
import numpy as np
import pytest

from segmentctscans_b200 import potts
from tests._cases import TAU, TAU_BASELINE, phantom_volume, random_volume

pytestmark = pytest.mark.gpu

V_REL_TOL_FP64 = 1e-5   # relative L2 of V against the FP64 oracle (128^3, 500 iterations)
V_REL_TOL_F32 = 1e-4    # relative L2 of V against the exact FP32 form on small random cases


def _same(m, a, b, what=("V", "Xi", "labels", "res")):
    mv = m.mask_values
    for name in what:
        x, y = mv(getattr(a, name)), mv(getattr(b, name))
        assert np.array_equal(x, y), f"{name} differs in {int(np.sum(x != y))} voxels"


CASES = [
    # n, rows, cols, r, K, iters
    (20, 18, 17, 7.9, 2, 25),
    (33, 21, 19, 9.3, 3, 30),
    (16, 24, 24, 11.2, 4, 20),
    (40, 15, 13, 6.4, 5, 15),
    (9, 17, 20, 8.1, 6, 20),
    (1, 9, 9, 4.0, 3, 5),      # a single slice
    (33, 6, 6, 2.6, 3, 12),    # n not a multiple of 32, short columns
    (5, 3, 40, 1.2, 2, 7),     # columns of one row
    (12, 10, 10, 4.3, 4, 1),   # one iteration
]


@pytest.mark.parametrize("case", CASES, ids=[f"K{c[4]}_n{c[0]}_it{c[5]}" for c in CASES])
def test_fast_fused_equals_fast_split(cuda_device, oracle_mod, case):
    n, rows, cols, r, K, iters = case
    m, u, ci = random_volume(n, rows, cols, r, K, seed=K + 7 * n)
    f = potts.solve(m, u, ci, 30.0, TAU, TAU, iters, variant=0, arith="fast")
    s = potts.solve(m, u, ci, 30.0, TAU, TAU, iters, variant=1, arith="fast")
    _same(m, f, s)
    np.testing.assert_array_equal(f.stats.dq_trace, s.stats.dq_trace)
    # and close to the exact FP32 form (same iteration, different rounding)
    o = oracle_mod.solve(m, u, ci, 30.0, TAU, TAU, iters, precision="f64")
    mv = m.mask_values
    if np.linalg.norm(mv(o.V)) > 0:
        rel = np.linalg.norm(mv(f.V) - mv(o.V)) / np.linalg.norm(mv(o.V))
        assert rel <= V_REL_TOL_F32, rel


TILE_SHAPES = {2: [(8, 128, 2), (8, 64, 4)], 3: [(16, 64, 2), (8, 128, 2), (8, 64, 2), (8, 128, 4)],
               4: [(8, 64, 2), (8, 64, 4), (4, 128, 4)], 5: [(4, 64, 4), (8, 64, 2)], 6: [(4, 64, 4)]}


@pytest.mark.parametrize("K", [2, 3, 4, 5, 6])
def test_fast_every_tile_shape_and_segment_length(cuda_device, K):
    """Partial n-tiles (n = 150), the n/row halos, segment starts and ends, against the split form."""
    m, u, ci = random_volume(150, 37, 35, 16.3, K, seed=40 + K)
    s = potts.solve(m, u, ci, 30.0, TAU, TAU, 9, variant=1, arith="fast")
    for rows, slices, vpt in TILE_SHAPES[K]:
        for seg in (1, 3, 32, 64):
            f = potts.solve(m, u, ci, 30.0, TAU, TAU, 9, variant=0, arith="fast", tile_rows=rows,
                            tile_slices=slices, tile_vpt=vpt, segment_cols=seg)
            _same(m, f, s)


@pytest.mark.parametrize("storage", ["bf16", "f16"])
@pytest.mark.parametrize("K", [3, 4])
def test_fast_16bit_fused_equals_split(cuda_device, storage, K):
    m, u, ci = random_volume(70, 22, 21, 9.9, K, seed=50 + K)
    f = potts.solve(m, u, ci, 30.0, TAU, TAU, 20, variant=0, arith="fast", storage=storage)
    s = potts.solve(m, u, ci, 30.0, TAU, TAU, 20, variant=1, arith="fast", storage=storage)
    _same(m, f, s)


def test_fast_slabs_and_padded_stride(cuda_device):
    m, u, ci = random_volume(100, 16, 16, 7.1, 3, seed=30)
    f = potts.solve(m, u, ci, 30.0, TAU, TAU, 7, variant=0, arith="fast", slab_w=40, want_state=False)
    s = potts.solve(m, u, ci, 30.0, TAU, TAU, 7, variant=1, arith="fast", slab_w=40, want_state=False)
    assert f.stats.n_slabs == 4
    _same(m, f, s, what=("labels", "res"))
    m, u, ci = random_volume(20, 12, 12, 5.5, 3, seed=13, nstride=96)
    _same(m, potts.solve(m, u, ci, 30.0, TAU, TAU, 15, variant=0, arith="fast"),
          potts.solve(m, u, ci, 30.0, TAU, TAU, 15, variant=1, arith="fast"))


def test_fast_on_phantom_equals_split(cuda_device):
    m, u, ci, _ = phantom_volume(48, 21.0, seed=3, radius_range=(3.0, 8.0))
    a = potts.solve(m, u, ci, 30.0, TAU_BASELINE, TAU_BASELINE, 120, variant=0, arith="fast", gap_every=40)
    b = potts.solve(m, u, ci, 30.0, TAU_BASELINE, TAU_BASELINE, 120, variant=1, arith="fast", gap_every=40)
    _same(m, a, b)
    np.testing.assert_array_equal(a.stats.energy_trace, b.stats.energy_trace)


def _tie_mask(V64):
    full = np.concatenate([V64, 1.0 - V64.sum(0, keepdims=True)])
    s = np.sort(full, axis=0)
    return s[-1] == s[-2]


def test_fast_config0_against_fp64_oracle(cuda_device, oracle_mod):
    """128^3, r = 60, K = 3, lam = 30, tau = tau' = 1/sqrt(12), 500 iterations."""
    from segmentctscans_b200.phantom import config0_phantom

    ph = config0_phantom(seed=0, device="cpu")
    m, u, ci = ph.mapping, ph.u.numpy().copy(), ph.ci
    iters = 500
    o = oracle_mod.solve(m, u, ci, 30.0, TAU_BASELINE, TAU_BASELINE, iters, precision="f64")
    mv = m.mask_values
    ties = _tie_mask(mv(o.V))
    for variant in (0, 1):
        g = potts.solve(m, u, ci, 30.0, TAU_BASELINE, TAU_BASELINE, iters, variant=variant, arith="fast")
        rel = np.linalg.norm(mv(g.V) - mv(o.V)) / np.linalg.norm(mv(o.V))
        assert rel <= V_REL_TOL_FP64, f"variant {variant}: V rel err {rel:.3e}"
        diff = mv(g.labels) != mv(o.labels)
        assert not np.any(diff & ~ties), f"variant {variant}: {int(np.sum(diff & ~ties))} label flips off ties"


def test_unknown_arith_is_rejected(cuda_device):
    m, u, ci = random_volume(16, 10, 10, 4.4, 3, seed=31)
    from segmentctscans_b200._native import PottsError

    with pytest.raises(PottsError) as e:
        potts.solve(m, u, ci, 30.0, TAU, TAU, 5, arith=2)
    assert e.value.status == 1
