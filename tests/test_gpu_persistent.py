"""The persistent form of the fused iteration (potts_options.persistent = 1).

One cooperative launch runs every iteration between two energy evaluations: the blocks take the
work items of an iteration from a counter and meet at a grid-wide barrier before the next one.
The order in which blocks take items does not change any voxel's arithmetic, so the persistent
launch must give the bits of one launch per iteration (persistent = 0) for every K, storage format,
arithmetic, tile shape and energy cadence, and a batch run as one persistent launch must give the
bits of its volumes' single solves.
"""
import numpy as np
import pytest

from segmentctscans_b200 import potts
from tests._cases import TAU, random_volume

pytestmark = pytest.mark.gpu


def _same(m, a, b):
    mv = m.mask_values
    for name in ("V", "Xi", "labels", "res"):
        x, y = mv(getattr(a, name)), mv(getattr(b, name))
        assert np.array_equal(x, y), f"{name} differs in {int(np.sum(x != y))} voxels"
    np.testing.assert_array_equal(a.stats.dq_trace, b.stats.dq_trace)


CASES = [
    # n, rows, cols, r, K, iters, gap_every
    (20, 18, 17, 7.9, 2, 25, 0),
    (33, 21, 19, 9.3, 3, 30, 7),
    (16, 24, 24, 11.2, 4, 20, 5),
    (40, 15, 13, 6.4, 5, 15, 0),
    (9, 17, 20, 8.1, 6, 20, 3),
    (70, 40, 38, 18.1, 3, 23, 5),
]


@pytest.mark.parametrize("arith", ["exact", "fast"])
@pytest.mark.parametrize("case", CASES, ids=[f"K{c[4]}_it{c[5]}_gap{c[6]}" for c in CASES])
def test_persistent_equals_one_launch_per_iteration(cuda_device, case, arith):
    n, rows, cols, r, K, iters, ge = case
    m, u, ci = random_volume(n, rows, cols, r, K, seed=K + 3 * n)
    a = potts.solve(m, u, ci, 30.0, TAU, TAU, iters, variant=0, arith=arith, gap_every=ge, persistent=1)
    b = potts.solve(m, u, ci, 30.0, TAU, TAU, iters, variant=0, arith=arith, gap_every=ge, persistent=0)
    _same(m, a, b)
    if ge:
        np.testing.assert_array_equal(a.stats.energy_trace, b.stats.energy_trace)
    # one launch per run of iterations between energy evaluations
    runs = 1 if not ge else len({(mm + ge - 1) // ge for mm in range(1, iters)})
    assert a.stats.loop_launches == runs and a.stats.loop_iters == iters - 1
    assert b.stats.loop_launches == iters - 1 and b.stats.loop_iters == iters - 1


@pytest.mark.parametrize("storage", ["bf16", "f16"])
def test_persistent_16bit_storage(cuda_device, storage):
    m, u, ci = random_volume(70, 22, 21, 9.9, 3, seed=52)
    a = potts.solve(m, u, ci, 30.0, TAU, TAU, 20, variant=0, storage=storage, persistent=1)
    b = potts.solve(m, u, ci, 30.0, TAU, TAU, 20, variant=0, storage=storage, persistent=0)
    _same(m, a, b)


def test_persistent_every_tile_shape_and_segment_length(cuda_device):
    m, u, ci = random_volume(150, 37, 35, 16.3, 3, seed=43)
    ref = potts.solve(m, u, ci, 30.0, TAU, TAU, 9, variant=1)
    for rows, slices, vpt in [(16, 64, 2), (8, 128, 2), (8, 64, 2), (8, 128, 4)]:
        for seg in (1, 3, 64):
            f = potts.solve(m, u, ci, 30.0, TAU, TAU, 9, variant=0, tile_rows=rows, tile_slices=slices,
                            tile_vpt=vpt, segment_cols=seg, persistent=1)
            _same(m, f, ref)


def test_persistent_slabs(cuda_device):
    m, u, ci = random_volume(100, 16, 16, 7.1, 3, seed=30)
    a = potts.solve(m, u, ci, 30.0, TAU, TAU, 7, variant=0, slab_w=40, want_state=False, persistent=1)
    b = potts.solve(m, u, ci, 30.0, TAU, TAU, 7, variant=1, slab_w=40, want_state=False)
    assert a.stats.n_slabs == 4
    mv = m.mask_values
    assert np.array_equal(mv(a.labels), mv(b.labels)) and np.array_equal(mv(a.res), mv(b.res))


def test_sync_monitor_runs_one_launch_per_iteration(cuda_device):
    m, u, ci = random_volume(33, 21, 19, 9.3, 3, seed=5)
    a = potts.solve(m, u, ci, 30.0, TAU, TAU, 12, variant=0, sync_monitor=1, persistent=1)
    b = potts.solve(m, u, ci, 30.0, TAU, TAU, 12, variant=0, persistent=1)
    _same(m, a, b)
    assert a.stats.loop_launches == 11 and b.stats.loop_launches == 1


def test_persistent_option_is_checked(cuda_device):
    from segmentctscans_b200._native import POTTS_EINVAL, PottsError

    m, u, ci = random_volume(16, 10, 10, 4.4, 3, seed=31)
    with pytest.raises(PottsError) as e:
        potts.solve(m, u, ci, 30.0, TAU, TAU, 5, persistent=2)
    assert e.value.status == POTTS_EINVAL
