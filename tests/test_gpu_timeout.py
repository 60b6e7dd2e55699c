"""The fused kernel's bounded waits run out without faulting the GPU.

potts_options.stall_plane makes the first work item's load warp skip the loads of one plane.  The
row warps' waits for that plane then give up after their limit, the block sets its abort flag,
drains its loads in flight and returns, and the solve reports POTTS_ETIMEOUT.  No wait is left
unbounded, nothing faults, and the same context then solves the same input bit for bit like the
FP32 oracle.
"""
import numpy as np
import pytest

from segmentctscans_b200 import _native, potts
from tests._cases import TAU, random_volume

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("arith", ["exact", "fast"])
def test_stalled_plane_times_out_and_context_stays_usable(cuda_device, oracle_mod, arith):
    import torch

    m, u, ci = random_volume(64, 24, 24, 11.0, 3, seed=60)
    iters = 2  # one fused launch
    with potts.make_context(0, stream=torch.cuda.current_stream().cuda_stream) as ctx:
        with pytest.raises(_native.PottsError) as e:
            potts.solve(m, u, ci, 30.0, TAU, TAU, iters, ctx=ctx, variant=0, arith=arith, stall_plane=2)
        assert e.value.status == _native.POTTS_ETIMEOUT
        g = potts.solve(m, u, ci, 30.0, TAU, TAU, iters, ctx=ctx, variant=0, arith=arith)
        s = potts.solve(m, u, ci, 30.0, TAU, TAU, iters, ctx=ctx, variant=1, arith=arith)
    mv = m.mask_values
    for name in ("V", "Xi", "labels"):
        assert np.array_equal(mv(getattr(g, name)), mv(getattr(s, name))), name
    if arith == "exact":
        o = oracle_mod.solve(m, u, ci, 30.0, TAU, TAU, iters, precision="f32")
        assert np.array_equal(mv(g.V), mv(o.V.astype(np.float32)))
        assert np.array_equal(mv(g.labels), mv(o.labels))


def test_stall_plane_must_not_be_negative(cuda_device):
    m, u, ci = random_volume(16, 10, 10, 4.4, 3, seed=61)
    with pytest.raises(_native.PottsError) as e:
        potts.solve(m, u, ci, 30.0, TAU, TAU, 3, stall_plane=-1)
    assert e.value.status == _native.POTTS_EINVAL
