"""Column sharding on the GPU (potts_shard_*): every shard of a volume held by one process on one
GPU, linked so that their halos move by device copies (the multi-GPU protocol without a second
GPU; the ranks' kernels never wait on one another).  The owned voxels of all shards together must
equal the single-volume fused solve bit for bit (V, labels), the reduced convergence trace must
equal its trace, and the summed FP64 energies must equal its energies within 1e-9 relative (same
per-voxel terms, different summation order)."""
import numpy as np
import pytest

from segmentctscans_b200 import potts
from segmentctscans_b200.sharding import Shard, native_bounds, native_cuts, run_shards, solve_local
from tests._cases import TAU, TAU_BASELINE, phantom_volume, random_volume

pytestmark = pytest.mark.gpu

ENERGY_REL_TOL = 1e-9


def _check(m, whole, labels, V, st, K, ge):
    mv = m.mask_values
    assert np.array_equal(mv(labels.cpu().numpy()), mv(whole.labels))
    assert np.array_equal(mv(V.cpu().numpy().reshape(K - 1, -1)), mv(whole.V))
    np.testing.assert_array_equal(st.dq_trace, whole.stats.dq_trace)
    if ge:
        np.testing.assert_allclose(st.energy_trace[:, :2], whole.stats.energy_trace[:, :2], rtol=ENERGY_REL_TOL)


@pytest.mark.parametrize("world", [1, 2, 3, 5])
@pytest.mark.parametrize("K", [3, 4])
def test_local_shards_equal_whole_volume(cuda_device, world, K):
    import torch

    iters, ge = 15, 7
    m, u, ci = random_volume(24, 26, 31, 11.8, K, seed=40 + K)
    whole = potts.solve(m, u, ci, 30.0, TAU, TAU, iters, variant=0, gap_every=ge)
    du = torch.from_numpy(u).cuda()
    with potts.make_context(0, stream=torch.cuda.current_stream().cuda_stream) as ctx:
        labels, V, st = solve_local(ctx, m, du, ci, 30.0, TAU, TAU, iters, world, gap_every=ge)
    _check(m, whole, labels, V, st, K, ge)
    assert st.n_slabs == world and st.loop_iters == iters - 1 and st.loop_launches == world * (iters - 1)


@pytest.mark.parametrize("arith,storage", [("fast", "f32"), ("exact", "bf16"), ("fast", "f16")])
def test_local_shards_other_forms(cuda_device, arith, storage):
    """The fast arithmetic and the 16-bit storage (the bfloat16 V's stochastic rounding is keyed by
    global line numbers, so shards give the single volume's bits)."""
    import torch

    iters = 12
    m, u, ci = random_volume(70, 30, 34, 14.2, 3, seed=11)
    whole = potts.solve(m, u, ci, 30.0, TAU, TAU, iters, variant=0, arith=arith, storage=storage)
    with potts.make_context(0, stream=torch.cuda.current_stream().cuda_stream) as ctx:
        labels, V, st = solve_local(ctx, m, torch.from_numpy(u).cuda(), ci, 30.0, TAU, TAU, iters, 3, arith=arith,
                                    storage=storage)
    _check(m, whole, labels, V, st, 3, 0)


def test_local_shards_on_phantom(cuda_device):
    import torch

    m, u, ci, _ = phantom_volume(48, 21.0, seed=3, radius_range=(3.0, 8.0))
    whole = potts.solve(m, u, ci, 30.0, TAU_BASELINE, TAU_BASELINE, 60, variant=0, gap_every=20)
    with potts.make_context(0, stream=torch.cuda.current_stream().cuda_stream) as ctx:
        labels, V, st = solve_local(ctx, m, torch.from_numpy(u).cuda(), ci, 30.0, TAU_BASELINE, TAU_BASELINE, 60, 4,
                                    gap_every=20)
    _check(m, whole, labels, V, st, 3, 20)


@pytest.mark.parametrize("iters", [0, 1, 2])
def test_local_shards_short_runs(cuda_device, iters):
    import torch

    m, u, ci = random_volume(16, 20, 22, 9.1, 3, seed=5)
    whole = potts.solve(m, u, ci, 30.0, TAU, TAU, iters, variant=0)
    with potts.make_context(0, stream=torch.cuda.current_stream().cuda_stream) as ctx:
        labels, V, st = solve_local(ctx, m, torch.from_numpy(u).cuda(), ci, 30.0, TAU, TAU, iters, 2)
    mv = m.mask_values
    assert np.array_equal(mv(labels.cpu().numpy()), mv(whole.labels))
    assert np.array_equal(mv(V.cpu().numpy()), mv(whole.V))


def test_shard_errors(cuda_device):
    import torch

    from segmentctscans_b200._native import POTTS_EINVAL, PottsError

    m, u, ci = random_volume(16, 20, 22, 9.1, 3, seed=5)
    du = torch.from_numpy(u).cuda()
    cuts = native_cuts(m, 2)
    with potts.make_context(0) as ctx:
        ptr = [du.data_ptr() + 4 * native_bounds(m, cuts, r)[1][0] for r in range(2)]
        with pytest.raises(PottsError) as e:  # the split form has no shard
            Shard(ctx, m, cuts, 0, ptr[0], ci, 30.0, TAU, TAU, variant=1)
        assert e.value.status == POTTS_EINVAL
        a = Shard(ctx, m, cuts, 0, ptr[0], ci, 30.0, TAU, TAU)
        b = Shard(ctx, m, cuts, 1, ptr[1], ci, 30.0, TAU, TAU)
        with pytest.raises(PottsError):  # not linked
            run_shards([a, b], 5)
        with pytest.raises(PottsError):  # a shard alone of a two-way split without NCCL
            run_shards([b], 5)
        with pytest.raises(PottsError):  # ranks out of order
            b.link(a)
        a.link(b)
        run_shards([a, b], 5)
        a.close()
        b.close()


def test_single_rank_nccl_shard(cuda_device):
    """The NCCL path on one GPU: a one-rank communicator of the library's own (the exchange has no
    peer; the trace and energies go through NCCL all-reduces)."""
    import ctypes

    import torch

    from segmentctscans_b200 import _native
    from segmentctscans_b200.sharding import destroy_comm

    lib = _native.host_lib()
    idbuf = (ctypes.c_uint8 * 128)()
    _native.check(lib.potts_nccl_unique_id(idbuf))
    comm = ctypes.c_void_p()
    _native.check(lib.potts_nccl_comm_create(idbuf, 1, 0, 0, ctypes.byref(comm)))
    try:
        iters, ge = 14, 5
        m, u, ci = random_volume(24, 26, 31, 11.8, 3, seed=9)
        whole = potts.solve(m, u, ci, 30.0, TAU, TAU, iters, variant=0, gap_every=ge)
        du = torch.from_numpy(u).cuda()
        cuts = native_cuts(m, 1)
        with potts.make_context(0, stream=torch.cuda.current_stream().cuda_stream) as ctx:
            s = Shard(ctx, m, cuts, 0, du.data_ptr(), ci, 30.0, TAU, TAU, gap_every=ge)
            s.use_nccl(comm)
            lab = torch.zeros(m.span, dtype=torch.uint8, device="cuda")
            V = torch.zeros((2, m.span), dtype=torch.float32, device="cuda")
            st = run_shards([s], iters, label_ptrs=[lab.data_ptr()], V_ptrs=[V.data_ptr()])
            s.close()
        _check(m, whole, lab, V, st, 3, ge)
    finally:
        destroy_comm(comm)
