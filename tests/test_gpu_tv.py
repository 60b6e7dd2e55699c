"""TV-L2 (ROF) denoising on the GPU (potts_tv_denoise, chambolle() of
totalvarmin/chambolle.cpp): bit-identical to the FP32 oracle (result and the per-iteration
max |dxi|^2), within 1e-5 relative L2 of the FP64 oracle."""
import numpy as np
import pytest

from segmentctscans_b200 import potts
from segmentctscans_b200._native import PottsError
from tests._cases import phantom_volume, random_volume

pytestmark = pytest.mark.gpu

TAU_TV = 0.99 / 6.0  # totalvarmin/totalvarmin.cpp:140


@pytest.mark.parametrize("geom", [
    (20, 18, 17, 7.9, 30),
    (33, 21, 19, 9.3, 25),
    (1, 9, 9, 4.0, 10),       # a single slice
    (5, 3, 40, 1.2, 12),      # columns of one row
    (12, 10, 10, 4.3, 0),     # zero iterations
])
@pytest.mark.parametrize("variant", [0, 1, 2], ids=["tiled", "plain", "fused_voxel"])
def test_tv_bitwise_equal_to_fp32_oracle(cuda_device, oracle_mod, geom, variant):
    n, rows, cols, r, iters = geom
    m, u, _ = random_volume(n, rows, cols, r, 3, seed=n + cols)
    out, st = potts.tv_denoise_host(m, u, 0.1, TAU_TV, iters, variant=variant)
    ref, dq = oracle_mod.tv(m, u, 0.1, TAU_TV, iters, "f32")
    mv = m.mask_values
    assert np.array_equal(mv(out), mv(ref))
    if iters:
        np.testing.assert_array_equal(st.dq_trace, dq)
        assert st.loop_launches == (2 if variant == 1 else 1) * iters


def test_tv_against_fp64_oracle_on_phantom(cuda_device, oracle_mod):
    m, u, ci, _ = phantom_volume(48, 21.0, seed=3, radius_range=(3.0, 8.0))
    out, _ = potts.tv_denoise_host(m, u, 0.05, TAU_TV, 150)
    ref, _ = oracle_mod.tv(m, u, 0.05, TAU_TV, 150, "f64")
    mv = m.mask_values
    assert np.linalg.norm(mv(out) - mv(ref)) <= 1e-5 * np.linalg.norm(mv(ref))
    # the field moved: denoising did something
    assert np.linalg.norm(mv(out) - mv(u)) > 1e-3 * np.linalg.norm(mv(u))


def test_tv_errors(cuda_device):
    m, u, _ = random_volume(8, 8, 8, 3.5, 3, seed=2)
    with potts.make_context(0) as ctx:
        fld = potts.upload(ctx, m, u)
        with pytest.raises(PottsError):
            potts.tv_denoise(ctx, m, fld.data_ptr(), 0.0, TAU_TV, 5)
        with pytest.raises(PottsError):
            potts.tv_denoise(ctx, m, fld.data_ptr(), 0.1, TAU_TV, -1)
        potts.tv_denoise(ctx, m, fld.data_ptr(), 0.1, TAU_TV, 3)


def test_tv_unaligned_field_pointer(cuda_device, oracle_mod):
    """A field that does not start on a 16-byte word (the tiled kernel reads g only through its
    difference planes): same bits."""
    import torch

    m, u, _ = random_volume(21, 14, 15, 6.2, 3, seed=9)
    ref, _ = oracle_mod.tv(m, u, 0.1, TAU_TV, 9, "f32")
    buf = torch.zeros(m.span + 1, dtype=torch.float32, device="cuda")
    buf[1:] = torch.from_numpy(u).cuda()
    with potts.make_context(0, stream=torch.cuda.current_stream().cuda_stream) as ctx:
        st = potts.tv_denoise(ctx, m, buf.data_ptr() + 4, 0.1, TAU_TV, 9, variant=0)
        ctx.synchronize()
    assert st.loop_launches == 9
    out = buf[1:].cpu().numpy()
    assert np.array_equal(m.mask_values(out), m.mask_values(ref))
