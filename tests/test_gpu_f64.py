"""The FP64 solve (potts_solve_device_f64, storage "f64") against the FP64 CPU oracle.

The FP64 kernels restate the oracle's double-precision operations in the same order (multiply-adds
fused at the same places, IEEE division and square root), so V, Xi, the labels and the convergence
trace must come out identical; the tolerance below only allows for that not to hold bit for bit on
some input (it is far below any difference between the FP64 and the FP32 solve).  This solve is
the yardstick of the FP32 and 16-bit forms on volumes too large for the CPU oracle.
"""
import numpy as np
import pytest

from segmentctscans_b200 import potts
from tests._cases import TAU, TAU_BASELINE, random_volume

pytestmark = pytest.mark.gpu

V_REL_TOL = 1e-12  # relative L2 of V (and Xi) against the FP64 oracle


def _check(m, g, o, iters):
    mv = m.mask_values
    for name in ("V", "Xi"):
        a, b = mv(getattr(g, name)), mv(getattr(o, name))
        assert a.dtype == np.float64
        scale = max(np.linalg.norm(b), 1e-300)
        assert np.linalg.norm(a - b) / scale <= V_REL_TOL, name
    assert np.array_equal(mv(g.labels), mv(o.labels))
    assert np.array_equal(mv(g.res), mv(o.res))
    if iters > 0:
        np.testing.assert_array_equal(g.stats.dq_trace, o.dq_trace)


CASES = [
    # n, rows, cols, r, K, iters
    (20, 18, 17, 7.9, 2, 25),
    (33, 21, 19, 9.3, 3, 30),
    (16, 24, 24, 11.2, 4, 20),
    (40, 15, 13, 6.4, 5, 15),
    (9, 17, 20, 8.1, 6, 20),
    (1, 9, 9, 4.0, 3, 5),      # a single slice
    (5, 3, 40, 1.2, 2, 7),     # columns of one row
    (12, 10, 10, 4.3, 3, 0),   # zero iterations: nearest label
]


@pytest.mark.parametrize("case", CASES, ids=[f"K{c[4]}_n{c[0]}_it{c[5]}" for c in CASES])
def test_f64_solve_equals_fp64_oracle(cuda_device, oracle_mod, case):
    n, rows, cols, r, K, iters = case
    m, u, ci = random_volume(n, rows, cols, r, K, seed=K + n)
    g = potts.solve(m, u, ci, 30.0, TAU, TAU, iters, storage="f64")
    o = oracle_mod.solve(m, u, ci, 30.0, TAU, TAU, iters, precision="f64")
    _check(m, g, o, iters)


def test_f64_ignores_the_variant_and_matches_forced_slabs(cuda_device, oracle_mod):
    m, u, ci = random_volume(90, 14, 15, 6.6, 3, seed=12)
    iters = 8
    g = potts.solve(m, u, ci, 30.0, TAU, TAU, iters, storage="f64", variant=0, slab_w=40, want_state=False)
    o = oracle_mod.solve(m, u, ci, 30.0, TAU, TAU, iters, precision="f64", slab_w=40, want_state=False)
    assert g.stats.n_slabs == 1 + (90 - 40 + 24 - 1) // 24
    mv = m.mask_values
    assert np.array_equal(mv(g.labels), mv(o.labels)) and np.array_equal(mv(g.res), mv(o.res))


def test_f64_energies_match_oracle(cuda_device, oracle_mod):
    m, u, ci = random_volume(24, 20, 20, 9.1, 3, seed=11)
    g = potts.solve(m, u, ci, 30.0, TAU, TAU, 40, storage="f64", gap_every=10, want_state=False)
    o = oracle_mod.solve(m, u, ci, 30.0, TAU, TAU, 40, precision="f64", gap_every=10, want_state=False)
    np.testing.assert_allclose(g.stats.energy_trace[:, :2], o.energy_trace[:, :2], rtol=1e-12)
    np.testing.assert_allclose(g.stats.energy_trace[:, 2], o.energy_trace[:, 2], rtol=1e-9, atol=1e-9)


def test_f64_config0_equals_fp64_oracle(cuda_device, oracle_mod):
    """128^3, r = 60, K = 3, lam = 30, tau = tau' = 1/sqrt(12), 500 iterations: the FP64 GPU solve is
    the FP64 oracle, and the FP32 solve is within the plain form's tolerance of it."""
    from segmentctscans_b200.phantom import config0_phantom

    ph = config0_phantom(seed=0, device="cpu")
    m, u, ci = ph.mapping, ph.u.numpy().copy(), ph.ci
    iters = 500
    o = oracle_mod.solve(m, u, ci, 30.0, TAU_BASELINE, TAU_BASELINE, iters, precision="f64")
    g = potts.solve(m, u, ci, 30.0, TAU_BASELINE, TAU_BASELINE, iters, storage="f64")
    _check(m, g, o, iters)
    f = potts.solve(m, u, ci, 30.0, TAU_BASELINE, TAU_BASELINE, iters, want_state=True)
    mv = m.mask_values
    rel = np.linalg.norm(mv(f.V) - mv(g.V)) / np.linalg.norm(mv(g.V))
    assert rel <= 1e-5, rel


def test_f64_device_outputs_rounded_through_solve_device(cuda_device):
    """potts_solve_device with storage f64 writes V rounded to FP32; potts_solve_device_f64 in FP64."""
    import torch

    m, u, ci = random_volume(20, 18, 17, 7.9, 3, seed=5)
    dev = cuda_device
    du = torch.from_numpy(u).to(dev)
    v32 = torch.zeros((2, m.span), dtype=torch.float32, device=dev)
    v64 = torch.zeros((2, m.span), dtype=torch.float64, device=dev)
    with potts.make_context(dev.index, stream=torch.cuda.current_stream(dev).cuda_stream) as ctx:
        potts.solve_device(ctx, m, du.data_ptr(), ci, 30.0, TAU, TAU, 12, V_ptr=v32.data_ptr(), storage="f64")
        potts.solve_device_f64(ctx, m, du.data_ptr(), ci, 30.0, TAU, TAU, 12, V_ptr=v64.data_ptr())
    torch.cuda.synchronize(dev)
    assert torch.equal(v64.to(torch.float32), v32)
