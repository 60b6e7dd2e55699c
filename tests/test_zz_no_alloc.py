"""potts_energies_static: the FP64 energies of a state without any device allocation.

It exists for callers that cannot call cudaMalloc (a host framework that owns
the device memory pool, a process whose device memory is reserved up front).
Its result must match the energies the solver itself reports for the same
state, on two calls in a row (the calls share the library's fixed working
memory).  This file is collected last, so a failure here comes after every
other test has run.
"""
import ctypes

import numpy as np
import pytest

from segmentctscans_b200 import _native, potts
from tests._cases import TAU, random_volume

pytestmark = pytest.mark.gpu

ENERGY_REL_TOL = 1e-9  # same per-voxel FP64 terms, different summation order


def _static_energies(m, du, ci, lam, dV, dX, stream):
    lib = _native.host_lib()
    out = (ctypes.c_double * 3)()
    c = np.ascontiguousarray(np.asarray(ci, np.float32))
    st = lib.potts_energies_static(ctypes.byref(m.as_c()), ctypes.c_void_p(du.data_ptr()), len(ci),
                                   c.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), float(lam),
                                   ctypes.c_void_p(dV.data_ptr()), ctypes.c_void_p(dX.data_ptr()),
                                   ctypes.c_void_p(stream), out)
    _native.check(st)
    return np.array(out[:])


@pytest.mark.parametrize("K,variant", [(3, 0), (4, 1)])
def test_static_energies_match_solver_energies(cuda_device, K, variant):
    import torch

    m, u, ci = random_volume(40, 26, 24, 11.7, K, seed=40 + K)
    iters = 30
    dev = cuda_device
    du = torch.from_numpy(u).to(dev)
    dV = torch.zeros((K - 1, m.span), dtype=torch.float32, device=dev)
    dX = torch.zeros((3 * (K - 1), m.span), dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    with potts.make_context(dev.index, stream=stream) as ctx:
        st = potts.solve_device(ctx, m, du.data_ptr(), ci, 30.0, TAU, TAU, iters, V_ptr=dV.data_ptr(),
                                Xi_ptr=dX.data_ptr(), variant=variant, gap_every=iters)
    want = st.energy_trace[-1]
    first = _static_energies(m, du, ci, 30.0, dV, dX, stream)
    # the second call allocates nothing: the device's free memory and torch's pool are unchanged
    torch.cuda.synchronize(dev)
    free_before, _ = torch.cuda.mem_get_info(dev)
    reserved_before = torch.cuda.memory_reserved(dev)
    second = _static_energies(m, du, ci, 30.0, dV, dX, stream)
    torch.cuda.synchronize(dev)
    free_after, _ = torch.cuda.mem_get_info(dev)
    assert free_after == free_before, (free_before, free_after)
    assert torch.cuda.memory_reserved(dev) == reserved_before
    for got in (first, second):
        np.testing.assert_allclose(got[:2], want[:2], rtol=ENERGY_REL_TOL)
        np.testing.assert_allclose(got[2], want[2], rtol=1e-6, atol=1e-9)
    assert np.array_equal(first, second)


def test_static_energies_reject_too_many_columns(cuda_device):
    import torch

    from segmentctscans_b200.layout import CylinderMapping

    cols = _native.STATIC_MAX_COLS + 1
    m = CylinderMapping.cylinder(4, 3, cols, 1.0, xc=2.0, yc=1.0)
    t = torch.zeros(max(m.span, 1), device=cuda_device)
    with pytest.raises(_native.PottsError) as e:
        _static_energies(m, t, [0.2, 0.8], 30.0, t, t, 0)
    assert e.value.status == _native.POTTS_EINVAL and "POTTS_STATIC_MAX_COLS" in str(e.value)
