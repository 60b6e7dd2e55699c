"""Differentiable solve (potts_forward_ckpt / potts_backward): the adjoint of the unrolled
iteration against FP64 central finite differences of the FP64 oracle.

Loss: L = -1/|mask| sum_x log(V_t(x) + 1e-3), t = the phantom's true label.  The finite
differences use a step of 1e-6 relative: at 1e-4 relative a change of c_i moves voxels
within 2e-4 of a nearest-label tie to the other initial label (the initial state is
piecewise constant in u and c), so those differences measure jumps, not the derivative.
The adjoint must agree within 1e-3 relative for c_1..c_K and lambda, and within 1e-3
relative L2 over 16 random in-mask coordinates of u.
"""
import numpy as np
import pytest

from segmentctscans_b200 import potts
from tests._cases import TAU, phantom_volume

pytestmark = pytest.mark.gpu

EPS = 1e-3
FD_REL_STEP = 1e-6
TOL = 1e-3


def fp64_loss(oracle_mod, m, u, truth, ci, lam, iters):
    r = oracle_mod.solve(m, u, ci, lam, TAU, TAU, iters, precision="f64")
    mv = m.mask_values
    Vm = mv(r.V)
    Vf = np.concatenate([Vm, 1.0 - Vm.sum(0, keepdims=True)])
    t = np.minimum(mv(truth).astype(np.int64), len(ci) - 1)
    vt = np.take_along_axis(Vf, t[None], 0)[0]
    return float(-np.mean(np.log(vt + EPS)))


def central_difference(fun, x, rel=FD_REL_STEP):
    h = rel * max(abs(x), 1e-2)
    xp, xm = np.float32(x + h), np.float32(x - h)  # the oracle reads FP32 inputs
    return (fun(float(xp)) - fun(float(xm))) / (float(xp) - float(xm))


@pytest.mark.parametrize("case", [(24, 10.0, 30, 8, 5), (32, 14.0, 60, 20, 6)], ids=["24^3", "32^3"])
def test_adjoint_matches_fp64_finite_differences(cuda_device, oracle_mod, case):
    size, r, iters, ckpt, seed = case
    m, u, ci, ph = phantom_volume(size, r, seed=seed)
    truth = ph.truth.numpy().astype(np.uint8)
    lam = 30.0
    loss, gu, gc, gl = potts.loss_and_grad(m, u, truth, ci, lam, TAU, TAU, iters, ckpt_every=ckpt, eps=EPS)
    L0 = fp64_loss(oracle_mod, m, u, truth, ci, lam, iters)
    assert abs(loss - L0) <= 1e-5 * abs(L0)
    for i in range(len(ci)):
        def f(v, i=i):
            c2 = list(ci)
            c2[i] = v
            return fp64_loss(oracle_mod, m, u, truth, c2, lam, iters)
        g = central_difference(f, ci[i])
        assert abs(gc[i] - g) <= TOL * abs(g), (i, gc[i], g)
    g = central_difference(lambda v: fp64_loss(oracle_mod, m, u, truth, ci, v, iters), lam)
    assert abs(gl - g) <= TOL * abs(g), (gl, g)
    rng = np.random.default_rng(seed)
    idx = np.arange(m.span).reshape(m.n_lines, m.nstride)[:, : m.n_images].reshape(-1)
    adj, fd = [], []
    for j in rng.choice(idx, 16, replace=False):
        def f(v, j=j):
            u2 = u.copy()
            u2[j] = v
            return fp64_loss(oracle_mod, m, u2, truth, ci, lam, iters)
        adj.append(gu[j])
        fd.append(central_difference(f, float(u[j])))
    adj, fd = np.array(adj), np.array(fd)
    assert np.linalg.norm(adj - fd) <= TOL * np.linalg.norm(fd) + 1e-12
    # outside the mask the gradient is zero
    pad = np.ones(m.span, bool)
    pad[idx] = False
    assert not np.any(gu[pad])


def test_backward_is_repeatable_and_checkpoint_independent(cuda_device):
    import torch

    m, u, ci, ph = phantom_volume(24, 10.0, seed=7)
    truth = ph.truth.numpy().astype(np.uint8)
    a = potts.loss_and_grad(m, u, truth, ci, 30.0, TAU, TAU, 25, ckpt_every=7, eps=EPS)
    b = potts.loss_and_grad(m, u, truth, ci, 30.0, TAU, TAU, 25, ckpt_every=25, eps=EPS)
    assert abs(a[0] - b[0]) <= 1e-12 * abs(a[0])  # an FP64 sum of atomics, in any order
    np.testing.assert_array_equal(a[1], b[1])
    # dL/dc and dL/dlambda are sums of FP64 atomics: the order (not the terms) differs
    np.testing.assert_allclose(a[2], b[2], rtol=1e-12)
    assert abs(a[3] - b[3]) <= 1e-12 * abs(a[3])
    with potts.make_context(0) as ctx:
        du = torch.from_numpy(u).cuda()
        dt = torch.from_numpy(truth).cuda()
        g1 = torch.zeros(m.span, device="cuda")
        g2 = torch.zeros(m.span, device="cuda")
        V = torch.zeros(2 * m.span, device="cuda")
        torch.cuda.synchronize()
        with potts.Tape(ctx, m, du.data_ptr(), dt.data_ptr(), ci, 30.0, TAU, TAU, 25, 7, EPS, V.data_ptr()) as t:
            c1, l1 = t.backward(g1.data_ptr())
            c2, l2 = t.backward(g2.data_ptr())
        ctx.synchronize()
        assert torch.equal(g1, g2)
        np.testing.assert_allclose(c1, c2, rtol=1e-12)
        assert abs(l1 - l2) <= 1e-12 * abs(l1)
        # the forward pass is the plain solve
        s = potts.solve(m, u, ci, 30.0, TAU, TAU, 25, variant=1)
        assert np.array_equal(m.mask_values(V.cpu().numpy().reshape(2, -1)), m.mask_values(s.V))


class GpuFp64Loss:
    """The FP64 loss through the FP64 GPU solve (potts_solve_device_f64: FP64 state and arithmetic,
    the same bits as the FP64 CPU oracle), for finite differences on volumes too large for the CPU."""

    def __init__(self, ctx, m, u, truth, iters, eps=EPS):
        import torch

        self.ctx, self.m, self.iters, self.eps = ctx, m, iters, eps
        self.dev = torch.device("cuda", ctx.device)
        self.u = torch.from_numpy(u).to(self.dev)
        idx = np.arange(m.span).reshape(m.n_lines, m.nstride)[:, : m.n_images].reshape(-1)
        self.idx = torch.from_numpy(idx).to(self.dev)
        self.t = torch.from_numpy(truth.astype(np.int64)).to(self.dev)[self.idx]
        self.V = None

    def __call__(self, ci, lam, u_override=None):
        import torch

        K = len(ci)
        self.t.clamp_(max=K - 1)
        if self.V is None or self.V.shape[0] != K - 1:
            self.V = torch.empty((K - 1, self.m.span), dtype=torch.float64, device=self.dev)
        u = self.u
        if u_override is not None:
            j, val = u_override
            u = self.u.clone()
            u[j] = val
        potts.solve_device_f64(self.ctx, self.m, u.data_ptr(), ci, lam, TAU, TAU, self.iters, V_ptr=self.V.data_ptr(),
                               stats=False)
        torch.cuda.synchronize(self.dev)
        Vm = self.V[:, self.idx]
        Vf = torch.cat([Vm, 1.0 - Vm.sum(0, keepdim=True)])
        vt = Vf.gather(0, self.t[None])[0]
        return float(-torch.log(vt + self.eps).mean().item())


def _init_label_flips(u_in, ci, c2):
    """In-mask voxels whose nearest label (the initial state) differs between labels ci and c2."""
    a = np.argmin(np.abs(np.asarray(ci, np.float32)[:, None] - u_in[None]), 0)
    b = np.argmin(np.abs(np.asarray(c2, np.float32)[:, None] - u_in[None]), 0)
    return int(np.sum(a != b))


def test_config4_192cubed_against_fp64_differences(cuda_device):
    """192^3, r = 90, K = 3, 200 unrolled iterations, checkpoints every 20; gradients of c_1..c_3,
    lambda and 64 random in-mask u coordinates against FP64 central differences (step 1e-6
    relative; for c_i shrunk where a step of 1e-6 would move a voxel's nearest label, which is a
    jump of the loss, not its derivative).  The 1e-4 step is also evaluated for u and reported."""
    import torch

    from segmentctscans_b200.phantom import make_phantom

    ph = make_phantom(192, 192, 192, 90.0, seed=0, radius_range=(4.0, 12.0), noise=7e-3, device="cpu")
    m, u, ci = ph.mapping, ph.u.numpy().copy(), ph.ci
    truth = ph.truth.numpy().astype(np.uint8)
    lam, iters = 30.0, 200
    with potts.make_context(0, stream=torch.cuda.current_stream().cuda_stream) as ctx:
        loss, gu, gc, gl = potts.loss_and_grad(m, u, truth, ci, lam, TAU, TAU, iters, ckpt_every=20, eps=EPS,
                                               ctx=ctx)
        f = GpuFp64Loss(ctx, m, u, truth, iters)
        L0 = f(ci, lam)
        assert abs(loss - L0) <= 1e-5 * abs(L0), (loss, L0)
        u_in = m.mask_values(u).reshape(-1)
        for i in range(len(ci)):
            rel = FD_REL_STEP
            while True:
                h = rel * abs(ci[i])
                cp, cm = list(ci), list(ci)
                cp[i], cm[i] = float(np.float32(ci[i] + h)), float(np.float32(ci[i] - h))
                if _init_label_flips(u_in, ci, cp) + _init_label_flips(u_in, ci, cm) == 0 or rel < 1e-8:
                    break
                rel /= 4.0
            assert cp[i] != cm[i]
            g = (f(cp, lam) - f(cm, lam)) / (cp[i] - cm[i])
            assert abs(gc[i] - g) <= TOL * abs(g), (i, rel, gc[i], g)
        g = central_difference(lambda v: f(ci, v), lam)
        assert abs(gl - g) <= TOL * abs(g), (gl, g)
        rng = np.random.default_rng(0)
        idx = np.arange(m.span).reshape(m.n_lines, m.nstride)[:, : m.n_images].reshape(-1)
        coords = rng.choice(idx, 64, replace=False)
        adj = np.array([gu[j] for j in coords])
        fd6 = np.array([central_difference(lambda v, j=j: f(ci, lam, (int(j), v)), float(u[j])) for j in coords])
        fd4 = np.array([central_difference(lambda v, j=j: f(ci, lam, (int(j), v)), float(u[j]), rel=1e-4)
                        for j in coords])
    err6 = np.linalg.norm(adj - fd6) / np.linalg.norm(fd6)
    err4 = np.linalg.norm(adj - fd4) / np.linalg.norm(fd4)
    print(f"config 4: u gradient relative L2 error over 64 coordinates: {err6:.3e} (step 1e-6), {err4:.3e} (1e-4)")
    assert err6 <= TOL
