"""CPU checks of the oracle: known answers, projection optimality, adjointness, slabs."""
import json
from pathlib import Path

import numpy as np
import pytest

from tests._cases import TAU, phantom_volume, random_volume

GOLDEN = Path(__file__).resolve().parent / "golden"


# --------------------------------------------------------------------------- simplex
def _simplex_numpy(q):
    """Independent restatement: Euclidean projection onto the probability simplex
    by bisection on the threshold (no sorting)."""
    q = np.asarray(q, np.float64)
    lo, hi = q.min() - 1.0, q.max()
    for _ in range(200):
        t = 0.5 * (lo + hi)
        if np.maximum(q - t, 0).sum() > 1:
            lo = t
        else:
            hi = t
    return np.maximum(q - 0.5 * (lo + hi), 0)


@pytest.mark.parametrize("K", [2, 3, 4, 5, 6])
def test_simplex_matches_independent_projection(oracle_mod, K):
    rng = np.random.default_rng(K)
    for _ in range(300):
        q = rng.normal(0, 2, K)
        p = oracle_mod.project_simplex(q, "f64")
        assert abs(p.sum() - 1) < 1e-12 and p.min() >= 0
        np.testing.assert_allclose(p, _simplex_numpy(q), atol=1e-10)


def test_simplex_known_answers(oracle_mod):
    kat = json.loads((GOLDEN / "kat.json").read_text())
    for case in kat["simplex"]:
        for prec, tol in (("f64", 1e-15), ("f32", 1e-7)):
            p = oracle_mod.project_simplex(case["q"], prec)
            np.testing.assert_allclose(p, case["p"], atol=tol, err_msg=str(case))


# --------------------------------------------------------------------------- Pi_K
def _pairs_ok(q, tol):
    K = q.shape[0]
    return all(np.linalg.norm(q[i] - q[j]) <= 1 + tol for i in range(K) for j in range(i + 1, K))


def _max_violation(q):
    K = q.shape[0]
    return max(np.linalg.norm(q[i] - q[j]) - 1 for i in range(K) for j in range(i + 1, K))


def test_project_K_known_answers(oracle_mod):
    kat = json.loads((GOLDEN / "kat.json").read_text())
    for case in kat["project_K"]:
        for prec, tol in (("f64", 1e-12), ("f32", 1e-6)):
            p, sw = oracle_mod.project_K(np.array(case["q"]), prec)
            np.testing.assert_allclose(p, np.array(case["p"]), atol=tol, err_msg=str(case))
            assert sw == case["sweeps"]


@pytest.mark.parametrize("K", [2, 3, 4, 6])
def test_project_K_feasible_and_optimal(oracle_mod, K):
    rng = np.random.default_rng(10 + K)
    for _ in range(100):
        q0 = rng.normal(0, 0.7, (K, 3))
        q0 -= q0.mean(0)
        p, sw = oracle_mod.project_K(q0, "f64")
        # feasibility: Dykstra stops when every step is < 1e-6 or after 20 sweeps; a
        # capped run is only closer to K than the input
        if sw < 20:
            assert _pairs_ok(p, 1e-4)
        else:
            assert _max_violation(p) < max(_max_violation(q0), 0.0) + 1e-12
        # sum of the vectors is preserved (each step moves a pair by +-delta)
        np.testing.assert_allclose(p.sum(0), q0.sum(0), atol=1e-12)
        if sw < 20:
            # variational inequality of the projection onto a convex set
            for _ in range(20):
                y = rng.normal(0, 0.2, (K, 3))
                if not _pairs_ok(y, 0):
                    continue
                assert np.sum((q0 - p) * (y - p)) <= 1e-4
        # a feasible point is a fixed point
        f = rng.normal(0, 0.05, (K, 3))
        pf, swf = oracle_mod.project_K(f, "f64")
        assert swf == 1 and np.array_equal(pf, f)


# --------------------------------------------------------------------------- grad / div
def _grad_np(m, Vfull):
    """Forward differences on the cylinder: [K, 3, span] (independent restatement)."""
    K = Vfull.shape[0]
    g = np.zeros((K, 3) + Vfull.shape[1:])
    rows, cols = m.lines()
    n = m.n_images
    for L, (r, c) in enumerate(zip(rows, cols)):
        o = L * m.nstride
        g[:, 0, o:o + n - 1] = Vfull[:, o + 1:o + n] - Vfull[:, o:o + n - 1]
        if r + 1 < m.row_end(c):
            g[:, 1, o:o + n] = Vfull[:, o + m.nstride:o + m.nstride + n] - Vfull[:, o:o + n]
        if c + 1 < m.col_end and m.row_begin(c + 1) <= r < m.row_end(c + 1):
            o2 = int(m.offset(0, r, c + 1))
            g[:, 2, o:o + n] = Vfull[:, o2:o2 + n] - Vfull[:, o:o + n]
    return g


def test_adjoint_identity_through_energies(oracle_mod):
    """With lam = 0 the oracle's Lagrangian is -<V, div Xi> = <grad V, Xi> (summed over all K labels)."""
    m, u, ci = random_volume(12, 15, 13, 6.2, 4, seed=3)
    K = 4
    rng = np.random.default_rng(0)
    span = m.span
    V = rng.normal(0, 1, (K - 1, span))
    Xi = rng.normal(0, 1, (3 * (K - 1), span))
    pad = np.ones(span, bool)
    pad.reshape(m.n_lines, m.nstride)[:, m.n_images:] = False
    V *= pad
    Xi *= pad
    Vfull = np.concatenate([V, (1 - V.sum(0, keepdims=True)) * pad])
    Xfull = np.concatenate([Xi.reshape(K - 1, 3, span), -Xi.reshape(K - 1, 3, span).sum(0, keepdims=True)])
    lag, dual, gap = oracle_mod.energies(m, K, Xi, V, u, ci, 0.0, "f64")
    rhs = float(np.sum(_grad_np(m, Vfull) * Xfull))
    assert abs(lag - rhs) <= 1e-9 * max(1.0, abs(rhs))


def test_grad_step_is_forward_difference_when_feasible(oracle_mod):
    m, u, ci = random_volume(10, 12, 12, 5.3, 3, seed=4)
    K = 3
    rng = np.random.default_rng(1)
    Vb = rng.uniform(0, 0.2, (K - 1, m.span))
    xi = oracle_mod.grad_step(m, K, np.zeros((3 * (K - 1), m.span)), Vb, 0.01, "f64")
    Vfull = np.concatenate([Vb, 1 - Vb.sum(0, keepdims=True)])
    g = _grad_np(m, Vfull)[: K - 1].reshape(3 * (K - 1), m.span)
    mv = m.mask_values
    np.testing.assert_allclose(mv(xi), mv(0.01 * g), atol=1e-15)


# --------------------------------------------------------------------------- solve
def test_zero_iterations_is_nearest_label(oracle_mod):
    m, u, ci = random_volume(9, 11, 10, 4.7, 5, seed=5)
    r = oracle_mod.solve(m, u, ci, 30.0, TAU, TAU, 0)
    mv = m.mask_values
    want = np.argmin(np.abs(np.asarray(ci, np.float32)[None, None, :] - mv(u)[..., None]), -1)
    assert np.array_equal(mv(r.labels), want)
    np.testing.assert_array_equal(mv(r.res), np.asarray(ci, np.float32)[want])


def test_fp32_mode_tracks_fp64(oracle_mod):
    m, u, ci, _ = phantom_volume(24, 10.0, seed=2)
    a = oracle_mod.solve(m, u, ci, 30.0, TAU, TAU, 60, precision="f64")
    b = oracle_mod.solve(m, u, ci, 30.0, TAU, TAU, 60, precision="f32")
    mv = m.mask_values
    rel = np.linalg.norm(mv(b.V) - mv(a.V)) / np.linalg.norm(mv(a.V))
    assert rel < 1e-5
    # the gap trace of a converging solve shrinks
    c = oracle_mod.solve(m, u, ci, 30.0, TAU, TAU, 60, precision="f64", gap_every=20, want_state=False)
    assert c.energy_trace.shape == (3, 3)
    assert np.all(c.energy_trace[:, 2] >= 0) and c.energy_trace[-1, 2] < c.energy_trace[0, 2]


def test_slab_interior_matches_whole_volume(oracle_mod):
    """The planner's halo = iters makes each slab's kept interior independent of the slab cut
    (potts-min-partition.cpp:563-569, 662-664)."""
    m, u, ci = random_volume(70, 14, 14, 6.1, 3, seed=6)
    whole = oracle_mod.solve(m, u, ci, 30.0, TAU, TAU, 6, want_state=False)
    sl = oracle_mod.solve(m, u, ci, 30.0, TAU, TAU, 6, slab_w=32, want_state=False)
    mv = m.mask_values
    assert np.array_equal(mv(sl.labels), mv(whole.labels))
    assert np.array_equal(mv(sl.res), mv(whole.res))


def test_slab_planner_rejects_too_narrow_slabs(oracle_mod):
    m, u, ci = random_volume(40, 10, 10, 4.2, 3, seed=7)
    with pytest.raises(RuntimeError):
        oracle_mod.solve(m, u, ci, 30.0, TAU, TAU, 10, slab_w=16)


def test_golden_small_solve(oracle_mod):
    """Regression pin of the oracle itself (fixture written by tests/golden/make_golden.py)."""
    from tests.golden.make_golden import golden_case

    z = np.load(GOLDEN / "potts_small.npz")
    m, u, ci, params = golden_case()
    assert np.array_equal(u, z["u"])
    r = oracle_mod.solve(m, u, ci, params["lam"], params["tau"], params["tau"], params["iters"])
    assert np.array_equal(r.labels, z["labels"])
    np.testing.assert_array_equal(r.V, z["V"])
    np.testing.assert_array_equal(r.dq_trace, z["dq_trace"])


# --------------------------------------------------------------------------- storage formats
def _bf16_representable(x):
    b = np.ascontiguousarray(x, np.float32).view(np.uint32)
    return np.all((b & 0xFFFF) == 0)


def test_store_formats_round_every_stored_value(oracle_mod):
    m, u, ci = random_volume(20, 14, 14, 6.3, 4, seed=40)
    mv = m.mask_values
    a = oracle_mod.solve(m, u, ci, 30.0, TAU, TAU, 12, precision="f32")
    f = oracle_mod.solve(m, u, ci, 30.0, TAU, TAU, 12, precision="f32", store="f32")
    assert np.array_equal(a.V, f.V) and np.array_equal(a.Xi, f.Xi)
    b = oracle_mod.solve(m, u, ci, 30.0, TAU, TAU, 12, precision="f32", store="bf16")
    assert _bf16_representable(mv(b.V)) and _bf16_representable(mv(b.Xi))
    h = oracle_mod.solve(m, u, ci, 30.0, TAU, TAU, 12, precision="f32", store="f16")
    for x in (mv(h.V), mv(h.Xi)):
        assert np.array_equal(x.astype(np.float16).astype(np.float32), x)
    # a solve close to the FP32 one, not identical to it
    for r, tol in ((b, 2e-2), (h, 3e-3)):
        rel = np.linalg.norm(mv(r.V) - mv(a.V)) / np.linalg.norm(mv(a.V))
        assert 0 < rel < tol


def test_bf16_store_is_reproducible_and_keyed_by_global_slice(oracle_mod):
    """The stochastic rounding of V depends on (line, global n, iteration, pair) only: slab cuts do
    not change the kept interior."""
    m, u, ci = random_volume(70, 14, 14, 6.1, 3, seed=6)
    mv = m.mask_values
    x = oracle_mod.solve(m, u, ci, 30.0, TAU, TAU, 6, precision="f32", store="bf16", want_state=False)
    y = oracle_mod.solve(m, u, ci, 30.0, TAU, TAU, 6, precision="f32", store="bf16", want_state=False)
    s = oracle_mod.solve(m, u, ci, 30.0, TAU, TAU, 6, precision="f32", store="bf16", slab_w=32,
                         want_state=False)
    assert np.array_equal(mv(x.res), mv(y.res)) and np.array_equal(mv(x.labels), mv(y.labels))
    assert np.array_equal(mv(s.labels), mv(x.labels))


# --------------------------------------------------------------------------- TV-L2 (ROF) denoising
def test_tv_oracle_properties(oracle_mod):
    """Constant fields are fixed points; the in-mask sum is preserved (div of a field whose
    missing-neighbour terms are zero sums to zero); FP32 mode tracks FP64."""
    m, u, _ = random_volume(16, 14, 15, 6.4, 3, seed=8)
    mv = m.mask_values
    c, dq = oracle_mod.tv(m, np.full(m.span, 0.37, np.float32), 0.1, 0.99 / 6, 20, "f64")
    assert np.array_equal(mv(c), np.full_like(mv(c), 0.37)) and not np.any(dq)
    a, dqa = oracle_mod.tv(m, u, 0.1, 0.99 / 6, 40, "f64")
    b, _ = oracle_mod.tv(m, u, 0.1, 0.99 / 6, 40, "f32")
    assert abs(mv(a).astype(np.float64).sum() - mv(u).astype(np.float64).sum()) <= 1e-4 * mv(u).size
    assert np.linalg.norm(mv(a) - mv(b)) <= 1e-5 * np.linalg.norm(mv(a))
    assert dqa[-1] < dqa[0]
    # smoothing lowers the total variation along n
    tv_in = np.abs(np.diff(mv(u), axis=-1)).sum()
    tv_out = np.abs(np.diff(mv(a), axis=-1)).sum()
    assert tv_out < tv_in
