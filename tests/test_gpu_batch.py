"""Batched solves (potts_batch_create / potts_batch_run): every volume of a batch gives
the bits of its own single-volume solve, for each storage format, with the iterations as one
persistent launch (the default) or one launch each, with the default tile and with the
autotuner's; replays reread u."""
import numpy as np
import pytest

from segmentctscans_b200 import potts
from segmentctscans_b200._native import PottsError
from tests._cases import TAU, random_volume
from tests.test_gpu_parity import assert_same

pytestmark = pytest.mark.gpu

# uneven volumes: (n, rows, cols, radius, lambda)
SHAPES = [(40, 30, 26, 12.1, 12.0), (17, 21, 33, 9.7, 55.0), (65, 18, 18, 7.9, 30.0), (9, 40, 38, 18.2, 90.0),
          (33, 25, 25, 11.6, 20.0)]


def _batch_inputs(K, seed0=100):
    import torch

    out = []
    for i, (n, rows, cols, r, lam) in enumerate(SHAPES):
        m, u, ci = random_volume(n, rows, cols, r, K, seed=seed0 + i)
        # volume 1 reads u from an address that is not 16-byte aligned (staged by the batch)
        off = 1 if i == 1 else 0
        du = torch.zeros(m.span + 4, dtype=torch.float32, device="cuda")
        du[off:off + m.span] = torch.from_numpy(u).cuda()
        out.append(dict(m=m, u=u, ci=ci, lam=lam, du=du, off=off,
                        res=torch.zeros(m.span, dtype=torch.float32, device="cuda"),
                        lab=torch.zeros(m.span, dtype=torch.uint8, device="cuda"),
                        V=torch.zeros((K - 1) * m.span, dtype=torch.float32, device="cuda")))
    return out


def _make(ctx, vols, iters, **opts):
    bv = [potts.BatchVolume(v["m"], v["du"].data_ptr() + 4 * v["off"], v["ci"], v["lam"], v["res"].data_ptr(),
                            v["lab"].data_ptr(), v["V"].data_ptr()) for v in vols]
    return potts.Batch(ctx, bv, TAU, TAU, iters, **opts)


def _check_against_single(vols, iters, **opts):
    for v in vols:
        g = potts.solve(v["m"], v["u"], v["ci"], v["lam"], TAU, TAU, iters, variant=0, **opts)
        mv = v["m"].mask_values
        K = len(v["ci"])
        assert np.array_equal(mv(v["lab"].cpu().numpy()), mv(g.labels))
        assert np.array_equal(mv(v["res"].cpu().numpy()), mv(g.res))
        assert np.array_equal(mv(v["V"].cpu().numpy().reshape(K - 1, -1)), mv(g.V))


@pytest.mark.parametrize("persistent", [1, 0])
@pytest.mark.parametrize("store", ["f32", "bf16", "f16"])
@pytest.mark.parametrize("K", [3, 4])
def test_batch_equals_single_volume_solves(cuda_device, store, K, persistent):
    iters = 14
    vols = _batch_inputs(K)
    with potts.make_context(0) as ctx:
        with _make(ctx, vols, iters, storage=store, persistent=persistent) as b:
            st = b.run()
            info = b.info()
            assert info.n_volumes == len(vols) and info.n_work > 0
            # set-up and finish launches per volume, plus the iterations: one persistent launch, or one each
            assert info.graph_launches >= (1 if persistent else iters - 1) + len(vols)
            assert st.loop_launches == (1 if persistent else iters - 1)
            assert st.loop_iters == iters - 1 and st.solve_ms > 0 and st.loop_ms > 0
            _check_against_single(vols, iters, storage=store)
            dq = b.dq()
            for i, v in enumerate(vols):
                g = potts.solve(v["m"], v["u"], v["ci"], v["lam"], TAU, TAU, iters, variant=0, storage=store)
                np.testing.assert_array_equal(dq[i], g.stats.dq_trace)
            np.testing.assert_array_equal(st.dq_trace, dq.max(axis=0))


def test_batch_autotuned_tile_gives_the_same_bits(cuda_device, oracle_mod):
    iters = 12
    vols = _batch_inputs(3, seed0=200)
    with potts.make_context(0) as ctx:
        with _make(ctx, vols, iters, autotune=1) as b:
            b.run()
            info = b.info()
            assert info.autotune_ms > 0 and info.tile[3] in (16, 32, 64)
            _check_against_single(vols, iters)
    v = vols[2]
    o = oracle_mod.solve(v["m"], v["u"], v["ci"], v["lam"], TAU, TAU, iters, precision="f32")
    mv = v["m"].mask_values
    assert np.array_equal(mv(v["lab"].cpu().numpy()), mv(o.labels))


def test_batch_replay_rereads_u(cuda_device):
    import torch

    iters = 10
    vols = _batch_inputs(3, seed0=300)
    with potts.make_context(0) as ctx:
        with _make(ctx, vols, iters) as b:
            b.run(stats=False)  # asynchronous on the context's stream
            ctx.synchronize()
            first = [v["res"].clone() for v in vols]
            b.run()
            for v, f in zip(vols, first):
                assert torch.equal(v["res"], f)
            # new intensities in volume 0: its result follows, the others stay
            rng = np.random.default_rng(7)
            v0 = vols[0]
            v0["u"] = np.clip(v0["u"] + rng.normal(0, 0.2, v0["u"].shape).astype(np.float32), 0, 1)
            v0["du"][: v0["m"].span] = torch.from_numpy(v0["u"]).cuda()
            b.run()
            _check_against_single(vols, iters)


def test_batch_errors(cuda_device):
    vols = _batch_inputs(3, seed0=400)[:2]
    with potts.make_context(0) as ctx:
        bad = dict(vols[0])
        bad["lam"] = float("nan")
        with pytest.raises(PottsError) as e:
            _make(ctx, [bad, vols[1]], 5)
        assert e.value.status == 1
        with pytest.raises(ValueError):
            potts.Batch(ctx, [], TAU, TAU, 5)
        # the context still solves
        with _make(ctx, vols, 3) as b:
            b.run()
