"""Column sharding (segmentctscans_b200/sharding.py, potts_shard_*) on CPU.

Two or three gloo ranks run the shard protocol of the library on the FP32 oracle's steps: each rank holds
its columns, the column before and the two after; per iteration it runs the dual step on all of
them, exchanges the Xi planes of one column with each neighbour, and runs the primal step (V at
the first column after its range comes out exact).  Every owned voxel must equal the
single-volume FP32 oracle solve bit for bit, the per-iteration max |dV|^2 reduced by max over the
ranks must equal the whole volume's trace, and the FP64 energies summed over the ranks must equal
the whole volume's (same terms, different summation order).
"""
import os
import socket

import numpy as np
import pytest

from segmentctscans_b200.sharding import make_shard, partition_columns
from tests._cases import TAU, random_volume

ENERGY_REL_TOL = 1e-9


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _nearest_onehot(u, ci, K):
    d = np.abs(u[None, :] - np.asarray(ci, np.float32)[:, None])
    lab = np.argmin(d, axis=0)  # first minimum wins, as the strict < of the reference
    V = np.zeros((K - 1, u.size), np.float32)
    for i in range(K - 1):
        V[i] = lab == i
    return V


def _exchange_xi(shard, xi):
    """The shard's Xi exchange: first owned column to the left rank (its right halo), last owned
    column to the right rank (its left halo); receive the halos the other way round."""
    import torch
    import torch.distributed as dist

    ops, fills = [], []
    if shard.left_halo:
        b, e = shard.col_span(shard.c_lo)
        ops.append(dist.P2POp(dist.isend, torch.from_numpy(np.ascontiguousarray(xi[:, b:e])), shard.rank - 1))
        b, e = shard.col_span(shard.c_lo - 1)
        buf = torch.empty((xi.shape[0], e - b), dtype=torch.float32)
        ops.append(dist.P2POp(dist.irecv, buf, shard.rank - 1))
        fills.append((b, e, buf))
    if shard.right_halo:
        b, e = shard.col_span(shard.c_hi - 1)
        ops.append(dist.P2POp(dist.isend, torch.from_numpy(np.ascontiguousarray(xi[:, b:e])), shard.rank + 1))
        b, e = shard.col_span(shard.c_hi)
        buf = torch.empty((xi.shape[0], e - b), dtype=torch.float32)
        ops.append(dist.P2POp(dist.irecv, buf, shard.rank + 1))
        fills.append((b, e, buf))
    if ops:
        for req in dist.batch_isend_irecv(ops):
            req.wait()
    for b, e, buf in fills:
        xi[:, b:e] = buf.numpy()


def _rank_main(rank, world, port, case, result_dir):
    import torch
    import torch.distributed as dist

    from oracle import oracle

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        n, rows, cols, r, K, iters, ge = case
        m, u, ci = random_volume(n, rows, cols, r, K, seed=K + n)
        shard = make_shard(m, world, rank)
        lm = shard.mapping
        lu = np.ascontiguousarray(shard.to_local(u))
        lo, hi = shard.local_col(shard.c_lo), shard.local_col(shard.c_hi)
        V = _nearest_onehot(lu, ci, K)
        Vb = V.copy()
        xi = np.zeros((3 * (K - 1), lm.span), np.float32)
        dq = np.zeros(iters, np.float32)
        en = []
        for it in range(iters):
            xi = oracle.grad_step(lm, K, xi, Vb, TAU, "f32")
            _exchange_xi(shard, xi)
            V, Vb, dq[it] = oracle.div_step_cols(lm, K, xi, V, lu, ci, 30.0, TAU, lo, hi, "f32")
            if ge and (it + 1) % ge == 0:
                en.append(oracle.energies_cols(lm, K, xi, V, lu, ci, 30.0, lo, hi, "f32"))
        t_dq = torch.from_numpy(dq.copy())
        dist.all_reduce(t_dq, op=dist.ReduceOp.MAX)
        en = np.asarray(en, np.float64).reshape(-1, 3)
        t_en = torch.from_numpy(en[:, :2].copy())
        dist.all_reduce(t_en, op=dist.ReduceOp.SUM)
        whole = oracle.solve(m, u, ci, 30.0, TAU, TAU, iters, precision="f32", gap_every=ge)
        b, e = shard.owned_span()
        gb, gend = shard.span_begin + b, shard.span_begin + e
        keep = (np.arange(lm.span)[b:e] % lm.nstride) < lm.n_images
        msgs = []
        if not np.array_equal(V[:, b:e][:, keep], whole.V[:, gb:gend][:, keep]):
            msgs.append("V")
        if not np.array_equal(xi[:, b:e][:, keep], whole.Xi[:, gb:gend][:, keep]):
            msgs.append("Xi")
        if not np.array_equal(t_dq.numpy(), whole.dq_trace):
            msgs.append("dq")
        if ge:
            got = t_en.numpy()
            want = np.asarray(whole.energy_trace).reshape(-1, 3)
            if got.shape[0] != want.shape[0] or not np.allclose(got, want[:, :2], rtol=ENERGY_REL_TOL, atol=0):
                msgs.append("energies")
        with open(os.path.join(result_dir, f"rank{rank}"), "w") as f:
            f.write("ok" if not msgs else "mismatch: " + ",".join(msgs))
    finally:
        dist.destroy_process_group()


# (n, rows, cols, r, K, iters, gap_every), ranks
CASES = [((20, 22, 21, 9.7, 3, 12, 4), 3), ((12, 18, 30, 8.4, 4, 9, 3), 2), ((9, 20, 26, 9.1, 2, 7, 0), 2)]


@pytest.mark.parametrize("case,world", CASES, ids=["K3_3ranks", "K4_2ranks", "K2_2ranks"])
def test_column_sharding_matches_whole_volume(oracle_mod, tmp_path, case, world):
    import torch.multiprocessing as mp

    mp.start_processes(_rank_main, args=(world, _free_port(), case, str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    for r in range(world):
        assert (tmp_path / f"rank{r}").read_text() == "ok"


def test_partition_balances_voxels():
    m, _, _ = random_volume(16, 60, 80, 28.0, 3, seed=1)
    for world in (2, 3, 5, 8):
        parts = partition_columns(m, world)
        assert parts[0][0] == m.col_begin and parts[-1][1] == m.col_end
        assert all(a[1] == b[0] for a, b in zip(parts, parts[1:]))
        vox = np.diff(np.asarray(m.base, np.int64)) // m.nstride
        loads = [vox[a:b].sum() for a, b in parts]
        assert max(loads) - min(loads) <= 2 * vox.max()
        for rank in range(world):
            s = make_shard(m, world, rank)
            assert s.left_halo == (rank > 0) and s.right_halo == (rank + 1 < world)
            assert s.last == (min(s.c_hi + 2, m.col_end) if rank + 1 < world else s.c_hi)
            assert s.mapping.span == int(m.base[s.last] - m.base[s.first])


def test_native_partition_and_bounds_match(native_lib):
    """potts_shard_partition / potts_shard_bounds (no GPU needed) agree with the Python restatement."""
    from segmentctscans_b200._native import PottsError
    from segmentctscans_b200.sharding import native_bounds, native_cuts

    m, _, _ = random_volume(16, 60, 80, 28.0, 3, seed=1)
    for world in (1, 2, 3, 7):
        cuts = native_cuts(m, world)
        parts = partition_columns(m, world)
        assert cuts == [p[0] for p in parts] + [parts[-1][1]]
        for rank in range(world):
            s = make_shard(m, world, rank)
            cols, span = native_bounds(m, cuts, rank)
            assert cols == (s.first, s.last, s.c_lo, s.c_hi)
            assert span == (s.span_begin, s.span_begin + s.mapping.span)
    with pytest.raises(PottsError):
        native_cuts(m, int(m.col_end - m.col_begin) + 1)
    with pytest.raises(PottsError):
        native_bounds(m, [int(m.col_begin), int(m.col_begin), int(m.col_end)], 0)
