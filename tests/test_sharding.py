"""Column sharding (segmentctscans_b200/sharding.py) on CPU: two gloo ranks run the FP32
oracle's steps on their local volumes with the two halo exchanges per iteration; every owned
voxel must equal the single-volume FP32 oracle solve bit for bit."""
import os
import socket

import numpy as np
import pytest

from segmentctscans_b200.sharding import make_shard, partition_columns
from tests._cases import TAU, random_volume


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


def _rank_main(rank, world, port, case, result_dir):
    import torch
    import torch.distributed as dist

    from oracle import oracle
    from segmentctscans_b200.sharding import HaloExchange, torch_exchange

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        n, rows, cols, r, K, iters = case
        m, u, ci = random_volume(n, rows, cols, r, K, seed=K + n)
        shard = make_shard(m, world, rank)
        lm = shard.mapping
        lu = np.ascontiguousarray(shard.to_local(u))
        # local state, as torch views of numpy arrays so that the exchange writes into them
        V = _nearest_onehot(lu, ci, K)
        Vb = V.copy()
        xi = np.zeros((3 * (K - 1), lm.span), np.float32)
        tV, tVb, txi = torch.from_numpy(V), torch.from_numpy(Vb), torch.from_numpy(xi)
        ex = HaloExchange(shard, torch_exchange)
        for it in range(iters):
            ex.vbar(tVb)
            xi[...] = oracle.grad_step(lm, K, xi, Vb, TAU, "f32")
            ex.xi(txi)
            Vn, Vbn, _ = oracle.div_step(lm, K, xi, V, lu, ci, 30.0, TAU, "f32")
            V[...] = Vn
            Vb[...] = Vbn
        whole = oracle.solve(m, u, ci, 30.0, TAU, TAU, iters, precision="f32")
        b, e = shard.owned_span()
        gb, ge = shard.span_begin + b, shard.span_begin + e
        # compare over in-mask slices of the owned lines
        keep = (np.arange(lm.span)[b:e] % lm.nstride) < lm.n_images
        ok = (np.array_equal(V[:, b:e][:, keep], whole.V[:, gb:ge][:, keep]) and
              np.array_equal(xi[:, b:e][:, keep], whole.Xi[:, gb:ge][:, keep]))
        with open(os.path.join(result_dir, f"rank{rank}"), "w") as f:
            f.write("ok" if ok else "mismatch")
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("case", [(20, 22, 21, 9.7, 3, 12), (12, 18, 30, 8.4, 4, 9)], ids=["K3", "K4"])
def test_two_rank_column_sharding_matches_whole_volume(oracle_mod, tmp_path, case):
    import torch.multiprocessing as mp

    mp.start_processes(_rank_main, args=(2, _free_port(), case, str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    for r in range(2):
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
            assert s.mapping.span == int(m.base[s.last] - m.base[s.first])
