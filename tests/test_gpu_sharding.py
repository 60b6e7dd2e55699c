"""Column sharding on the GPU: shards held by one process, stepped with potts_stepper and
exchanged by device copies (the protocol of the multi-GPU path, without a second GPU); the
owned columns must equal the single-volume split solve bit for bit."""
import numpy as np
import pytest

from segmentctscans_b200 import potts
from segmentctscans_b200.sharding import Stepper, exchange_in_process, make_shard
from tests._cases import TAU, random_volume

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("world", [1, 2, 3])
@pytest.mark.parametrize("K", [3, 4])
def test_sharded_steps_equal_whole_volume(cuda_device, world, K):
    import torch

    iters = 15
    m, u, ci = random_volume(24, 26, 31, 11.8, K, seed=40 + K)
    whole = potts.solve(m, u, ci, 30.0, TAU, TAU, iters, variant=1)
    shards = [make_shard(m, world, r) for r in range(world)]
    du = torch.from_numpy(u).cuda()
    with potts.make_context(0, stream=torch.cuda.current_stream().cuda_stream) as ctx:
        locs = [du[s.span_begin:s.span_begin + s.mapping.span].contiguous() for s in shards]
        steppers = [Stepper(ctx, s.mapping, lu.data_ptr(), ci, 30.0, TAU, TAU) for s, lu in zip(shards, locs)]
        for it in range(iters):
            exchange_in_process(shards, [st.vb for st in steppers], "vbar")
            for st in steppers:
                st.dual()
            exchange_in_process(shards, [st.xi for st in steppers], "xi")
            for st in steppers:
                st.primal(it)
        for s, st in zip(shards, steppers):
            lab = torch.zeros(s.mapping.span, dtype=torch.uint8, device="cuda")
            V = torch.zeros((K - 1, s.mapping.span), dtype=torch.float32, device="cuda")
            st.finish(labels_ptr=lab.data_ptr(), V_ptr=V.data_ptr())
            ctx.synchronize()
            b, e = s.owned_span()
            gb, ge = s.span_begin + b, s.span_begin + e
            keep = (np.arange(b, e) % m.nstride) < m.n_images
            assert np.array_equal(lab.cpu().numpy()[b:e][keep], whole.labels[gb:ge][keep])
            assert np.array_equal(V.cpu().numpy()[:, b:e][:, keep], whole.V[:, gb:ge][:, keep])
            st.close()
