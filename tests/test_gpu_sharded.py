"""Target sharding on one GPU: the ensemble's targets split over several
shard handles (qg_shard_create), stepped in turn in one process (no kernel
waits on another shard's), with the new rho01 slices gathered and imported
after every step (quest_b200.sharded.LocalGroup; across GPUs ShardDriver
does the same with an NCCL all-gather).  Each shard's targets get the
unsharded handle's sums term for term, so the rho01 of every dot at every
step must equal the unsharded on-the-fly run's, bit for bit."""
import numpy as np
import pytest

from quest_b200 import capi, inputs as I, sharded

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("world,precision", [(2, capi.PREC_FP64), (3, capi.PREC_FP64), (2, capi.PREC_MIXED)])
def test_shards_reproduce_the_unsharded_run(golden_weights, world, precision):
    import torch

    wl = I.plain_small(n=300, steps=160, pulse_delay=0.12)
    wl.dots[:, 6:9] *= 0.5
    T = 160
    with capi.Simulation(wl.dots, wl.pulse, wl.constants, weights=golden_weights, precision=precision,
                         coef_mode=capi.COEF_ON_THE_FLY) as sim:
        ref = sim.run(T)
    shards = [sharded.GpuShard(wl.dots, wl.pulse, wl.constants, r, world, weights=golden_weights,
                               precision=precision) for r in range(world)]
    try:
        grp = sharded.LocalGroup(shards, device="cuda")
        got = np.empty((T, wl.n), dtype=np.complex128)
        for t in range(T):
            grp.step()
            got[t] = grp.rho01_user()
        torch.cuda.synchronize()
        assert np.abs(ref[..., 1]).max() > 1e-5  # excited
        np.testing.assert_array_equal(got, ref[..., 1])
        # each shard's own dots' final rho (both components) as well
        first_counts = [s.layout() for s in shards]
        for s, (f, c, n_pad, user) in zip(shards, first_counts):
            mine = user[f: f + c]
            mine = mine[mine >= 0]
            np.testing.assert_array_equal(s.state()[mine], ref[-1][mine])
            assert s.bad_step() == -1
    finally:
        for s in shards:
            s.close()


def test_shard_arguments_are_checked(golden_weights):
    wl = I.plain_small(n=64, steps=16)
    with pytest.raises(capi.QuestError):
        sharded.GpuShard(wl.dots, wl.pulse, wl.constants, 2, 2, weights=golden_weights)
    with pytest.raises(capi.QuestError):  # 2 blocks of 32 dots cannot make 3 shards
        sharded.GpuShard(wl.dots, wl.pulse, wl.constants, 0, 3, weights=golden_weights)
