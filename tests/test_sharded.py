"""Target sharding's host logic on CPU: two gloo ranks (separate processes,
rendezvous on 127.0.0.1) each step their own contiguous range of target dots
with the oracle's faithful step restricted to that range, and all-gather the
new rho01 slices through quest_b200.sharded.ShardDriver after every step.
Each rank's history must be the one-rank faithful run's, bit for bit, for its
own dots (rho and rho-dot) and for the others' rho01 it imported.  The GPU
form of the same loop is tests/test_gpu_sharded.py."""
import json
import os
import socket
import subprocess
import sys

import numpy as np

from tests.conftest import ROOT

CHILD = r"""
import json, os, sys
sys.path.insert(0, os.environ["QG_ROOT"])
import numpy as np
import torch
import torch.distributed as dist
from oracle import oracle as O
from quest_b200 import inputs as I, sharded

dist.init_process_group("gloo")
rank, world = dist.get_rank(), dist.get_world_size()
ps, cs, fc = I.load_pc_weights(os.path.join(os.environ["QG_ROOT"], "tests", "golden", "pc_weights_18_22_3.15.txt"))
W = O.Weights(ps, cs, fc)
T = int(os.environ["QG_T"])
wl = I.plain_small(n=int(os.environ["QG_N"]), steps=T, pulse_delay=0.12)
c = wl.constants
delays, coefs = O.build_table(wl.dots, c)


class OracleShard:
    # dots [lo, hi) of the user order; the history array holds every dot
    def __init__(self):
        n = wl.n
        self.lo, self.hi = n * rank // world, n * (rank + 1) // world
        self.hist = O.init_history(n, T)
        self.t = 0

    def layout(self):
        return self.lo, self.hi - self.lo, wl.n, np.arange(wl.n, dtype=np.int32)

    def step(self, out):
        O.faithful_step_range(wl.dots, wl.pulse, c, W, T, delays, coefs, self.hist, self.t, self.lo, self.hi)
        v = self.hist[self.lo: self.hi, self.t + O.WINDOW, 0, 1]
        out.copy_(torch.from_numpy(np.stack([v.real, v.imag], axis=1)))

    def import_full(self, full):
        f = full.numpy()
        z = f[:, 0] + 1j * f[:, 1]
        mask = np.ones(wl.n, dtype=bool)
        mask[self.lo: self.hi] = False
        self.hist[mask, self.t + O.WINDOW, 0, 1] = z[mask]
        self.t += 1


sh = OracleShard()
drv = sharded.ShardDriver(sh, sharded.DistExchange())
drv.run(T)
ref, bad = O.run_faithful(wl.dots, wl.pulse, c, W, T)
own = slice(sh.lo, sh.hi)
other = np.ones(wl.n, dtype=bool)
other[own] = False
out = {"rank": rank, "range": [sh.lo, sh.hi], "bad": bad,
       "own_equal": bool(np.array_equal(sh.hist[own], ref[own])),
       "others_rho01_equal": bool(np.array_equal(sh.hist[other, :, 0, 1], ref[other, :, 0, 1])),
       "last_user_equal": bool(np.array_equal(drv.rho01_user(), ref[:, T - 1 + O.WINDOW, 0, 1])),
       "excited": float(np.abs(ref[:, O.WINDOW:, 0, 1]).max()),
       "counts": drv.counts}
dist.destroy_process_group()
print(json.dumps(out))
"""


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_two_gloo_ranks_reproduce_the_one_rank_run():
    port = free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), QG_ROOT=ROOT, QG_N="48", QG_T="150", CUDA_VISIBLE_DEVICES="",
                   OMP_NUM_THREADS="1")
        procs.append(subprocess.Popen([sys.executable, "-c", CHILD], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        o, e = p.communicate(timeout=300)
        assert p.returncode == 0, e
        outs.append(json.loads(o.strip().splitlines()[-1]))
    a, b = sorted(outs, key=lambda d: d["rank"])
    assert a["range"] == [0, 24] and b["range"] == [24, 48]
    assert a["counts"] == b["counts"] == [24, 24]
    for r in (a, b):
        assert r["bad"] is None and r["excited"] > 1e-4
        assert r["own_equal"] and r["others_rho01_equal"] and r["last_user_equal"]


def test_shard_ranges_tile_the_blocks():
    from quest_b200 import sharded
    for nb, world in [(128, 2), (7, 3), (2048, 8), (5, 5)]:
        rs = sharded.shard_ranges(nb, world)
        assert rs[0][0] == 0 and rs[-1][1] == nb
        assert all(rs[i][1] == rs[i + 1][0] for i in range(world - 1))
        sizes = [hi - lo for lo, hi in rs]
        assert max(sizes) - min(sizes) <= 1
