"""bench.py's multi-rank logic on CPU: two gloo ranks started as separate
processes (rendezvous on 127.0.0.1), each with its own ensemble; the timing
is the maximum over ranks and the whole-job throughput counts every rank's
ensemble (weak scaling, no data-path collective)."""
import json
import os
import socket
import subprocess
import sys

import pytest

from tests.conftest import ROOT

CHILD = r"""
import json, os, sys
sys.path.insert(0, os.environ["QG_ROOT"])
import argparse
import bench
args = bench.parse_args(["--n", "64", "--steps", "10", "--warmup", "3"])
world, rank, local = bench.dist_setup(args, backend="gloo")
warm, timed = bench.main_window(args)
wl = bench.workload(args, rank, warm + timed)
ms = 10.0 + 5.0 * rank            # this rank's (pretend) device time
ms_max = bench.max_over_ranks(ms, world)
bench.barrier(world)
value = bench.job_throughput(world, wl.n, timed, ms_max)
out = {"rank": rank, "world": world, "ms_max": ms_max, "value": value,
       "first_dot": [float(x) for x in wl.dots[0, :3]],
       "timed": timed, "parallelism": bench.config_dict(args, warm, timed)["parallelism"]}
import torch.distributed as dist
dist.destroy_process_group()
print(json.dumps(out))
"""


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_two_gloo_ranks():
    port = free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), QG_ROOT=ROOT, CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", CHILD], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        o, e = p.communicate(timeout=120)
        assert p.returncode == 0, e
        outs.append(json.loads(o.strip().splitlines()[-1]))
    a, b = sorted(outs, key=lambda d: d["rank"])
    assert a["world"] == b["world"] == 2
    assert a["ms_max"] == b["ms_max"] == 15.0          # the slower rank
    assert a["timed"] == b["timed"] == 16                # whole 16-step blocks
    assert a["value"] == b["value"] == pytest.approx(2 * 64 * 64 * 16 / 0.015)
    assert a["first_dot"] != b["first_dot"]            # each rank its own ensemble
    assert a["parallelism"] == "independent ensemble per GPU"
