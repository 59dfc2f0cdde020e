"""Target sharding of one ensemble over several GPUs, one process per GPU.

The reference sums every pair in one loop on one core
(src/interactions/history_interaction.cpp:47-70).  For an ensemble whose pair
sum is too much for one GPU, each rank takes a contiguous range of the
library's internal 32-dot blocks as its targets (qg_shard_create: every group
of dots coupled at delay 0 lies inside one block, so the current-step
coupling stays on one rank) and keeps every dot's rho01 history, which its
far and mid terms read.  The one exchange is after each step: the ranks'
new rho01 slices are all-gathered (NCCL over NVLink on GPUs; the gathered
vector lands in each rank's own memory) and imported into every rank's
history.  A sharded run gives the unsharded run's results bit for bit.

ShardDriver holds the host logic (slice sizes, padding for the all-gather,
reassembly in rank order) over two interfaces, so that it runs the same on
GPUs and in the CPU tests:

* a backend: layout() -> (first, count, n_pad, user), step(out) writes this
  rank's new slice, import_full(full) takes the step's whole vector;
* an exchange: all_gather(x) -> the ranks' x stacked in rank order.
"""
from __future__ import annotations

import ctypes
from typing import Sequence

import numpy as np

from . import capi


class DistExchange:
    """all_gather over torch.distributed (NCCL for CUDA tensors, gloo for CPU
    ones)."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.world = dist.get_world_size(group)
        self.rank = dist.get_rank(group)

    def all_gather(self, x):
        import torch
        # the ranks' tensors concatenated along the first dimension, then
        # viewed as (world, *x.shape)
        out = torch.empty((self.world * x.shape[0],) + tuple(x.shape[1:]), dtype=x.dtype, device=x.device)
        self.dist.all_gather_into_tensor(out, x.contiguous(), group=self.group)
        return out.view((self.world,) + tuple(x.shape))


class ShardDriver:
    """Steps one rank's shard and exchanges its new rho01 slice each step."""

    def __init__(self, backend, exchange, device="cpu"):
        import torch
        self.backend = backend
        self.exchange = exchange
        self.first, self.count, self.n_pad, self.user = backend.layout()
        # every rank's slice (count complex as count x 2 float64), padded to
        # the largest for the all-gather
        counts = exchange.all_gather(torch.tensor([self.first, self.count], dtype=torch.int64, device=device))
        counts = counts.cpu().numpy().reshape(-1, 2)
        self.firsts = [int(f) for f in counts[:, 0]]
        self.counts = [int(c) for c in counts[:, 1]]
        if sum(self.counts) != self.n_pad or self.firsts != list(np.cumsum([0] + self.counts[:-1])):
            raise ValueError(f"shard ranges {list(zip(self.firsts, self.counts))} do not tile 0..{self.n_pad}")
        self.max_count = max(self.counts)
        self.slice = torch.zeros((self.max_count, 2), dtype=torch.float64, device=device)
        self.full = torch.zeros((self.n_pad, 2), dtype=torch.float64, device=device)

    def step(self) -> None:
        self.backend.step(self.slice[: self.count])
        parts = self.exchange.all_gather(self.slice)
        for r, (f, c) in enumerate(zip(self.firsts, self.counts)):
            self.full[f: f + c] = parts[r, :c]
        self.backend.import_full(self.full)

    def run(self, n_steps: int) -> None:
        for _ in range(n_steps):
            self.step()

    def rho01_user(self) -> np.ndarray:
        """The last exchanged step's rho01 of every dot, user order."""
        full = self.full.cpu().numpy()
        out = np.zeros(int((self.user >= 0).sum()), dtype=np.complex128)
        live = self.user >= 0
        out[self.user[live]] = full[live, 0] + 1j * full[live, 1]
        return out


class GpuShard:
    """Backend over the library's shard handle (qg_shard_*); tensors on the
    handle's GPU."""

    def __init__(self, dots: np.ndarray, pulse: np.ndarray, constants, rank: int, world: int, weights=None,
                 precision=capi.PREC_FP64):
        L = capi.lib()
        self.n = int(dots.shape[0])
        self._dots = capi.dots_array(dots)
        self._pulse = capi.pulse_struct(pulse)
        self._params = capi.make_params(constants, precision, capi.COEF_ON_THE_FLY)
        self._w = capi.make_weights(*weights) if weights is not None else None
        h = ctypes.c_void_p()
        capi._check(L.qg_shard_create(self._dots, self.n, ctypes.byref(self._pulse), ctypes.byref(self._params),
                                      ctypes.byref(self._w) if self._w is not None else None, rank, world,
                                      ctypes.byref(h)))
        self.h = h

    def layout(self):
        first, count, n_pad = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        capi._check(capi.lib().qg_shard_layout(self.h, ctypes.byref(first), ctypes.byref(count),
                                               ctypes.byref(n_pad), None))
        user = np.empty(n_pad.value, dtype=np.int32)
        capi._check(capi.lib().qg_shard_layout(self.h, None, None, None,
                                               user.ctypes.data_as(ctypes.POINTER(ctypes.c_int))))
        return first.value, count.value, n_pad.value, user

    def step(self, out) -> None:
        assert out.is_cuda and out.is_contiguous()
        capi._check(capi.lib().qg_shard_step(self.h, ctypes.cast(out.data_ptr(), ctypes.POINTER(ctypes.c_double))))

    def import_full(self, full) -> None:
        assert full.is_cuda and full.is_contiguous()
        capi._check(capi.lib().qg_shard_import(self.h, ctypes.cast(full.data_ptr(),
                                                                   ctypes.POINTER(ctypes.c_double))))

    def state(self) -> np.ndarray:
        """(N, 2) rho after the last step; only this shard's dots are current."""
        out = np.empty((self.n, 2), dtype=np.complex128)
        capi._check(capi.lib().qg_get_state(self.h, capi._dp(out.view(np.float64))))
        return out

    def bad_step(self) -> int:
        b = ctypes.c_int()
        capi._check(capi.lib().qg_bad_step(self.h, ctypes.byref(b)))
        return b.value

    def close(self) -> None:
        if getattr(self, "h", None) is not None and self.h.value:
            capi.lib().qg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class LocalGroup:
    """Several shards stepped in one process in turn (no device waits on
    another): step() runs every shard's step, then hands the gathered vector
    to every shard.  For testing the sharded path on one GPU."""

    def __init__(self, backends: Sequence, device="cpu"):
        import torch
        self.backends = list(backends)
        lay = [b.layout() for b in self.backends]
        self.n_pad = lay[0][2]
        self.user = lay[0][3]
        self.ranges = [(f, c) for f, c, _, _ in lay]
        if sorted(self.ranges) != self.ranges or sum(c for _, c in self.ranges) != self.n_pad:
            raise ValueError(f"shard ranges {self.ranges} do not tile 0..{self.n_pad}")
        self.full = torch.zeros((self.n_pad, 2), dtype=torch.float64, device=device)

    def step(self) -> None:
        for b, (f, c) in zip(self.backends, self.ranges):
            b.step(self.full[f: f + c])
        for b in self.backends:
            b.import_full(self.full)

    def run(self, n_steps: int) -> None:
        for _ in range(n_steps):
            self.step()

    def rho01_user(self) -> np.ndarray:
        full = self.full.cpu().numpy()
        live = self.user >= 0
        out = np.zeros(int(live.sum()), dtype=np.complex128)
        out[self.user[live]] = full[live, 0] + 1j * full[live, 1]
        return out


def shard_ranges(n_blocks: int, world: int) -> list[tuple[int, int]]:
    """The blocks [lo, hi) of each rank, as qg_shard_create splits them."""
    return [(n_blocks * r // world, n_blocks * (r + 1) // world) for r in range(world)]
