"""A batch of envs split over several GPUs, one process per GPU.

Envs are independent, so a global batch of N envs is cut into contiguous
ranges, one per rank; each rank steps its own MineEnv and nothing crosses
the ranks in the step itself.  The one coupling the reference has between
envs - "any env done (or reset) -> every world is regenerated"
(minecu/__init__.py:290-300, 356-358, 439-441) - would otherwise apply per
rank only.  With `sync_regen`, after every step (or reset) each rank
all-reduces a one-byte any-done flag (MAX) and regenerates its worlds when
the flag is set anywhere, on the device, without a host synchronisation
(`MineEnv.regenerate_if`).  The result is the same as one MineEnv holding
the whole batch.  The all-reduce is only needed when episodes can end or
masked resets happen; a run with neither leaves `sync_regen` off.

`gather` brings every rank's rewards and dones to every rank in global env
order (one all-gather), for a single consumer of the whole batch.

Actions for a rank's envs come from the global action stream with the rank's
first env as the offset (Philox counter = (global env, step)), so the job is
independent of the number of ranks:

    shard = ShardedEnv(MineEnv(batch_size=count, ...), global_batch=N)
    _C.philox_actions(acts, shard.start, step0, seed)
"""
from __future__ import annotations

from typing import Optional, Tuple

import torch
import torch.distributed as dist


def shard_range(global_batch: int, world: int, rank: int) -> Tuple[int, int]:
    """(first env, number of envs) of `rank` when `global_batch` envs are cut
    into `world` contiguous ranges whose sizes differ by at most one."""
    if world < 1 or not 0 <= rank < world or global_batch < 0:
        raise ValueError(f"bad shard request: {global_batch} envs, world {world}, rank {rank}")
    base, extra = divmod(global_batch, world)
    start = rank * base + min(rank, extra)
    return start, base + (1 if rank < extra else 0)


def max_over_ranks(x: float, device: Optional[torch.device] = None) -> float:
    """The maximum of a per-rank number (e.g. a timed region) over all ranks."""
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return x
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class ShardedEnv:
    """One rank's contiguous slice of a global batch.  `env` holds this
    rank's envs (its batch size must be the rank's count) and provides
    step/reset, a `do_reset` bool tensor and `regenerate_if(flag)`."""

    def __init__(self, env, global_batch: int, sync_regen: bool = True, group=None,
                 flag_device: Optional[torch.device] = None):
        self.env = env
        self.group = group
        self.world = dist.get_world_size(group) if dist.is_initialized() else 1
        self.rank = dist.get_rank(group) if dist.is_initialized() else 0
        self.start, self.count = shard_range(global_batch, self.world, self.rank)
        n = getattr(env, "batch_size", None)
        if n is not None and n != self.count:
            raise ValueError(f"rank {self.rank} holds envs [{self.start}, {self.start + self.count}); "
                             f"its env has batch_size {n}")
        self.global_batch = global_batch
        self._sync_requested = sync_regen and self.world > 1
        self.flag_device = flag_device if flag_device is not None else getattr(env, "device", torch.device("cpu"))
        self._flag = torch.zeros(1, dtype=torch.uint8, device=self.flag_device)

    @property
    def sync_regen(self) -> bool:
        """Whether a step or reset all-reduces the any-done flag: asked for,
        more than one rank, and the env's regeneration rule is "all" (read at
        every step, so `env.set_regen` after construction takes effect; per-env
        regeneration couples no envs and needs nothing)."""
        return self._sync_requested and getattr(self.env, "regen", "all") == "all"

    def set_regen(self, mode: str) -> None:
        """Switch the env's regeneration rule ("all" or "per_env").  Every
        rank must make the same switch between the same two steps, since the
        all-reduce runs on every rank or on none."""
        self.env.set_regen(mode)

    def _sync(self, local_any: torch.Tensor) -> None:
        self._flag.copy_(local_any.reshape(1).to(device=self.flag_device, dtype=torch.uint8))
        dist.all_reduce(self._flag, op=dist.ReduceOp.MAX, group=self.group)
        self.env.regenerate_if(self._flag)

    def step(self, *args):
        out = self.env.step(*args)
        if self.sync_regen:
            self._sync(torch.as_tensor(self.env.do_reset).any())
        return out

    def gather(self, rewards: torch.Tensor, dones: torch.Tensor) -> Tuple[torch.Tensor, torch.Tensor]:
        """Every rank's rewards and dones of a step, in global env order, on
        every rank (for a single consumer such as a learner): one all-gather
        of a [2, n] float32 block per rank (rewards, dones as 0/1), each
        padded to the largest range.  Returns (rewards float32 [N], dones
        bool [N]) on this rank's flag device."""
        dev = self.flag_device
        if self.world == 1:
            return rewards.to(dev, torch.float32), dones.to(dev).bool()
        counts = [shard_range(self.global_batch, self.world, r)[1] for r in range(self.world)]
        n = max(counts)
        block = torch.zeros((2, n), dtype=torch.float32, device=dev)
        block[0, :self.count] = rewards.reshape(-1).to(dev, torch.float32)
        block[1, :self.count] = dones.reshape(-1).to(dev, torch.float32)
        parts = [torch.empty_like(block) for _ in range(self.world)]
        dist.all_gather(parts, block, group=self.group)
        rew = torch.cat([p[0, :c] for p, c in zip(parts, counts)])
        done = torch.cat([p[1, :c] for p, c in zip(parts, counts)]) != 0
        return rew, done

    def reset(self, mask: Optional[torch.Tensor] = None):
        obs = self.env.reset(mask)
        if self.sync_regen:
            local = torch.ones(1, dtype=torch.bool) if mask is None else torch.as_tensor(mask).any()
            self._sync(local)
            if mask is not None:
                obs = self.env.get_obs()  # a world regenerated for another rank changes this rank's view
        return obs
