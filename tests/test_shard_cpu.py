"""A batch split over ranks (minecu.shard) equals the same batch in one env.

Two gloo ranks on the CPU, each stepping its contiguous slice of a global
batch with the CPU oracle as its env, against one oracle env holding the
whole batch: the same actions (the global Philox stream, offset by each
rank's first env), masked resets on one rank only, and episodes that end on
one rank before the other.  With the any-done flag all-reduced every step
(sync_regen) every world is regenerated wherever the single env would
regenerate it, so worlds, observations, rewards, dones and agent state must
match exactly; without it the ranks drift apart (checked too).
"""
import os
import socket
import tempfile

import numpy as np
import pytest
import torch

from minecu.shard import shard_range

GLOBAL_B, STEPS, EPISODE = 10, 14, 5
RESET_AT, RESET_MASK = 3, (0, 1, 2)  # global envs reset at step 3: all on rank 0


def test_shard_range_covers_the_batch():
    for n in (0, 1, 7, 10, 32768, 32769):
        for world in (1, 2, 3, 8):
            parts = [shard_range(n, world, r) for r in range(world)]
            assert parts[0][0] == 0 and sum(c for _, c in parts) == n
            for (s0, c0), (s1, _) in zip(parts, parts[1:]):
                assert s0 + c0 == s1
            assert max(c for _, c in parts) - min(c for _, c in parts) <= 1
    with pytest.raises(ValueError):
        shard_range(4, 2, 2)


class _OracleShard:
    """The CPU oracle env with the interface ShardedEnv needs."""

    def __init__(self, n):
        import oracle as O
        self.e = O.OracleEnv(batch_size=n, world_size=16, render_width=16, render_height=16, obs_dtype="uint8",
                             episode_length=EPISODE)
        self.batch_size = n
        self.device = torch.device("cpu")
        self.regen = "all"  # the oracle env applies the all-world rule; ShardedEnv reads this mode

    def set_regen(self, mode):
        self.regen = mode

    @property
    def do_reset(self):
        return torch.from_numpy(self.e.do_reset.copy())

    def step(self, btn, look):
        return self.e.step(btn, look)

    def reset(self, mask=None):
        return self.e.reset(None if mask is None else np.asarray(mask))

    def get_obs(self):
        return self.e.get_obs()

    def regenerate_if(self, flag):
        if int(flag.reshape(-1)[0]):
            self.e._generate_world()


def _trajectory(env, start, count, sharded):
    import oracle as O
    out = {"obs": [], "rewards": [], "dones": [], "voxels": [], "positions": []}
    env.reset()
    for s in range(STEPS):
        if s == RESET_AT:
            mask = np.array([start + i in RESET_MASK for i in range(count)])
            env.reset(mask)
        a = O.philox_actions(count, s, 17, env_offset=start, break_half=True)
        btn, look = O.discrete_to_buttons(a, 0.1)
        env.step(btn, look)
        e = env.env.e if sharded else env.e
        out["obs"].append(e.obs.copy())
        out["rewards"].append(e.rewards.copy())
        out["dones"].append(e.do_reset.copy())
        out["voxels"].append(e.voxels.copy())
        out["positions"].append(e.positions.copy())
    return {k: np.stack(v) for k, v in out.items()}


def _rank_main(rank, world, port, out_dir, sync, switch=False):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    for sub in ("mine.cu_b200", "oracle", "tests"):
        sys.path.insert(0, os.path.join(root, sub))
    import torch.distributed as dist
    from minecu.shard import ShardedEnv, shard_range as sr
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        start, count = sr(GLOBAL_B, world, rank)
        inner = _OracleShard(count)
        if switch:
            inner.regen = "per_env"  # built under the per-env rule, switched before the first step
        env = ShardedEnv(inner, GLOBAL_B, sync_regen=sync)
        if switch:
            assert not env.sync_regen
            env.set_regen("all")
            assert env.sync_regen
        traj = _trajectory(env, start, count, True)
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), start=start, **traj)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _gather_main(rank, world, port, out_dir, global_b):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.join(root, "mine.cu_b200"))
    import torch.distributed as dist
    from minecu.shard import ShardedEnv, shard_range as sr

    class _Env:
        def __init__(self, n):
            self.batch_size = n
            self.device = torch.device("cpu")

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        start, count = sr(global_b, world, rank)
        env = ShardedEnv(_Env(count), global_b, sync_regen=False)
        rew = torch.arange(start, start + count, dtype=torch.float32) * 0.5
        done = (torch.arange(start, start + count) % 3) == 0
        g_rew, g_done = env.gather(rew, done)
        np.savez(os.path.join(out_dir, f"gather{rank}.npz"), rew=g_rew.numpy(), done=g_done.numpy())
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(300)
@pytest.mark.parametrize("global_b", [10, 7])
def test_gather_brings_every_ranks_results_in_env_order(global_b):
    """ShardedEnv.gather on two gloo ranks, even and uneven ranges."""
    import torch.multiprocessing as mp
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_gather_main, args=(2, _free_port(), d, global_b), nprocs=2, start_method="spawn",
                           join=True)
        for r in range(2):
            got = np.load(os.path.join(d, f"gather{r}.npz"))
            assert np.array_equal(got["rew"], np.arange(global_b, dtype=np.float32) * 0.5)
            assert np.array_equal(got["done"], np.arange(global_b) % 3 == 0)


def _run_ranks(sync, switch=False):
    import torch.multiprocessing as mp
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_rank_main, args=(2, _free_port(), d, sync, switch), nprocs=2, start_method="spawn",
                           join=True)
        parts = [dict(np.load(os.path.join(d, f"rank{r}.npz"))) for r in range(2)]
    return {k: np.concatenate([p[k] for p in parts], axis=1) for k in parts[0] if k != "start"}


@pytest.mark.timeout(300)
def test_two_ranks_equal_one_env_with_synced_regeneration():
    whole = _trajectory(_OracleShard(GLOBAL_B), 0, GLOBAL_B, False)
    split = _run_ranks(sync=True)
    for k in whole:
        assert np.array_equal(whole[k], split[k]), k
    # the scenario exercises the cross-rank rule: some step has dones on one rank only
    d = whole["dones"]
    half = GLOBAL_B // 2
    assert any(d[s, :half].any() != d[s, half:].any() for s in range(STEPS))


@pytest.mark.timeout(300)
def test_two_ranks_without_sync_drift_apart():
    whole = _trajectory(_OracleShard(GLOBAL_B), 0, GLOBAL_B, False)
    split = _run_ranks(sync=False)
    assert not np.array_equal(whole["voxels"], split["voxels"])


@pytest.mark.timeout(300)
def test_regen_mode_switched_after_construction_takes_effect():
    """A ShardedEnv built while its env regenerates per env, then switched to
    the all-world rule with set_regen, all-reduces the any-done flag from
    the next step on: the ranks again equal one env holding the batch."""
    whole = _trajectory(_OracleShard(GLOBAL_B), 0, GLOBAL_B, False)
    split = _run_ranks(sync=True, switch=True)
    for k in whole:
        assert np.array_equal(whole[k], split[k]), k
