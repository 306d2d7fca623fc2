"""Ragged batches: several MineEnv groups (different world sizes,
resolutions, episode lengths) stepped by one persistent launch.

Each group must end every step bit-identical (floats compared as int32 bit
patterns; tolerance none) to the same MineEnv stepped on its own with the
fused form, which the other parity tests tie to the CPU oracle (ieee) and to
the reference's CUDA build (ref_fast).  The ieee case is also compared with
the CPU oracle directly.
"""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

KEYS = ("voxels", "positions", "velocities", "yaws", "pitches", "on_ground", "step_count", "do_reset", "cameras",
        "rewards", "obs_buffer")

# (batch, world, (res_w, res_h), ground_height, episode_length)
GROUPS = [
    (37, 8, (16, 16), 4, None),
    (50, 16, (32, 32), 8, 9),
    (23, 24, (24, 16), 8, None),
    (19, 32, (64, 64), 8, 6),
]


def _bits(torch, t):
    return t.view(torch.int32) if t.dtype == torch.float32 else t


def _make(torch, cuda, groups, obs_dtype, numerics):
    from minecu import MineEnv
    return [MineEnv(batch_size=b, world_size=w, render_width=r[0], render_height=r[1], ground_height=gh,
                    episode_length=el, obs_dtype=obs_dtype, numerics=numerics, device=cuda)
            for b, w, r, gh, el in groups]


def _actions(torch, cuda, total, steps, seed):
    from minecu import _C
    a = torch.empty((steps, total), dtype=torch.uint8, device=cuda)
    _C.philox_actions(a, 0, 0, seed)
    return a


def _assert_same(torch, ea, eb, what):
    for g, (a, b) in enumerate(zip(ea, eb)):
        for k in KEYS:
            x, y = getattr(a, k), getattr(b, k)
            if not torch.equal(_bits(torch, x), _bits(torch, y)):
                n = int((_bits(torch, x) != _bits(torch, y)).sum())
                raise AssertionError(f"{what}: group {g} field {k}: {n} elements differ")


def _run_vs_separate(cuda, obs_dtype, numerics, config=None, steps=14, seed=3, groups=GROUPS):
    import torch
    from minecu.ragged import RaggedBatch
    ra = _make(torch, cuda, groups, obs_dtype, numerics)
    sb = _make(torch, cuda, groups, obs_dtype, numerics)
    batch = RaggedBatch(ra)
    if config is not None:
        batch.set_launch_config(*config)
    batch.reset()
    for e in sb:
        e.reset()
    acts = _actions(torch, cuda, batch.total, steps, seed)
    for s in range(steps):
        batch.step(acts[s])
        for g, e in enumerate(sb):
            e.step(acts[s, batch.group_slice(g)])
        torch.cuda.synchronize()
        _assert_same(torch, ra, sb, f"step {s}")
    batch.check_error()
    return ra


@pytest.mark.parametrize("obs_dtype", ["uint8", "float32", "uint8_minimal", "uint8_prebasis_full"])
def test_ragged_equals_separate_fused_ref_fast(cuda, obs_dtype):
    _run_vs_separate(cuda, obs_dtype, "ref_fast")


# (warps_per_cta, ctas_per_sm, stage, tile_w, team_warps, coop)
@pytest.mark.parametrize("config", [
    (8, 4, [1, 1, 1, 0], [4, 4, 4, 4], 1, [0, 0, 0, 0]),
    (4, 2, [0, 0, 0, 0], [8, 16, 32, 8], 2, [0, 0, 0, 0]),
    (3, 1, [1, 0, 1, 1], [16, 4, 8, 32], 1, [0, 0, 0, 0]),
    (6, 3, [0, 1, 0, 1], [32, 8, 16, 4], 2, [1, 0, 1, 0]),
    (8, 3, [1, 1, 1, 1], [4, 8, 8, 8], 8, [0, 1, 1, 1]),
    (8, 2, [0, 0, 1, 1], [4, 4, 16, 4], 4, [1, 1, 1, 1]),
    (4, 4, [1, 1, 0, 1], [8, 4, 4, 16], 4, [1, 0, 0, 1]),
    # staging depth 2: the next unit's world is copied while the current one renders
    (8, 2, [2, 2, 2, 2], [4, 8, 8, 8], 4, [0, 1, 1, 1]),
    (4, 2, [2, 0, 2, 2], [8, 4, 16, 8], 2, [0, 0, 1, 1]),
    (4, 2, [2, 2, 0, 0], [4, 4, 8, 16], 1, [0, 0, 0, 0]),
    (8, 1, [2, 2, 2, 2], [4, 8, 4, 8], 8, [1, 1, 1, 1]),
])
def test_ragged_launch_configs_bit_exact(cuda, config):
    """Every launch shape, team shape, tile shape and staging choice gives the same bits."""
    wpc, cps, stage, tile_w, team, coop = config
    _run_vs_separate(cuda, "uint8", "ref_fast", config=(wpc, cps, stage, tile_w, team, coop), steps=10)


@pytest.mark.parametrize("obs_dtype", ["uint8", "float32", "uint8_fast", "uint8_prebasis_full"])
def test_ragged_teams_all_families(cuda, obs_dtype):
    """Cooperative teams in every render family."""
    _run_vs_separate(cuda, obs_dtype, "ref_fast", config=(8, 3, [1, 0, 1, 0], [4, 8, 16, 8], 4, [1, 1, 0, 1]),
                     steps=10)


@pytest.mark.parametrize("mode", ["uint8", "float32", "uint8_minimal", "uint8_prebasis_full"])
@pytest.mark.parametrize("team", [(2, 1, 1, 4), (8, 1, 0, 8), (8, 0, 1, 16), (4, 1, 1, 32), (4, 1, 2, 8),
                                  (2, 0, 2, 4)])
def test_env_team_form_equals_per_warp(cuda, mode, team):
    """MineEnv with the team kernel (teams_warps, coop, stage, tile_w) equals the per-warp kernel."""
    import torch
    from minecu import MineEnv
    tw, coop, stage, tile = team
    kw = dict(batch_size=45, world_size=16, render_width=40, render_height=24, obs_dtype=mode, device=cuda,
              episode_length=7)
    a, b = MineEnv(**kw), MineEnv(**kw)
    b.set_launch_config(stage, 8, 3, tile, team_warps=tw, coop=coop)
    a.reset()
    b.reset()
    acts = _actions(torch, cuda, 45, 16, 9)
    for s in range(16):
        a.step(acts[s])
        b.step(acts[s])
        torch.cuda.synchronize()
        _assert_same(torch, [a], [b], f"step {s}")
    b.check_error()


def test_ragged_ieee_vs_oracle(cuda):
    """ieee numerics: every group equals the CPU oracle env of its config."""
    import torch
    from minecu.ragged import RaggedBatch
    from mc_harness import diff_report
    groups = [(9, 8, (16, 16), 4, None), (7, 16, (32, 32), 8, 5), (5, 24, (24, 16), 8, None)]
    envs = _make(torch, cuda, groups, "uint8", "ieee")
    batch = RaggedBatch(envs)
    orcs = [O.OracleEnv(batch_size=b, world_x=w, world_y=w, world_z=w, render_width=r[0], render_height=r[1],
                        ground_height=gh, episode_length=el, obs_dtype="uint8")
            for b, w, r, gh, el in groups]
    batch.reset()
    for o in orcs:
        o.reset()
    steps = 12
    acts = _actions(torch, cuda, batch.total, steps, 3)
    host = acts.cpu().numpy()
    for s in range(steps):
        batch.step(acts[s])
        torch.cuda.synchronize()
        for g, (e, o) in enumerate(zip(envs, orcs)):
            btn, look = O.discrete_to_buttons(host[s, batch.group_slice(g)], 0.1)
            o.step(btn, look)
            mine = {"voxels": e.voxels.cpu().numpy(), "positions": e.positions.cpu().numpy(),
                    "obs": e.obs_buffer.cpu().numpy(), "rewards": e.rewards.cpu().numpy(),
                    "do_reset": e.do_reset.cpu().numpy(), "step_count": e.step_count.cpu().numpy()}
            ref = {"voxels": o.voxels, "positions": o.positions, "obs": o.obs, "rewards": o.rewards,
                   "do_reset": o.do_reset, "step_count": o.step_count}
            d = diff_report(mine, ref)
            assert not d, f"step {s} group {g}: {d}"


def test_ragged_rollout_equals_steps(cuda):
    import torch
    from minecu.ragged import RaggedBatch
    ea = _make(torch, cuda, GROUPS, "uint8", "ref_fast")
    eb = _make(torch, cuda, GROUPS, "uint8", "ref_fast")
    ba, bb = RaggedBatch(ea), RaggedBatch(eb)
    ba.reset()
    bb.reset()
    acts = _actions(torch, cuda, ba.total, 16, 4)
    ba.rollout(acts[:8])
    ba.rollout(acts[8:])
    for s in range(16):
        bb.step(acts[s])
    torch.cuda.synchronize()
    _assert_same(torch, ea, eb, "after 16 steps")


def test_ragged_buttons_and_look(cuda):
    """The continuous action form, concatenated in group order."""
    import torch
    from minecu.ragged import RaggedBatch
    ra = _make(torch, cuda, GROUPS[:3], "uint8", "ref_fast")
    sb = _make(torch, cuda, GROUPS[:3], "uint8", "ref_fast")
    batch = RaggedBatch(ra)
    batch.reset()
    for e in sb:
        e.reset()
    rng = np.random.default_rng(11)
    for s in range(8):
        btn = torch.from_numpy(rng.integers(0, 2, (batch.total, 8), dtype=np.int8)).to(cuda)
        look = torch.from_numpy(rng.uniform(-0.3, 0.3, (batch.total, 2)).astype(np.float32)).to(cuda)
        batch.step(btn, look)
        for g, e in enumerate(sb):
            sl = batch.group_slice(g)
            e.step(btn[sl].contiguous(), look[sl].contiguous())
        torch.cuda.synchronize()
        _assert_same(torch, ra, sb, f"step {s}")


def test_ragged_rejects_invalid(cuda):
    import torch
    from minecu import MineEnv
    from minecu.ragged import RaggedBatch
    a = MineEnv(batch_size=4, world_size=16, render_width=16, render_height=16, obs_dtype="uint8", device=cuda)
    b = MineEnv(batch_size=4, world_size=16, render_width=16, render_height=16, obs_dtype="float32", device=cuda)
    with pytest.raises(RuntimeError, match="observation kind"):
        RaggedBatch([a, b])
    odd = MineEnv(batch_size=4, world_x=9, world_y=9, world_z=9, render_width=16, render_height=16,
                  obs_dtype="uint8", device=cuda)
    batch = RaggedBatch([a, odd])
    with pytest.raises(RuntimeError, match="stage needs"):
        batch.set_launch_config(8, 4, [1, 1], [4, 4])
    with pytest.raises(RuntimeError, match="tile_w"):
        batch.set_launch_config(8, 4, [1, 0], [4, 5])
    with pytest.raises(RuntimeError, match="team_warps"):
        batch.set_launch_config(6, 4, [1, 0], [4, 4], team_warps=4)
    with pytest.raises(RuntimeError, match="shared memory"):
        big = MineEnv(batch_size=2, world_size=48, render_width=16, render_height=16, obs_dtype="uint8", device=cuda)
        RaggedBatch([a, big]).set_launch_config(8, 1, [0, 1], [4, 4], team_warps=1, coop=[0, 0])
    with pytest.raises(ValueError):
        RaggedBatch([a] * 17)
    with pytest.raises(RuntimeError, match="repeats"):
        RaggedBatch([a, a])
    del torch


@pytest.mark.parametrize("config", [None, (8, 3, [1, 1, 1, 1], [4, 8, 8, 8], 4, [0, 1, 1, 1])],
                         ids=["default", "teams"])
def test_ragged_per_env_regen_equals_separate(cuda, config):
    """Per-env regeneration (regen="per_env") through one ragged launch equals
    the same groups stepped alone with it.  A masked reset of a third of each
    group's envs at step 4 offsets their episodes, so envs of one group end
    on different steps and only their own worlds regenerate; half the actions
    break blocks, so the worlds left alone differ from the start world."""
    import torch
    from minecu import _C
    from minecu.ragged import RaggedBatch
    ra = _make(torch, cuda, GROUPS, "uint8", "ref_fast")
    sb = _make(torch, cuda, GROUPS, "uint8", "ref_fast")
    for e in ra + sb:
        e.set_regen("per_env")
    batch = RaggedBatch(ra)
    if config is not None:
        batch.set_launch_config(*config)
    batch.reset()
    for e in sb:
        e.reset()
    steps = 18
    acts = torch.empty((steps, batch.total), dtype=torch.uint8, device=cuda)
    _C.philox_actions(acts, 0, 0, 9, True)
    for s in range(steps):
        if s == 4:
            for a, b in zip(ra, sb):
                m = (torch.arange(a.batch_size, device=cuda) % 3) == 0
                a.reset(m)
                b.reset(m)
        batch.step(acts[s])
        for g, e in enumerate(sb):
            e.step(acts[s, batch.group_slice(g)])
        torch.cuda.synchronize()
        _assert_same(torch, ra, sb, f"step {s}")
    batch.check_error()
