"""The launch-shape autotuner (minecu.autotune): it times candidate shapes on
the caller's envs from one restored snapshot, sets the fastest, restores the
envs' state, caches the result, and never changes what a step computes (the
tuned env stays bit-identical to an untuned one)."""
import os

import pytest

pytestmark = pytest.mark.gpu


def _bits(torch, t):
    return t.view(torch.int32) if t.dtype == torch.float32 else t


def test_tune_env_restores_state_and_caches(cuda, tmp_path, monkeypatch):
    import torch
    from minecu import MineEnv, _C, autotune
    monkeypatch.setenv("MINECU_TUNE_CACHE", str(tmp_path / "tune.json"))
    kw = dict(batch_size=256, world_size=16, render_width=32, render_height=32, obs_dtype="uint8", device=cuda)
    a, b = MineEnv(**kw), MineEnv(**kw)
    a.reset()
    b.reset()
    before = a.state_dict()
    cands = [(1, 8, 4, 4, 1, 0), (0, 8, 4, 8, 1, 0), (1, 8, 3, 8, 4, 1), (1, 8, 4, 5, 1, 0)]  # the last is invalid
    out = autotune.tune_env(a, steps=4, warm_steps=3, candidates=cands, use_cache=True)
    assert tuple(out["config"]) in [c for c in cands[:3]] and out["trials"] == 3
    cfg = a.launch_config()
    assert [cfg[k] for k in ("stage", "warps_per_cta", "ctas_per_sm", "tile_w", "team_warps", "coop")] == \
        list(out["config"])
    after = a.state_dict()
    for k in before:
        assert torch.equal(_bits(torch, before[k]), _bits(torch, after[k])), k
    assert os.path.exists(tmp_path / "tune.json")
    again = autotune.tune_env(b, steps=4, warm_steps=3, candidates=cands, use_cache=True)
    assert again["config"] == out["config"]  # from the cache
    acts = torch.empty((6, 256), dtype=torch.uint8, device=cuda)
    _C.philox_actions(acts, 0, 0, 5)
    c = MineEnv(**kw)
    c.reset()
    for s in range(6):
        a.step(acts[s])
        c.step(acts[s])
    torch.cuda.synchronize()
    for k in ("voxels", "positions", "obs_buffer", "rewards"):
        assert torch.equal(_bits(torch, getattr(a, k)), _bits(torch, getattr(c, k))), k


def test_tune_ragged_sets_a_valid_config(cuda, tmp_path, monkeypatch):
    import torch
    from minecu import MineEnv, autotune
    from minecu.ragged import RaggedBatch
    monkeypatch.setenv("MINECU_TUNE_CACHE", str(tmp_path / "tune.json"))
    envs = [MineEnv(batch_size=128, world_size=8, render_width=16, render_height=16, ground_height=4,
                    obs_dtype="uint8", device=cuda),
            MineEnv(batch_size=64, world_size=32, render_width=64, render_height=64, obs_dtype="uint8", device=cuda)]
    batch = RaggedBatch(envs)
    batch.reset()
    before = batch.state_dict()
    out = autotune.tune_ragged(batch, steps=3, warm_steps=2, rounds=1, use_cache=False)
    cfg = batch.launch_config()
    assert cfg["team_warps"] == out["config"]["team_warps"] and cfg["coop"] == out["config"]["coop"]
    assert out["trials"] > 5
    after = batch.state_dict()
    for sb, sa in zip(before, after):
        for k in sb:
            assert torch.equal(_bits(torch, sb[k]), _bits(torch, sa[k])), k
