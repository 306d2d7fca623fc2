"""The device side of a sharded batch: two MineEnvs holding the two halves
of a batch, with the any-done flag combined as the all-reduce would combine
it (max) and applied with MineEnv.regenerate_if, equal one MineEnv holding
the whole batch - worlds, observations, rewards, dones and agent state, bit
for bit.  (The multi-process exchange itself is tested on CPU ranks in
test_shard_cpu.py; this run has one GPU.)"""
import pytest

pytestmark = pytest.mark.gpu

B, HALF, STEPS, EPISODE = 12, 6, 16, 5
KEYS = ("voxels", "positions", "velocities", "yaws", "pitches", "step_count", "do_reset", "obs_buffer", "rewards")


def _bits(torch, t):
    return t.view(torch.int32) if t.dtype == torch.float32 else t


def test_halves_with_combined_flag_equal_whole_batch(cuda):
    import torch
    from minecu import MineEnv, _C
    kw = dict(world_size=16, render_width=16, render_height=16, obs_dtype="uint8", episode_length=EPISODE,
              device=cuda)
    whole = MineEnv(batch_size=B, **kw)
    halves = [MineEnv(batch_size=HALF, **kw), MineEnv(batch_size=HALF, **kw)]
    acts = torch.empty((STEPS, B), dtype=torch.uint8, device=cuda)
    _C.philox_actions(acts, 0, 0, 23, True)
    whole.reset()
    for h in halves:
        h.reset()
    flag = torch.zeros(1, dtype=torch.uint8, device=cuda)
    one_sided = 0
    for s in range(STEPS):
        if s == 2:  # a masked reset on the first half only: episodes end at different steps
            m = torch.zeros(B, dtype=torch.bool, device=cuda)
            m[:3] = True
            whole.reset(m)
            halves[0].reset(m[:HALF].clone())
            halves[1].reset(m[HALF:].clone())
            flag.fill_(1)
            for h in halves:
                h.regenerate_if(flag)
                h.get_obs()
        whole.step(acts[s])
        for i, h in enumerate(halves):
            h.step(acts[s, i * HALF:(i + 1) * HALF].contiguous())
        anys = [h.do_reset.any() for h in halves]
        one_sided += int(bool(anys[0]) != bool(anys[1]))
        flag.copy_(torch.stack(anys).any().reshape(1).to(torch.uint8))
        for h in halves:
            h.regenerate_if(flag)
        torch.cuda.synchronize()
        for k in KEYS:
            cat = torch.cat([getattr(h, k) for h in halves])
            assert torch.equal(_bits(torch, cat), _bits(torch, getattr(whole, k))), f"step {s}: {k}"
    assert one_sided > 0
