"""MineEnv.step_host (mc_env_step_host): the discrete step with host buffers,
whose uploads and read-backs overlap the neighbouring steps.

Two envs built alike take the same actions: one through step(actions) with
device tensors, the other through step_host with pinned host tensors.  After
join_host and a synchronisation, every step's rewards and dones in host
memory, and the final state of the two envs, must be identical (floats
compared as int32 bit patterns; tolerance none).  Short episodes and half of
the actions forced to "break" make rewards, dones and world regeneration
happen inside the window.
"""
import pytest

pytestmark = pytest.mark.gpu

KEYS = ("voxels", "positions", "velocities", "yaws", "pitches", "on_ground", "step_count", "do_reset", "cameras",
        "rewards", "obs_buffer")


def _pair(cuda, form, **kw):
    from minecu import MineEnv
    envs = [MineEnv(device=cuda, **kw) for _ in range(2)]
    for e in envs:
        e.form = form
        e.reset()
    return envs


@pytest.mark.parametrize("form", ["fused", "plain"])
@pytest.mark.parametrize("shape", [dict(batch_size=300, world_size=16, render_width=32, render_height=32,
                                        episode_length=7, obs_dtype="uint8"),
                                   dict(batch_size=77, world_size=32, render_width=24, render_height=16,
                                        episode_length=5, obs_dtype="float32")])
def test_step_host_matches_step(cuda, form, shape):
    import torch
    from minecu import _C
    ref, host = _pair(cuda, form, **shape)
    B, K = shape["batch_size"], 23
    acts = torch.empty((K, B), dtype=torch.uint8, device=cuda)
    _C.philox_actions(acts, 0, 0, 11, True)
    h_acts = acts.cpu().pin_memory()
    h_rew = torch.zeros((K, B), dtype=torch.float32).pin_memory()
    h_done = torch.zeros((K, B), dtype=torch.bool).pin_memory()
    want_rew, want_done = [], []
    for s in range(K):
        _, r, d = ref.step(acts[s])
        want_rew.append(r.clone())
        want_done.append(d.clone())
        host.step_host(h_acts[s], h_rew[s], h_done[s])
    host.join_host()
    torch.cuda.synchronize()
    want_rew = torch.stack(want_rew).cpu()
    want_done = torch.stack(want_done).cpu()
    assert torch.equal(h_rew.view(torch.int32), want_rew.view(torch.int32))
    assert torch.equal(h_done, want_done.to(torch.bool))
    assert bool(want_done.any()), "the window should end episodes"
    assert bool((want_rew != 0).any()), "the window should earn rewards"
    for k in KEYS:
        a, b = getattr(ref, k), getattr(host, k)
        if a.dtype == torch.float32:
            a, b = a.view(torch.int32), b.view(torch.int32)
        assert torch.equal(a, b), k


@pytest.mark.parametrize("launch,wait0", [((0, 8, 4, 4, 1, 0), False), ((2, 8, 4, 4, 1, 0), False),
                                          ((1, 8, 4, 4, 1, 0), True), ((2, 8, 4, 4, 1, 0), True)],
                         ids=["depth0", "depth2", "depth1_timeouts", "depth2_timeouts"])
def test_step_host_per_warp_launches(cuda, launch, wait0):
    """The per-warp fused kernel writes every env's reward and done into the
    read-back buffer itself (no copy kernel): at staging depth 0 and 2, and
    with every bulk-copy wait made to run out, where the global-memory path
    steps the envs.  The host results equal step(actions)'s."""
    import torch
    from minecu import _C
    shape = dict(batch_size=300, world_size=16, render_width=32, render_height=32, episode_length=7,
                 obs_dtype="uint8")
    ref, host = _pair(cuda, "fused", **shape)
    host.set_launch_config(*launch)
    if wait0:
        host.set_wait_limit(0)
    B, K = shape["batch_size"], 15
    acts = torch.empty((K, B), dtype=torch.uint8, device=cuda)
    _C.philox_actions(acts, 0, 0, 13, True)
    h_acts = acts.cpu().pin_memory()
    h_rew = torch.zeros((K, B), dtype=torch.float32).pin_memory()
    h_done = torch.zeros((K, B), dtype=torch.bool).pin_memory()
    want_rew, want_done = [], []
    for s in range(K):
        _, r, d = ref.step(acts[s])
        want_rew.append(r.clone())
        want_done.append(d.clone())
        host.step_host(h_acts[s], h_rew[s], h_done[s])
    host.join_host()
    torch.cuda.synchronize()
    assert torch.equal(h_rew.view(torch.int32), torch.stack(want_rew).cpu().view(torch.int32))
    assert torch.equal(h_done, torch.stack(want_done).cpu().to(torch.bool))
    assert bool(torch.stack(want_done).any()) and bool((torch.stack(want_rew) != 0).any())
    if wait0:
        with pytest.raises(RuntimeError, match="timed out"):
            host.check_error()
    else:
        host.check_error()
    for k in KEYS:
        a, b = getattr(ref, k), getattr(host, k)
        if a.dtype == torch.float32:
            a, b = a.view(torch.int32), b.view(torch.int32)
        assert torch.equal(a, b), k


def test_step_host_rejects_device_and_pageable_buffers(cuda):
    import torch
    from minecu import MineEnv
    env = MineEnv(batch_size=8, world_size=8, render_width=8, render_height=8, ground_height=4, device=cuda)
    env.reset()
    rew = torch.zeros(8, dtype=torch.float32).pin_memory()
    done = torch.zeros(8, dtype=torch.bool).pin_memory()
    with pytest.raises(RuntimeError, match="pinned"):
        env.step_host(torch.zeros(8, dtype=torch.uint8), rew, done)
    with pytest.raises(RuntimeError, match="host"):
        env.step_host(torch.zeros(8, dtype=torch.uint8, device=cuda), rew, done)
    with pytest.raises(RuntimeError, match="entries"):
        env.step_host(torch.zeros(9, dtype=torch.uint8).pin_memory(), rew, done)


def test_ragged_step_host_matches_step(cuda):
    """RaggedBatch.step_host against RaggedBatch.step on a twin batch of four
    groups (different worlds, resolutions and episode lengths)."""
    import torch
    from minecu import MineEnv, _C
    from minecu.ragged import RaggedBatch
    groups = [(37, 8, 16, 4, None), (50, 16, 32, 8, 9), (23, 24, 24, 8, None), (19, 32, 64, 8, 6)]

    def make():
        envs = [MineEnv(batch_size=b, world_size=w, render_width=r, render_height=r, ground_height=gh,
                        episode_length=el, obs_dtype="uint8", device=cuda) for b, w, r, gh, el in groups]
        batch = RaggedBatch(envs)
        batch.reset()
        return batch

    ref, host = make(), make()
    total, K = sum(g[0] for g in groups), 19
    acts = torch.empty((K, total), dtype=torch.uint8, device=cuda)
    _C.philox_actions(acts, 0, 0, 5, True)
    h_acts = acts.cpu().pin_memory()
    h_rew = torch.zeros((K, total), dtype=torch.float32).pin_memory()
    h_done = torch.zeros((K, total), dtype=torch.bool).pin_memory()
    want_rew, want_done = [], []
    for s in range(K):
        res = ref.step(acts[s])
        want_rew.append(torch.cat([r.clone() for _, r, _ in res]))
        want_done.append(torch.cat([d.clone().to(torch.bool) for _, _, d in res]))
        host.step_host(h_acts[s], h_rew[s], h_done[s])
    host.join_host()
    torch.cuda.synchronize()
    want_rew = torch.stack(want_rew).cpu()
    want_done = torch.stack(want_done).cpu()
    assert torch.equal(h_rew.view(torch.int32), want_rew.view(torch.int32))
    assert torch.equal(h_done, want_done)
    assert bool(want_done.any()) and bool((want_rew != 0).any())
    for ga, gb in zip(ref.envs, host.envs):
        for k in KEYS:
            a, b = getattr(ga, k), getattr(gb, k)
            if a.dtype == torch.float32:
                a, b = a.view(torch.int32), b.view(torch.int32)
            assert torch.equal(a, b), k
