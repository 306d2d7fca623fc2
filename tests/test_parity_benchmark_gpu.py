"""ref_fast numerics against the reference's own CUDA build at the sizes the
benchmark measures, in the launch shapes and code paths it times.

* peak shape: B=32768, 16^3, 32x32 uint8, discrete actions from seed 1 (the
  benchmark's), stepped through `MineEnv.rollout` (the K-step CUDA graph of
  the per-warp fused kernel): every step of 0..30, the whole window 31..699
  as one 669-step graph (rewards and dones of every step, the full state at
  its end), then every step of the late window 700..709;
* render-dominated: B=4096, 32^3, 64x64, half the actions breaking blocks
  (seed 2), 60 steps in the default team launch (cooperative teams over
  staged 32 KB worlds);
* ragged: the six groups of the ragged workload in one persistent launch
  (default and autotuned shapes) against six reference envs;
* big images at a batch that gives every resident warp two envs (B=9472,
  16^3, 64x64), where the default is one warp per env.

The reference side is oracle/_ref/libminecu_ref.so (the reference's
src/kernels.cu compiled unmodified) driven in MineEnv's order by
oracle/ref_driver.py.  Tolerance: none; floats are compared as int32 bit
patterns, on the device.
"""
import pytest

ref_driver = pytest.importorskip("ref_driver")

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref_driver.available(), reason="oracle/_ref/libminecu_ref.so not built")]

# MineEnv attribute -> RefEnv attribute
FIELDS = {"voxels": "voxels", "positions": "positions", "velocities": "velocities", "yaws": "yaws",
          "pitches": "pitches", "on_ground": "on_ground", "step_count": "step_count", "do_reset": "do_reset",
          "cameras": "cameras", "obs_buffer": "obs_buffer", "rewards": "rewards"}


def _bits(torch, t):
    return t.view(torch.int32) if t.dtype == torch.float32 else t


def _same(torch, a, b, what):
    a, b = _bits(torch, a), _bits(torch, b)
    if not torch.equal(a, b):
        n = int((a != b).sum())
        raise AssertionError(f"{what}: {n} of {a.numel()} elements differ")


def _assert_env_equal(torch, env, ref, what):
    for mine, theirs in FIELDS.items():
        _same(torch, getattr(env, mine), getattr(ref, theirs), f"{what}: {mine}")


class _Buttons:
    """Device buttons/look of discrete actions (the workload's adapter, look
    step 0.1 rad), in persistent buffers."""

    def __init__(self, torch, B, dev):
        from minecu import _C
        self._C = _C
        self.btn = torch.empty((B, 8), dtype=torch.int8, device=dev)
        self.look = torch.empty((B, 2), dtype=torch.float32, device=dev)

    def __call__(self, actions):
        self._C.discrete_to_buttons(actions, 0.1, self.btn, self.look)
        return self.btn, self.look


def test_peak_shape_full_batch_vs_reference_build(cuda):
    import torch
    from minecu import MineEnv, _C
    B, seed = 32768, 1
    env = MineEnv(batch_size=B, world_size=16, render_width=32, render_height=32, obs_dtype="uint8", device=cuda)
    cfg = env.launch_config()
    assert (cfg["stage"], cfg["team_warps"], cfg["coop"]) == (1, 1, 0), cfg  # the benchmarked per-warp kernel
    ref = ref_driver.RefEnv(batch_size=B, world_size=16, render_width=32, render_height=32, obs_dtype="uint8",
                            device=cuda, target_block=3)
    env.reset()
    ref.reset()
    torch.cuda.synchronize()
    _assert_env_equal(torch, env, ref, "after reset")
    steps = 710
    acts = torch.empty((steps, B), dtype=torch.uint8, device=cuda)
    _C.philox_actions(acts, 0, 0, seed)
    to_btn = _Buttons(torch, B, cuda)
    a1 = torch.empty((1, B), dtype=torch.uint8, device=cuda)
    r1 = torch.empty((1, B), dtype=torch.float32, device=cuda)
    d1 = torch.empty((1, B), dtype=torch.bool, device=cuda)

    def one_step(s):
        a1.copy_(acts[s:s + 1])
        env.rollout(a1, r1, d1)
        ref.step(*to_btn(acts[s]))
        torch.cuda.synchronize()
        _assert_env_equal(torch, env, ref, f"step {s}")
        _same(torch, r1[0], ref.rewards, f"step {s}: rollout rewards")
        _same(torch, d1[0], ref.do_reset, f"step {s}: rollout dones")

    for s in range(31):
        one_step(s)
    # one 669-step graph, as the benchmark replays its window
    s0, s1 = 31, 700
    rk = torch.empty((s1 - s0, B), dtype=torch.float32, device=cuda)
    dk = torch.empty((s1 - s0, B), dtype=torch.bool, device=cuda)
    env.rollout(acts[s0:s1].contiguous(), rk, dk)
    ref_r = torch.empty_like(rk)
    ref_d = torch.empty_like(dk)
    for s in range(s0, s1):
        ref.step(*to_btn(acts[s]))
        ref_r[s - s0].copy_(ref.rewards)
        ref_d[s - s0].copy_(ref.do_reset)
    torch.cuda.synchronize()
    _same(torch, rk, ref_r, f"rewards of steps {s0}..{s1 - 1}")
    _same(torch, dk, ref_d, f"dones of steps {s0}..{s1 - 1}")
    _assert_env_equal(torch, env, ref, f"after step {s1 - 1}")
    assert int((ref_r != 0).sum()) > 0, "no block broken in the window: the test would not see the interaction"
    for s in range(s1, steps):
        one_step(s)
    env.check_error()


def test_render_dominated_vs_reference_build(cuda):
    import torch
    from minecu import MineEnv, _C
    B, seed, steps = 4096, 2, 60
    env = MineEnv(batch_size=B, world_size=32, render_width=64, render_height=64, obs_dtype="uint8", device=cuda)
    cfg = env.launch_config()
    assert (cfg["stage"], cfg["coop"]) == (1, 1), cfg  # teams over staged worlds, as benchmarked
    ref = ref_driver.RefEnv(batch_size=B, world_size=32, render_width=64, render_height=64, obs_dtype="uint8",
                            device=cuda, target_block=3)
    env.reset()
    ref.reset()
    acts = torch.empty((steps, B), dtype=torch.uint8, device=cuda)
    _C.philox_actions(acts, 0, 0, seed, True)  # half the actions break blocks
    to_btn = _Buttons(torch, B, cuda)
    a1 = torch.empty((1, B), dtype=torch.uint8, device=cuda)
    changed = 0
    for s in range(steps):
        a1.copy_(acts[s:s + 1])
        env.rollout(a1)
        ref.step(*to_btn(acts[s]))
        torch.cuda.synchronize()
        _assert_env_equal(torch, env, ref, f"step {s}")
        changed += int((ref.rewards != 0).sum())
    assert changed > 0
    env.check_error()


RAGGED_GROUPS = [(8192, 8, 16), (6144, 16, 32), (4096, 16, 64), (3072, 24, 32), (2048, 32, 32), (1024, 32, 64)]


@pytest.mark.parametrize("shape", ["default", "autotuned"])
def test_ragged_workload_vs_reference_build(cuda, shape):
    import torch
    from minecu import MineEnv, _C, autotune
    from minecu.ragged import RaggedBatch
    ground = lambda w: min(8, w // 2)  # noqa: E731  (the ragged workload's ground heights)
    envs = [MineEnv(batch_size=b, world_size=w, render_width=r, render_height=r, ground_height=ground(w),
                    obs_dtype="uint8", device=cuda) for b, w, r in RAGGED_GROUPS]
    batch = RaggedBatch(envs)
    if shape == "autotuned":
        autotune.tune_ragged(batch, steps=8, warm_steps=20, use_cache=False, rounds=1)
    refs = [ref_driver.RefEnv(batch_size=b, world_size=w, render_width=r, render_height=r, ground_height=ground(w),
                              obs_dtype="uint8", device=cuda, target_block=3) for b, w, r in RAGGED_GROUPS]
    batch.reset()
    for r in refs:
        r.reset()
    steps = 30
    acts = torch.empty((steps, batch.total), dtype=torch.uint8, device=cuda)
    _C.philox_actions(acts, 0, 0, 3)
    to_btn = [_Buttons(torch, b, cuda) for b, _, _ in RAGGED_GROUPS]
    for s in range(steps):
        batch.step(acts[s])
        for g, r in enumerate(refs):
            r.step(*to_btn[g](acts[s, batch.group_slice(g)].contiguous()))
        torch.cuda.synchronize()
        for g, (e, r) in enumerate(zip(envs, refs)):
            _assert_env_equal(torch, e, r, f"{shape} step {s} group {g}")
    batch.check_error()


def test_big_images_one_warp_per_env_vs_reference_build(cuda):
    """16^3 worlds with 64x64 images at B=9472 = 2 x 148 SMs x 32 warps: the
    default launch is one warp per env (staged worlds, 64-pixel bands)."""
    import torch
    from minecu import MineEnv, _C
    B, steps = 9472, 20
    env = MineEnv(batch_size=B, world_size=16, render_width=64, render_height=64, obs_dtype="uint8", device=cuda)
    props = torch.cuda.get_device_properties(cuda)
    if B >= 2 * props.multi_processor_count * 32:
        cfg = env.launch_config()
        assert (cfg["team_warps"], cfg["coop"], cfg["stage"]) == (1, 0, 1), cfg
    ref = ref_driver.RefEnv(batch_size=B, world_size=16, render_width=64, render_height=64, obs_dtype="uint8",
                            device=cuda, target_block=3)
    env.reset()
    ref.reset()
    acts = torch.empty((steps, B), dtype=torch.uint8, device=cuda)
    _C.philox_actions(acts, 0, 0, 4, True)
    to_btn = _Buttons(torch, B, cuda)
    for s in range(steps):
        env.step(acts[s])
        ref.step(*to_btn(acts[s]))
        torch.cuda.synchronize()
        _assert_env_equal(torch, env, ref, f"step {s}")
    env.check_error()
