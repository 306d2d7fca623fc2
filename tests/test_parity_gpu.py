"""Parity of the CUDA path (called through the C-ABI) with the oracles.

* "ieee" numerics  vs the CPU oracle (oracle/mc_oracle.c): bit-exact, every
  state field, every observation byte, the world grids, and the debug
  outputs (interaction voxel index per env, hit block/face per pixel).
* "ref_fast" numerics vs the reference's own CUDA build (oracle/_ref, run
  through its launchers in MineEnv's order): bit-exact.
* plain form vs fused form, and staged vs unstaged worlds: bit-exact.
Tolerance: none.  Every comparison below is bitwise (floats compared as
their int32 bit patterns).
"""
import numpy as np
import pytest

from minecu import capi
import oracle as O
from mc_harness import GpuEnv, actions_for, diff_report, oracle_state

pytestmark = pytest.mark.gpu

PLAIN, FUSED = capi.FORM_PLAIN, capi.FORM_FUSED


def run_vs_oracle(cuda, steps, seed, form, obs_dtype="uint8", B=64, world=16, res=(32, 32), stage=None,
                  break_half=False, look_delta=0.1, episode_length=None, world_xyz=None, reset_every=None,
                  fused_cfg=None, debug=True, regen="all", **kw):
    wx, wy, wz = world_xyz or (world, world, world)
    g = GpuEnv(cuda, B, world_x=wx, world_y=wy, world_z=wz, render_width=res[0], render_height=res[1],
               obs_dtype=obs_dtype, numerics="ieee", look_delta=look_delta, episode_length=episode_length,
               debug=debug, **kw)
    if stage is not None:
        g.set_fused(stage)
    if fused_cfg is not None:
        g.set_fused(*fused_cfg)
    if regen != "all":
        g.set_regen(True)
    o = O.OracleEnv(batch_size=B, world_x=wx, world_y=wy, world_z=wz, render_width=res[0], render_height=res[1],
                    obs_dtype=obs_dtype, debug=True, episode_length=episode_length, regen=regen, **kw)
    g.reset()
    o.reset()
    d = diff_report(g.state(), oracle_state(o), ["voxels", "positions", "obs", "cameras", "do_reset", "step_count"])
    assert not d, f"after reset: {d}"
    rng = np.random.default_rng(seed)
    for s in range(steps):
        if reset_every and s and s % reset_every == 0:
            mask = rng.random(B) < 0.3
            g.reset(mask)
            o.reset(mask)
        _, btn, look = actions_for(B, s, seed, look_delta, break_half)
        # exercise place and sprint too, which the discrete table never sets
        btn[:, 6] = (rng.random(B) < 0.1).astype(np.int8)
        btn[:, 7] = (rng.random(B) < 0.3).astype(np.int8)
        g.step(btn, look, form)
        o.step(btn, look)
        d = diff_report(g.state(), oracle_state(o))
        assert not d, f"step {s}: differing elements {d}"
    g.check_error()
    g.close()


@pytest.mark.parametrize("form", [PLAIN, FUSED])
def test_c1_uint8_ieee_bit_exact(cuda, form):
    """Config 1: B=64, 16^3, 32x32 uint8, 100 steps, seed 0."""
    run_vs_oracle(cuda, 100, 0, form)


@pytest.mark.parametrize("stage", [0, 1, 2])
def test_fused_staged_and_direct_bit_exact(cuda, stage):
    run_vs_oracle(cuda, 40, 5, FUSED, stage=stage, B=40)


@pytest.mark.parametrize("mode", ["float32", "uint8_minimal", "uint8_fp16", "uint8_prebasis", "uint8_smem",
                                  "uint8_fast"])
@pytest.mark.parametrize("form", [PLAIN, FUSED])
def test_modes_ieee_bit_exact(cuda, mode, form):
    run_vs_oracle(cuda, 30, 11, form, obs_dtype=mode, B=37, res=(24, 20))


@pytest.mark.parametrize("form", [PLAIN, FUSED])
def test_prebasis_full_episodes_bit_exact(cuda, form):
    """Kernel-side episode rule and the all-world regeneration."""
    run_vs_oracle(cuda, 40, 3, form, obs_dtype="uint8_prebasis_full", B=33, episode_length=7, break_half=True)


@pytest.mark.parametrize("form", [PLAIN, FUSED])
def test_episode_length_and_masked_reset(cuda, form):
    run_vs_oracle(cuda, 45, 4, form, B=50, episode_length=9, reset_every=13, break_half=True)


@pytest.mark.parametrize("form", [PLAIN, FUSED])
def test_w32_render_dominated_bit_exact(cuda, form):
    """Config 3 shape, reduced: 32^3 world, 64x64, half the actions break."""
    run_vs_oracle(cuda, 12, 2, form, B=24, world=32, res=(64, 64), break_half=True)


@pytest.mark.parametrize("form", [PLAIN, FUSED])
def test_small_and_odd_sizes(cuda, form):
    """8^3 world (the camera spawns above the world), 7x5 image (3-byte rows
    not 16-byte aligned), one env."""
    run_vs_oracle(cuda, 25, 6, form, B=1, world=8, res=(7, 5))
    run_vs_oracle(cuda, 25, 7, form, B=3, world=5, res=(16, 16), obs_dtype="float32")


@pytest.mark.parametrize("mode", ["uint8", "uint8_prebasis"])
def test_noncubic_world_bit_exact(cuda, mode):
    run_vs_oracle(cuda, 25, 8, FUSED, obs_dtype=mode, B=17, world_xyz=(24, 16, 20), res=(16, 16))


# Shapes for the march without debug outputs (kwargs of run_vs_oracle).
EARLY_EXIT_CASES = {
    "c1": dict(steps=30, seed=0, B=40),
    "one_env_8cube_7x5": dict(steps=25, seed=6, B=1, world=8, res=(7, 5)),
    "world5_f32": dict(steps=25, seed=7, B=3, world=5, res=(16, 16), obs_dtype="float32"),
    "noncubic": dict(steps=25, seed=8, B=17, world_xyz=(24, 16, 20), res=(16, 16)),
    "w32_64x64_break": dict(steps=12, seed=2, B=24, world=32, res=(64, 64), break_half=True),
    "steps3_vd2.5": dict(steps=10, seed=9, B=9, max_steps=3, view_distance=2.5),
    "steps20_vd6": dict(steps=15, seed=10, B=30, max_steps=20, view_distance=6.0),
    "episodes_masked_reset": dict(steps=45, seed=4, B=50, episode_length=9, reset_every=13, break_half=True),
    "wide_flat_32x8x32": dict(steps=20, seed=12, B=21, world_xyz=(32, 8, 32), res=(8, 8), ground_height=4,
                              break_half=True),
}


@pytest.mark.parametrize("case", sorted(EARLY_EXIT_CASES))
@pytest.mark.parametrize("mode", ["uint8", "uint8_minimal"])
@pytest.mark.parametrize("cfg", [(1, 8, 4, 4, 1, 0), (1, 8, 3, 8, 4, 1), (2, 8, 2, 8, 4, 1), (2, 8, 4, 4, 1, 0)],
                         ids=["per_warp", "team", "team_depth2", "per_warp_depth2"])
def test_early_exit_march_vs_oracle(cuda, case, mode, cfg):
    """The fused kernels without debug outputs, where the march over a
    staged world ends rays early (left the box, above the highest solid
    layer, view distance tested at the hit) in PTX loops, against the CPU
    oracle: bit-exact on every state field and observation byte."""
    kw = dict(EARLY_EXIT_CASES[case])
    kw.setdefault("obs_dtype", mode)
    wx, wy, wz = kw.get("world_xyz") or (kw.get("world", 16),) * 3
    if (wx * wy * wz) % 16:
        cfg = (0,) + tuple(cfg[1:])  # a bulk copy needs whole 16-byte chunks: march the global world
    elif cfg[4] == 1 and wx * wy * wz > 16384:
        cfg = (1, 4, 1, 4, 1, 0)  # one 32 KB world per warp: 4 warps fit in a CTA's shared memory
    run_vs_oracle(cuda, kw.pop("steps"), kw.pop("seed"), FUSED, fused_cfg=cfg, debug=False, **kw)


@pytest.mark.parametrize("form", [PLAIN, FUSED])
@pytest.mark.parametrize("debug", [True, False])
def test_per_env_regen_vs_oracle(cuda, form, debug):
    """Opt-in per-env regeneration (MC_REGEN_PER_ENV): with short episodes,
    masked resets and half the actions breaking blocks, only the worlds of
    the envs done or reset return to the start world; every other world
    keeps its broken blocks.  Bit-exact against the oracle's per-env rule."""
    run_vs_oracle(cuda, 45, 14, form, B=50, episode_length=9, reset_every=13, break_half=True, regen="per_env",
                  debug=debug)


@pytest.mark.parametrize("cfg", [(1, 8, 4, 4, 1, 0), (1, 8, 3, 8, 4, 1)], ids=["per_warp", "team"])
def test_per_env_regen_fused_configs(cuda, cfg):
    run_vs_oracle(cuda, 30, 15, FUSED, B=33, episode_length=7, break_half=True, regen="per_env", debug=False,
                  fused_cfg=cfg)


@pytest.mark.parametrize("mode", ["uint8", "uint8_minimal"])
@pytest.mark.parametrize("cfg", [(1, 8, 4, 4, 1, 0), (1, 8, 3, 8, 4, 1)], ids=["per_warp", "team"])
def test_wide_flat_world_staged(cuda, mode, cfg):
    """A 32x8x32 world (1 KB layers) with 8x8 images, staged: the march
    loads one voxel past the box before its exit test, and the layouts keep
    one world layer allocated in front of the first staged world and after
    the last; here the tables and bands in front of the first world are
    shorter than a layer, so both layouts add that room."""
    run_vs_oracle(cuda, 20, 12, FUSED, obs_dtype=mode, B=21, world_xyz=(32, 8, 32), res=(8, 8), ground_height=4,
                  break_half=True, fused_cfg=cfg)


def test_limits_max_steps_and_view_distance(cuda):
    run_vs_oracle(cuda, 10, 9, FUSED, B=9, max_steps=0)
    run_vs_oracle(cuda, 10, 9, FUSED, B=9, max_steps=3, view_distance=2.5)
    run_vs_oracle(cuda, 10, 9, PLAIN, B=9, view_distance=0.0)
    run_vs_oracle(cuda, 10, 9, FUSED, B=9, target_block=-1, reward_value=2.5)


@pytest.mark.parametrize("mode", ["uint8", "float32", "uint8_minimal", "uint8_prebasis_full"])
def test_ref_fast_fused_equals_plain(cuda, mode):
    B = 200
    kw = dict(episode_length=17) if mode == "uint8_prebasis_full" else {}
    a = GpuEnv(cuda, B, obs_dtype=mode, numerics="ref_fast", **kw)
    b = GpuEnv(cuda, B, obs_dtype=mode, numerics="ref_fast", **kw)
    a.reset()
    b.reset()
    for s in range(40):
        _, btn, look = actions_for(B, s, 21, break_half=(s % 2 == 0))
        a.step(btn, look, PLAIN)
        b.step(btn, look, FUSED)
        d = diff_report(a.state(), b.state())
        assert not d, f"step {s}: {d}"


def test_rollout_graph_equals_single_steps(cuda):
    import torch
    B, K = 300, 12
    a = GpuEnv(cuda, B, numerics="ref_fast", episode_length=5)
    b = GpuEnv(cuda, B, numerics="ref_fast", episode_length=5)
    a.reset()
    b.reset()
    acts = np.stack([actions_for(B, s, 31)[0] for s in range(K)])
    dev_acts = torch.from_numpy(acts).to(cuda)
    rew = torch.zeros((K, B), dtype=torch.float32, device=cuda)
    dones = torch.zeros((K, B), dtype=torch.bool, device=cuda)
    for _ in range(2):  # second call replays the cached graph
        capi.check(capi.lib().mc_env_rollout(a.h, dev_acts.data_ptr(), K, rew.data_ptr(), dones.data_ptr(), None))
        torch.cuda.synchronize()
        for s in range(K):
            b.step_discrete(acts[s], FUSED)
            assert np.array_equal(rew[s].cpu().numpy(), b.state()["rewards"])
            assert np.array_equal(dones[s].cpu().numpy().astype(np.uint8), b.state()["do_reset"])
        d = diff_report(a.state(), b.state())
        assert not d, d


def test_full_size_sampled_envs_bit_exact(cuda):
    """Config 2 shape (B=32768, 16^3, 32x32): every env is independent when
    no episode limit is set, so a sample of envs is checked against the
    oracle started from the GPU's own state."""
    B = 32768
    g = GpuEnv(cuda, B, numerics="ieee", debug=False)
    g.reset()
    rng = np.random.default_rng(1)
    sample = np.sort(rng.choice(B, 96, replace=False))
    for s in range(6):
        _, btn, look = actions_for(B, s, 1)
        before = g.state()
        g.step(btn, look, FUSED)
        after = g.state()
        o = O.OracleEnv(batch_size=len(sample), world_size=16, render_width=32, render_height=32, obs_dtype="uint8")
        for k in ("voxels", "positions", "velocities", "yaws", "pitches", "on_ground", "step_count"):
            getattr(o, k)[...] = before[k][sample]
        o.step(btn[sample], look[sample])
        sub = {k: v[sample] for k, v in after.items()}
        d = diff_report(sub, oracle_state(o), ["voxels", "positions", "velocities", "yaws", "pitches", "obs",
                                              "rewards", "cameras"])
        assert not d, f"step {s}: {d}"


# ---------------------------------------------------------------------------
# ref_fast numerics vs the reference's own CUDA build
# ---------------------------------------------------------------------------
ref_driver = pytest.importorskip("ref_driver")


def _ref_available():
    return ref_driver.available()


@pytest.mark.skipif(not _ref_available(), reason="oracle/_ref/libminecu_ref.so not built")
@pytest.mark.parametrize("mode", ["uint8", "float32", "uint8_minimal", "uint8_fp16", "uint8_prebasis",
                                  "uint8_prebasis_full", "uint8_fast"])
@pytest.mark.parametrize("form", [PLAIN, FUSED])
def test_ref_fast_vs_reference_build(cuda, mode, form):
    import torch
    B, steps = 64, 60
    kw = dict(episode_length=23) if mode in ("uint8", "uint8_prebasis_full") else {}
    ref = ref_driver.RefEnv(batch_size=B, world_size=16, render_width=32, render_height=32, obs_dtype=mode,
                            target_block=3, **kw)
    g = GpuEnv(cuda, B, obs_dtype=mode, numerics="ref_fast", debug=False, **kw)
    ref.reset()
    g.reset()
    torch.cuda.synchronize()

    def ref_state():
        s = dict(voxels=ref.voxels, positions=ref.positions, velocities=ref.velocities, yaws=ref.yaws,
                 pitches=ref.pitches, on_ground=ref.on_ground, step_count=ref.step_count, do_reset=ref.do_reset,
                 cameras=ref.cameras, obs=ref.obs_buffer, rewards=ref.rewards)
        out = {}
        for k, v in s.items():
            a = v.cpu().numpy()
            out[k] = a.astype(np.uint8) if a.dtype == np.bool_ else a
        return out

    d = diff_report(g.state(), ref_state())
    assert not d, f"after reset: {d}"
    rng = np.random.default_rng(12)
    for s in range(steps):
        _, btn, look = actions_for(B, s, 40, break_half=(s % 3 == 0))
        btn[:, 6] = (rng.random(B) < 0.1).astype(np.int8)
        btn[:, 7] = (rng.random(B) < 0.3).astype(np.int8)
        ref.step(torch.from_numpy(btn).to(cuda), torch.from_numpy(look).to(cuda))
        g.step(btn, look, form)
        torch.cuda.synchronize()
        d = diff_report(g.state(), ref_state())
        assert not d, f"step {s}: differing elements {d}"
