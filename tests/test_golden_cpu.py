"""The CPU oracle (oracle/mc_oracle.c, IEEE numerics) against the golden
fixtures recorded from the reference's own CUDA build (tests/golden/*.npz).

The reference build computes with fast-math intrinsics (approximate
sin/cos, division and square root, contracted multiply-adds); the oracle with
correctly rounded IEEE operations.  Pinned here, per step of every fixture:
  exact:      rewards, dones, step counts, on_ground, yaw, pitch, every
              changed voxel at the end, uint8 observations
  positions:  within 8 ulp (the two arithmetics drift by about an ulp per
              landing or collision; 6 ulp is the largest seen over C1's 100 steps)
  velocities: within 1e-6 absolute (a landing can leave -1.5e-8 against 0.0)
  float32 observations: within 1e-6 absolute
The GPU path is pinned to the same fixtures bit for bit in test_golden_gpu.py.
"""
import numpy as np
import pytest

import golden_cases as GC
import oracle as O

POS_ULP = 8
VEL_ABS = 1e-6
OBS_F32_ABS = 1e-6


def test_fixtures_present_and_well_formed():
    paths = GC.fixtures()
    assert len(paths) >= 4
    for p in paths:
        fx = GC.load(p)
        K, B = fx["actions"].shape
        assert fx["config"]["batch_size"] == B and fx["config"]["steps"] == K
        for f in GC.FIELDS:
            assert fx[f].shape[:2] == (K, B), f
        assert fx["obs"].shape[0] == len(fx["obs_steps"])
        assert fx["actions"].max() <= 10


@pytest.mark.parametrize("path", GC.fixtures(), ids=[p.split("/")[-1][:-4] for p in GC.fixtures()])
def test_oracle_matches_reference_fixture(path):
    fx = GC.load(path)
    cfg = fx["config"]
    a = GC.env_args(cfg)
    env = O.OracleEnv(batch_size=a["batch_size"], world_size=a["world_size"], render_width=a["render_width"],
                      render_height=a["render_height"], obs_dtype=a["obs_dtype"],
                      episode_length=a.get("episode_length"), target_block=cfg["target_block"])
    world0 = env.voxels.copy()
    env.reset()
    k = 0

    def check_obs(what):
        ref = fx["obs"][k]
        if ref.dtype == np.uint8:
            assert np.array_equal(env.obs, ref), what
        else:
            assert np.abs(env.obs - ref).max() <= OBS_F32_ABS, what

    if fx["obs_steps"][0] == -1:
        check_obs("obs after reset")
        k = 1
    for s in range(fx["actions"].shape[0]):
        btn, look = O.discrete_to_buttons(fx["actions"][s], cfg["look_delta"])
        env.step(btn, look)
        for f, mine in (("rewards", env.rewards), ("dones", env.do_reset), ("step_count", env.step_count),
                        ("on_ground", env.on_ground), ("yaws", env.yaws), ("pitches", env.pitches)):
            ref = fx[f][s]
            if ref.dtype == np.float32:
                assert np.array_equal(mine.view(np.int32), ref.view(np.int32)), f"step {s}: {f}"
            else:
                assert np.array_equal(mine.astype(ref.dtype), ref), f"step {s}: {f}"
        ulp = np.abs(env.positions.view(np.int32).astype(np.int64) - fx["positions"][s].view(np.int32).astype(np.int64))
        assert ulp.max() <= POS_ULP, f"step {s}: positions differ by {ulp.max()} ulp"
        assert np.abs(env.velocities - fx["velocities"][s]).max() <= VEL_ABS, f"step {s}: velocities"
        if s in fx["obs_steps"]:
            check_obs(f"obs after step {s}")
            k += 1
    vox = env.voxels.ravel()
    diff = np.flatnonzero(vox != world0.ravel())
    assert np.array_equal(diff, fx["vox_idx"]) and np.array_equal(vox[diff], fx["vox_val"])
