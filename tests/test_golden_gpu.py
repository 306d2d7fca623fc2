"""The CUDA path against the golden fixtures recorded from the reference's
own CUDA build (tests/golden/*.npz, made by tests/golden/make_golden.py).

ref_fast numerics, fused and plain forms: every recorded field after every
step (agent state, step counters, rewards, dones), the observations at the
recorded steps and the changed voxels at the end must equal the reference's
bit for bit (floats compared as int32 patterns; tolerance none).
"""
import os

import numpy as np
import pytest

import golden_cases as GC

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("form", ["fused", "plain"])
@pytest.mark.parametrize("path", GC.fixtures(), ids=[os.path.basename(p)[:-4] for p in GC.fixtures()])
def test_cuda_path_equals_reference_fixture(cuda, path, form):
    import torch
    from minecu import MineEnv
    fx = GC.load(path)
    cfg = fx["config"]
    env = MineEnv(device=cuda, numerics="ref_fast", form=form, look_delta=cfg["look_delta"],
                  target_block=cfg["target_block"], **GC.env_args(cfg))
    world0 = env.voxels.clone()
    env.reset()
    k = 0
    steps = list(fx["obs_steps"])
    if steps[0] == -1:
        assert np.array_equal(env.obs_buffer.cpu().numpy(), fx["obs"][0]), "obs after reset"
        k = 1
    for s in range(fx["actions"].shape[0]):
        _, rew, done = env.step(torch.from_numpy(fx["actions"][s]).to(cuda))
        state = {f: getattr(env, f).cpu().numpy() for f in GC.FIELDS if f not in ("rewards", "dones")}
        state["rewards"] = rew.cpu().numpy()
        state["dones"] = done.cpu().numpy()
        d = GC.compare(fx, s, state)
        assert not d, f"step {s}: {d}"
        if s in steps:
            assert np.array_equal(env.obs_buffer.cpu().numpy(), fx["obs"][k]), f"obs after step {s}"
            k += 1
    vox = env.voxels.cpu().numpy().ravel()
    diff = np.flatnonzero(vox != world0.cpu().numpy().ravel())
    assert np.array_equal(diff, fx["vox_idx"]) and np.array_equal(vox[diff], fx["vox_val"])
