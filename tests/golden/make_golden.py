"""Generate the golden fixtures of tests/golden/ from the reference itself.

The reference ships no golden vectors or known-answer tests, so these are
made by running the reference's own CUDA build - oracle/_ref/libminecu_ref.so,
its src/kernels.cu compiled unmodified by oracle/Makefile - through
oracle/ref_driver.RefEnv, which issues the reference MineEnv's launch
sequence (minecu/__init__.py:141-466).  It needs a CUDA GPU:

    python tests/golden/make_golden.py [out_dir]     # default: tests/golden

Each case is one .npz (compressed) with:
  config      JSON of the MineEnv arguments and the action stream
  actions     uint8 [K, B] discrete actions (Philox4x32-10, seed, counter (env, step))
  rewards, dones                       [K, B] after every step
  positions, velocities, yaws, pitches, on_ground, step_count   after every step
  obs_steps   the steps whose observation is stored (-1 = after reset())
  obs         [len(obs_steps), B, H, W, 3]
  vox_idx, vox_val   voxels (flat index into [B, Y, X, Z]) that differ, after
                     the last step, from the freshly generated worlds, and their values
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

# name -> (MineEnv arguments, steps, action seed, break_half, steps whose obs is kept)
CASES = {
    "c1_uint8": (dict(batch_size=64, world_size=16, render_width=32, render_height=32, obs_dtype="uint8"),
                 100, 0, False, (-1, 0, 1, 9, 49, 99)),
    "float32_small": (dict(batch_size=16, world_size=16, render_width=24, render_height=20, obs_dtype="float32"),
                      12, 7, False, (-1, 0, 5, 11)),
    "minimal_ep9": (dict(batch_size=24, world_size=16, render_width=32, render_height=32, obs_dtype="uint8_minimal",
                         episode_length=9), 30, 11, True, (-1, 8, 9, 29)),
    "prebasis_full_ep7": (dict(batch_size=24, world_size=16, render_width=32, render_height=32,
                               obs_dtype="uint8_prebasis_full", episode_length=7), 30, 3, True, (-1, 6, 7, 29)),
}
LOOK_DELTA = 0.1


def run_case(name, args, steps, seed, break_half, obs_steps):
    import torch
    import oracle as O
    import ref_driver
    dev = torch.device("cuda", 0)
    env = ref_driver.RefEnv(device=str(dev), target_block=3, **args)
    B = args["batch_size"]
    env.reset()
    world0 = env.voxels.cpu().numpy().copy()
    rec = {k: [] for k in ("rewards", "dones", "positions", "velocities", "yaws", "pitches", "on_ground",
                           "step_count")}
    obs = []
    if -1 in obs_steps:
        obs.append(env.obs_buffer.cpu().numpy().copy())
    acts = np.stack([O.philox_actions(B, s, seed, break_half=break_half) for s in range(steps)])
    for s in range(steps):
        btn, look = O.discrete_to_buttons(acts[s], LOOK_DELTA)
        _, rew, done = env.step(torch.from_numpy(btn).to(dev), torch.from_numpy(look).to(dev))
        torch.cuda.synchronize()
        rec["rewards"].append(rew.cpu().numpy().copy())
        rec["dones"].append(done.cpu().numpy().copy())
        for k in ("positions", "velocities", "yaws", "pitches", "on_ground", "step_count"):
            rec[k].append(getattr(env, k).cpu().numpy().copy())
        if s in obs_steps:
            obs.append(env.obs_buffer.cpu().numpy().copy())
    vox = env.voxels.cpu().numpy()
    diff = np.flatnonzero(vox.ravel() != world0.ravel())
    config = dict(args, steps=steps, seed=seed, break_half=break_half, look_delta=LOOK_DELTA, target_block=3,
                  actions="philox4x32-10 (seed, counter (env, step)), uniform over 11, expanded by the "
                          "discrete adapter")
    out = dict(config=np.array(json.dumps(config)), actions=acts.astype(np.uint8),
               obs_steps=np.array(obs_steps, dtype=np.int32), obs=np.stack(obs),
               vox_idx=diff.astype(np.int64), vox_val=vox.ravel()[diff].astype(np.int8))
    for k, v in rec.items():
        out[k] = np.stack(v)
    return out


def main(out_dir=HERE):
    import ref_driver
    if not ref_driver.available():
        raise SystemExit("oracle/_ref/libminecu_ref.so is not built (make -C oracle)")
    os.makedirs(out_dir, exist_ok=True)
    for name, (args, steps, seed, bh, obs_steps) in CASES.items():
        data = run_case(name, args, steps, seed, bh, obs_steps)
        path = os.path.join(out_dir, f"{name}.npz")
        np.savez_compressed(path, **data)
        print(f"{path}: {os.path.getsize(path)} bytes, {len(data['vox_idx'])} changed voxels, "
              f"{int(data['rewards'].sum())} reward, {int(data['dones'].sum())} dones")


if __name__ == "__main__":
    main(*sys.argv[1:])
