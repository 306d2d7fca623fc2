"""This build against the reference package itself.

`baseline/_ref` holds the reference's `minecu` package built by its own
setup.py (`pip install --target`, see `__graft_entry__.build`): its
`_C` extension and its Python `MineEnv`, unmodified.  A child process (both
packages are named `minecu`) steps the reference's `MineEnv` with the
buttons and looks of seeded discrete actions, through persistent action
buffers as its CUDA graphs require (src/kernels.cu:2526-2542), and saves
every step's rewards and dones and the final state.  This process steps
`MineEnv` of this build (default numerics "ref_fast", default launch
shapes) with the same discrete actions and compares everything bit for bit
(floats as int32 patterns).  Tolerance: none.

Cases: the small plain-method configuration (B=64, 16^3, 32x32 uint8, seed
0, 100 steps), every other observation mode of the reference's baseline
list (uint8_minimal and uint8_prebasis_full with episode limits: resets and
world regeneration inside the window), and a render-dominated shape (32^3
worlds, 64x64, half the actions breaking blocks).
"""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_PKG = os.path.join(ROOT, "baseline", "_ref")

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not os.path.exists(os.path.join(REF_PKG, "minecu", "__init__.py")),
                                 reason="baseline/_ref (the reference package) is not installed")]

STATE = ("voxels", "positions", "velocities", "yaws", "pitches", "on_ground", "step_count", "do_reset",
         "cameras", "rewards", "obs_buffer")

CASES = [
    dict(name="plain_small", B=64, world=16, res=32, obs="uint8", steps=100, seed=0, ep=None, brk=False),
    # float32 without an episode limit: the reference's float32 step graph keeps
    # the first do_reset pointer while MineEnv.step rebinds do_reset every step
    # (minecu/__init__.py:364), so its resets under a limit are stale
    dict(name="float32", B=256, world=16, res=32, obs="float32", steps=40, seed=4, ep=None, brk=False),
    dict(name="minimal_episodes", B=256, world=16, res=32, obs="uint8_minimal", steps=40, seed=5, ep=7, brk=False),
    dict(name="prebasis_full_episodes", B=256, world=16, res=32, obs="uint8_prebasis_full", steps=40, seed=6,
         ep=7, brk=False),
    dict(name="render_break", B=512, world=32, res=64, obs="uint8", steps=30, seed=2, ep=None, brk=True),
]

# The reference side, run with only the reference package (and the numpy
# action stream of oracle/) on sys.path.
CHILD = r"""
import json, sys, numpy as np, torch
sys.path.insert(0, sys.argv[1])
sys.path.insert(1, sys.argv[2])
import minecu
assert minecu.__file__.startswith(sys.argv[1]), minecu.__file__
import oracle as O
cases = json.loads(sys.argv[3])
out = {}
dev = torch.device("cuda", 0)
for c in cases:
    env = minecu.MineEnv(batch_size=c["B"], world_size=c["world"], render_width=c["res"], render_height=c["res"],
                         device="cuda:0", obs_dtype=c["obs"], episode_length=c["ep"], target_block=3)
    pb = torch.zeros((c["B"], 8), dtype=torch.int8, device=dev)
    pl = torch.zeros((c["B"], 2), dtype=torch.float32, device=dev)
    env.reset()
    rew, done = [], []
    for s in range(c["steps"]):
        b, l = O.discrete_to_buttons(O.philox_actions(c["B"], s, c["seed"], break_half=c["brk"]), 0.1)
        pb.copy_(torch.from_numpy(b))
        pl.copy_(torch.from_numpy(l))
        _, r, d = env.step(pb, pl)
        rew.append(r.cpu().numpy().copy())
        done.append(d.cpu().numpy().copy())
    n = c["name"]
    out[n + "/step_rewards"] = np.stack(rew)
    out[n + "/step_dones"] = np.stack(done)
    for k in %(state)r:
        out[n + "/" + k] = getattr(env, k).cpu().numpy()
np.savez(sys.argv[4], **out)
print("CHILD OK")
""" % {"state": STATE}


@pytest.fixture(scope="module")
def reference_states(tmp_path_factory):
    path = str(tmp_path_factory.mktemp("stock") / "states.npz")
    r = subprocess.run([sys.executable, "-c", CHILD, REF_PKG, os.path.join(ROOT, "oracle"), json.dumps(CASES), path],
                       capture_output=True, text=True, timeout=900)
    assert r.returncode == 0 and "CHILD OK" in r.stdout, r.stderr[-3000:]
    return dict(np.load(path))


def _bits(a):
    return a.view(np.int32) if a.dtype == np.float32 else a


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_mineenv_equals_reference_package(cuda, reference_states, case):
    import torch
    import oracle as O
    from minecu import MineEnv
    c = case
    env = MineEnv(batch_size=c["B"], world_size=c["world"], render_width=c["res"], render_height=c["res"],
                  device=cuda, obs_dtype=c["obs"], episode_length=c["ep"], look_delta=0.1)
    env.reset()
    ref = {k.split("/", 1)[1]: v for k, v in reference_states.items() if k.startswith(c["name"] + "/")}
    for s in range(c["steps"]):
        a = torch.from_numpy(O.philox_actions(c["B"], s, c["seed"], break_half=c["brk"])).to(cuda)
        _, r, d = env.step(a)
        assert np.array_equal(_bits(r.cpu().numpy()), _bits(ref["step_rewards"][s])), f"rewards differ at step {s}"
        assert np.array_equal(d.cpu().numpy(), ref["step_dones"][s]), f"dones differ at step {s}"
    env.check_error()
    if c["ep"] is not None:
        assert ref["step_dones"].any(), "the window should hold episode ends"
    for k in STATE:
        mine = getattr(env, k).cpu().numpy()
        assert mine.shape == ref[k].shape and mine.dtype == ref[k].dtype, k
        diff = int((_bits(mine) != _bits(ref[k])).sum())
        assert diff == 0, f"{k}: {diff} of {mine.size} elements differ"
