"""Loading and replaying the golden fixtures of tests/golden/ (made from the
reference's own CUDA build by tests/golden/make_golden.py)."""
import glob
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FIELDS = ("positions", "velocities", "yaws", "pitches", "on_ground", "step_count", "rewards", "dones")


def fixtures():
    return sorted(glob.glob(os.path.join(GOLDEN, "*.npz")))


def load(path):
    d = dict(np.load(path, allow_pickle=False))
    d["config"] = json.loads(str(d["config"]))
    return d


def env_args(cfg):
    keys = ("batch_size", "world_size", "render_width", "render_height", "obs_dtype", "episode_length")
    return {k: cfg[k] for k in keys if k in cfg}


def compare(fx, s, state):
    """Differences between the fixture after step s and `state` (arrays by
    fixture field name): {field: number of differing elements}, floats
    compared as their bit patterns."""
    out = {}
    for k in FIELDS:
        a, b = fx[k][s], state[k]
        if a.dtype.kind == "f":
            a, b = a.view(np.int32), np.ascontiguousarray(b, dtype=np.float32).view(np.int32)
        n = int(np.count_nonzero(a.astype(np.int64) != b.astype(np.int64)))
        if n:
            out[k] = n
    return out
