"""Rays going up end early once they pass the bounds of their quadrant's
solid voxels (the per-env scan of the staged world, staged_up_bounds).

Random scenes: sparse blocks of every kind above a solid ground, eyes
anywhere in the open (above and below the blocks, next to the box's faces),
every yaw and a wide range of pitches, stepped through both fused kernels
(per-warp, and cooperative teams of 2, 4 and 8 warps that share the scan;
staging depth 1 and 2) without debug outputs, so that the common-case loop
runs.  World shapes cover rows of 16 and 32 bytes (32-bit masks), 48 bytes
(64-bit masks) and 20 bytes (no scan: the top layer only).  Compared with
the CPU oracle bit for bit: every state field and observation byte.
"""
import zlib

import numpy as np
import pytest

from minecu import capi
import oracle as O
from mc_harness import GpuEnv, diff_report, oracle_state

pytestmark = pytest.mark.gpu

FUSED = capi.FORM_FUSED

SHAPES = {
    "16cube": (16, 16, 16),
    "32cube": (32, 32, 32),
    "24x16x48": (24, 16, 48),
    "16x20x32": (16, 20, 32),
    "24x16x20": (24, 16, 20),
}
CFGS = {
    "per_warp": (1, 8, 4, 4, 1, 0),
    "team": (1, 8, 3, 8, 4, 1),
    # the team's warps share the scan (team_up_bounds): teams of 2 and 8 too
    "team2": (1, 8, 3, 8, 2, 1),
    "team8": (1, 8, 2, 16, 8, 1),
    "team_depth2": (2, 8, 2, 8, 4, 1),
    "per_warp_depth2": (2, 8, 4, 4, 1, 0),
}


def random_scene(rng, B, wx, wy, wz, gh, density):
    """Worlds [B, y, x, z]: a solid ground below gh and random blocks above
    it; agents whose eye voxel (position + 1.6 in y) holds air."""
    vox = np.full((B, wy, wx, wz), -1, np.int8)
    vox[:, :gh] = rng.integers(0, 13, size=(B, gh, wx, wz), dtype=np.int8)
    above = rng.random((B, wy - gh, wx, wz)) < density
    vox[:, gh:][above] = rng.integers(0, 13, size=int(above.sum()), dtype=np.int8)
    pos = np.zeros((B, 3), np.float32)
    for b in range(B):
        while True:
            ex, ey, ez = rng.integers(0, wx), rng.integers(gh, wy), rng.integers(0, wz)
            if vox[b, ey, ex, ez] < 0:
                break
        f = rng.uniform(0.05, 0.95, 3)
        pos[b] = (ex + f[0], ey + f[1] - 1.6, ez + f[2])
    yaws = rng.uniform(-3.1, 3.1, B).astype(np.float32)
    pitches = rng.uniform(-1.4, 1.4, B).astype(np.float32)
    return vox, pos, yaws, pitches


@pytest.mark.parametrize("shape", sorted(SHAPES))
@pytest.mark.parametrize("mode", ["uint8", "uint8_minimal", "uint8_prebasis"])
@pytest.mark.parametrize("cfg", sorted(CFGS))
def test_up_bounds_random_scenes(cuda, shape, mode, cfg):
    wx, wy, wz = SHAPES[shape]
    fused = CFGS[cfg]
    if fused[4] == 1 and wx * wy * wz > 16384:
        fused = (fused[0], 4, 1, 4, 1, 0)  # one big world per warp: 4 warps fit in a CTA's shared memory
    B, gh = 48, 4
    rng = np.random.default_rng(zlib.crc32(f"{shape}/{mode}/{cfg}".encode()))
    vox, pos, yaws, pitches = random_scene(rng, B, wx, wy, wz, gh, density=0.03)
    g = GpuEnv(cuda, B, world_x=wx, world_y=wy, world_z=wz, render_width=16, render_height=16, obs_dtype=mode,
               numerics="ieee", debug=False, ground_height=gh)
    g.set_fused(*fused)
    o = O.OracleEnv(batch_size=B, world_x=wx, world_y=wy, world_z=wz, render_width=16, render_height=16,
                    obs_dtype=mode, ground_height=gh)
    st = dict(voxels=vox, positions=pos, velocities=np.zeros((B, 3), np.float32), yaws=yaws, pitches=pitches,
              on_ground=np.zeros(B, np.uint8))
    g.load(st)
    for k, a in st.items():
        getattr(o, k)[...] = a
    for s in range(3):
        btn = np.zeros((B, 8), np.int8)
        look = rng.uniform(-0.3, 0.3, (B, 2)).astype(np.float32)
        g.step(btn, look, FUSED)
        o.step(btn, look)
        d = diff_report(g.state(), oracle_state(o))
        assert not d, f"step {s}: differing elements {d}"
    g.check_error()
    g.close()
