"""Policy input (mc_obs_to_policy, MineEnv.policy_obs): a uint8 observation
as float32 obs / 255 in NCHW or NHWC.  Compared with numpy's float32
division on the host: bit-exact (tolerance none), for the vectorised path
(H*W a multiple of 4, aligned buffers) and the per-pixel path."""
import ctypes

import numpy as np
import pytest

from minecu import capi

pytestmark = pytest.mark.gpu


def _want(obs_u8: np.ndarray, layout: str) -> np.ndarray:
    v = obs_u8.astype(np.float32) / np.float32(255.0)
    return np.ascontiguousarray(v.transpose(0, 3, 1, 2)) if layout == "nchw" else v


@pytest.mark.parametrize("layout", ["nchw", "nhwc"])
@pytest.mark.parametrize("shape", [(6, 8, 8), (5, 7, 9), (3, 32, 32), (1, 1, 1)])
def test_c_abi_matches_numpy(cuda, layout, shape):
    import torch
    B, H, W = shape
    rng = np.random.default_rng(B * 1000 + H * 10 + W)
    obs = rng.integers(0, 256, size=(B, H, W, 3), dtype=np.uint8)
    d_obs = torch.from_numpy(obs).to(cuda)
    out = torch.full((B * H * W * 3,), -1.0, dtype=torch.float32, device=cuda)
    rc = capi.lib().mc_obs_to_policy(ctypes.c_void_p(d_obs.data_ptr()), ctypes.c_void_p(out.data_ptr()), B, H, W,
                                     0 if layout == "nchw" else 1, None)
    capi.check(rc, "mc_obs_to_policy")
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    assert np.array_equal(got.view(np.int32), _want(obs, layout).reshape(-1).view(np.int32))


def test_unaligned_output_takes_the_per_pixel_path(cuda):
    import torch
    from minecu import _C
    obs = np.random.default_rng(1).integers(0, 256, size=(4, 8, 8, 3), dtype=np.uint8)
    d_obs = torch.from_numpy(obs).to(cuda)
    big = torch.zeros(4 * 8 * 8 * 3 + 1, dtype=torch.float32, device=cuda)
    out = big[1:]  # 4-byte offset: not 16-byte aligned
    _C.obs_to_policy(d_obs, out, 0)
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy().view(np.int32), _want(obs, "nchw").reshape(-1).view(np.int32))
    assert float(big[0]) == 0.0


@pytest.mark.parametrize("layout", ["nchw", "nhwc"])
def test_mine_env_policy_obs(cuda, layout):
    import torch
    from minecu import MineEnv, _C
    env = MineEnv(batch_size=40, world_size=16, render_width=24, render_height=20, obs_dtype="uint8", device=cuda)
    env.reset()
    acts = torch.empty((5, 40), dtype=torch.uint8, device=cuda)
    _C.philox_actions(acts, 0, 0, 7, False)
    for s in range(5):
        env.step(acts[s])
    got = env.policy_obs(layout=layout)
    torch.cuda.synchronize()
    want = _want(env.obs_buffer.cpu().numpy(), layout)
    assert tuple(got.shape) == want.shape
    assert np.array_equal(got.cpu().numpy().view(np.int32), want.view(np.int32))
    # a caller's buffer is filled in place
    out = torch.empty_like(got)
    assert env.policy_obs(out=out, layout=layout) is out
    assert torch.equal(out, got)


def test_float32_observations_are_permuted_only(cuda):
    import torch
    from minecu import MineEnv
    env = MineEnv(batch_size=9, world_size=16, render_width=16, render_height=12, obs_dtype="float32", device=cuda)
    env.reset()
    got = env.policy_obs()
    assert torch.equal(got, env.obs_buffer.permute(0, 3, 1, 2))
    assert got.is_contiguous()
