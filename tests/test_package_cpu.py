"""Host-side behaviour of the minecu package (no GPU needed)."""
import pytest
import torch

import minecu
from minecu import BlockType, EnvConfig, MineEnv
from minecu.config import FAST_ENV, QUALITY_ENV


def test_extension_is_the_in_tree_build():
    import os
    assert os.path.dirname(minecu._C.__file__) == os.path.dirname(minecu.__file__)
    assert minecu._C.ABI_VERSION == 2
    for name in ("render", "render_uint8", "physics", "raycast_break", "reset", "generate_world", "place_tree",
                 "place_house", "step", "step_uint8", "step_uint8_fast", "step_uint8_minimal", "step_uint8_fp16",
                 "step_uint8_prebasis", "step_uint8_prebasis_full", "step_uint8_smem", "precompute_camera_basis",
                 "render_uint8_prebasis", "render_uint8_coalesced"):
        assert hasattr(minecu._C, name), name


def test_reference_api_surface():
    assert MineEnv.button_dim == 8 and MineEnv.look_dim == 2 and MineEnv.action_dim == 11
    assert BlockType.OAKLOG == 3 and BlockType.AIR == -1 and BlockType.BEDROCK == 12
    assert FAST_ENV.batch_size == 32768 and FAST_ENV.render_width == 32 and FAST_ENV.max_steps == 32
    assert QUALITY_ENV.view_distance == 64.0
    assert EnvConfig().episode_length == 60
    assert set(minecu.OBS_MODES) >= {"float32", "uint8", "uint8_minimal", "uint8_fp16", "uint8_prebasis",
                                     "uint8_prebasis_full", "uint8_smem"}


def test_mine_env_argument_checks():
    with pytest.raises(AssertionError):
        MineEnv(batch_size=4, device="cpu")
    with pytest.raises(ValueError):
        MineEnv(batch_size=4, obs_dtype="bf16")
    with pytest.raises(ValueError):
        MineEnv(batch_size=4, numerics="fast")


def test_memory_estimate():
    assert EnvConfig(batch_size=32768, world_size=16, render_width=32, render_height=32).memory_mb() > 500
