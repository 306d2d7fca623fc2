"""Environment configuration: the reference's EnvConfig and presets
(minecu/config.py:11-101), same field names and defaults, so
`MineEnv.from_config(FAST_ENV)` builds the same environment."""
from dataclasses import dataclass
from typing import Optional


@dataclass
class EnvConfig:
    """Constructor arguments of MineEnv (reference minecu/config.py:11-66)."""

    batch_size: int = 4096
    world_size: int = 32
    render_width: int = 64
    render_height: int = 64
    max_steps: int = 64
    view_distance: float = 32.0
    fov_degrees: float = 70.0
    dt: float = 0.05
    gravity: float = -20.0
    walk_speed: float = 4.0
    jump_vel: float = 8.0
    ground_height: int = 8
    seed: int = 42
    target_block: int = 3
    reward_value: float = 1.0
    episode_length: Optional[int] = 60
    device: str = "cuda"

    def memory_bytes(self) -> int:
        """Device bytes of the env state (reference minecu/config.py:47-61,
        which counts float32 observations)."""
        B, W = self.batch_size, self.world_size
        H, WW = self.render_height, self.render_width
        voxels = B * W * W * W
        agent = B * (3 * 4 + 3 * 4 + 4 + 4 + 1)
        obs = B * H * WW * 3 * 4
        cameras = B * 5 * 4
        action_buffers = B * 4 * 5 + B * 2
        return voxels + agent + obs + cameras + action_buffers

    def memory_mb(self) -> float:
        return self.memory_bytes() / (1024 * 1024)


@dataclass
class TrainConfig:
    """Training hyper-parameters (reference minecu/config.py:69-82); kept for
    import compatibility, nothing in the package reads it."""

    lr: float = 3e-4
    gamma: float = 0.99
    total_steps: int = 10_000_000
    log_interval: int = 100_000
    hidden_dim: int = 256


DEFAULT_ENV = EnvConfig()
FAST_ENV = EnvConfig(batch_size=32768, render_width=32, render_height=32, max_steps=32)
QUALITY_ENV = EnvConfig(batch_size=4096, render_width=128, render_height=128, max_steps=128, view_distance=64.0)
