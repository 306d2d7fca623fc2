"""mine.cu environment step on B200.

Drop-in for the reference's `minecu.MineEnv` (minecu/__init__.py:65-479):
same constructor arguments, same state tensors (zero-copy torch tensors on
the device), same `reset(mask)` / `step(buttons, look)` and, in addition,
the discrete `step(actions)` of docs/environment.md (11 actions,
`action_dim`).  All work runs in the CUDA kernels of libminecu_b200.so,
reached through the torch extension `minecu._C`; there is no Python or CPU
fallback.

    env = MineEnv(batch_size=32768, world_size=16, render_width=32,
                  render_height=32, obs_dtype="uint8")
    obs = env.reset()
    obs, rewards, dones = env.step(actions)         # actions: int [B] in 0..10
    obs, rewards, dones = env.step(buttons, look)   # int8 [B,8], float32 [B,2]

Extra keyword arguments (not in the reference):
    numerics  "ref_fast" (default): the reference build's fast-math CUDA
              calls, bit-identical to it; "ieee": IEEE-754 arithmetic,
              bit-identical to the CPU checker.
    form      "fused" (default): one persistent kernel per step;
              "plain": the reference's kernel sequence.
    look_delta  radians turned by one discrete look action (default 0.1).
    debug     also keep per-pixel hit codes and per-env interaction indices.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional, Tuple

import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "libminecu_b200.so")

try:
    # make the C-ABI library resolvable for the extension even when the
    # extension's rpath is not honoured
    ctypes.CDLL(_LIB, mode=ctypes.RTLD_GLOBAL)
    from minecu import _C  # noqa: E402
except (ImportError, OSError) as exc:  # fail loudly: there is no fallback
    raise ImportError(
        "minecu native extension not built: run `python mine.cu_b200/build.py` "
        f"(or __graft_entry__.build()); cause: {exc}"
    ) from exc

from minecu.config import EnvConfig, TrainConfig, DEFAULT_ENV, FAST_ENV, QUALITY_ENV  # noqa: E402

__version__ = "0.2.0"
__all__ = ["MineEnv", "BlockType", "EnvConfig", "TrainConfig", "OBS_MODES", "NUMERICS", "REGEN_MODES", "lib_path"]

# obs_dtype -> C-ABI MC_OBS_* (include/minecu_b200.h); the reference accepts
# the first seven (minecu/__init__.py:167-169), uint8_fast exposes its
# step_uint8_fast binding (src/bindings.cpp:1112-1139) as a mode
OBS_MODES = {
    "float32": 0,
    "uint8": 1,
    "uint8_minimal": 2,
    "uint8_fp16": 3,
    "uint8_prebasis": 4,
    "uint8_prebasis_full": 5,
    "uint8_smem": 6,
    "uint8_fast": 7,
}

# which worlds dones and masked resets regenerate (C-ABI MC_REGEN_*)
REGEN_MODES = {"all": 0, "per_env": 1}
NUMERICS = {"ref_fast": 0, "ieee": 1}
FORMS = {"plain": 0, "fused": 1}


def lib_path() -> str:
    """Path of the C-ABI library (include/minecu_b200.h)."""
    return _LIB


class BlockType:
    """Block ids (reference src/kernels.cu:11-24, minecu/__init__.py:47-62)."""
    AIR = -1
    GRASS = 0
    DIRT = 1
    STONE = 2
    OAKLOG = 3
    LEAVES = 4
    SAND = 5
    WATER = 6
    GLASS = 7
    BRICK = 8
    COBBLESTONE = 9
    PLANKS = 10
    SNOW = 11
    BEDROCK = 12


class MineEnv:
    """Batched voxel environment (reference minecu/__init__.py:65-479).

    Actions: `step(buttons, look)` with buttons int8[B, 8] multi-hot
    (forward, back, left, right, jump, break, place, sprint) and look
    float32[B, 2] (delta yaw, + = left; delta pitch, + = up); or
    `step(actions)` with actions an integer tensor [B] over the 11 discrete
    actions of docs/environment.md.

    Returns (obs, rewards, dones): obs [B, H, W, 3] and rewards [B] are the
    env's own buffers, overwritten by the next step (as in the reference);
    dones is a fresh bool tensor.
    """

    button_dim = 8
    look_dim = 2
    action_dim = 11

    @classmethod
    def from_config(cls, config: EnvConfig, **kw) -> "MineEnv":
        """reference minecu/__init__.py:114-139"""
        return cls(
            batch_size=config.batch_size,
            world_size=getattr(config, "world_size", 32),
            world_x=getattr(config, "world_x", None),
            world_y=getattr(config, "world_y", None),
            world_z=getattr(config, "world_z", None),
            render_width=config.render_width,
            render_height=config.render_height,
            device=config.device,
            max_steps=config.max_steps,
            view_distance=config.view_distance,
            fov_degrees=config.fov_degrees,
            dt=config.dt,
            gravity=config.gravity,
            walk_speed=config.walk_speed,
            sprint_mult=getattr(config, "sprint_mult", 1.5),
            jump_vel=config.jump_vel,
            ground_height=config.ground_height,
            target_block=config.target_block,
            reward_value=config.reward_value,
            episode_length=config.episode_length,
            seed=config.seed,
            **kw,
        )

    def __init__(
        self,
        batch_size: int = 4096,
        world_size: int = 32,
        world_x: Optional[int] = None,
        world_y: Optional[int] = None,
        world_z: Optional[int] = None,
        render_width: int = 64,
        render_height: int = 64,
        device: str = "cuda",
        max_steps: int = 64,
        view_distance: float = 32.0,
        fov_degrees: float = 70.0,
        dt: float = 0.05,
        gravity: float = -20.0,
        walk_speed: float = 4.0,
        sprint_mult: float = 1.5,
        jump_vel: float = 8.0,
        ground_height: int = 8,
        target_block: int = BlockType.OAKLOG,
        reward_value: float = 1.0,
        episode_length: Optional[int] = None,
        seed: int = 42,
        obs_dtype: str = "float32",
        *,
        numerics: str = "ref_fast",
        form: str = "fused",
        look_delta: float = 0.1,
        debug: bool = False,
        regen: str = "all",
    ):
        assert "cuda" in str(device), "MineEnv requires CUDA device"
        if obs_dtype not in OBS_MODES:
            raise ValueError(f"obs_dtype must be one of {sorted(OBS_MODES)}, got {obs_dtype!r}")
        if numerics not in NUMERICS:
            raise ValueError(f"numerics must be one of {sorted(NUMERICS)}")
        if form not in FORMS:
            raise ValueError(f"form must be one of {sorted(FORMS)}")
        if regen not in REGEN_MODES:
            raise ValueError(f"regen must be one of {sorted(REGEN_MODES)}")
        self.device = torch.device(device)
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        self.batch_size = batch_size
        self.world_x = world_x if world_x is not None else world_size
        self.world_y = world_y if world_y is not None else world_size
        self.world_z = world_z if world_z is not None else world_size
        self.world_size = world_size
        self.render_width = render_width
        self.render_height = render_height
        self.max_steps = max_steps
        self.view_distance = view_distance
        self.fov_degrees = fov_degrees
        self.dt = dt
        self.gravity = gravity
        self.walk_speed = walk_speed
        self.sprint_mult = sprint_mult
        self.jump_vel = jump_vel
        self.ground_height = ground_height
        self.target_block = target_block
        self.reward_value = reward_value
        self.episode_length = episode_length
        self.seed = seed
        self.obs_dtype = obs_dtype
        self.numerics = numerics
        self.form = form
        self.look_delta = look_delta
        self.debug = debug

        # spawn, tree and house (reference minecu/__init__.py:195-206)
        self.spawn_x = self.world_x / 2.0
        self.spawn_y = float(ground_height + 2)
        self.spawn_z = self.world_z / 2.0
        self.tree_x = int(self.spawn_x)
        self.tree_z = int(self.spawn_z) + 2
        self.house_x = int(self.spawn_x) + 6
        self.house_z = int(self.spawn_z) - 2

        self._allocate_state()
        with torch.cuda.device(self.device):
            self._env = _C.env_create(self._config_dict(), self._state_dict_ptrs())
            self._generate_world()
        self.regen = "all"
        self.set_regen(regen)

    # ------------------------------------------------------------------
    def _config_dict(self) -> dict:
        prebasis_full = self.obs_dtype == "uint8_prebasis_full"
        if prebasis_full:
            has_limit, L = 1, (self.episode_length if self.episode_length is not None else 0)
        else:
            has_limit, L = (0, 0) if self.episode_length is None else (1, int(self.episode_length))
        return dict(
            batch_size=self.batch_size, world_x=self.world_x, world_y=self.world_y, world_z=self.world_z,
            render_width=self.render_width, render_height=self.render_height, max_steps=self.max_steps,
            view_distance=float(self.view_distance), fov_degrees=float(self.fov_degrees), dt=float(self.dt),
            gravity=float(self.gravity), walk_speed=float(self.walk_speed), sprint_mult=float(self.sprint_mult),
            jump_vel=float(self.jump_vel), ground_height=int(self.ground_height),
            target_block=int(self.target_block), reward_value=float(self.reward_value),
            has_episode_limit=has_limit, episode_length=int(L), obs_mode=OBS_MODES[self.obs_dtype],
            numerics=NUMERICS[self.numerics], look_delta=float(self.look_delta),
        )

    def _allocate_state(self):
        """State tensors of the reference (minecu/__init__.py:214-256)."""
        B = self.batch_size
        dev = self.device
        WX, WY, WZ = self.world_x, self.world_y, self.world_z
        H, WW = self.render_height, self.render_width
        self.voxels = torch.zeros((B, WY, WX, WZ), dtype=torch.int8, device=dev)
        self.positions = torch.zeros((B, 3), dtype=torch.float32, device=dev)
        self.velocities = torch.zeros((B, 3), dtype=torch.float32, device=dev)
        self.yaws = torch.zeros((B,), dtype=torch.float32, device=dev)
        self.pitches = torch.zeros((B,), dtype=torch.float32, device=dev)
        self.on_ground = torch.ones((B,), dtype=torch.bool, device=dev)
        obs_t = torch.float32 if self.obs_dtype == "float32" else torch.uint8
        self.obs_buffer = torch.zeros((B, H, WW, 3), dtype=obs_t, device=dev)
        self.cameras = torch.zeros((B, 5), dtype=torch.float32, device=dev)
        if self.obs_dtype in ("uint8_prebasis", "uint8_prebasis_full", "uint8_smem"):
            self.basis = torch.zeros((B, 14), dtype=torch.float32, device=dev)
        else:
            self.basis = None
        self.rewards = torch.zeros((B,), dtype=torch.float32, device=dev)
        self.step_count = torch.zeros((B,), dtype=torch.int32, device=dev)
        self.do_reset = torch.zeros((B,), dtype=torch.bool, device=dev)
        if self.debug:
            self.dbg_interact = torch.full((B,), -1, dtype=torch.int32, device=dev)
            self.dbg_pixel = torch.zeros((B, H, WW), dtype=torch.int16, device=dev)
        else:
            self.dbg_interact = None
            self.dbg_pixel = None

    _STATE_KEYS = ("voxels", "positions", "velocities", "yaws", "pitches", "on_ground", "step_count", "do_reset",
                   "cameras", "basis", "obs_buffer", "rewards", "dbg_interact", "dbg_pixel")

    def _state_dict_ptrs(self) -> dict:
        return {k: getattr(self, k) for k in self._STATE_KEYS}

    def _generate_world(self):
        """reference minecu/__init__.py:258-268 (one template world broadcast)."""
        _C.env_generate_world(self._env)

    # ------------------------------------------------------------------
    def reset(self, mask: Optional[torch.Tensor] = None) -> torch.Tensor:
        """reference minecu/__init__.py:270-302.  The `mask.any()` test runs
        on the device, so no host synchronisation happens here."""
        with torch.cuda.device(self.device):
            if mask is None:
                _C.env_reset(self._env, None)
            else:
                m = mask.to(device=self.device, dtype=torch.bool).contiguous().reshape(self.batch_size)
                _C.env_reset(self._env, m)
        return self.obs_buffer

    def step(self, buttons: torch.Tensor, look: Optional[torch.Tensor] = None,
             ) -> Tuple[torch.Tensor, torch.Tensor, torch.Tensor]:
        """reference minecu/__init__.py:304-444 (buttons + look), or the
        discrete form when `look` is omitted."""
        form = FORMS[self.form]
        with torch.cuda.device(self.device):
            if look is None:
                a = buttons
                if a.dtype != torch.uint8 or a.device != self.device or not a.is_contiguous():
                    a = a.to(device=self.device, dtype=torch.uint8).contiguous()
                if a.numel() != self.batch_size:
                    raise ValueError(f"actions must have {self.batch_size} entries, got {a.numel()}")
                _C.env_step_discrete(self._env, a.reshape(self.batch_size), form)
            else:
                b = buttons
                if b.dtype != torch.int8 or b.device != self.device or not b.is_contiguous():
                    b = b.to(device=self.device, dtype=torch.int8).contiguous()
                lk = look
                if lk.dtype != torch.float32 or lk.device != self.device or not lk.is_contiguous():
                    lk = lk.to(device=self.device, dtype=torch.float32).contiguous()
                if b.shape != (self.batch_size, 8) or lk.shape != (self.batch_size, 2):
                    raise ValueError(f"buttons must be [{self.batch_size}, 8] and look [{self.batch_size}, 2]")
                _C.env_step(self._env, b, lk, form)
            return self.obs_buffer, self.rewards, self.do_reset.clone()

    def step_host(self, actions: torch.Tensor, rewards_out: torch.Tensor, dones_out: torch.Tensor) -> torch.Tensor:
        """The discrete step for a host-side policy: actions uint8 [B] read
        from pinned host memory, rewards float32 [B] and dones bool [B]
        written to pinned host memory.  Returns the (device) observation
        buffer.  The copies overlap the device steps of the neighbouring
        calls, so a call's host tensors stay in use until `join_host()` and
        a synchronisation of the current stream (e.g.
        torch.cuda.synchronize()): its actions must not be overwritten, nor
        its rewards and dones read, before then."""
        form = FORMS[self.form]
        with torch.cuda.device(self.device):
            _C.env_step_host(self._env, actions, rewards_out, dones_out, self.batch_size, form)
        return self.obs_buffer

    def join_host(self) -> None:
        """Make the current stream wait for the host copies of every
        step_host call so far."""
        with torch.cuda.device(self.device):
            _C.env_host_join(self._env)

    def rollout(self, actions: torch.Tensor, rewards_out: Optional[torch.Tensor] = None,
                dones_out: Optional[torch.Tensor] = None) -> None:
        """K fused steps of discrete actions [K, B] (uint8, on the device),
        captured once in a CUDA graph and replayed.  rewards_out float32
        [K, B] and dones_out bool [K, B], if given, receive every step's
        rewards and dones; obs_buffer holds the last step's observation."""
        if actions.dtype != torch.uint8 or actions.dim() != 2 or actions.shape[1] != self.batch_size:
            raise ValueError("actions must be uint8 [K, B]")
        with torch.cuda.device(self.device):
            _C.env_rollout(self._env, actions.contiguous(), rewards_out, dones_out)

    def prepare_rollout(self, actions: torch.Tensor, rewards_out: Optional[torch.Tensor] = None,
                        dones_out: Optional[torch.Tensor] = None) -> None:
        """Capture the rollout graph for these buffers without running it."""
        with torch.cuda.device(self.device):
            _C.env_rollout_prepare(self._env, actions.contiguous(), rewards_out, dones_out)

    def _render(self) -> torch.Tensor:
        """reference minecu/__init__.py:446-466"""
        with torch.cuda.device(self.device):
            _C.env_render(self._env)
        return self.obs_buffer

    def policy_obs(self, out: Optional[torch.Tensor] = None, layout: str = "nchw") -> torch.Tensor:
        """The current observation as a policy takes it: float32 in [0, 1],
        [B, 3, H, W] ("nchw", what the reference's example policy permutes
        its input to) or [B, H, W, 3] ("nhwc").  One pass over the uint8
        observation (obs / 255, IEEE division); for "float32" observations,
        which already hold those values, the permuted buffer."""
        if layout not in ("nchw", "nhwc"):
            raise ValueError("layout must be 'nchw' or 'nhwc'")
        B, H, W = self.batch_size, self.render_height, self.render_width
        shape = (B, 3, H, W) if layout == "nchw" else (B, H, W, 3)
        if self.obs_buffer.dtype == torch.float32:
            src = self.obs_buffer.permute(0, 3, 1, 2) if layout == "nchw" else self.obs_buffer
            if out is None:
                return src.contiguous()
            out.copy_(src)
            return out
        if out is None:
            out = torch.empty(shape, dtype=torch.float32, device=self.device)
        elif tuple(out.shape) != shape or out.dtype != torch.float32 or not out.is_contiguous():
            raise ValueError(f"out must be a contiguous float32 tensor of shape {shape}")
        with torch.cuda.device(self.device):
            _C.obs_to_policy(self.obs_buffer, out, 0 if layout == "nchw" else 1)
        return out

    def set_regen(self, mode: str) -> None:
        """Which worlds a step's dones (and reset(mask)) regenerate: "all"
        (the reference's rule: every world when any env is done or reset) or
        "per_env" (opt-in: only the worlds of the envs done or reset, each
        back to the start world)."""
        if mode not in REGEN_MODES:
            raise ValueError(f"regen must be one of {sorted(REGEN_MODES)}")
        _C.env_set_regen_mode(self._env, REGEN_MODES[mode])
        self.regen = mode

    def set_wait_limit(self, polls: int) -> None:
        """Budget of the fused kernels' bounded waits for a world's bulk copy
        into shared memory: polls > 0 polls, 0 = give up at once (every wait
        runs out: a test of the timeout path, after which the kernel renders
        from global memory and check_error() reports the timeout), < 0 = the
        default."""
        _C.env_set_wait_limit(self._env, int(polls))

    def regenerate_if(self, flag: torch.Tensor) -> None:
        """Regenerate every world when the one-byte device tensor `flag` is
        non-zero, with no host synchronisation (the all-reduced any-done
        flag of a batch sharded over several GPUs; see minecu.shard)."""
        with torch.cuda.device(self.device):
            _C.env_regenerate_if(self._env, flag)

    def get_obs(self) -> torch.Tensor:
        return self._render()

    def close(self):
        self._env = None

    @property
    def observation_shape(self) -> Tuple[int, int, int]:
        return (self.render_height, self.render_width, 3)

    # ------------------------------------------------------------------
    def set_launch_config(self, stage: int, warps_per_cta: int, ctas_per_sm: int, tile_w: int,
                          team_warps: int = 1, coop: int = 0) -> None:
        """Launch shape of the fused step (see minecu.autotune).  team_warps=1,
        coop=0: one warp steps and renders each env; coop=1: a team of
        team_warps warps renders each env together."""
        _C.env_set_fused(self._env, int(stage), int(warps_per_cta), int(ctas_per_sm), int(tile_w), int(team_warps),
                         int(coop))

    def launch_config(self) -> dict:
        return _C.env_get_fused(self._env)

    def check_error(self) -> None:
        """Raise if a kernel recorded an error (synchronises)."""
        with torch.cuda.device(self.device):
            _C.env_check_error(self._env)

    def state_dict(self) -> dict:
        """Env state for checkpointing: the reference keeps its state in
        plain tensors (minecu/__init__.py:214-256)."""
        keys = ("voxels", "positions", "velocities", "yaws", "pitches", "on_ground", "step_count", "do_reset",
                "cameras", "rewards", "obs_buffer")
        return {k: getattr(self, k).clone() for k in keys}

    def load_state_dict(self, sd: dict) -> None:
        for k, v in sd.items():
            t = getattr(self, k)
            if t.shape != v.shape or t.dtype != v.dtype:
                raise ValueError(f"{k}: expected {tuple(t.shape)} {t.dtype}, got {tuple(v.shape)} {v.dtype}")
            t.copy_(v)
