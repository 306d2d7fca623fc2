"""ctypes binding of the C-ABI in include/minecu_b200.h.

The torch extension minecu._C is the usual way in; this module reaches the
same library without torch's C++ headers, with raw device pointers
(e.g. `tensor.data_ptr()`) and an explicit stream handle (an int, 0 = the
legacy default stream).  Every function returns the C status; `check()`
raises on a non-zero one with mc_last_error()'s message.
"""
from __future__ import annotations

import ctypes
import os
import re
from typing import List

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libminecu_b200.so")
# the same library with every index bounds-checked (a debug build; see
# mc_build_checks_bounds in the header)
CHECKED_LIB_PATH = os.path.join(_HERE, "libminecu_b200_checked.so")
HEADER = os.path.join(os.path.dirname(os.path.dirname(_HERE)), "include", "minecu_b200.h")

MC_OK, MC_ERR_INVALID, MC_ERR_CUDA, MC_ERR_KERNEL, MC_ERR_UNSUPPORTED = 0, -1, -2, -3, -4
MC_ERR_BUDGET, MC_ERR_TIMEOUT, MC_ERR_BUSY = -5, -6, -7
REQ_STEP, REQ_RESET = 0, 1
NOALLOC_MAX_ENVS = 65536
NUMERICS_REF_FAST, NUMERICS_IEEE = 0, 1
FORM_PLAIN, FORM_FUSED = 0, 1
OBS = dict(float32=0, uint8=1, uint8_minimal=2, uint8_fp16=3, uint8_prebasis=4, uint8_prebasis_full=5,
           uint8_smem=6, uint8_fast=7)

c_int32, c_float, c_void_p = ctypes.c_int32, ctypes.c_float, ctypes.c_void_p


class EnvConfig(ctypes.Structure):
    _fields_ = [
        ("batch_size", c_int32), ("world_x", c_int32), ("world_y", c_int32), ("world_z", c_int32),
        ("render_width", c_int32), ("render_height", c_int32), ("max_steps", c_int32),
        ("view_distance", c_float), ("fov_degrees", c_float), ("dt", c_float), ("gravity", c_float),
        ("walk_speed", c_float), ("sprint_mult", c_float), ("jump_vel", c_float),
        ("ground_height", c_int32), ("target_block", c_int32), ("reward_value", c_float),
        ("has_episode_limit", c_int32), ("episode_length", c_int32), ("obs_mode", c_int32),
        ("numerics", c_int32), ("look_delta", c_float),
        ("spawn_override", c_int32), ("spawn_x", c_float), ("spawn_y", c_float), ("spawn_z", c_float),
    ]


class EnvState(ctypes.Structure):
    _fields_ = [(n, c_void_p) for n in (
        "voxels", "positions", "velocities", "yaws", "pitches", "on_ground", "step_count", "do_reset",
        "cameras", "basis", "obs", "rewards", "dbg_interact", "dbg_pixel")]


class FusedConfig(ctypes.Structure):
    _fields_ = [("stage", c_int32), ("warps_per_cta", c_int32), ("ctas_per_sm", c_int32),
                ("tile_w", c_int32), ("team_warps", c_int32), ("coop", c_int32)]


class DecodeBuffers(ctypes.Structure):
    _fields_ = [(n, c_void_p) for n in (
        "forward_in", "strafe_in", "delta_yaw_in", "delta_pitch_in", "jump_in", "do_break", "do_place",
        "speed_mult")]


RAGGED_MAX_GROUPS = 16


class RaggedConfig(ctypes.Structure):
    _fields_ = [("warps_per_cta", c_int32), ("ctas_per_sm", c_int32), ("team_warps", c_int32),
                ("stage", c_int32 * RAGGED_MAX_GROUPS), ("tile_w", c_int32 * RAGGED_MAX_GROUPS),
                ("coop", c_int32 * RAGGED_MAX_GROUPS)]


class ServerConfig(ctypes.Structure):
    _fields_ = [("hbm_budget_bytes", ctypes.c_int64), ("numerics", c_int32), ("batching", c_int32),
                ("max_inflight", c_int32), ("max_envs_per_launch", c_int32)]


class ServerStats(ctypes.Structure):
    _fields_ = [("step_requests", ctypes.c_int64), ("reset_requests", ctypes.c_int64),
                ("env_steps", ctypes.c_int64), ("launches", ctypes.c_int64), ("elapsed_s", ctypes.c_double),
                ("env_steps_per_s", ctypes.c_double), ("p50_us", ctypes.c_double), ("p90_us", ctypes.c_double),
                ("p99_us", ctypes.c_double), ("max_us", ctypes.c_double), ("mean_us", ctypes.c_double),
                ("reset_p50_us", ctypes.c_double), ("reset_p99_us", ctypes.c_double),
                ("mean_jobs_per_launch", ctypes.c_double), ("jobs", c_int32), ("bytes_admitted", ctypes.c_int64)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class LoadJob(ctypes.Structure):
    _fields_ = [("job", c_int32), ("rate_hz", ctypes.c_double), ("episode_steps", c_int32),
                ("seed", ctypes.c_uint32)]


class LoadConfig(ctypes.Structure):
    _fields_ = [("seconds", ctypes.c_double), ("closed_loop", c_int32), ("njobs", c_int32),
                ("jobs", ctypes.POINTER(LoadJob))]


P, I, F, U32, U64 = c_void_p, c_int32, c_float, ctypes.c_uint32, ctypes.c_uint64
PCFG, PST = ctypes.POINTER(EnvConfig), ctypes.POINTER(EnvState)

_PROTOS = {
    "mc_abi_version": (I, []),
    "mc_last_error": (ctypes.c_char_p, []),
    "mc_env_create": (I, [PCFG, PST, ctypes.POINTER(c_void_p)]),
    "mc_env_destroy": (I, [P]),
    "mc_env_set_state": (I, [P, PST]),
    "mc_env_generate_world": (I, [P, P]),
    "mc_env_reset": (I, [P, P, P]),
    "mc_env_step": (I, [P, P, P, ctypes.c_int, P]),
    "mc_env_step_discrete": (I, [P, P, ctypes.c_int, P]),
    "mc_env_step_host": (I, [P, P, P, P, ctypes.c_int, P]),
    "mc_env_host_join": (I, [P, P]),
    "mc_env_render": (I, [P, P]),
    "mc_env_set_regen_mode": (I, [P, ctypes.c_int32]),
    "mc_obs_to_policy": (I, [P, P, ctypes.c_int64, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, P]),
    "mc_env_get_regen_mode": (I, [P]),
    "mc_env_set_wait_limit": (I, [P, ctypes.c_int32]),
    "mc_env_regenerate_if": (I, [P, P, P]),
    "mc_env_rollout": (I, [P, P, I, P, P, P]),
    "mc_env_rollout_prepare": (I, [P, P, I, P, P]),
    "mc_env_set_fused_config": (I, [P, ctypes.POINTER(FusedConfig)]),
    "mc_env_get_fused_config": (I, [P, ctypes.POINTER(FusedConfig)]),
    "mc_env_check_error": (I, [P, P]),
    "mc_build_checks_bounds": (I, []),
    "mc_debug_bounds_report": (I, [c_int32, P, P]),
    "mc_debug_bounds_selftest": (I, [c_int32, P]),
    "mc_env_fused_smem_bytes": (ctypes.c_int64, [P]),
    "mc_default_fused_config": (I, [PCFG, c_int32, c_int32, P, P]),
    "mc_ragged_create": (I, [ctypes.POINTER(c_void_p), I, ctypes.POINTER(c_void_p)]),
    "mc_ragged_destroy": (I, [P]),
    "mc_ragged_set_config": (I, [P, ctypes.POINTER(RaggedConfig)]),
    "mc_ragged_get_config": (I, [P, ctypes.POINTER(RaggedConfig)]),
    "mc_ragged_total_envs": (ctypes.c_int64, [P]),
    "mc_ragged_smem_bytes": (ctypes.c_int64, [P]),
    "mc_ragged_step": (I, [P, P, P, P]),
    "mc_ragged_step_discrete": (I, [P, P, P]),
    "mc_ragged_step_host": (I, [P, P, P, P, P]),
    "mc_ragged_host_join": (I, [P, P]),
    "mc_ragged_rollout": (I, [P, P, I, P]),
    "mc_ragged_rollout_prepare": (I, [P, P, I]),
    "mc_ragged_check_error": (I, [P, P]),
    "mc_server_create": (I, [ctypes.POINTER(ServerConfig), ctypes.POINTER(c_void_p)]),
    "mc_server_destroy": (I, [P]),
    "mc_server_set_rounds": (I, [P, c_int32]),
    "mc_server_job_bytes": (ctypes.c_int64, [PCFG]),
    "mc_server_admit": (I, [P, PCFG, ctypes.POINTER(c_int32)]),
    "mc_server_release": (I, [P, I]),
    "mc_server_job_state": (I, [P, I, PST]),
    "mc_server_submit": (I, [P, I, I, P, ctypes.POINTER(ctypes.c_int64)]),
    "mc_server_wait": (I, [P, ctypes.c_int64, P, P, ctypes.c_int64]),
    "mc_server_get_stats": (I, [P, ctypes.POINTER(ServerStats)]),
    "mc_server_reset_stats": (I, [P]),
    "mc_server_drive": (I, [P, ctypes.POINTER(LoadConfig), ctypes.POINTER(ServerStats)]),
    "mc_generate_world": (I, [P, I, I, I, I, I, U32, P]),
    "mc_place_tree": (I, [P, I, I, I, I, I, I, I, P]),
    "mc_place_house": (I, [P, I, I, I, I, I, I, I, P]),
    "mc_reset_agents": (I, [P, P, P, P, P, P, I, F, F, F, P]),
    "mc_render": (I, [PCFG, PST, I, P]),
    "mc_precompute_camera_basis": (I, [P, P, I, I, I, F, I, P]),
    "mc_render_uint8_prebasis": (I, [P, P, P, I, I, I, I, I, I, I, I, P]),
    "mc_render_uint8_coalesced": (I, [P, P, P, I, I, I, I, I, I, P]),
    "mc_step_stateless": (I, [PCFG, PST, P, P, ctypes.POINTER(DecodeBuffers), I, P]),
    "mc_physics": (I, [P, P, P, P, P, P, P, P, P, P, P, I, I, F, F, F, F, I, P]),
    "mc_raycast_break": (I, [P, P, P, P, P, P, I, I, I, F, I, P]),
    "mc_step_plain_noalloc": (I, [PCFG, PST, P, P, P]),
    "mc_philox_actions": (I, [P, I, I, I, I, U64, I, P]),
    "mc_discrete_to_buttons": (I, [P, I, F, P, P, P]),
}

_lib = None
_checked_lib = None


def _bind(L: ctypes.CDLL) -> ctypes.CDLL:
    for name, (res, args) in _PROTOS.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    return L


def lib(checked: bool = False) -> ctypes.CDLL:
    """Load libminecu_b200.so, or with checked=True the bounds-checked debug
    build libminecu_b200_checked.so (raises OSError if it is not built).
    Both link with -Bsymbolic, so the two can be loaded in one process."""
    global _lib, _checked_lib
    if checked:
        if _checked_lib is None:
            _checked_lib = _bind(ctypes.CDLL(CHECKED_LIB_PATH, mode=ctypes.RTLD_LOCAL))
        return _checked_lib
    if _lib is None:
        _lib = _bind(ctypes.CDLL(LIB_PATH, mode=ctypes.RTLD_GLOBAL))
    return _lib


def header_functions() -> List[str]:
    """Names of every function include/minecu_b200.h declares."""
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(mc_[a-z0-9_]+)\s*\(", src)))


def last_error(L: ctypes.CDLL = None) -> str:
    return (L or lib()).mc_last_error().decode(errors="replace")


def check(rc: int, what: str = "call", L: ctypes.CDLL = None) -> None:
    if rc != MC_OK:
        raise RuntimeError(f"{what} failed ({rc}): {last_error(L)}")


def make_config(batch_size, world_x, world_y, world_z, render_width, render_height, obs_dtype="uint8",
                numerics="ref_fast", max_steps=64, view_distance=32.0, fov_degrees=70.0, dt=0.05, gravity=-20.0,
                walk_speed=4.0, sprint_mult=1.5, jump_vel=8.0, ground_height=8, target_block=3, reward_value=1.0,
                episode_length=None, look_delta=0.1, spawn=None) -> EnvConfig:
    """An EnvConfig with MineEnv's defaults and episode rule."""
    c = EnvConfig()
    c.batch_size, c.world_x, c.world_y, c.world_z = batch_size, world_x, world_y, world_z
    c.render_width, c.render_height, c.max_steps = render_width, render_height, max_steps
    c.view_distance, c.fov_degrees, c.dt, c.gravity = view_distance, fov_degrees, dt, gravity
    c.walk_speed, c.sprint_mult, c.jump_vel = walk_speed, sprint_mult, jump_vel
    c.ground_height, c.target_block, c.reward_value = ground_height, target_block, reward_value
    if obs_dtype == "uint8_prebasis_full":
        c.has_episode_limit, c.episode_length = 1, (episode_length or 0)
    else:
        c.has_episode_limit, c.episode_length = (0, 0) if episode_length is None else (1, episode_length)
    c.obs_mode = OBS[obs_dtype]
    c.numerics = NUMERICS_IEEE if numerics == "ieee" else NUMERICS_REF_FAST
    c.look_delta = look_delta
    if spawn is not None:
        c.spawn_override = 1
        c.spawn_x, c.spawn_y, c.spawn_z = spawn
    return c
