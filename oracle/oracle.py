"""TEST INFRASTRUCTURE ONLY: numpy front end of the CPU checker (liboracle.so).

The CPU restatement of mine.cu's environment step lives in mc_oracle.c
(reference: src/kernels.cu, minecu/__init__.py).  This module mirrors the
reference's MineEnv constructor arguments and state tensors with numpy arrays
so that tests can run the oracle and the CUDA product on identical inputs.
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle.so")

RENDER_SHADED, RENDER_SHADED_FAST, RENDER_MINIMAL, RENDER_FP16, RENDER_PREBASIS = range(5)

# obs_dtype -> (render family used by step(), float32 obs)
# (minecu/__init__.py:304-444 dispatch; reset()/get_obs() always use the
# shaded kernel, minecu/__init__.py:455-464)
OBS_MODES = {
    "float32": (RENDER_SHADED, True),
    "uint8": (RENDER_SHADED, False),
    "uint8_fast": (RENDER_SHADED_FAST, False),
    "uint8_minimal": (RENDER_MINIMAL, False),
    "uint8_fp16": (RENDER_FP16, False),
    "uint8_prebasis": (RENDER_PREBASIS, False),
    "uint8_prebasis_full": (RENDER_PREBASIS, False),
    "uint8_smem": (RENDER_PREBASIS, False),
}


class OrcCfg(ctypes.Structure):
    _fields_ = [
        ("B", ctypes.c_int), ("wx", ctypes.c_int), ("wy", ctypes.c_int), ("wz", ctypes.c_int),
        ("width", ctypes.c_int), ("height", ctypes.c_int), ("max_steps", ctypes.c_int),
        ("view_distance", ctypes.c_float), ("fov_degrees", ctypes.c_float),
        ("dt", ctypes.c_float), ("gravity", ctypes.c_float), ("walk_speed", ctypes.c_float),
        ("sprint_mult", ctypes.c_float), ("jump_vel", ctypes.c_float),
        ("ground_height", ctypes.c_int), ("target_block", ctypes.c_int),
        ("reward_value", ctypes.c_float),
        ("spawn_x", ctypes.c_float), ("spawn_y", ctypes.c_float), ("spawn_z", ctypes.c_float),
        ("tree_x", ctypes.c_int), ("tree_z", ctypes.c_int),
        ("house_x", ctypes.c_int), ("house_z", ctypes.c_int),
        ("episode_rule", ctypes.c_int), ("has_limit", ctypes.c_int), ("episode_length", ctypes.c_int),
        ("render", ctypes.c_int), ("obs_f32", ctypes.c_int), ("regen_per_env", ctypes.c_int),
    ]


class OrcState(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in (
        "voxels", "positions", "velocities", "yaws", "pitches", "on_ground", "step_count",
        "do_reset", "cameras", "basis", "obs", "rewards", "dbg_interact", "dbg_pixel")]


def build() -> None:
    """Compile liboracle.so (and oracle/_ref when the reference sources exist)."""
    subprocess.run(["make", "-C", _HERE, "-s"], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        L = ctypes.CDLL(_LIB)
        P, I, F = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
        L.orc_env_step.restype = I
        L.orc_env_step.argtypes = [ctypes.POINTER(OrcCfg), ctypes.POINTER(OrcState), P, P, I]
        L.orc_env_reset.restype = None
        L.orc_env_reset.argtypes = [ctypes.POINTER(OrcCfg), ctypes.POINTER(OrcState), P, I]
        L.orc_env_render.restype = None
        L.orc_env_render.argtypes = [ctypes.POINTER(OrcCfg), ctypes.POINTER(OrcState), I]
        L.orc_render.restype = None
        L.orc_render.argtypes = [ctypes.POINTER(OrcCfg), I, I, P, P, P, P, I]
        for n in ("orc_generate_world",):
            getattr(L, n).argtypes = [P, I, I, I, I, I]
        for n in ("orc_place_tree", "orc_place_house"):
            getattr(L, n).argtypes = [P, I, I, I, I, I, I, I]
        L.orc_philox_actions.argtypes = [P, I, I, I, ctypes.c_uint64, I]
        L.orc_discrete_to_buttons.argtypes = [P, I, F, P, P]
        for n in ("orc_sinf", "orc_cosf", "orc_tanf"):
            getattr(L, n).restype = F
            getattr(L, n).argtypes = [F]
        L.orc_philox4x32_10.argtypes = [P, ctypes.c_uint32, ctypes.c_uint32]
        _lib = L
    return _lib


def _p(a: Optional[np.ndarray]):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.c_void_p)


class OracleEnv:
    """numpy mirror of the reference MineEnv (minecu/__init__.py:65-479)."""

    def __init__(self, batch_size=4096, world_size=32, world_x=None, world_y=None, world_z=None,
                 render_width=64, render_height=64, max_steps=64, view_distance=32.0,
                 fov_degrees=70.0, dt=0.05, gravity=-20.0, walk_speed=4.0, sprint_mult=1.5,
                 jump_vel=8.0, ground_height=8, target_block=3, reward_value=1.0,
                 episode_length=None, seed=42, obs_dtype="float32", debug=False, threads=0, regen="all"):
        self.B = batch_size
        self.wx = world_x if world_x is not None else world_size
        self.wy = world_y if world_y is not None else world_size
        self.wz = world_z if world_z is not None else world_size
        self.W, self.H = render_width, render_height
        self.obs_dtype = obs_dtype
        self.threads = threads
        fam, f32 = OBS_MODES[obs_dtype]
        # spawn / tree / house (minecu/__init__.py:195-206)
        sx, sy, sz = self.wx / 2.0, float(ground_height + 2), self.wz / 2.0
        c = OrcCfg()
        c.B, c.wx, c.wy, c.wz = self.B, self.wx, self.wy, self.wz
        c.width, c.height, c.max_steps = self.W, self.H, max_steps
        c.view_distance, c.fov_degrees = view_distance, fov_degrees
        c.dt, c.gravity, c.walk_speed, c.sprint_mult, c.jump_vel = dt, gravity, walk_speed, sprint_mult, jump_vel
        c.ground_height, c.target_block, c.reward_value = ground_height, target_block, reward_value
        c.spawn_x, c.spawn_y, c.spawn_z = sx, sy, sz
        c.tree_x, c.tree_z = int(sx), int(sz) + 2
        c.house_x, c.house_z = int(sx) + 6, int(sz) - 2
        c.episode_rule = 1 if obs_dtype == "uint8_prebasis_full" else 0
        if obs_dtype == "uint8_prebasis_full":
            c.has_limit, c.episode_length = 1, (episode_length if episode_length is not None else 0)
        else:
            c.has_limit, c.episode_length = (0, 0) if episode_length is None else (1, episode_length)
        c.render, c.obs_f32 = fam, int(f32)
        c.regen_per_env = 1 if regen == "per_env" else 0
        self.cfg = c
        B = self.B
        self.voxels = np.zeros((B, self.wy, self.wx, self.wz), np.int8)
        self.positions = np.zeros((B, 3), np.float32)
        self.velocities = np.zeros((B, 3), np.float32)
        self.yaws = np.zeros((B,), np.float32)
        self.pitches = np.zeros((B,), np.float32)
        self.on_ground = np.ones((B,), np.uint8)  # minecu/__init__.py:228
        self.step_count = np.zeros((B,), np.int32)
        self.do_reset = np.zeros((B,), np.uint8)
        self.cameras = np.zeros((B, 5), np.float32)
        self.basis = np.zeros((B, 14), np.float32) if fam == RENDER_PREBASIS else None
        self.obs = np.zeros((B, self.H, self.W, 3), np.float32 if f32 else np.uint8)
        self.rewards = np.zeros((B,), np.float32)
        self.dbg_interact = np.full((B,), -1, np.int32) if debug else None
        self.dbg_pixel = np.zeros((B, self.H, self.W), np.int16) if debug else None
        self._generate_world()

    def _state(self) -> OrcState:
        s = OrcState()
        for n in ("voxels", "positions", "velocities", "yaws", "pitches", "on_ground", "step_count",
                  "do_reset", "cameras", "basis", "rewards", "dbg_interact", "dbg_pixel"):
            setattr(s, n, _p(getattr(self, n)))
        s.obs = _p(self.obs)
        return s

    def _generate_world(self):
        L, c = lib(), self.cfg
        L.orc_generate_world(_p(self.voxels), c.B, c.wx, c.wy, c.wz, c.ground_height)
        L.orc_place_tree(_p(self.voxels), c.B, c.wx, c.wy, c.wz, c.tree_x, c.tree_z, c.ground_height)
        L.orc_place_house(_p(self.voxels), c.B, c.wx, c.wy, c.wz, c.house_x, c.house_z, c.ground_height)

    def reset(self, mask: Optional[np.ndarray] = None) -> np.ndarray:
        m = None if mask is None else np.ascontiguousarray(mask.astype(np.uint8))
        lib().orc_env_reset(ctypes.byref(self.cfg), ctypes.byref(self._state()), _p(m), self.threads)
        return self.obs

    def step(self, buttons: np.ndarray, look: np.ndarray):
        b = np.ascontiguousarray(buttons, dtype=np.int8)
        lk = np.ascontiguousarray(look, dtype=np.float32)
        assert b.shape == (self.B, 8) and lk.shape == (self.B, 2)
        lib().orc_env_step(ctypes.byref(self.cfg), ctypes.byref(self._state()), _p(b), _p(lk), self.threads)
        return self.obs, self.rewards, self.do_reset.astype(bool)

    def get_obs(self) -> np.ndarray:
        lib().orc_env_render(ctypes.byref(self.cfg), ctypes.byref(self._state()), self.threads)
        return self.obs


def render(family: int, obs_f32: bool, voxels: np.ndarray, cameras: np.ndarray, width: int, height: int,
           max_steps=64, view_distance=32.0, fov_degrees=70.0, ground_height=8, debug=False, threads=0):
    """Stand-alone render of one kernel family from a [B,5] camera buffer."""
    B, wy, wx, wz = voxels.shape
    c = OrcCfg()
    c.B, c.wx, c.wy, c.wz = B, wx, wy, wz
    c.width, c.height, c.max_steps = width, height, max_steps
    c.view_distance, c.fov_degrees, c.ground_height = view_distance, fov_degrees, ground_height
    obs = np.zeros((B, height, width, 3), np.float32 if obs_f32 else np.uint8)
    dbg = np.zeros((B, height, width), np.int16) if debug else None
    lib().orc_render(ctypes.byref(c), family, int(obs_f32), _p(np.ascontiguousarray(voxels)),
                     _p(np.ascontiguousarray(cameras, dtype=np.float32)), _p(obs), _p(dbg), threads)
    return (obs, dbg) if debug else obs


def philox_actions(B: int, step: int, seed: int, env_offset: int = 0, break_half: bool = False) -> np.ndarray:
    out = np.zeros((B,), np.uint8)
    lib().orc_philox_actions(_p(out), B, env_offset, step, seed, int(break_half))
    return out


def discrete_to_buttons(actions: np.ndarray, look_delta: float):
    a = np.ascontiguousarray(actions, dtype=np.uint8)
    B = a.shape[0]
    btn = np.zeros((B, 8), np.int8)
    look = np.zeros((B, 2), np.float32)
    lib().orc_discrete_to_buttons(_p(a), B, look_delta, _p(btn), _p(look))
    return btn, look


def philox4x32_10(ctr, key):
    """One Philox4x32-10 block (the action stream's generator): 4 counter
    words and 2 key words in, 4 words out."""
    c = np.ascontiguousarray(np.array(ctr, dtype=np.uint32))
    lib().orc_philox4x32_10(c.ctypes.data, int(key[0]), int(key[1]))
    return tuple(int(v) for v in c)


def sinf(x: float) -> float:
    return lib().orc_sinf(x)


def cosf(x: float) -> float:
    return lib().orc_cosf(x)


def tanf(x: float) -> float:
    return lib().orc_tanf(x)
