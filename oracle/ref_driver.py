"""TEST INFRASTRUCTURE ONLY: the reference implementation, run on a GPU.

`oracle/_ref/libminecu_ref.so` is the reference's own src/kernels.cu,
compiled unmodified with its own flags (nvcc -O3 --use_fast_math, see
oracle/Makefile).  Its `extern "C"` launchers are the reference's native
interface (src/kernels.cu:2076-3245).  `RefEnv` drives them in the order
the reference's Python MineEnv does (minecu/__init__.py:141-466), with
torch tensors for the state, so tests, golden-fixture generation and the
benchmark's reference arm run the reference's stock kernels and launch
sequence.  The Python glue below is a restatement of MineEnv's (that file
is not shipped); every step cites the lines it follows.

As the reference's CUDA graphs bake in the action pointers
(src/kernels.cu:2526-2542), actions are always copied into persistent
buffers before a step.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional

import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(_HERE, "_ref", "libminecu_ref.so")

P, I, F = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
I8 = ctypes.c_int8

_STEP_COMMON = [P, P, P, P, P, P, P, P, P, P, P, P, P, P, P, P, P, P]  # voxels..cameras (18 pointers)
_TAIL = [F, F, F, F, F, F, F, F, I8, F, F, F, F]  # vd, fov, dt, g, walk, sprint, jump, target, reward, sx, sy, sz
_PROTOS = {
    # launch_step*(..., obs, rewards, B, ws, W, H, max_steps, vd, ...) (src/kernels.cu:2497-2834)
    "launch_step": _STEP_COMMON + [P, P, I, I, I, I, I] + [F, F, F, F, F, F, F, I8, F, F, F, F],
    "launch_step_uint8": _STEP_COMMON + [P, P, I, I, I, I, I] + [F, F, F, F, F, F, F, I8, F, F, F, F],
    "launch_step_uint8_minimal": _STEP_COMMON + [P, P, I, I, I, I, I] + [F, F, F, F, F, F, F, I8, F, F, F, F],
    "launch_step_uint8_fp16": _STEP_COMMON + [P, P, I, I, I, I, I] + [F, F, F, F, F, F, F, I8, F, F, F, F],
    "launch_step_uint8_fast": _STEP_COMMON + [P, P, I, I, I, I, I] + [F, F, F, F, F, F, F, I8, F, F, F, F, I],
    # prebasis: + basis, wx/wy/wz (src/kernels.cu:2993-3076)
    "launch_step_uint8_prebasis": _STEP_COMMON + [P, P, P, I, I, I, I, I, I, I] + [F, F, F, F, F, F, F, I8, F, F, F, F],
    # prebasis_full: step_count after do_reset (src/kernels.cu:3081-3168)
    "launch_step_uint8_prebasis_full": [P, P, P, P, P, P, P, P, P, P] + [P] * 9 + [P, P, P, I, I, I, I, I, I, I]
                                       + [F, F, F, F, F, F, F, I8, F, F, F, F, I],
    "launch_generate_world": [P, I, I, I, I, I, ctypes.c_uint],
    "launch_place_tree": [P, I, I, I, I, I, I, I],
    "launch_place_house": [P, I, I, I, I, I, I, I],
    "launch_reset": [P, P, P, P, P, P, I, F, F, F],
    "launch_render": [P, P, P, I, I, I, I, I, F, F],
    "launch_render_uint8": [P, P, P, I, I, I, I, I, F, F],
    "launch_render_uint8_minimal": [P, P, P, I, I, I, I, I, F, F],
    "launch_render_uint8_fp16": [P, P, P, I, I, I, I, I, F, F],
    "launch_render_uint8_fast": [P, P, P, I, I, I, I, I, F, F, I],
    "launch_precompute_camera_basis": [P, P, I, I, I, F],
    "launch_render_uint8_prebasis": [P, P, P, I, I, I, I, I],
    "launch_render_uint8_coalesced": [P, P, P, I, I, I, I, I],
    "launch_physics": [P, P, P, P, P, P, P, P, P, P, P, I, I, F, F, F, F],
    "launch_raycast_break": [P, P, P, P, P, P, I, I, I8, F],
    "launch_decode_actions": [P, P, P, P, P, P, P, P, P, P, I, F],
}

_lib = None


def available() -> bool:
    return os.path.exists(REF_LIB)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        L = ctypes.CDLL(REF_LIB)
        for n, args in _PROTOS.items():
            fn = getattr(L, n)
            fn.restype = None
            fn.argtypes = args
        _lib = L
    return _lib


def _p(t: Optional[torch.Tensor]):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


class RefEnv:
    """The reference MineEnv (minecu/__init__.py:65-479) over its own kernels."""

    MODES = ("float32", "uint8", "uint8_minimal", "uint8_fp16", "uint8_prebasis", "uint8_prebasis_full",
             "uint8_fast")

    def __init__(self, batch_size=4096, world_size=32, world_x=None, world_y=None, world_z=None, render_width=64,
                 render_height=64, device="cuda", max_steps=64, view_distance=32.0, fov_degrees=70.0, dt=0.05,
                 gravity=-20.0, walk_speed=4.0, sprint_mult=1.5, jump_vel=8.0, ground_height=8, target_block=3,
                 reward_value=1.0, episode_length=None, seed=42, obs_dtype="float32"):
        # uint8_smem is left out: its launcher's C declaration in
        # src/bindings.cpp:195-210 does not match the definition in
        # src/kernels.cu:3170-3184, so its arguments arrive shifted
        assert obs_dtype in self.MODES, obs_dtype
        self.dev = torch.device(device)
        self.B = batch_size
        self.wx = world_x if world_x is not None else world_size
        self.wy = world_y if world_y is not None else world_size
        self.wz = world_z if world_z is not None else world_size
        self.W, self.H = render_width, render_height
        self.max_steps, self.vd, self.fov = max_steps, view_distance, fov_degrees
        self.dt, self.g, self.walk, self.sprint, self.jump = dt, gravity, walk_speed, sprint_mult, jump_vel
        self.gh, self.target, self.reward_value = ground_height, target_block, reward_value
        self.episode_length, self.seed, self.obs_dtype = episode_length, seed, obs_dtype
        # minecu/__init__.py:195-206
        self.spawn_x, self.spawn_y, self.spawn_z = self.wx / 2.0, float(ground_height + 2), self.wz / 2.0
        self.tree_x, self.tree_z = int(self.spawn_x), int(self.spawn_z) + 2
        self.house_x, self.house_z = int(self.spawn_x) + 6, int(self.spawn_z) - 2
        # minecu/__init__.py:214-256
        B, d = self.B, self.dev
        z = lambda *s, dt=torch.float32: torch.zeros(s, dtype=dt, device=d)  # noqa: E731
        self.voxels = z(B, self.wy, self.wx, self.wz, dt=torch.int8)
        self.positions, self.velocities = z(B, 3), z(B, 3)
        self.yaws, self.pitches = z(B), z(B)
        self.on_ground = torch.ones(B, dtype=torch.bool, device=d)
        self.obs_buffer = z(B, self.H, self.W, 3, dt=torch.float32 if obs_dtype == "float32" else torch.uint8)
        self.cameras = z(B, 5)
        self.basis = z(B, 14) if obs_dtype.startswith("uint8_prebasis") else None
        self.forward_in, self.strafe_in, self.delta_yaw_in, self.delta_pitch_in = z(B), z(B), z(B), z(B)
        self.jump_in, self.do_break, self.do_place = (z(B, dt=torch.bool) for _ in range(3))
        self.speed_mult = torch.ones(B, dtype=torch.float32, device=d)
        self.rewards = z(B)
        self.step_count = z(B, dt=torch.int32)
        self.do_reset = z(B, dt=torch.bool)
        # persistent action buffers (the graph modes bake their pointers in)
        self.buttons = z(B, 8, dt=torch.int8)
        self.look = z(B, 2)
        self._generate_world()

    def _generate_world(self):
        """minecu/__init__.py:258-268"""
        L = lib()
        L.launch_generate_world(_p(self.voxels), self.B, self.wx, self.wy, self.wz, self.gh, self.seed)
        L.launch_place_tree(_p(self.voxels), self.B, self.wx, self.wy, self.wz, self.tree_x, self.tree_z, self.gh)
        L.launch_place_house(_p(self.voxels), self.B, self.wx, self.wy, self.wz, self.house_x, self.house_z, self.gh)

    def reset(self, mask: Optional[torch.Tensor] = None) -> torch.Tensor:
        """minecu/__init__.py:270-302"""
        if mask is None:
            self.do_reset.fill_(True)
        else:
            self.do_reset.copy_(mask)
        lib().launch_reset(_p(self.positions), _p(self.velocities), _p(self.yaws), _p(self.pitches),
                           _p(self.on_ground), _p(self.do_reset), self.B, self.spawn_x, self.spawn_y, self.spawn_z)
        self.step_count.masked_fill_(self.do_reset, 0)
        if mask is None or bool(mask.any()):
            self._generate_world()
        return self._render()

    def _render(self) -> torch.Tensor:
        """minecu/__init__.py:446-466"""
        self.cameras[:, 0] = self.positions[:, 0]
        self.cameras[:, 1] = self.positions[:, 1]
        self.cameras[:, 2] = self.positions[:, 2]
        self.cameras[:, 3] = self.yaws
        self.cameras[:, 4] = self.pitches
        fn = lib().launch_render if self.obs_dtype == "float32" else lib().launch_render_uint8
        fn(_p(self.voxels), _p(self.cameras), _p(self.obs_buffer), self.B, self.wy, self.W, self.H,
           self.max_steps, self.vd, self.fov)
        return self.obs_buffer

    def get_obs(self):
        return self._render()

    def _common(self):
        return [_p(self.voxels), _p(self.positions), _p(self.velocities), _p(self.yaws), _p(self.pitches),
                _p(self.on_ground), _p(self.buttons), _p(self.look), _p(self.do_reset)]

    def _decode(self):
        return [_p(self.forward_in), _p(self.strafe_in), _p(self.delta_yaw_in), _p(self.delta_pitch_in),
                _p(self.jump_in), _p(self.do_break), _p(self.do_place), _p(self.speed_mult), _p(self.cameras)]

    def _params(self):
        return [self.max_steps, self.vd, self.fov, self.dt, self.g, self.walk, self.sprint, self.jump,
                self.target, self.reward_value, self.spawn_x, self.spawn_y, self.spawn_z]

    def step(self, buttons: torch.Tensor, look: torch.Tensor):
        """minecu/__init__.py:304-444"""
        self.buttons.copy_(buttons)
        self.look.copy_(look)
        L = lib()
        if self.obs_dtype == "uint8_prebasis_full":
            L.launch_step_uint8_prebasis_full(
                *self._common()[:9], _p(self.step_count), *self._decode(), _p(self.basis), _p(self.obs_buffer),
                _p(self.rewards), self.B, self.wx, self.wy, self.wz, self.W, self.H, *self._params(),
                self.episode_length if self.episode_length is not None else 0)
            if bool(self.do_reset.any()):
                self._generate_world()
            return self.obs_buffer, self.rewards, self.do_reset.clone()
        if self.episode_length is not None:
            # the reference rebinds do_reset to a new tensor here
            # (minecu/__init__.py:364); writing in place is equivalent
            torch.ge(self.step_count, self.episode_length, out=self.do_reset)
        else:
            self.do_reset.zero_()
        head = self._common() + self._decode()
        if self.obs_dtype == "uint8_prebasis":
            L.launch_step_uint8_prebasis(*head, _p(self.basis), _p(self.obs_buffer), _p(self.rewards), self.B,
                                         self.wx, self.wy, self.wz, self.W, self.H, *self._params())
        else:
            fn = {"float32": L.launch_step, "uint8": L.launch_step_uint8, "uint8_minimal": L.launch_step_uint8_minimal,
                  "uint8_fp16": L.launch_step_uint8_fp16, "uint8_fast": L.launch_step_uint8_fast}[self.obs_dtype]
            extra = [self.gh] if self.obs_dtype == "uint8_fast" else []
            fn(*head, _p(self.obs_buffer), _p(self.rewards), self.B, self.wy, self.W, self.H, *self._params(), *extra)
        self.step_count += 1
        self.step_count.masked_fill_(self.do_reset, 1)
        if bool(self.do_reset.any()):
            self._generate_world()
        return self.obs_buffer, self.rewards, self.do_reset.clone()
