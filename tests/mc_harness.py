"""Test harness: run the CUDA product through its C-ABI (minecu.capi) and
the CPU oracle (oracle/oracle.py) side by side on identical inputs."""
from __future__ import annotations

import ctypes
from typing import Dict, Optional

import numpy as np

from minecu import capi
import oracle as O

STATE_FIELDS = ("voxels", "positions", "velocities", "yaws", "pitches", "on_ground", "step_count", "do_reset",
                "cameras", "obs", "rewards")


class GpuEnv:
    """An mc_env over torch-allocated state, driven through the C-ABI."""

    def __init__(self, device, batch_size, world_size=16, world_x=None, world_y=None, world_z=None,
                 render_width=32, render_height=32, obs_dtype="uint8", numerics="ieee", debug=True, checked=False,
                 **kw):
        import torch
        self.torch = torch
        self.L = capi.lib(checked=checked)  # checked: the bounds-checked debug build
        self.B = batch_size
        self.wx = world_x or world_size
        self.wy = world_y or world_size
        self.wz = world_z or world_size
        self.W, self.H = render_width, render_height
        self.obs_dtype = obs_dtype
        self.cfg = capi.make_config(batch_size, self.wx, self.wy, self.wz, render_width, render_height,
                                    obs_dtype=obs_dtype, numerics=numerics, **kw)
        B, d = batch_size, device
        z = lambda *s, dt=torch.float32: torch.zeros(s, dtype=dt, device=d)  # noqa: E731
        self.t = dict(
            voxels=z(B, self.wy, self.wx, self.wz, dt=torch.int8), positions=z(B, 3), velocities=z(B, 3),
            yaws=z(B), pitches=z(B), on_ground=torch.ones(B, dtype=torch.bool, device=d),
            step_count=z(B, dt=torch.int32), do_reset=z(B, dt=torch.bool), cameras=z(B, 5),
            obs=z(B, self.H, self.W, 3, dt=torch.float32 if obs_dtype == "float32" else torch.uint8),
            rewards=z(B),
        )
        self.t["basis"] = z(B, 14) if obs_dtype in ("uint8_prebasis", "uint8_prebasis_full", "uint8_smem") else None
        self.t["dbg_interact"] = torch.full((B,), -1, dtype=torch.int32, device=d) if debug else None
        self.t["dbg_pixel"] = z(B, self.H, self.W, dt=torch.int16) if debug else None
        self.st = capi.EnvState()
        for k, v in self.t.items():
            setattr(self.st, k, None if v is None or v.numel() == 0 else v.data_ptr())
        self.h = ctypes.c_void_p()
        capi.check(self.L.mc_env_create(ctypes.byref(self.cfg), ctypes.byref(self.st), ctypes.byref(self.h)),
                   "mc_env_create", L=self.L)
        self.buttons = z(B, 8, dt=torch.int8)
        self.look = z(B, 2)
        self.actions = z(B, dt=torch.uint8)
        capi.check(self.L.mc_env_generate_world(self.h, None), "generate_world", L=self.L)

    def close(self):
        if self.h:
            self.L.mc_env_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_regen(self, per_env: bool):
        capi.check(self.L.mc_env_set_regen_mode(self.h, 1 if per_env else 0), "set_regen_mode", L=self.L)
        assert self.L.mc_env_get_regen_mode(self.h) == (1 if per_env else 0)

    def set_fused(self, stage, warps_per_cta=8, ctas_per_sm=4, tile_w=8, team_warps=1, coop=0):
        f = capi.FusedConfig(stage, warps_per_cta, ctas_per_sm, tile_w, team_warps, coop)
        capi.check(self.L.mc_env_set_fused_config(self.h, ctypes.byref(f)), "set_fused_config", L=self.L)

    def reset(self, mask: Optional[np.ndarray] = None):
        m = None
        if mask is not None:
            m = self.torch.as_tensor(mask.astype(bool), device=self.t["voxels"].device)
        capi.check(self.L.mc_env_reset(self.h, None if m is None else m.data_ptr(), None), "reset", L=self.L)
        self.torch.cuda.synchronize()

    def step(self, buttons: np.ndarray, look: np.ndarray, form: int):
        self.buttons.copy_(self.torch.from_numpy(np.ascontiguousarray(buttons, np.int8)))
        self.look.copy_(self.torch.from_numpy(np.ascontiguousarray(look, np.float32)))
        capi.check(self.L.mc_env_step(self.h, self.buttons.data_ptr(), self.look.data_ptr(), form, None), "step", L=self.L)
        self.torch.cuda.synchronize()

    def step_discrete(self, actions: np.ndarray, form: int):
        self.actions.copy_(self.torch.from_numpy(np.ascontiguousarray(actions, np.uint8)))
        capi.check(self.L.mc_env_step_discrete(self.h, self.actions.data_ptr(), form, None), "step", L=self.L)
        self.torch.cuda.synchronize()

    def render(self):
        capi.check(self.L.mc_env_render(self.h, None), "render", L=self.L)
        self.torch.cuda.synchronize()

    def check_error(self):
        capi.check(self.L.mc_env_check_error(self.h, None), "check_error", L=self.L)

    def state(self) -> Dict[str, np.ndarray]:
        out = {}
        for k, v in self.t.items():
            if v is not None:
                a = v.cpu().numpy()
                out[k] = a.astype(np.uint8) if a.dtype == np.bool_ else a
        return out

    def load(self, st: Dict[str, np.ndarray]):
        for k, a in st.items():
            if self.t.get(k) is not None:
                src = self.torch.from_numpy(np.ascontiguousarray(a))
                if self.t[k].dtype == self.torch.bool:
                    src = src.bool()
                self.t[k].copy_(src)
        self.torch.cuda.synchronize()


def oracle_state(e: "O.OracleEnv") -> Dict[str, np.ndarray]:
    s = dict(voxels=e.voxels, positions=e.positions, velocities=e.velocities, yaws=e.yaws, pitches=e.pitches,
             on_ground=e.on_ground, step_count=e.step_count, do_reset=e.do_reset, cameras=e.cameras, obs=e.obs,
             rewards=e.rewards)
    if e.basis is not None:
        s["basis"] = e.basis
    if e.dbg_interact is not None:
        s["dbg_interact"] = e.dbg_interact
        s["dbg_pixel"] = e.dbg_pixel
    return s


def diff_report(a: Dict[str, np.ndarray], b: Dict[str, np.ndarray], fields=None) -> Dict[str, int]:
    """Number of differing elements per field (bitwise for floats)."""
    out = {}
    for k in (fields or a.keys()):
        if k not in a or k not in b:
            continue
        x, y = a[k], b[k]
        if x.dtype.kind == "f":
            x, y = x.view(np.int32 if x.dtype == np.float32 else np.int64), y.view(np.int32 if y.dtype == np.float32 else np.int64)
        n = int(np.count_nonzero(x != y))
        if n:
            out[k] = n
    return out


def actions_for(B: int, step: int, seed: int, look_delta: float = 0.1, break_half: bool = False, env_offset=0):
    a = O.philox_actions(B, step, seed, env_offset=env_offset, break_half=break_half)
    btn, look = O.discrete_to_buttons(a, look_delta)
    return a, btn, look
