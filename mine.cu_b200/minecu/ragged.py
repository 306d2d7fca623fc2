"""Ragged batches: several MineEnv groups stepped by one persistent launch.

The reference runs one world size and one resolution per MineEnv
(minecu/__init__.py:141-212), one kernel sequence per env per step.  A
`RaggedBatch` takes up to 16 MineEnv objects ("groups") that differ in batch
size, world size, resolution and parameters (same `numerics` and the same
observation kind) and steps all of them with one launch of the team kernel:
teams of warps claim work from one counter across every group, the groups
with the most expensive envs first.  Per group, a whole team renders each env
(big images or worlds) or each warp its own env (small ones), with the
group's own pixel-tile shape and shared-memory staging.  Each group's state,
observation, rewards and dones are exactly those of stepping that MineEnv on
its own with the fused form, including the regeneration of all of a group's
worlds when one of its envs is done.

    envs = [MineEnv(batch_size=8192, world_size=8, render_width=16, render_height=16, obs_dtype="uint8"),
            MineEnv(batch_size=1024, world_size=32, render_width=64, render_height=64, obs_dtype="uint8")]
    batch = RaggedBatch(envs)
    batch.reset()
    results = batch.step(actions)            # actions uint8 [total]; [(obs, rewards, dones) per group]
    batch.rollout(actions_k)                 # [K, total], one CUDA graph
"""
from __future__ import annotations

from typing import List, Optional, Sequence, Tuple

import torch

from minecu import MineEnv, _C

MAX_GROUPS = 16


class RaggedBatch:
    def __init__(self, envs: Sequence[MineEnv]):
        envs = list(envs)
        if not 1 <= len(envs) <= MAX_GROUPS:
            raise ValueError(f"a ragged batch holds 1..{MAX_GROUPS} groups, got {len(envs)}")
        e0 = envs[0]
        for g, e in enumerate(envs):
            if e.device != e0.device:
                raise ValueError(f"group {g} is on {e.device}, group 0 on {e0.device}")
            if e.numerics != e0.numerics:
                raise ValueError(f"group {g}: numerics {e.numerics!r} differs from {e0.numerics!r}")
        self.envs: List[MineEnv] = envs
        self.device = e0.device
        self.sizes = [e.batch_size for e in envs]
        self.offsets = [0]
        for n in self.sizes:
            self.offsets.append(self.offsets[-1] + n)
        self.total = self.offsets[-1]
        with torch.cuda.device(self.device):
            self._r = _C.ragged_create([e._env for e in envs])

    # ------------------------------------------------------------------
    def reset(self, masks: Optional[Sequence[Optional[torch.Tensor]]] = None) -> List[torch.Tensor]:
        """MineEnv.reset of every group (masks: one per group, or None)."""
        masks = masks if masks is not None else [None] * len(self.envs)
        return [e.reset(m) for e, m in zip(self.envs, masks)]

    def _u8(self, a: torch.Tensor) -> torch.Tensor:
        if a.dtype != torch.uint8 or a.device != self.device or not a.is_contiguous():
            a = a.to(device=self.device, dtype=torch.uint8).contiguous()
        return a

    def step(self, actions: torch.Tensor, look: Optional[torch.Tensor] = None
             ) -> List[Tuple[torch.Tensor, torch.Tensor, torch.Tensor]]:
        """One step of every group.  `actions` is uint8 [total] (discrete
        actions 0..10, concatenated in group order), or int8 buttons
        [total, 8] together with float32 `look` [total, 2]."""
        with torch.cuda.device(self.device):
            if look is None:
                a = self._u8(actions)
                if a.numel() != self.total:
                    raise ValueError(f"actions must have {self.total} entries, got {a.numel()}")
                _C.ragged_step_discrete(self._r, a.reshape(self.total))
            else:
                b = actions.to(device=self.device, dtype=torch.int8).contiguous()
                lk = look.to(device=self.device, dtype=torch.float32).contiguous()
                if b.shape != (self.total, 8) or lk.shape != (self.total, 2):
                    raise ValueError(f"buttons must be [{self.total}, 8] and look [{self.total}, 2]")
                _C.ragged_step(self._r, b, lk)
        return [(e.obs_buffer, e.rewards, e.do_reset.clone()) for e in self.envs]

    def step_host(self, actions: torch.Tensor, rewards_out: torch.Tensor, dones_out: torch.Tensor
                  ) -> List[torch.Tensor]:
        """One discrete step of every group with host buffers, as
        MineEnv.step_host: actions uint8 [total] from pinned host memory,
        rewards float32 [total] and dones bool [total] (group order) to
        pinned host memory, valid after `join_host()` and a synchronisation
        of the current stream.  Returns each group's (device) observation
        buffer."""
        with torch.cuda.device(self.device):
            _C.ragged_step_host(self._r, actions, rewards_out, dones_out)
        return [e.obs_buffer for e in self.envs]

    def join_host(self) -> None:
        """Make the current stream wait for the host copies of every
        step_host call so far."""
        with torch.cuda.device(self.device):
            _C.ragged_host_join(self._r)

    def rollout(self, actions: torch.Tensor) -> None:
        """K steps of discrete actions uint8 [K, total] captured once in a
        CUDA graph and replayed."""
        if actions.dtype != torch.uint8 or actions.dim() != 2 or actions.shape[1] != self.total:
            raise ValueError(f"actions must be uint8 [K, {self.total}]")
        with torch.cuda.device(self.device):
            _C.ragged_rollout(self._r, actions.contiguous(), False)

    def prepare_rollout(self, actions: torch.Tensor) -> None:
        with torch.cuda.device(self.device):
            _C.ragged_rollout(self._r, actions.contiguous(), True)

    def group_slice(self, g: int) -> slice:
        return slice(self.offsets[g], self.offsets[g + 1])

    # ------------------------------------------------------------------
    def set_launch_config(self, warps_per_cta: int, ctas_per_sm: int, stage: Sequence[int],
                          tile_w: Sequence[int], team_warps: int = 1, coop: Optional[Sequence[int]] = None) -> None:
        """Launch shape (warps per CTA, CTAs per SM, warps per team) and, per
        group, shared-memory staging depth (0: none, 1: one world buffer per
        stepping warp, 2: two, the next unit's world copied while the current
        one renders; the launch stages every staged group at the largest depth
        asked), pixel-tile width and whether a whole team renders each env
        (coop 1) or each warp its own (0)."""
        coop = [0] * len(self.envs) if coop is None else coop
        _C.ragged_set_config(self._r, int(warps_per_cta), int(ctas_per_sm), int(team_warps),
                             [int(s) for s in stage], [int(t) for t in tile_w], [int(c) for c in coop])

    def launch_config(self) -> dict:
        return _C.ragged_get_config(self._r)

    def check_error(self) -> None:
        with torch.cuda.device(self.device):
            _C.ragged_check_error(self._r)

    def state_dict(self) -> List[dict]:
        return [e.state_dict() for e in self.envs]

    def load_state_dict(self, sds: Sequence[dict]) -> None:
        for e, sd in zip(self.envs, sds):
            e.load_state_dict(sd)

    def algorithmic_bytes_per_step(self) -> int:
        """World bytes read plus observation bytes written, summed over groups."""
        total = 0
        for e in self.envs:
            px = e.render_width * e.render_height * 3 * (4 if e.obs_dtype == "float32" else 1)
            total += e.batch_size * (e.world_x * e.world_y * e.world_z + px)
        return total
