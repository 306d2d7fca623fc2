"""Env server: many client jobs stepped together on one GPU.

The reference has one MineEnv per Python process, stepped by its owner
(minecu/__init__.py:65-479).  `EnvServer` wraps the C-ABI server of
libminecu_b200.so (mc_server_*): jobs (env configurations) are admitted
against an HBM budget and keep their worlds and agents resident on the
device; client threads submit step/reset requests, and a native launcher
batches the oldest request of every job with work into one team-kernel
launch (one actions upload, one rewards/dones read-back).  Each step's
results equal MineEnv.step on that job alone with the fused form.

    srv = EnvServer(hbm_budget_bytes=150e9)
    job = srv.admit(batch_size=1024, world_size=16, render_width=32, render_height=32)
    t = srv.submit(job, actions)              # uint8 [batch] (host), returns a ticket
    rewards, dones = srv.wait(t)              # numpy arrays
    obs = srv.state(job)["obs"]               # torch tensor on the device, zero-copy
    stats = srv.drive([(job, 500.0, 200, 1)], seconds=2.0)   # Poisson load generator
"""
from __future__ import annotations

import ctypes
from typing import Dict, Optional, Sequence, Tuple

import numpy as np
import torch

from minecu import capi

_TYPESTR = {torch.uint8: "|u1", torch.int8: "|i1", torch.bool: "|b1", torch.int32: "<i4", torch.float32: "<f4"}


class _DeviceArray:
    """A device buffer owned by the server, seen by torch without a copy."""

    def __init__(self, owner, ptr: int, shape: Tuple[int, ...], dtype: torch.dtype):
        self._owner = owner
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": _TYPESTR[dtype], "data": (ptr, False),
                                         "version": 3}


class EnvServer:
    def __init__(self, hbm_budget_bytes: float = 150e9, numerics: str = "ref_fast", batching: bool = True,
                 max_inflight: int = 2, max_envs_per_launch: int = 0, device: Optional[torch.device] = None,
                 rounds: int = 1):
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.numerics = numerics
        self._L = capi.lib()
        cfg = capi.ServerConfig(int(hbm_budget_bytes), capi.NUMERICS_IEEE if numerics == "ieee" else
                                capi.NUMERICS_REF_FAST, 1 if batching else 0, int(max_inflight),
                                int(max_envs_per_launch))
        self._h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            torch.cuda.init()
            capi.check(self._L.mc_server_create(ctypes.byref(cfg), ctypes.byref(self._h)), "mc_server_create")
        if rounds != 1:
            self.set_rounds(rounds)
        self._jobs: Dict[int, capi.EnvConfig] = {}
        self._tickets: Dict[int, int] = {}  # ticket -> batch size of its results

    def set_rounds(self, rounds: int) -> None:
        """Step requests of one job a batching launch may run, one round
        after another (1..8): a burst of a job's requests then waits for one
        launch instead of one launch per request."""
        capi.check(self._L.mc_server_set_rounds(self._h, int(rounds)), "mc_server_set_rounds")

    # ------------------------------------------------------------------
    def _config(self, batch_size: int, world_size: int = 16, render_width: int = 32, render_height: int = 32,
                obs_dtype: str = "uint8", **kw) -> capi.EnvConfig:
        return capi.make_config(batch_size, kw.pop("world_x", world_size), kw.pop("world_y", world_size),
                                kw.pop("world_z", world_size), render_width, render_height, obs_dtype=obs_dtype,
                                numerics=self.numerics, **kw)

    def job_bytes(self, batch_size: int, **kw) -> int:
        """Device bytes a job of this configuration is charged at admission."""
        cfg = self._config(batch_size, **kw)
        return int(self._L.mc_server_job_bytes(ctypes.byref(cfg)))

    def admit(self, batch_size: int, **kw) -> int:
        """Admit a job (MineEnv constructor arguments; its worlds are
        generated and its agents spawned); raises MemoryError when it does
        not fit the HBM budget."""
        cfg = self._config(batch_size, **kw)
        job = ctypes.c_int32(-1)
        with torch.cuda.device(self.device):
            rc = self._L.mc_server_admit(self._h, ctypes.byref(cfg), ctypes.byref(job))
        if rc == capi.MC_ERR_BUDGET:
            raise MemoryError(capi.last_error())
        capi.check(rc, "mc_server_admit")
        self._jobs[job.value] = cfg
        return job.value

    def release(self, job: int) -> None:
        capi.check(self._L.mc_server_release(self._h, int(job)), "mc_server_release")
        self._jobs.pop(job, None)

    def state(self, job: int) -> Dict[str, torch.Tensor]:
        """The job's state as device tensors (zero-copy, MineEnv's names and shapes)."""
        st = capi.EnvState()
        capi.check(self._L.mc_server_job_state(self._h, int(job), ctypes.byref(st)), "mc_server_job_state")
        c = self._jobs[job]
        B, H, W = c.batch_size, c.render_height, c.render_width
        obs_t = torch.float32 if c.obs_mode == capi.OBS["float32"] else torch.uint8
        spec = {"voxels": ((B, c.world_y, c.world_x, c.world_z), torch.int8), "positions": ((B, 3), torch.float32),
                "velocities": ((B, 3), torch.float32), "yaws": ((B,), torch.float32),
                "pitches": ((B,), torch.float32), "on_ground": ((B,), torch.bool), "step_count": ((B,), torch.int32),
                "do_reset": ((B,), torch.bool), "cameras": ((B, 5), torch.float32), "obs": ((B, H, W, 3), obs_t),
                "rewards": ((B,), torch.float32)}
        out = {}
        for name, (shape, dt) in spec.items():
            ptr = getattr(st, name)
            out[name] = torch.as_tensor(_DeviceArray(self, ptr, shape, dt), device=self.device)
        return out

    # ------------------------------------------------------------------
    def submit(self, job: int, actions=None, reset: bool = False) -> int:
        """Queue a step (actions: uint8 [batch] on the host) or a reset; returns a ticket."""
        ticket = ctypes.c_int64(0)
        ptr = None
        if not reset:
            a = actions.cpu().numpy() if isinstance(actions, torch.Tensor) else np.asarray(actions)
            a = np.ascontiguousarray(a, dtype=np.uint8)
            if a.size != self._jobs[job].batch_size:
                raise ValueError(f"actions must have {self._jobs[job].batch_size} entries, got {a.size}")
            ptr = a.ctypes.data
        capi.check(self._L.mc_server_submit(self._h, int(job), capi.REQ_RESET if reset else capi.REQ_STEP, ptr,
                                            ctypes.byref(ticket)), "mc_server_submit")
        self._tickets[ticket.value] = 0 if reset else self._jobs[job].batch_size
        return ticket.value

    def wait(self, ticket: int, timeout_s: Optional[float] = None) -> Tuple[np.ndarray, np.ndarray]:
        """Results of a step request: (rewards float32 [batch], dones bool [batch]);
        empty arrays for a reset.  Raises TimeoutError after timeout_s."""
        if ticket not in self._tickets:
            raise KeyError(f"unknown ticket {ticket}")
        n = self._tickets[ticket]
        rew = np.zeros(n, dtype=np.float32)
        done = np.zeros(n, dtype=np.uint8)
        t_us = -1 if timeout_s is None else int(timeout_s * 1e6)
        rc = self._L.mc_server_wait(self._h, int(ticket), rew.ctypes.data, done.ctypes.data, t_us)
        if rc == capi.MC_ERR_TIMEOUT:
            raise TimeoutError(capi.last_error())
        del self._tickets[ticket]
        capi.check(rc, "mc_server_wait")
        return rew, done.astype(bool)

    def step(self, job: int, actions) -> Tuple[torch.Tensor, np.ndarray, np.ndarray]:
        """Submit a step and wait for it: (obs on the device, rewards, dones)."""
        rew, done = self.wait(self.submit(job, actions))
        return self.state(job)["obs"], rew, done

    def reset(self, job: int) -> torch.Tensor:
        self.wait(self.submit(job, reset=True))
        return self.state(job)["obs"]

    def stats(self) -> dict:
        s = capi.ServerStats()
        capi.check(self._L.mc_server_get_stats(self._h, ctypes.byref(s)), "mc_server_get_stats")
        return s.as_dict()

    def reset_stats(self) -> None:
        capi.check(self._L.mc_server_reset_stats(self._h), "mc_server_reset_stats")

    def drive(self, jobs: Sequence[Tuple[int, float, int, int]], seconds: float, closed_loop: bool = False) -> dict:
        """Native load generator: one client thread per (job, rate_hz,
        episode_steps, seed), Poisson arrivals (or closed loop) for `seconds`;
        returns the window's statistics (latency of the requests issued in it,
        env-steps completed in it)."""
        arr = (capi.LoadJob * len(jobs))(*[capi.LoadJob(int(j), float(r), int(ep), int(sd)) for j, r, ep, sd in jobs])
        cfg = capi.LoadConfig(float(seconds), 1 if closed_loop else 0, len(jobs), arr)
        out = capi.ServerStats()
        with torch.cuda.device(self.device):
            capi.check(self._L.mc_server_drive(self._h, ctypes.byref(cfg), ctypes.byref(out)), "mc_server_drive")
        return out.as_dict()

    def close(self) -> None:
        if self._h:
            self._L.mc_server_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
