"""The allocation-free step (mc_step_plain_noalloc) against the allocating one.

mc_step_plain_noalloc is for callers that cannot allocate device memory:
its scratch is a static array inside libminecu_b200.so instead of buffers
the caller passes or the library allocates.  This file checks, through the
C-ABI, that two calls in a row give exactly the output of the existing
plain entry point mc_step_stateless (same tolerance as every parity test
here: none, floats compared bit for bit), and that batches above the stated
maximum are refused.  It is named to be collected last and works both alone
in a fresh process and after the other tests.
"""
import ctypes

import numpy as np
import pytest

from minecu import capi


def _make_state(torch, dev, B, ws, res, mode):
    z = lambda *s, dt=torch.float32: torch.zeros(s, dtype=dt, device=dev)  # noqa: E731
    t = dict(voxels=z(B, ws, ws, ws, dt=torch.int8), positions=z(B, 3), velocities=z(B, 3), yaws=z(B),
             pitches=z(B), on_ground=torch.ones(B, dtype=torch.bool, device=dev), step_count=z(B, dt=torch.int32),
             do_reset=z(B, dt=torch.bool), cameras=z(B, 5),
             obs=z(B, res, res, 3, dt=torch.float32 if mode == "float32" else torch.uint8), rewards=z(B))
    L = capi.lib()
    sx, sy, sz = ws / 2.0, 10.0, ws / 2.0
    capi.check(L.mc_generate_world(t["voxels"].data_ptr(), B, ws, ws, ws, 8, 0, None))
    capi.check(L.mc_place_tree(t["voxels"].data_ptr(), B, ws, ws, ws, int(sx), int(sz) + 2, 8, None))
    capi.check(L.mc_place_house(t["voxels"].data_ptr(), B, ws, ws, ws, int(sx) + 6, int(sz) - 2, 8, None))
    everyone = torch.ones(B, dtype=torch.bool, device=dev)
    capi.check(L.mc_reset_agents(t["positions"].data_ptr(), t["velocities"].data_ptr(), t["yaws"].data_ptr(),
                                 t["pitches"].data_ptr(), t["on_ground"].data_ptr(), everyone.data_ptr(), B, sx, sy,
                                 sz, None))
    return t


def _state_struct(t):
    st = capi.EnvState()
    for k, v in t.items():
        setattr(st, k, v.data_ptr())
    return st


def _bits(torch, v):
    return v.view(torch.int32) if v.dtype == torch.float32 else v


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["uint8", "float32"])
def test_noalloc_step_matches_allocating_step(cuda, mode):
    import torch
    B, ws, res = 96, 16, 32
    cfg = capi.make_config(B, ws, ws, ws, res, res, obs_dtype=mode, numerics="ref_fast")
    a = _make_state(torch, cuda, B, ws, res, mode)
    b = {k: v.clone() for k, v in a.items()}
    dec = {k: torch.zeros(B, dtype=dt, device=cuda) for k, dt in
           (("forward_in", torch.float32), ("strafe_in", torch.float32), ("delta_yaw_in", torch.float32),
            ("delta_pitch_in", torch.float32), ("jump_in", torch.bool), ("do_break", torch.bool),
            ("do_place", torch.bool), ("speed_mult", torch.float32))}
    db = capi.DecodeBuffers()
    for k, v in dec.items():
        setattr(db, k, v.data_ptr())
    rng = np.random.default_rng(7)
    L = capi.lib()
    for call in range(2):  # two calls in a row share the static scratch
        btn = torch.from_numpy(rng.integers(0, 2, (B, 8), dtype=np.int8)).to(cuda)
        look = torch.from_numpy(rng.uniform(-0.3, 0.3, (B, 2)).astype(np.float32)).to(cuda)
        do_reset = torch.from_numpy(rng.random(B) < 0.1).to(cuda)
        a["do_reset"].copy_(do_reset)
        b["do_reset"].copy_(do_reset)
        capi.check(L.mc_step_stateless(ctypes.byref(cfg), ctypes.byref(_state_struct(a)), btn.data_ptr(),
                                       look.data_ptr(), ctypes.byref(db), capi.FORM_PLAIN, None), "mc_step_stateless")
        capi.check(L.mc_step_plain_noalloc(ctypes.byref(cfg), ctypes.byref(_state_struct(b)), btn.data_ptr(),
                                           look.data_ptr(), None), "mc_step_plain_noalloc")
        torch.cuda.synchronize()
        for k in a:
            assert torch.equal(_bits(torch, a[k]), _bits(torch, b[k])), f"call {call}: {k} differs"
    # the step did real work: agents moved and something was broken
    assert not torch.equal(a["positions"], _make_state(torch, cuda, B, ws, res, mode)["positions"])


def test_noalloc_rejects_batches_above_the_maximum():
    L = capi.lib()
    cfg = capi.make_config(capi.NOALLOC_MAX_ENVS + 1, 16, 16, 16, 32, 32)
    st = capi.EnvState()
    rc = L.mc_step_plain_noalloc(ctypes.byref(cfg), ctypes.byref(st), None, None, None)
    assert rc == capi.MC_ERR_INVALID
    assert "MC_NOALLOC_MAX_ENVS" in capi.last_error()
