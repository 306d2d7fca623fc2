"""Kernel-level parity with the reference's own CUDA kernels (oracle/_ref,
src/kernels.cu compiled unmodified with its fast-math flags) on random
worlds, cameras and agent states, through the C-ABI in "ref_fast" numerics.

Float outputs are compared as bit patterns; float32 renders expose 1-ulp
differences, the uint8 and flat-colour renders are checked on tens of
millions of rays over worlds of random block ids (so a different voxel or
face shows up as a different byte).  Tolerance: none.
"""
import ctypes

import numpy as np
import pytest

from minecu import capi

ref_driver = pytest.importorskip("ref_driver")
pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref_driver.available(), reason="oracle/_ref/libminecu_ref.so not built")]

VP = ctypes.c_void_p


def _world(torch, dev, B, ws, density, seed):
    g = torch.Generator().manual_seed(seed)
    ids = torch.randint(0, 13, (B, ws, ws, ws), generator=g)
    keep = torch.rand(B, ws, ws, ws, generator=g) < density
    return torch.where(keep, ids, torch.full_like(ids, -1)).to(torch.int8).to(dev)


def _cams(torch, dev, B, ws, seed, y_lo=0.0, y_hi=None):
    g = torch.Generator().manual_seed(seed)
    y_hi = ws - 2.0 if y_hi is None else y_hi
    return torch.stack([torch.rand(B, generator=g) * (ws - 2) + 1,
                        torch.rand(B, generator=g) * (y_hi - y_lo) + y_lo,
                        torch.rand(B, generator=g) * (ws - 2) + 1,
                        (torch.rand(B, generator=g) * 2 - 1) * 6.0,
                        (torch.rand(B, generator=g) * 2 - 1) * 1.56], 1).float().to(dev)


def _mine_render(torch, vox, cams, out, obs_dtype, shaded, max_steps=64, vd=32.0, fov=70.0, gh=8):
    B, ws = vox.shape[0], vox.shape[1]
    H, W = out.shape[1], out.shape[2]
    cfg = capi.make_config(B, ws, ws, ws, W, H, obs_dtype=obs_dtype, numerics="ref_fast", max_steps=max_steps,
                           view_distance=vd, fov_degrees=fov, ground_height=gh)
    st = capi.EnvState()
    st.voxels, st.cameras, st.obs = vox.data_ptr(), cams.data_ptr(), out.data_ptr()
    capi.check(capi.lib().mc_render(ctypes.byref(cfg), ctypes.byref(st), int(shaded), None), "mc_render")


@pytest.mark.parametrize("ws,res,density", [(16, 32, 0.25), (32, 64, 0.03), (16, 48, 0.6)])
def test_shaded_float32_render(cuda, ws, res, density):
    import torch
    B = 2048
    vox = _world(torch, cuda, B, ws, density, 1)
    cams = _cams(torch, cuda, B, ws, 2)
    ref = torch.zeros(B, res, res, 3, device=cuda)
    mine = torch.zeros_like(ref)
    ref_driver.lib().launch_render(VP(vox.data_ptr()), VP(cams.data_ptr()), VP(ref.data_ptr()), B, ws, res, res, 64,
                                   32.0, 70.0)
    _mine_render(torch, vox, cams, mine, "float32", True)
    torch.cuda.synchronize()
    n = int((mine.view(torch.int32) != ref.view(torch.int32)).sum())
    assert n == 0, f"{n} of {ref.numel()} floats differ"


@pytest.mark.parametrize("fn,mode,shaded", [("launch_render_uint8", "uint8", True),
                                            ("launch_render_uint8_minimal", "uint8_minimal", False),
                                            ("launch_render_uint8_fp16", "uint8_fp16", False)])
def test_uint8_renders(cuda, fn, mode, shaded):
    import torch
    B, ws, res = 8192, 16, 64
    vox = _world(torch, cuda, B, ws, 0.3, 3)
    cams = _cams(torch, cuda, B, ws, 4)
    ref = torch.zeros(B, res, res, 3, dtype=torch.uint8, device=cuda)
    mine = torch.zeros_like(ref)
    getattr(ref_driver.lib(), fn)(VP(vox.data_ptr()), VP(cams.data_ptr()), VP(ref.data_ptr()), B, ws, res, res, 64,
                                  32.0, 70.0)
    _mine_render(torch, vox, cams, mine, mode, shaded)
    torch.cuda.synchronize()
    n = int((mine != ref).any(-1).sum())
    assert n == 0, f"{n} of {B * res * res} pixels differ"


def test_uint8_fast_render(cuda):
    import torch
    B, ws, res = 8192, 16, 64
    vox = _world(torch, cuda, B, ws, 0.3, 5)
    cams = _cams(torch, cuda, B, ws, 6)
    ref = torch.zeros(B, res, res, 3, dtype=torch.uint8, device=cuda)
    mine = torch.zeros_like(ref)
    ref_driver.lib().launch_render_uint8_fast(VP(vox.data_ptr()), VP(cams.data_ptr()), VP(ref.data_ptr()), B, ws,
                                              res, res, 64, 32.0, 70.0, 5)
    _mine_render(torch, vox, cams, mine, "uint8_fast", True, gh=5)
    torch.cuda.synchronize()
    n = int((mine != ref).any(-1).sum())
    assert n == 0, f"{n} pixels differ"


def test_basis_and_prebasis_render(cuda):
    import torch
    B, ws, res = 8192, 16, 64
    vox = _world(torch, cuda, B, ws, 0.3, 7)
    cams = _cams(torch, cuda, B, ws, 8)
    rb = torch.zeros(B, 14, device=cuda)
    mb = torch.zeros(B, 14, device=cuda)
    L = ref_driver.lib()
    L.launch_precompute_camera_basis(VP(cams.data_ptr()), VP(rb.data_ptr()), B, res, res, 70.0)
    capi.check(capi.lib().mc_precompute_camera_basis(cams.data_ptr(), mb.data_ptr(), B, res, res, 70.0, 0, None))
    torch.cuda.synchronize()
    assert int((rb[:, :13].view(torch.int32) != mb[:, :13].view(torch.int32)).sum()) == 0
    ref = torch.zeros(B, res, res, 3, dtype=torch.uint8, device=cuda)
    mine = torch.zeros_like(ref)
    L.launch_render_uint8_prebasis(VP(vox.data_ptr()), VP(rb.data_ptr()), VP(ref.data_ptr()), B, ws, res, res, 64)
    capi.check(capi.lib().mc_render_uint8_prebasis(vox.data_ptr(), mb.data_ptr(), mine.data_ptr(), B, ws, ws, ws, res,
                                                   res, 64, 0, None))
    torch.cuda.synchronize()
    n = int((mine != ref).any(-1).sum())
    assert n == 0, f"{n} pixels differ"
    # the [Y,X,Z,B] layout variant
    vt = vox.permute(1, 2, 3, 0).contiguous()
    ref2 = torch.zeros_like(ref)
    mine2 = torch.zeros_like(ref)
    L.launch_render_uint8_coalesced(VP(vt.data_ptr()), VP(rb.data_ptr()), VP(ref2.data_ptr()), B, ws, res, res, 64)
    capi.check(capi.lib().mc_render_uint8_coalesced(vt.data_ptr(), mb.data_ptr(), mine2.data_ptr(), B, ws, res, res,
                                                    64, 0, None))
    torch.cuda.synchronize()
    assert int((mine2 != ref2).any(-1).sum()) == 0
    assert torch.equal(ref2, ref)


def test_physics_and_break(cuda):
    import torch
    B, ws = 1 << 20, 16
    g = torch.Generator().manual_seed(9)
    r = lambda *s: torch.rand(*s, generator=g)  # noqa: E731
    pos = torch.stack([r(B) * 18 - 1, r(B) * 14 - 1, r(B) * 18 - 1], 1).float()
    vel = (r(B, 3) * 20 - 10).float()
    yaw = ((r(B) * 2 - 1) * 40).float()
    pitch = ((r(B) * 2 - 1) * 2).float()
    og = r(B) < 0.5
    fwd = torch.randint(-3, 4, (B,), generator=g).float()
    strafe = torch.randint(-3, 4, (B,), generator=g).float()
    dyaw = ((r(B) * 2 - 1) * 0.7).float()
    dpitch = ((r(B) * 2 - 1) * 0.7).float()
    jump = r(B) < 0.5
    speed = torch.where(r(B) < 0.5, torch.tensor(1.5), torch.tensor(1.0)).float()
    dev = [t.to(cuda) for t in (pos, vel, yaw, pitch, og, fwd, strafe, dyaw, dpitch, jump, speed)]
    mine = [t.clone() for t in dev[:5]]
    ref_driver.lib().launch_physics(*[VP(t.data_ptr()) for t in dev], B, ws, 0.05, -20.0, 4.0, 8.0)
    capi.check(capi.lib().mc_physics(*[t.data_ptr() for t in mine], *[t.data_ptr() for t in dev[5:]], B, ws, 0.05,
                                     -20.0, 4.0, 8.0, 0, None))
    torch.cuda.synchronize()
    for a, b, name in zip(dev[:5], mine, ("positions", "velocities", "yaws", "pitches", "on_ground")):
        if a.dtype == torch.float32:
            a, b = a.view(torch.int32), b.view(torch.int32)
        assert torch.equal(a, b), f"{name}: {int((a != b).sum())} differ"
    # raycast break from the moved agents, random worlds
    Bb = 1 << 16
    vox = _world(torch, cuda, Bb, ws, 0.15, 10)
    vox2 = vox.clone()
    brk = (torch.rand(Bb, generator=g) < 0.8).to(cuda)
    rew, rew2 = torch.zeros(Bb, device=cuda), torch.zeros(Bb, device=cuda)
    p, yw, pt = dev[0][:Bb].contiguous(), dev[2][:Bb].contiguous(), dev[3][:Bb].contiguous()
    ref_driver.lib().launch_raycast_break(VP(vox.data_ptr()), VP(p.data_ptr()), VP(yw.data_ptr()), VP(pt.data_ptr()),
                                          VP(brk.data_ptr()), VP(rew.data_ptr()), Bb, ws, 3, 1.0)
    capi.check(capi.lib().mc_raycast_break(vox2.data_ptr(), p.data_ptr(), yw.data_ptr(), pt.data_ptr(),
                                           brk.data_ptr(), rew2.data_ptr(), Bb, ws, 3, 1.0, 0, None))
    torch.cuda.synchronize()
    assert torch.equal(vox, vox2), f"{int((vox != vox2).sum())} voxels differ"
    assert torch.equal(rew, rew2)
    assert int((vox != _world(torch, cuda, Bb, ws, 0.15, 10)).sum()) > Bb // 4  # many blocks were broken
