"""The bounds-checked debug build, libminecu_b200_checked.so.

The same library compiled with every voxel, shared-memory world, table and
observation index checked against its buffer before the access; a failed
check skips the access and is recorded (mc_debug_bounds_report), never
trapped.  The checks that matter most are the PTX marches': each of their
loads happens before the exit test, so the load of the step that leaves the
box reads up to one world layer before or after the staged world, and the
shared-memory layouts keep that much allocated.  The debug build checks
every such load address against the staged world plus one layer on either
side, and against the CTA's dynamic shared memory.

Each case runs in the debug build against the CPU oracle (ieee numerics,
bit for bit, tolerance none) and then requires a zero record: the edge
shapes of the early-exit march tests in both fused kernels, and the plain
form and debug outputs on small shapes.  A self-test records one violation
with no memory access behind it, to show that a violation reaches the
record.
"""
import ctypes

import numpy as np
import pytest

from minecu import capi
import oracle as O
from mc_harness import GpuEnv, actions_for, diff_report, oracle_state
from test_parity_gpu import EARLY_EXIT_CASES

pytestmark = pytest.mark.gpu


def _checked():
    try:
        return capi.lib(checked=True)
    except OSError as exc:
        pytest.fail(f"the debug build is missing (build() makes it): {exc}")


def _report(L):
    out = (ctypes.c_int32 * 4)()
    capi.check(L.mc_debug_bounds_report(capi.NUMERICS_IEEE, out, None), "bounds report", L=L)
    return list(out)


def _run_checked(cuda, steps, seed, form, fused_cfg=None, debug=False, obs_dtype="uint8", B=64, world=16,
                 res=(32, 32), world_xyz=None, break_half=False, episode_length=None, reset_every=None, **kw):
    L = _checked()
    assert L.mc_build_checks_bounds() == 1
    _report(L)  # start from an empty record
    wx, wy, wz = world_xyz or (world, world, world)
    g = GpuEnv(cuda, B, world_x=wx, world_y=wy, world_z=wz, render_width=res[0], render_height=res[1],
               obs_dtype=obs_dtype, numerics="ieee", debug=debug, checked=True, episode_length=episode_length, **kw)
    if fused_cfg is not None:
        g.set_fused(*fused_cfg)
    o = O.OracleEnv(batch_size=B, world_x=wx, world_y=wy, world_z=wz, render_width=res[0], render_height=res[1],
                    obs_dtype=obs_dtype, debug=debug, episode_length=episode_length, **kw)
    g.reset()
    o.reset()
    rng = np.random.default_rng(seed)
    for s in range(steps):
        if reset_every and s and s % reset_every == 0:
            mask = rng.random(B) < 0.3
            g.reset(mask)
            o.reset(mask)
        _, btn, look = actions_for(B, s, seed, 0.1, break_half)
        btn[:, 6] = (rng.random(B) < 0.1).astype(np.int8)
        btn[:, 7] = (rng.random(B) < 0.3).astype(np.int8)
        g.step(btn, look, form)
        o.step(btn, look)
        d = diff_report(g.state(), oracle_state(o))
        assert not d, f"step {s}: {d}"
    rec = _report(L)
    assert rec[0] == 0, f"bounds violations: {rec[0]}, first at site {rec[1]}, index {rec[2]} of limit {rec[3]}"
    g.check_error()  # the step kernels also report violations in the env's error word
    g.close()


@pytest.mark.parametrize("case", sorted(EARLY_EXIT_CASES))
@pytest.mark.parametrize("mode", ["uint8", "uint8_minimal"])
@pytest.mark.parametrize("cfg", [(1, 8, 4, 4, 1, 0), (1, 8, 3, 8, 4, 1)], ids=["per_warp", "team"])
def test_checked_build_early_exit_marches(cuda, case, mode, cfg):
    kw = dict(EARLY_EXIT_CASES[case])
    kw.setdefault("obs_dtype", mode)
    wx, wy, wz = kw.get("world_xyz") or (kw.get("world", 16),) * 3
    if (wx * wy * wz) % 16:
        cfg = (0,) + tuple(cfg[1:])
    elif cfg[4] == 1 and wx * wy * wz > 16384:
        cfg = (1, 4, 1, 4, 1, 0)
    _run_checked(cuda, kw.pop("steps"), kw.pop("seed"), capi.FORM_FUSED, fused_cfg=cfg, **kw)


@pytest.mark.parametrize("mode", ["uint8", "float32", "uint8_minimal", "uint8_prebasis", "uint8_fp16", "uint8_fast"])
@pytest.mark.parametrize("form", [capi.FORM_PLAIN, capi.FORM_FUSED])
def test_checked_build_modes_with_debug_outputs(cuda, mode, form):
    _run_checked(cuda, 12, 11, form, debug=True, obs_dtype=mode, B=37, res=(24, 20))


def test_checked_build_wide_flat_world_and_odd_image(cuda):
    _run_checked(cuda, 15, 12, capi.FORM_FUSED, fused_cfg=(1, 8, 4, 4, 1, 0), B=21, world_xyz=(32, 8, 32),
                 res=(8, 8), ground_height=4, break_half=True)
    _run_checked(cuda, 15, 6, capi.FORM_FUSED, B=1, world=8, res=(7, 5))


def test_checked_build_records_a_violation(cuda):
    L = _checked()
    _report(L)
    capi.check(L.mc_debug_bounds_selftest(capi.NUMERICS_IEEE, None), "self-test", L=L)
    rec = _report(L)
    assert rec == [1, 0, -1, 1], rec
    assert _report(L) == [0, 0, 0, 0]  # reading cleared it
