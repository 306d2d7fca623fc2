"""The C-ABI library loads, exports every function include/minecu_b200.h
declares, and rejects bad arguments on the host (no GPU needed)."""
import ctypes

import pytest

from minecu import capi


def test_library_exports_every_declared_symbol():
    L = capi.lib()
    names = capi.header_functions()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert L.mc_abi_version() == 2


def test_prototypes_cover_header():
    assert set(capi.header_functions()) == set(capi._PROTOS)


def _cfg(**kw):
    base = dict(batch_size=4, world_x=16, world_y=16, world_z=16, render_width=8, render_height=8)
    base.update(kw)
    return capi.make_config(**base)


@pytest.mark.parametrize("bad", [dict(batch_size=-1), dict(world_x=0), dict(render_width=0),
                                 dict(target_block=300), dict(world_z=4)])
def test_env_create_rejects_bad_config(bad):
    L = capi.lib()
    c = _cfg(**bad)
    st = capi.EnvState()
    for f, _ in capi.EnvState._fields_:
        setattr(st, f, 16)  # never dereferenced: validation fails first
    h = ctypes.c_void_p()
    rc = L.mc_env_create(ctypes.byref(c), ctypes.byref(st), ctypes.byref(h))
    assert rc == capi.MC_ERR_INVALID, capi.last_error()
    assert capi.last_error()
    assert not h.value


def test_bad_enums_and_null_state():
    L = capi.lib()
    c = _cfg()
    c.obs_mode = 42
    st = capi.EnvState()
    h = ctypes.c_void_p()
    assert L.mc_env_create(ctypes.byref(c), ctypes.byref(st), ctypes.byref(h)) == capi.MC_ERR_INVALID
    c = _cfg()
    c.numerics = 9
    assert L.mc_env_create(ctypes.byref(c), ctypes.byref(st), ctypes.byref(h)) == capi.MC_ERR_INVALID
    c = _cfg()
    assert L.mc_env_create(ctypes.byref(c), ctypes.byref(st), ctypes.byref(h)) == capi.MC_ERR_INVALID
    assert "NULL" in capi.last_error()


def test_stateless_entry_points_validate_before_launch():
    L = capi.lib()
    assert L.mc_place_tree(None, 1, 8, 8, 8, 9, 2, 4, None) == capi.MC_ERR_INVALID  # tree outside
    assert L.mc_generate_world(None, 1, 0, 8, 8, 4, 0, None) == capi.MC_ERR_INVALID
    assert L.mc_precompute_camera_basis(None, None, 1, 8, 8, 70.0, 7, None) == capi.MC_ERR_INVALID
    assert L.mc_philox_actions(None, -1, 1, 0, 0, 0, 0, None) == capi.MC_ERR_INVALID
    # zero-sized work is a no-op, not an error
    assert L.mc_generate_world(None, 0, 8, 8, 8, 4, 0, None) == capi.MC_OK
    assert L.mc_env_destroy(None) == capi.MC_OK


def test_ragged_entry_points_validate_before_launch():
    L = capi.lib()
    out = ctypes.c_void_p()
    assert L.mc_ragged_create(None, 2, ctypes.byref(out)) == capi.MC_ERR_INVALID
    groups = (ctypes.c_void_p * 17)()
    assert L.mc_ragged_create(groups, 17, ctypes.byref(out)) == capi.MC_ERR_INVALID
    assert "ngroups" in capi.last_error()
    assert L.mc_ragged_create(groups, 2, ctypes.byref(out)) == capi.MC_ERR_INVALID  # NULL groups
    assert not out.value
    assert L.mc_ragged_step_discrete(None, None, None) == capi.MC_ERR_INVALID
    assert L.mc_ragged_rollout(None, None, 4, None) == capi.MC_ERR_INVALID
    assert L.mc_ragged_set_config(None, None) == capi.MC_ERR_INVALID
    assert L.mc_ragged_total_envs(None) == -1
    assert L.mc_ragged_destroy(None) == capi.MC_OK


def test_server_admission_arithmetic_and_config_checks():
    L = capi.lib()
    c = capi.make_config(1000, 16, 16, 16, 32, 32)
    al = lambda n: (n + 255) // 256 * 256  # noqa: E731
    state = (al(1000 * 4096) + 2 * al(12000) + 2 * al(4000) + al(1000) + al(4000) + al(1000) + al(20000)
             + al(1000 * 3072) + al(4000))
    assert L.mc_server_job_bytes(ctypes.byref(c)) == state + al(4096) + 4096
    c.world_x = 0
    assert L.mc_server_job_bytes(ctypes.byref(c)) == -1
    out = ctypes.c_void_p()
    bad = capi.ServerConfig(0, 0, 1, 2, 0)  # no budget
    assert L.mc_server_create(ctypes.byref(bad), ctypes.byref(out)) == capi.MC_ERR_INVALID
    bad = capi.ServerConfig(1 << 30, 0, 1, 9, 0)  # max_inflight
    assert L.mc_server_create(ctypes.byref(bad), ctypes.byref(out)) == capi.MC_ERR_INVALID
    assert "max_inflight" in capi.last_error()
    assert L.mc_server_destroy(None) == capi.MC_OK


def _default_shape(B, W, H, world, obs_dtype, sms=148, aligned=1):
    L = capi.lib()
    c = capi.make_config(B, world, world, world, W, H, obs_dtype=obs_dtype)
    f = capi.FusedConfig()
    smem = ctypes.c_int64(-1)
    rc = L.mc_default_fused_config(ctypes.byref(c), sms, aligned, ctypes.byref(f), ctypes.byref(smem))
    assert rc == capi.MC_OK, capi.last_error()
    return f, smem.value


@pytest.mark.parametrize("B,W,H,world,mode", [
    (32768, 32, 32, 16, "uint8"), (4096, 64, 64, 32, "uint8"), (9472, 64, 64, 16, "uint8"),
    (9472, 320, 320, 16, "float32"), (9472, 1280, 8, 16, "uint8"), (4096, 320, 320, 16, "float32"),
    (20000, 512, 512, 16, "float32"), (2048, 1024, 1024, 16, "float32"), (64, 7, 5, 8, "uint8_minimal"),
    (100, 16, 16, 64, "uint8"),
])
def test_default_launch_shape_fits_shared_memory(B, W, H, world, mode):
    """The default shape of every configuration validates (mc_env_create
    launches it unchanged), including wide float32 images at batches that
    pick one warp per env, whose image band alone can exceed 227 KB."""
    f, smem = _default_shape(B, W, H, world, mode)
    assert 0 < smem <= 227 * 1024, (f.stage, f.warps_per_cta, f.team_warps, f.coop, smem)


def test_default_launch_shape_choices():
    f, _ = _default_shape(32768, 32, 32, 16, "uint8")
    assert (f.stage, f.team_warps, f.coop, f.tile_w) == (1, 1, 0, 4)  # one warp per env, staged
    f, _ = _default_shape(4096, 64, 64, 32, "uint8")
    assert (f.stage, f.team_warps, f.coop) == (1, 4, 1)  # teams over staged 32 KB worlds
    f, _ = _default_shape(9472, 64, 64, 16, "uint8")
    assert (f.team_warps, f.coop) == (1, 0)  # two envs per resident warp: one warp per env
    f, _ = _default_shape(9472, 320, 320, 16, "float32")
    assert f.coop == 1  # the one-warp band does not fit: team shape
    f, _ = _default_shape(32768, 32, 32, 16, "uint8", aligned=0)
    assert f.stage == 0  # bulk copies need 16-byte aligned worlds


def test_normal_build_checks_no_bounds():
    L = capi.lib()
    assert L.mc_build_checks_bounds() == 0
    out = (ctypes.c_int32 * 4)()
    assert L.mc_debug_bounds_report(capi.NUMERICS_IEEE, out, None) == capi.MC_ERR_UNSUPPORTED
    assert L.mc_debug_bounds_selftest(capi.NUMERICS_IEEE, None) == capi.MC_ERR_UNSUPPORTED


def test_checked_build_loads_beside_the_normal_one():
    """The bounds-checked debug build exports the same functions and says it
    checks; loading it does not change which build the normal handle calls."""
    import os
    if not os.path.exists(capi.CHECKED_LIB_PATH):
        pytest.skip("debug build not built")
    C = capi.lib(checked=True)
    missing = [n for n in capi.header_functions() if not hasattr(C, n)]
    assert not missing, missing
    assert C.mc_build_checks_bounds() == 1
    assert capi.lib().mc_build_checks_bounds() == 0
