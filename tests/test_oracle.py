"""The CPU oracle against known answers derived from the reference source
(there are no reference tests or golden vectors; see tests/golden for
fixtures generated by running the reference's own CUDA build)."""
import math

import numpy as np
import pytest

import oracle as O

BLK = dict(AIR=-1, GRASS=0, DIRT=1, OAKLOG=3, LEAVES=4, BRICK=8, COBBLESTONE=9, PLANKS=10, BEDROCK=12)


def test_ieee_trig_accuracy():
    xs = np.linspace(-60.0, 60.0, 4001, dtype=np.float32)
    e_s = max(abs(O.sinf(float(x)) - math.sin(float(x))) for x in xs)
    e_c = max(abs(O.cosf(float(x)) - math.cos(float(x))) for x in xs)
    assert e_s < 2e-7 and e_c < 2e-7
    assert O.sinf(0.0) == 0.0 and O.cosf(0.0) == 1.0
    assert abs(O.tanf(0.6108652) - math.tan(0.6108652)) < 3e-7
    assert math.isnan(O.sinf(float("nan"))) and math.isnan(O.cosf(float("inf")))


def test_ieee_trig_within_one_ulp():
    """The ieee trig (mc_ieee_math.h, one source for the kernels' ieee mode and
    this checker) against the correctly rounded value (float64 math rounded
    to float32) on seeded random inputs: pitches, yaws after many look
    actions, and the whole range the header documents (|x| < 6000).  sin and
    cos are within 1 ulp, tan within 2: the shared source is accurate, not
    only identical on both sides."""
    rng = np.random.default_rng(12)

    def worst_ulp(fn, ref, lo, hi, n=4000):
        worst = 0.0
        for x in rng.uniform(lo, hi, n).astype(np.float32):
            got, want = np.float32(fn(float(x))), np.float32(ref(float(x)))
            worst = max(worst, abs(float(got) - float(want)) / float(np.spacing(np.abs(want))))
        return worst

    for lo, hi in ((-1.6, 1.6), (-math.pi, math.pi), (-100.0, 100.0), (-6000.0, 6000.0)):
        assert worst_ulp(O.sinf, math.sin, lo, hi) <= 1.0, (lo, hi)
        assert worst_ulp(O.cosf, math.cos, lo, hi) <= 1.0, (lo, hi)
    assert worst_ulp(O.tanf, math.tan, 0.01, 1.2) <= 2.0


def test_philox_known_answers():
    """The action stream's block function (mc_philox.h, shared by the kernels
    and this checker) against the published Philox4x32-10 known-answer
    vectors of Salmon et al. (SC'11, the Random123 library)."""
    kat = [((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
           ((0xFFFFFFFF,) * 4, (0xFFFFFFFF, 0xFFFFFFFF), (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
           ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
            (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1))]
    for ctr, key, want in kat:
        assert O.philox4x32_10(ctr, key) == want


def test_world_census_and_structures():
    """generate_world + tree + house (kernels.cu:1793-1946), W=16, gh=8."""
    e = O.OracleEnv(batch_size=2, world_size=16, render_width=4, render_height=4, obs_dtype="uint8")
    v = e.voxels[0]
    assert np.array_equal(e.voxels[0], e.voxels[1])
    assert (v[0] == BLK["BEDROCK"]).all()
    assert (v[1:7] == BLK["DIRT"]).all()
    assert (v[7] == BLK["GRASS"]).all()
    # tree at (x=8, z=10): logs y=8..10, leaves y=11
    assert [v[y, 8, 10] for y in range(8, 12)] == [3, 3, 3, 4]
    # house corner (x=14, z=6), clipped at x=16: floor cobblestone, corner logs,
    # door opening at dx=2 is outside the world here
    assert v[8, 14, 6] == BLK["COBBLESTONE"] and v[8, 15, 9] == BLK["COBBLESTONE"]
    assert v[9, 14, 6] == BLK["OAKLOG"] and v[11, 14, 9] == BLK["OAKLOG"]
    assert v[9, 15, 6] == BLK["PLANKS"] and v[12, 15, 7] == BLK["BRICK"]
    assert v[10, 15, 7] == BLK["AIR"]  # inside the house
    census = {b: int((v[8:] == b).sum()) for b in (3, 4, 8, 9, 10)}
    assert census == {3: 3 + 6, 4: 1, 8: 8, 9: 8, 10: 12}


def test_house_door_in_w32():
    e = O.OracleEnv(batch_size=1, world_size=32, render_width=4, render_height=4, obs_dtype="uint8")
    v = e.voxels[0]
    hx, hz = 22, 14
    assert v[9, hx + 2, hz] == -1 and v[10, hx + 2, hz] == -1 and v[11, hx + 2, hz] == 10  # door 1x2
    assert v[9, hx + 1, hz] == 10 and v[9, hx, hz] == 3


@pytest.mark.parametrize("W,land_y,steps", [(16, 4.0, 15), (32, 8.0, 9)])
def test_fall_trajectory(W, land_y, steps):
    """Physics clamps feet to world_y/4 (kernels.cu:1566): from the spawn at
    y=10 the agent lands at y=W/4 after `steps` steps."""
    e = O.OracleEnv(batch_size=1, world_size=W, render_width=4, render_height=4, obs_dtype="uint8")
    e.reset()
    z8, z2 = np.zeros((1, 8), np.int8), np.zeros((1, 2), np.float32)
    ys = []
    for _ in range(20):
        e.step(z8, z2)
        ys.append(float(e.positions[0, 1]))
    assert ys.index(land_y) + 1 == steps
    assert ys[-1] == land_y and e.on_ground[0] == 1


def test_break_reward_known_answers():
    """At W=32 after landing, breaking at yaw=pitch=0 hits the OAKLOG at
    (16, 9, 18) and pays; before landing the eye at y=11.6 hits LEAVES."""
    z2 = np.zeros((1, 2), np.float32)
    brk = np.zeros((1, 8), np.int8)
    brk[0, 5] = 1
    e = O.OracleEnv(batch_size=1, world_size=32, render_width=4, render_height=4, obs_dtype="uint8", debug=True)
    e.reset()
    e.step(brk, z2)
    y, r = divmod(int(e.dbg_interact[0]), 32 * 32)
    assert (r // 32, y, r % 32) == (16, 11, 18) and e.rewards[0] == 0.0
    e = O.OracleEnv(batch_size=1, world_size=32, render_width=4, render_height=4, obs_dtype="uint8", debug=True)
    e.reset()
    for _ in range(9):
        e.step(np.zeros((1, 8), np.int8), z2)
    e.step(brk, z2)
    y, r = divmod(int(e.dbg_interact[0]), 32 * 32)
    assert (r // 32, y, r % 32) == (16, 9, 18) and e.rewards[0] == 1.0
    assert e.voxels[0, 9, 16, 18] == -1


def test_place_puts_dirt_before_hit():
    e = O.OracleEnv(batch_size=1, world_size=32, render_width=4, render_height=4, obs_dtype="uint8", debug=True)
    e.reset()
    z2 = np.zeros((1, 2), np.float32)
    for _ in range(9):
        e.step(np.zeros((1, 8), np.int8), z2)
    pl = np.zeros((1, 8), np.int8)
    pl[0, 6] = 1
    e.step(pl, z2)
    y, r = divmod(int(e.dbg_interact[0]), 32 * 32)
    assert (r // 32, y, r % 32) == (16, 9, 17) and e.voxels[0, 9, 16, 17] == 1


def test_sky_and_flat_colours():
    """Sky: (135,206,234) truncated in the shaded kernels, (135,206,235) in
    the flat table (kernels.cu:462-469 vs 495)."""
    vox = np.full((1, 16, 16, 16), -1, np.int8)
    cam = np.array([[8, 30, 8, 0, 1.0]], np.float32)
    assert tuple(O.render(O.RENDER_SHADED, False, vox, cam, 4, 4)[0, 0, 0]) == (135, 206, 234)
    assert tuple(O.render(O.RENDER_MINIMAL, False, vox, cam, 4, 4)[0, 0, 0]) == (135, 206, 235)
    f = O.render(O.RENDER_SHADED, True, vox, cam, 4, 4)[0, 0, 0]
    assert np.array_equal(f, np.array([0.53, 0.81, 0.92], np.float32))


def test_buried_camera_sees_dirt():
    """At W=16 the landed eye (y=5.6) is inside DIRT: every shaded pixel is
    the DIRT colour with shade 1 and no fog, every flat pixel the table's."""
    e = O.OracleEnv(batch_size=1, world_size=16, render_width=8, render_height=8, obs_dtype="uint8")
    e.reset()
    for _ in range(16):
        e.step(np.zeros((1, 8), np.int8), np.zeros((1, 2), np.float32))
    assert (e.obs[0] == np.array([140, 89, 51], np.uint8)).all()  # (0.55,0.35,0.20)*255 truncated


def test_episode_rules():
    z8 = np.zeros((4, 8), np.int8)
    z2 = np.zeros((4, 2), np.float32)
    e = O.OracleEnv(batch_size=4, world_size=16, render_width=4, render_height=4, obs_dtype="uint8", episode_length=3)
    e.reset()
    dones = [bool(e.step(z8, z2)[2][0]) for _ in range(9)]
    assert dones == [False, False, False, True, False, False, True, False, False]
    assert list(e.step_count) == [3] * 4
    # kernel rule: episode_length 0 means no limit (kernels.cu:1963)
    e = O.OracleEnv(batch_size=4, world_size=16, render_width=4, render_height=4, obs_dtype="uint8_prebasis_full",
                    episode_length=None)
    e.reset()
    assert not any(bool(e.step(z8, z2)[2][0]) for _ in range(5))


def test_done_regenerates_every_world():
    B = 3
    e = O.OracleEnv(batch_size=B, world_size=16, render_width=4, render_height=4, obs_dtype="uint8", episode_length=2)
    e.reset()
    fresh = e.voxels.copy()
    e.voxels[:, 10, 3, 3] = 5  # a SAND block everywhere
    z2 = np.zeros((B, 2), np.float32)
    e.step(np.zeros((B, 8), np.int8), z2)
    assert (e.voxels[:, 10, 3, 3] == 5).all()
    e.step(np.zeros((B, 8), np.int8), z2)
    e.step(np.zeros((B, 8), np.int8), z2)  # step_count 2 -> done -> regen
    assert np.array_equal(e.voxels, fresh)


def test_philox_stream_is_pure_and_uniform():
    a = O.philox_actions(10000, 7, 1)
    b = O.philox_actions(10000, 7, 1)
    assert np.array_equal(a, b)
    assert a.max() == 10 and a.min() == 0
    counts = np.bincount(a, minlength=11)
    assert counts.min() > 800
    assert not np.array_equal(a, O.philox_actions(10000, 8, 1))
    assert np.array_equal(O.philox_actions(100, 3, 5, env_offset=50), O.philox_actions(150, 3, 5)[50:])
    h = O.philox_actions(20000, 0, 2, break_half=True)
    assert 0.5 < (h == 6).mean() < 0.6


def test_discrete_adapter_table():
    btn, look = O.discrete_to_buttons(np.arange(12, dtype=np.uint8), 0.25)
    assert btn[0].sum() == 0 and (look[0] == 0).all()
    for a, col in zip(range(1, 7), range(6)):
        assert btn[a, col] == 1 and btn[a].sum() == 1
    assert list(look[7]) == [0.25, 0] and list(look[8]) == [-0.25, 0]
    assert list(look[9]) == [0, 0.25] and list(look[10]) == [0, -0.25]
    assert btn[11].sum() == 0 and (look[11] == 0).all()


def test_per_env_regen_rule_on_masked_reset():
    """The oracle's per-env rule (the build's opt-in MC_REGEN_PER_ENV): a
    masked reset returns only the masked envs' worlds to the start world;
    the other worlds keep the blocks broken in them.  Under the reference's
    rule every world returns to the start world."""
    import numpy as np
    from mc_harness import actions_for
    for regen in ("per_env", "all"):
        e = O.OracleEnv(batch_size=6, world_size=16, render_width=8, render_height=8, obs_dtype="uint8",
                        regen=regen)
        e.reset()
        start = e.voxels[0].copy()
        for s in range(8):
            _, btn, look = actions_for(6, s, 3, break_half=True)
            e.step(btn, look)
        before = e.voxels.copy()
        changed = [i for i in range(6) if not np.array_equal(before[i], start)]
        mask = np.array([1, 0, 1, 0, 0, 0], np.uint8)
        assert any(not mask[i] for i in changed), "an unmasked env should have broken a block"
        e.reset(mask)
        for i in range(6):
            if regen == "all" or mask[i]:
                assert np.array_equal(e.voxels[i], start), (regen, i)
            else:
                assert np.array_equal(e.voxels[i], before[i]), (regen, i)
