"""The reference-shaped surface of minecu._C, run on a GPU.

`minecu._C` keeps the reference module's function names, argument order and
defaults (src/bindings.cpp:985-1269), so that the reference's own Python
MineEnv could call it unchanged.  `CStepEnv` below is that Python glue
(minecu/__init__.py:258-444: world generation, reset, the per-mode step
calls with positional arguments, the Python episode rule and counter, the
any-done regeneration), calling this build's `_C` on state tensors laid out
as the reference allocates them (minecu/__init__.py:214-256).  Each step
mode is compared bit for bit with the reference's own CUDA build
(oracle/_ref, driven by oracle/ref_driver.RefEnv) over 30 steps, with an
episode limit so the regeneration path runs.  Tolerance: none.
"""
import pytest

ref_driver = pytest.importorskip("ref_driver")

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref_driver.available(), reason="oracle/_ref/libminecu_ref.so not built")]

STEP_MODES = ["float32", "uint8", "uint8_minimal", "uint8_fp16", "uint8_prebasis", "uint8_prebasis_full",
              "uint8_fast"]


class CStepEnv(ref_driver.RefEnv):
    """The reference MineEnv's glue over this build's minecu._C."""

    def __init__(self, **kw):
        from minecu import _C
        self._C = _C
        super().__init__(**kw)

    def _generate_world(self):
        # minecu/__init__.py:258-268
        C = self._C
        C.generate_world(self.voxels, self.gh, self.seed)
        C.place_tree(self.voxels, self.tree_x, self.tree_z, self.gh)
        C.place_house(self.voxels, self.house_x, self.house_z, self.gh)

    def reset(self, mask=None):
        # minecu/__init__.py:270-302
        if mask is None:
            self.do_reset.fill_(True)
        else:
            self.do_reset.copy_(mask)
        self._C.reset(self.positions, self.velocities, self.yaws, self.pitches, self.on_ground, self.do_reset,
                      self.spawn_x, self.spawn_y, self.spawn_z)
        self.step_count.masked_fill_(self.do_reset, 0)
        if mask is None or mask.any():
            self._generate_world()
        return self._render()

    def _render(self):
        # minecu/__init__.py:446-466
        self.cameras[:, 0] = self.positions[:, 0]
        self.cameras[:, 1] = self.positions[:, 1]
        self.cameras[:, 2] = self.positions[:, 2]
        self.cameras[:, 3] = self.yaws
        self.cameras[:, 4] = self.pitches
        fn = self._C.render if self.obs_dtype == "float32" else self._C.render_uint8
        fn(self.voxels, self.cameras, self.obs_buffer, self.max_steps, self.vd, self.fov)
        return self.obs_buffer

    def _tail(self):
        return (self.obs_buffer, self.rewards, self.W, self.H, self.max_steps, self.vd, self.fov, self.dt, self.g,
                self.walk, self.sprint, self.jump, self.target, self.reward_value, self.spawn_x, self.spawn_y,
                self.spawn_z)

    def _dec(self):
        return (self.forward_in, self.strafe_in, self.delta_yaw_in, self.delta_pitch_in, self.jump_in,
                self.do_break, self.do_place, self.speed_mult, self.cameras)

    def step(self, buttons, look):
        # minecu/__init__.py:304-444, positional arguments as the reference passes them
        C = self._C
        head = (self.voxels, self.positions, self.velocities, self.yaws, self.pitches, self.on_ground, buttons, look)
        if self.obs_dtype == "uint8_prebasis_full":
            C.step_uint8_prebasis_full(*head, self.do_reset, self.step_count, *self._dec(), self.basis,
                                       *self._tail(),
                                       self.episode_length if self.episode_length is not None else 0)
            if self.do_reset.any():
                self._generate_world()
            return self.obs_buffer, self.rewards, self.do_reset.clone()
        if self.episode_length is not None:
            self.do_reset = self.step_count >= self.episode_length  # rebinds, as the reference does
        else:
            self.do_reset.zero_()
        if self.obs_dtype == "uint8_prebasis":
            C.step_uint8_prebasis(*head, self.do_reset, *self._dec(), self.basis, *self._tail())
        elif self.obs_dtype == "uint8_fast":
            C.step_uint8_fast(*head, self.do_reset, *self._dec(), *self._tail(), self.gh)
        else:
            fn = {"uint8_fp16": C.step_uint8_fp16, "uint8_minimal": C.step_uint8_minimal, "uint8": C.step_uint8,
                  "float32": C.step}[self.obs_dtype]
            fn(*head, self.do_reset, *self._dec(), *self._tail())
        self.step_count += 1
        self.step_count.masked_fill_(self.do_reset, 1)
        if self.do_reset.any():
            self._generate_world()
        return self.obs_buffer, self.rewards, self.do_reset.clone()


FIELDS = ("voxels", "positions", "velocities", "yaws", "pitches", "on_ground", "step_count", "do_reset", "cameras",
          "obs_buffer", "rewards", "forward_in", "strafe_in", "delta_yaw_in", "delta_pitch_in", "jump_in",
          "do_break", "do_place", "speed_mult")


@pytest.mark.parametrize("mode", STEP_MODES)
def test_reference_order_step_vs_reference_build(cuda, mode):
    import numpy as np
    import torch
    import oracle as O
    B, steps = 96, 30
    kw = dict(batch_size=B, world_size=16, render_width=32, render_height=24, obs_dtype=mode, device=cuda,
              target_block=3, episode_length=11)
    mine, ref = CStepEnv(**kw), ref_driver.RefEnv(**kw)
    fields = FIELDS + (("basis",) if mode.startswith("uint8_prebasis") else ())

    def compare(what):
        torch.cuda.synchronize()
        for f in fields:
            a, b = getattr(mine, f), getattr(ref, f)
            if a.dtype == torch.float32:
                a, b = a.view(torch.int32), b.view(torch.int32)
            assert torch.equal(a, b), f"{mode} {what}: {f} differs in {int((a != b).sum())} elements"

    mine.reset()
    ref.reset()
    compare("after reset")
    rng = np.random.default_rng(7)
    for s in range(steps):
        if s == 17:
            mask = torch.from_numpy(rng.random(B) < 0.25).to(cuda)
            mine.reset(mask)
            ref.reset(mask)
            compare("after masked reset")
        a = O.philox_actions(B, s, 8, break_half=(s % 2 == 0))
        btn, look = O.discrete_to_buttons(a, 0.1)
        btn[:, 6] = (rng.random(B) < 0.15).astype(np.int8)  # place and sprint, which the discrete table never sets
        btn[:, 7] = (rng.random(B) < 0.3).astype(np.int8)
        b_t, l_t = torch.from_numpy(btn).to(cuda), torch.from_numpy(look).to(cuda)
        _, r_m, d_m = mine.step(b_t, l_t)
        _, r_r, d_r = ref.step(b_t, l_t)
        compare(f"step {s}")
        assert torch.equal(d_m, d_r)


def test_render_entry_points_vs_reference_build(cuda):
    """_C.render / render_uint8 / render_uint8_prebasis / precompute_camera_basis
    with the reference's argument order, on a stepped state."""
    import torch
    import oracle as O
    from minecu import _C
    B = 64
    ref = ref_driver.RefEnv(batch_size=B, world_size=16, render_width=32, render_height=32, obs_dtype="uint8",
                            device=cuda, target_block=3)
    ref.reset()
    for s in range(12):
        btn, look = O.discrete_to_buttons(O.philox_actions(B, s, 5, break_half=True), 0.1)
        ref.step(torch.from_numpy(btn).to(cuda), torch.from_numpy(look).to(cuda))
    L = ref_driver.lib()
    P = ref_driver._p
    for f32 in (False, True):
        out_m = torch.zeros((B, 32, 32, 3), dtype=torch.float32 if f32 else torch.uint8, device=cuda)
        out_r = torch.zeros_like(out_m)
        (_C.render if f32 else _C.render_uint8)(ref.voxels, ref.cameras, out_m, 64, 32.0, 70.0)
        (L.launch_render if f32 else L.launch_render_uint8)(P(ref.voxels), P(ref.cameras), P(out_r), B, 16, 32, 32,
                                                             64, 32.0, 70.0)
        torch.cuda.synchronize()
        a, b = (out_m.view(torch.int32), out_r.view(torch.int32)) if f32 else (out_m, out_r)
        assert torch.equal(a, b), f"render f32={f32}"
    bm = torch.zeros((B, 14), dtype=torch.float32, device=cuda)
    br = torch.zeros_like(bm)
    _C.precompute_camera_basis(ref.cameras, bm, 32, 32, 70.0)
    L.launch_precompute_camera_basis(P(ref.cameras), P(br), B, 32, 32, 70.0)
    torch.cuda.synchronize()
    assert torch.equal(bm.view(torch.int32), br.view(torch.int32))
    om = torch.zeros((B, 32, 32, 3), dtype=torch.uint8, device=cuda)
    orr = torch.zeros_like(om)
    _C.render_uint8_prebasis(ref.voxels, bm, om, 64)
    L.launch_render_uint8_prebasis(P(ref.voxels), P(br), P(orr), B, 16, 32, 32, 64)
    torch.cuda.synchronize()
    assert torch.equal(om, orr)
