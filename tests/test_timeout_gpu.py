"""The bounded wait for a world's bulk copy into shared memory, made to run
out on purpose (mc_env_set_wait_limit(env, 0): every wait gives up at once,
while the copies are still in flight).

A warp whose wait runs out records MC_KERR_TMA_TIMEOUT in the env's error
word, renders that env and every later one from the world in global memory,
and before it leaves waits (with the default bound) for the copy it gave up
on, so no copy lands in shared memory that another CTA may own.  The results
must not change: every state field and observation byte is compared with
the CPU oracle bit for bit (ieee numerics; tolerance none), and
mc_env_check_error must report the timeout.  With the default budget again
no error is recorded.  Nothing here faults, traps or hangs the GPU: the
waits are bounded and the copies are ordinary 4 KB copies that complete.
"""
import pytest

from minecu import capi
import oracle as O
from mc_harness import GpuEnv, actions_for, diff_report, oracle_state

pytestmark = pytest.mark.gpu

CONFIGS = {
    "per_warp": (1, 8, 4, 4, 1, 0),
    "per_warp_depth2": (2, 8, 4, 4, 1, 0),
    "team_coop": (1, 8, 3, 8, 4, 1),
    "team_per_warp": (1, 8, 3, 4, 2, 0),
    "team_coop_depth2": (2, 8, 2, 8, 4, 1),
    "team_per_warp_depth2": (2, 8, 2, 4, 2, 0),
}


@pytest.mark.parametrize("name", sorted(CONFIGS))
@pytest.mark.parametrize("mode", ["uint8", "uint8_minimal"])
def test_copy_timeout_keeps_results_exact(cuda, name, mode):
    L = capi.lib()
    B, steps = 40, 12  # the cameras are above the ground (so their worlds are staged) for the first ~11 steps
    g = GpuEnv(cuda, B, numerics="ieee", obs_dtype=mode, debug=False)
    g.set_fused(*CONFIGS[name])
    o = O.OracleEnv(batch_size=B, world_size=16, render_width=32, render_height=32, obs_dtype=mode)
    capi.check(L.mc_env_set_wait_limit(g.h, 0), "set_wait_limit")
    g.reset()
    o.reset()

    def run(s0, s1):
        for s in range(s0, s1):
            _, btn, look = actions_for(B, s, 23, break_half=True)
            g.step(btn, look, capi.FORM_FUSED)
            o.step(btn, look)
            d = diff_report(g.state(), oracle_state(o))
            assert not d, f"step {s}: {d}"

    run(0, steps)
    rc = L.mc_env_check_error(g.h, None)
    assert rc == capi.MC_ERR_KERNEL, "the waits were made to run out, but no timeout was recorded"
    assert "timed out" in capi.last_error()
    assert L.mc_env_check_error(g.h, None) == capi.MC_OK  # reading the error word cleared it
    capi.check(L.mc_env_set_wait_limit(g.h, -1), "set_wait_limit")  # the default budget
    run(steps, steps + 4)
    g.check_error()
    g.close()


def test_copy_timeout_in_a_ragged_launch(cuda):
    """Ragged groups with one group's waits made to run out: every group
    still equals the same env stepped alone with the default budget."""
    import torch
    from minecu import MineEnv, _C
    from minecu.ragged import RaggedBatch
    groups = [(37, 16, 32), (19, 32, 64), (50, 16, 16)]

    def make():
        return [MineEnv(batch_size=b, world_size=w, render_width=r, render_height=r, obs_dtype="uint8",
                        device=cuda) for b, w, r in groups]

    ra, sb = make(), make()
    batch = RaggedBatch(ra)
    batch.set_launch_config(8, 3, [1, 1, 1], [4, 8, 4], 4, [0, 1, 0])
    ra[1].set_wait_limit(0)
    batch.reset()
    for e in sb:
        e.reset()
    acts = torch.empty((10, batch.total), dtype=torch.uint8, device=cuda)
    _C.philox_actions(acts, 0, 0, 29, True)
    for s in range(10):
        batch.step(acts[s])
        for gi, e in enumerate(sb):
            e.step(acts[s, batch.group_slice(gi)])
        torch.cuda.synchronize()
        for gi, (a, b) in enumerate(zip(ra, sb)):
            for k in ("voxels", "positions", "obs_buffer", "rewards", "do_reset"):
                x, y = getattr(a, k), getattr(b, k)
                if x.dtype == torch.float32:
                    x, y = x.view(torch.int32), y.view(torch.int32)
                assert torch.equal(x, y), f"step {s} group {gi} {k}"
    with pytest.raises(RuntimeError, match="timed out"):
        batch.check_error()
    for e in sb:
        e.check_error()


def test_copy_timeout_depth2_keeps_claimed_envs(cuda):
    """Staging depth 2 with more envs than the grid has warps: every warp
    claims its next env one ahead, so each warp whose wait runs out holds a
    claimed env that it must still step and render from global memory.  The
    result equals the same envs stepped with the default budget (no
    timeouts), bit for bit, at every step."""
    from mc_harness import GpuEnv
    L = capi.lib()
    B = 9600  # above 148 SMs x 4 CTAs x 8 warps: two or more envs per warp
    envs = []
    for limit in (0, -1):
        g = GpuEnv(cuda, B, numerics="ieee", obs_dtype="uint8", debug=False)
        g.set_fused(2, 8, 4, 4, 1, 0)
        capi.check(L.mc_env_set_wait_limit(g.h, limit), "set_wait_limit")
        g.reset()
        envs.append(g)
    timed_out, normal = envs
    for s in range(12):
        _, btn, look = actions_for(B, s, 31, break_half=True)
        timed_out.step(btn, look, capi.FORM_FUSED)
        normal.step(btn, look, capi.FORM_FUSED)
        d = diff_report(timed_out.state(), normal.state())
        assert not d, f"step {s}: {d}"
    assert L.mc_env_check_error(timed_out.h, None) == capi.MC_ERR_KERNEL
    assert "timed out" in capi.last_error()
    normal.check_error()
    for g in envs:
        g.close()
