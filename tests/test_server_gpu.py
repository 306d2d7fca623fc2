"""Env server (mc_server_*): jobs admitted against an HBM budget, step and
reset requests from client threads batched into team-kernel launches.

Every step a job gets from the server must equal MineEnv.step on that job
alone (fused form), bit for bit (floats compared as int32 patterns; the
rewards and dones the server hands back too), with batching on and off.
Failure handling is exercised on the host: over-budget admission, malformed
requests, a client that never collects its results, a busy release.
"""
import threading
import time

import numpy as np
import pytest

from minecu import capi

pytestmark = pytest.mark.gpu

# (batch, world, (res_w, res_h), ground_height, episode_length)
JOBS = [(33, 16, (32, 32), 8, None), (17, 32, (64, 64), 8, 5), (20, 8, (16, 16), 4, None), (9, 24, (24, 16), 8, 7)]
KEYS = ("voxels", "positions", "velocities", "yaws", "pitches", "on_ground", "step_count", "do_reset", "cameras",
        "rewards")


def _bits(torch, t):
    return t.view(torch.int32) if t.dtype == torch.float32 else t


def _env(cuda, b, w, r, gh, el):
    from minecu import MineEnv
    return MineEnv(batch_size=b, world_size=w, render_width=r[0], render_height=r[1], ground_height=gh,
                   episode_length=el, obs_dtype="uint8", device=cuda)


def _admit(srv, b, w, r, gh, el):
    return srv.admit(b, world_size=w, render_width=r[0], render_height=r[1], ground_height=gh, episode_length=el)


@pytest.mark.parametrize("batching", [True, False])
def test_server_steps_equal_mineenv(cuda, batching):
    import torch
    from minecu.server import EnvServer
    srv = EnvServer(hbm_budget_bytes=4e9, batching=batching)
    jobs = [_admit(srv, *j) for j in JOBS]
    envs = [_env(cuda, *j) for j in JOBS]
    for e in envs:
        e.reset()
    rng = np.random.default_rng(5)
    for s in range(12):
        acts = [rng.integers(0, 11, j[0], dtype=np.uint8) for j in JOBS]
        tickets = [srv.submit(job, a) for job, a in zip(jobs, acts)]
        results = [srv.wait(t) for t in tickets]
        for g, (job, e, a, (rew, done)) in enumerate(zip(jobs, envs, acts, results)):
            _, r_ref, d_ref = e.step(torch.from_numpy(a).to(cuda))
            st = srv.state(job)
            torch.cuda.synchronize()
            for k in KEYS:
                assert torch.equal(_bits(torch, st[k]), _bits(torch, getattr(e, k))), f"step {s} job {g}: {k}"
            assert torch.equal(st["obs"], e.obs_buffer), f"step {s} job {g}: obs"
            assert np.array_equal(rew.view(np.int32), r_ref.cpu().numpy().view(np.int32)), f"step {s} job {g}"
            assert np.array_equal(done, d_ref.cpu().numpy()), f"step {s} job {g}: dones"
    # a reset request = MineEnv.reset()
    srv.reset(jobs[0])
    envs[0].reset()
    torch.cuda.synchronize()
    assert torch.equal(srv.state(jobs[0])["obs"], envs[0].obs_buffer)
    st = srv.stats()
    assert st["step_requests"] == 12 * len(JOBS) and st["reset_requests"] == 1
    if batching:
        assert st["mean_jobs_per_launch"] > 1.0
    srv.close()


def test_server_budget_admission_and_release(cuda):
    from minecu.server import EnvServer
    probe = EnvServer(hbm_budget_bytes=1e9)
    a = dict(world_size=16, render_width=32, render_height=32)
    b = dict(world_size=32, render_width=64, render_height=64)
    need = probe.job_bytes(512, **a) + probe.job_bytes(256, **b)
    probe.close()
    srv = EnvServer(hbm_budget_bytes=need - 1)
    ja = srv.admit(512, **a)
    with pytest.raises(MemoryError, match="budget"):
        srv.admit(256, **b)
    assert srv.stats()["bytes_admitted"] == srv.job_bytes(512, **a)
    srv.release(ja)
    assert srv.stats()["bytes_admitted"] == 0
    jb = srv.admit(256, **b)
    srv.step(jb, np.zeros(256, dtype=np.uint8))
    srv.close()


def test_server_rejects_malformed_requests(cuda):
    import ctypes
    from minecu.server import EnvServer
    srv = EnvServer(hbm_budget_bytes=1e9)
    job = srv.admit(16)
    L = capi.lib()
    t = ctypes.c_int64()
    assert L.mc_server_submit(srv._h, 999, capi.REQ_STEP, None, ctypes.byref(t)) == capi.MC_ERR_INVALID
    assert L.mc_server_submit(srv._h, job, 7, None, ctypes.byref(t)) == capi.MC_ERR_INVALID
    assert L.mc_server_submit(srv._h, job, capi.REQ_STEP, None, ctypes.byref(t)) == capi.MC_ERR_INVALID
    assert L.mc_server_wait(srv._h, 12345, None, None, 0) == capi.MC_ERR_INVALID
    assert L.mc_server_release(srv._h, 999) == capi.MC_ERR_INVALID
    with pytest.raises(ValueError):
        srv.submit(job, np.zeros(15, dtype=np.uint8))
    cfg = capi.make_config(16, 16, 16, 16, 32, 32, numerics="ieee")
    jid = ctypes.c_int32()
    assert L.mc_server_admit(srv._h, ctypes.byref(cfg), ctypes.byref(jid)) == capi.MC_ERR_INVALID  # numerics
    # the server still serves well-formed requests
    _, rew, done = srv.step(job, np.ones(16, dtype=np.uint8))
    assert rew.shape == (16,) and done.shape == (16,)
    srv.close()


def test_server_busy_release_and_dropped_client(cuda):
    from minecu.server import EnvServer
    srv = EnvServer(hbm_budget_bytes=8e9)
    big = srv.admit(4096, world_size=32, render_width=64, render_height=64)
    small = srv.admit(64)
    acts = np.zeros(4096, dtype=np.uint8)
    for _ in range(40):  # a client that never collects its results
        srv.submit(big, acts)
    with pytest.raises(RuntimeError, match="queued"):
        srv.release(big)  # requests still queued or running
    # other clients keep being served meanwhile
    _, rew, _ = srv.step(small, np.zeros(64, dtype=np.uint8))
    assert rew.shape == (64,)
    deadline = time.time() + 30
    while True:
        try:
            srv.release(big)
            break
        except RuntimeError:
            assert time.time() < deadline, "the dropped client's requests never drained"
            time.sleep(0.01)
    assert srv.stats()["jobs"] == 1
    srv.close()


def test_server_threads_and_load_generator(cuda):
    from minecu.server import EnvServer
    srv = EnvServer(hbm_budget_bytes=4e9)
    jobs = [srv.admit(256 * (i + 1), world_size=16 if i % 2 else 32, render_width=32, render_height=32)
            for i in range(4)]
    errors = []

    def client(job, n):
        try:
            rng = np.random.default_rng(job)
            for _ in range(n):
                srv.step(job, rng.integers(0, 11, 256 * (job + 1), dtype=np.uint8))
        except Exception as ex:  # reported below
            errors.append(ex)

    th = [threading.Thread(target=client, args=(j, 20)) for j in jobs]
    for t in th:
        t.start()
    for t in th:
        t.join()
    assert not errors
    assert srv.stats()["step_requests"] == 80
    open_loop = srv.drive([(j, 200.0, 50, j + 1) for j in jobs], seconds=0.5)
    assert open_loop["step_requests"] > 0 and open_loop["env_steps"] > 0
    assert 0 < open_loop["p50_us"] <= open_loop["p99_us"] <= open_loop["max_us"]
    closed = srv.drive([(j, 0.0, 0, j + 1) for j in jobs], seconds=0.5, closed_loop=True)
    assert closed["env_steps_per_s"] > 0 and closed["reset_requests"] == 0
    srv.close()


def test_server_rounds_run_a_burst_in_one_launch(cuda):
    """With rounds, a burst of one job's queued requests runs in one launch,
    one round after another: every step's rewards and dones, and each job's
    state afterwards, equal MineEnv stepping the same actions in order (a
    reset request in the middle of a burst included)."""
    import torch
    from minecu.server import EnvServer
    srv = EnvServer(hbm_budget_bytes=4e9, batching=True, rounds=4, max_inflight=1)
    jobs = [_admit(srv, *j) for j in JOBS]
    envs = [_env(cuda, *j) for j in JOBS]
    for e in envs:
        e.reset()
    rng = np.random.default_rng(11)
    for burst in range(4):
        plan = []  # per job: list of ("step", actions) / ("reset", None)
        for g, j in enumerate(JOBS):
            reqs = [("step", rng.integers(0, 11, j[0], dtype=np.uint8)) for _ in range(3)]
            if burst == 2 and g == 1:
                reqs.insert(1, ("reset", None))
            plan.append(reqs)
        tickets = []
        for g, reqs in enumerate(plan):  # every request queued before any runs finishes
            tickets.append([srv.submit(jobs[g], a) if kind == "step" else srv.submit(jobs[g], reset=True)
                            for kind, a in reqs])
        for g, (reqs, ts) in enumerate(zip(plan, tickets)):
            for (kind, a), t in zip(reqs, ts):
                if kind == "reset":
                    srv.wait(t)
                    envs[g].reset()
                    continue
                rew, done = srv.wait(t)
                _, r_ref, d_ref = envs[g].step(torch.from_numpy(a).to(cuda))
                assert np.array_equal(rew.view(np.int32), r_ref.cpu().numpy().view(np.int32)), f"burst {burst} job {g}"
                assert np.array_equal(done, d_ref.cpu().numpy()), f"burst {burst} job {g}: dones"
        torch.cuda.synchronize()
        for g, (job, e) in enumerate(zip(jobs, envs)):
            st = srv.state(job)
            for k in KEYS:
                assert torch.equal(_bits(torch, st[k]), _bits(torch, getattr(e, k))), f"burst {burst} job {g}: {k}"
            assert torch.equal(st["obs"], e.obs_buffer), f"burst {burst} job {g}: obs"
    st = srv.stats()
    assert st["step_requests"] == 4 * 3 * len(JOBS)
    assert st["launches"] < st["step_requests"] / len(JOBS)  # bursts ran in fewer launches than requests per job
    srv.close()
