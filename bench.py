"""Benchmark of the mine.cu environment step on B200.

Workload (the headline "peak shape"): B=32768 envs per GPU, world 16^3,
32x32 RGB uint8 observations (obs_dtype "uint8", the shaded kernels),
max_steps 64, view distance 32, fov 70, target block OAKLOG, no episode
limit; synthetic discrete actions uniform over the 11 actions from a seeded
Philox4x32-10 stream (seed 1; counter = (global env, step)).

Metric: env-steps/s (B x steps x GPUs / time), higher is better.
  value  the fused step (one persistent kernel per step) of K steps captured
         in a CUDA graph, actions resident in HBM, timed with CUDA events on
         the launching stream, max over ranks.
  e2e    MineEnv.step(actions) through the public API, every step copying
         that step's actions from pinned host memory and the step's rewards
         and dones back to pinned host memory (asynchronously, read after the
         timed loop).
  plain  the reference's kernel sequence (one kernel per reference kernel).
The per-step working set (worlds 134 MB + observations 101 MB) exceeds the
126 MB L2, so no flush is done between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W]
  python bench.py --impl reference   # the reference's own CUDA build, same workload

With --gpus N > 1 launch one process per GPU with torch.distributed.run;
each rank steps its own B envs (weak scaling, no collective in the step).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "mine.cu_b200"))

WORKLOAD = dict(workload="peak shape: B=32768 envs/GPU, world 16^3, 32x32x3 uint8 obs (shaded), "
                "uniform discrete actions seed 1", batch_size=32768, world=16, res=32, obs_dtype="uint8",
                max_steps=64, seed=1, look_delta=0.1, break_half=False)
# Render-dominated shape: B=4096, world 32^3, 64x64 uint8, half of the
# actions forced to "break" (world mutation), seed 2, 500 steps.
RENDER_WORKLOAD = dict(workload="render-dominated: B=4096 envs/GPU, world 32^3, 64x64x3 uint8 obs (shaded), "
                       "discrete actions seed 2 with half forced to break", batch_size=4096, world=32, res=64,
                       obs_dtype="uint8", max_steps=64, seed=2, look_delta=0.1, break_half=True)
METRIC = "env-steps/s at B=32K, W=16, 32x32 (fused step, CUDA graph)"
RENDER_METRIC = "env-steps/s at B=4096, W=32, 64x64, half break actions (fused step, CUDA graph)"
# DRAM bytes (read + written) of one launch of the workload's step kernel,
# from the ncu captures summarised in profiles/ (cold caches under ncu)
TRAFFIC = {
    "peak": (113.2e6 + 60.8e6, "k_step_fused, step 701, profiles/k_step_fused_peak_late_full.md"),
    "render": (135.3e6 + 28.4e6, "k_step_team, step 301, profiles/k_step_team_B4096_w32_r64_full.md"),
    "ragged": (70.7e6 + 15.3e6, "k_step_team, mean of its 75 launches, profiles/k_step_team_ragged_launches.md"),
}


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        try:
            d = json.load(open(p))
            return float(d["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle samples while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                if out:
                    self.samples.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.1)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i, v in enumerate(s[5:9]) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


CLOCK_HOLD_S = 0.6


def hold_load(fn, seconds):
    """Replay fn (one timed region's work) for about `seconds`, so that the
    clock sampler sees the GPU under the same load as the timed region."""
    import torch
    t0 = time.perf_counter()
    while time.perf_counter() - t0 < seconds:
        fn()
        torch.cuda.synchronize()


def dist_setup(n_gpus):
    import torch
    import torch.distributed as dist
    if n_gpus > 1 or "RANK" in os.environ:
        rank = int(os.environ.get("RANK", 0))
        world = int(os.environ.get("WORLD_SIZE", 1))
        local = int(os.environ.get("LOCAL_RANK", 0))
        torch.cuda.set_device(local)
        if world > 1:
            import datetime
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                    device_id=torch.device("cuda", local))
        return rank, world, local
    torch.cuda.set_device(0)
    return 0, 1, 0


def barrier(world):
    import torch.distributed as dist
    if world > 1:
        dist.barrier()


def max_over_ranks(x: float, world: int) -> float:
    import torch
    import torch.distributed as dist
    if world == 1:
        return x
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def workload(args):
    """The peak-shape (or render-dominated) workload, or the shape --shape B,W,R asks for (profiling runs)."""
    W = dict(RENDER_WORKLOAD if getattr(args, "workload", "peak") == "render" else WORKLOAD)
    if getattr(args, "shape", ""):
        b, w, r = (int(x) for x in args.shape.split(","))
        W.update(batch_size=b, world=w, res=r,
                 workload=f"B={b} envs/GPU, world {w}^3, {r}x{r}x3 uint8 obs (shaded), uniform discrete actions "
                          f"seed 1")
    return W


def cpu_baseline(seconds=12.0, B=2048, W=WORKLOAD):
    """The CPU restatement of the step (oracle/mc_oracle.c, IEEE numerics,
    OpenMP over envs) on this host's cores, on a bounded sample: B envs of
    the same workload stepped until `seconds` have passed."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    cores = os.cpu_count() or 1
    e = O.OracleEnv(batch_size=B, world_size=W["world"], render_width=W["res"], render_height=W["res"],
                    obs_dtype=W["obs_dtype"], max_steps=W["max_steps"], threads=cores)
    e.reset()
    acts = [O.discrete_to_buttons(O.philox_actions(B, s, W["seed"], break_half=W["break_half"]), W["look_delta"])
            for s in range(64)]
    for s in range(3):  # warm-up
        e.step(*acts[s])
    n, t0 = 0, time.perf_counter()
    while True:
        e.step(*acts[(n + 3) % 64])
        n += 1
        el = time.perf_counter() - t0
        if el >= seconds or n >= 500:
            break
    return {"value": B * n / el, "unit": "env-steps/s", "cores": cores, "kind": "port",
            "sample": f"{B} envs x {n} steps of the same workload ({el:.1f} s), oracle/mc_oracle.c with "
                      f"{cores} OpenMP threads"}


def run_mine(args):
    import torch
    from minecu import MineEnv, _C

    rank, world, local = dist_setup(args.gpus)
    W = workload(args)
    B, K, Wm = W["batch_size"], args.steps, args.warmup
    bytes_per_env_step = W["world"] ** 3 + W["res"] ** 2 * 3
    dev = torch.device("cuda", local)
    env = MineEnv(batch_size=B, world_size=W["world"], render_width=W["res"], render_height=W["res"],
                  device=str(dev), max_steps=W["max_steps"], obs_dtype=W["obs_dtype"], numerics="ref_fast",
                  form="fused", look_delta=W["look_delta"])
    if args.launch:
        env.set_launch_config(*(int(x) for x in args.launch.split(",")))
    stream = torch.cuda.current_stream()
    # every arm below replays steps [0, Wm) untimed and [Wm, Wm+K) timed of
    # the same seeded trajectory, starting from reset(); with --start-state
    # every arm instead starts from a saved state at step Wm (profiling runs
    # of late steps with few launches before the captured one)
    saved = None
    if args.start_state and os.path.exists(args.start_state):
        saved = torch.load(args.start_state, map_location=dev)
        Wm = int(saved["step"])
    acts_w = torch.empty((Wm, B), dtype=torch.uint8, device=dev)
    acts_t = torch.empty((K, B), dtype=torch.uint8, device=dev)
    _C.philox_actions(acts_w, rank * B, 0, W["seed"], W["break_half"])
    _C.philox_actions(acts_t, rank * B, Wm, W["seed"], W["break_half"])

    def start(eager=False):
        """Bring the env to the first timed step of the window."""
        if saved is not None:
            env.load_state_dict(saved["state"])
            return
        env.reset()
        if eager:
            for s in range(Wm):
                env.step(acts_w[s])
        else:
            env.rollout(acts_w)
        if args.start_state and not os.path.exists(args.start_state):
            torch.save({"step": Wm, "state": env.state_dict()}, args.start_state)
    if Wm:
        env.prepare_rollout(acts_w)
    env.prepare_rollout(acts_t)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn):
        torch.cuda.synchronize()
        barrier(world)
        ev0.record(stream)
        fn()
        ev1.record(stream)
        torch.cuda.synchronize()
        barrier(world)
        return max_over_ranks(ev0.elapsed_time(ev1) / 1e3, world)

    # ---- fused step, K steps in one CUDA graph (value) ----------------------
    start()
    with ClockSampler(local) as clk:
        t_fused = timed(lambda: env.rollout(acts_t))
        # a short timed region sees few nvidia-smi samples: keep the same
        # load running under the sampler for a while (not part of the value)
        hold_load(lambda: env.rollout(acts_t), CLOCK_HOLD_S)
    env.check_error()
    value = B * K * world / t_fused

    # ---- same, L2 flushed (a 256 MB write) before every step ----------------
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    start()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    torch.cuda.synchronize()
    for s in range(K):
        flush.fill_(s & 255)
        starts[s].record(stream)
        _C.env_step_discrete(env._env, acts_t[s], 1)
        ends[s].record(stream)
    torch.cuda.synchronize()
    t_flushed = max_over_ranks(sum(a.elapsed_time(b) for a, b in zip(starts, ends)) / 1e3, world)
    del flush

    # ---- plain form (the reference's kernel sequence, eager) ---------------
    env.form = "plain"
    start(eager=True)
    t_plain = timed(lambda: [env.step(acts_t[s]) for s in range(K)])
    plain_value = B * K * world / t_plain
    env.form = "fused"

    # ---- e2e through the public API with host buffers ------------------------
    h_acts = torch.cat([acts_w, acts_t]).cpu().pin_memory()
    h_rew = torch.empty((K, B), dtype=torch.float32).pin_memory()
    h_done = torch.empty((K, B), dtype=torch.bool).pin_memory()
    d_act = torch.empty((B,), dtype=torch.uint8, device=dev)
    start(eager=True)

    def e2e_loop():
        for s in range(K):
            d_act.copy_(h_acts[Wm + s], non_blocking=True)
            obs, rew, done = env.step(d_act)
            h_rew[s].copy_(rew, non_blocking=True)
            h_done[s].copy_(done, non_blocking=True)

    t_e2e_step = timed(e2e_loop)
    _ = float(h_rew.sum())  # the host reads the results

    # the same through MineEnv.step_host: uploads and read-backs on the env's
    # own streams, overlapping the neighbouring steps
    start(eager=True)
    snap = env.state_dict()
    env.step_host(h_acts[Wm], h_rew[0], h_done[0])  # the first call allocates the host-I/O buffers
    env.join_host()
    torch.cuda.synchronize()
    env.load_state_dict(snap)
    del snap
    h_rew.zero_()

    def e2e_host_loop():
        for s in range(K):
            env.step_host(h_acts[Wm + s], h_rew[s], h_done[s])
        env.join_host()

    t_e2e = timed(e2e_host_loop)
    e2e_value = B * K * world / t_e2e
    _ = float(h_rew.sum())

    # the policy input a trainer takes (float32 NCHW obs / 255): one pass over
    # the step's uint8 observation, timed on its own
    policy = None
    if W["obs_dtype"] != "float32":
        pol_out = torch.empty((B, 3, W["res"], W["res"]), dtype=torch.float32, device=dev)
        env.policy_obs(out=pol_out)
        torch.cuda.synchronize()
        n_pol = 20
        e_a, e_b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e_a.record(stream)
        for _ in range(n_pol):
            env.policy_obs(out=pol_out)
        e_b.record(stream)
        torch.cuda.synchronize()
        ms_pol = e_a.elapsed_time(e_b) / n_pol
        pol_bytes = B * W["res"] ** 2 * 3 * 5  # uint8 read + float32 written
        policy = {"ms": ms_pol, "GB_per_s": pol_bytes / (ms_pol * 1e-3) / 1e9, "layout": "NCHW float32 obs/255",
                  "path": "MineEnv.policy_obs (mc_obs_to_policy)"}
        del pol_out

    # the reference's published headline configuration is this shape with
    # float32 observations (49.6 M env-steps/s on an RTX 3090): the same
    # trajectory window with float32 observations, for comparison
    f32 = None
    if args.workload == "peak" and not args.shape and saved is None:
        env32 = MineEnv(batch_size=B, world_size=W["world"], render_width=W["res"], render_height=W["res"],
                        device=str(dev), max_steps=W["max_steps"], obs_dtype="float32", numerics="ref_fast",
                        form="fused", look_delta=W["look_delta"])
        env32.reset()
        if Wm:
            env32.rollout(acts_w)
        env32.prepare_rollout(acts_t)
        t32 = timed(lambda: env32.rollout(acts_t))
        env32.check_error()
        f32 = {"obs_dtype": "float32", "value": B * K * world / t32, "unit": "env-steps/s",
               "ms_per_step": t32 / K * 1e3, "published_rtx3090": 49.6e6,
               "note": "the reference's published number is float32 obs on an RTX 3090 (README.md:11,50)"}
        del env32

    # the other observation modes of the reference's baseline list, same shape and window
    modes = {}
    if f32 is not None:
        modes["float32"] = {"value": f32["value"], "ms_per_step": f32["ms_per_step"]}
        for mode in ("uint8_minimal", "uint8_prebasis_full"):
            env_m = MineEnv(batch_size=B, world_size=W["world"], render_width=W["res"], render_height=W["res"],
                            device=str(dev), max_steps=W["max_steps"], obs_dtype=mode, numerics="ref_fast",
                            form="fused", look_delta=W["look_delta"])
            env_m.reset()
            if Wm:
                env_m.rollout(acts_w)
            env_m.prepare_rollout(acts_t)
            t_m = timed(lambda: env_m.rollout(acts_t))
            env_m.check_error()
            modes[mode] = {"value": B * K * world / t_m, "ms_per_step": t_m / K * 1e3}
            del env_m

    legs = None
    if args.workload == "peak" and not args.shape and saved is None and world == 1 and not args.no_legs:
        legs = mine_legs(args, dev, env, W)

    peak, peak_kind = load_peaks()
    achieved = bytes_per_env_step * B / (t_fused / K) / 1e9
    line = {
        "metric": RENDER_METRIC if args.workload == "render" else METRIC, "value": value, "unit": "env-steps/s",
        "n_gpus": world, "steps": K, "warmup": Wm,
        "ms_per_step": t_fused / K * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (reference world generator, Philox actions)",
        "config": {"workload": W["workload"], "global_batch": B * world, "world": "{0}x{0}x{0}".format(W["world"]),
                   "render": "{0}x{0}x3 uint8".format(W["res"]), "obs_dtype": W["obs_dtype"], "numerics": "ref_fast",
                   "form": "fused persistent kernel, K-step CUDA graph", "launch": env.launch_config(),
                   "parallelism": f"env-sharded x{world} (no collective)",
                   "trajectory": f"steps {Wm}..{Wm + K - 1} after reset(), every arm",
                   "l2": f"per-step working set {bytes_per_env_step * B / 1e6:.0f} MB (worlds + obs); the peak shape's "
                         "235 MB exceeds the 126 MB L2: no flush (l2_flushed: 256 MB write before every step)"},
        "l2_flushed": {"value": B * K * world / t_flushed, "unit": "env-steps/s",
                       "ms_per_step": t_flushed / K * 1e3},
        "plain": {"value": plain_value, "unit": "env-steps/s", "ms_per_step": t_plain / K * 1e3,
                  "fused_speedup": value / plain_value},
        "e2e": {"value": e2e_value, "unit": "env-steps/s", "h2d_bytes_per_step": B,
                "d2h_bytes_per_step": B * 4 + B,
                "path": "MineEnv.step_host per step: pinned host actions in, pinned host rewards+dones out; "
                        "uploads and read-backs overlap the neighbouring steps",
                "step_with_copies": {"value": B * K * world / t_e2e_step, "unit": "env-steps/s",
                                     "path": "MineEnv.step(actions) per step; H2D actions, D2H rewards+dones, "
                                             "one stream"}},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": float(args.traffic_bytes) if args.traffic_bytes else
                     (TRAFFIC[args.workload][0] if not args.shape else None),
                     "traffic_source": "--traffic-bytes" if args.traffic_bytes else
                     (TRAFFIC[args.workload][1] if not args.shape else None), "peak_kind": peak_kind,
                     "algorithmic_bytes_per_env_step": bytes_per_env_step,
                     "kernel": "k_step_fused (avg over the timed region)"},
        "gpu_launches": K,
        "clocks": clk.summary(),
    }
    if f32 is not None:
        line["float32_obs"] = f32
    if modes:
        line["modes"] = modes
    if policy is not None:
        line["policy_obs"] = policy
    if legs is not None:
        line["workloads"] = legs
        line["late_window"] = legs["late_window"]
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args.cpu_seconds, B=min(2048, B // 2) if B > 1 else 1, W=W)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


# Ragged batch: 24,576 envs in 6 uneven groups (batch, world edge, square
# resolution), uint8 shaded observations, discrete actions seed 3.  The
# 8^3 group uses ground height 4 (half its height); with the default 8 its
# whole world would be solid ground.
RAGGED_GROUPS = [(8192, 8, 16), (6144, 16, 32), (4096, 16, 64), (3072, 24, 32), (2048, 32, 32), (1024, 32, 64)]
RAGGED_SEED = 3
RAGGED_METRIC = "env-steps/s, ragged batch of 24,576 envs in 6 groups (one persistent launch, CUDA graph)"


def ragged_ground(w: int) -> int:
    return min(8, w // 2)


def ragged_bytes_per_step(groups=RAGGED_GROUPS) -> int:
    return sum(b * (w ** 3 + r * r * 3) for b, w, r in groups)


def ragged_cpu_baseline(seconds=12.0, scale=16):
    """The oracle (IEEE numerics, OpenMP over envs) on a bounded sample of
    the ragged workload: every group at 1/`scale` of its batch, stepped
    until `seconds` have passed; env-steps/s summed over the groups."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    cores = os.cpu_count() or 1
    envs = []
    for b, w, r in RAGGED_GROUPS:
        e = O.OracleEnv(batch_size=b // scale, world_size=w, render_width=r, render_height=r,
                        ground_height=ragged_ground(w), obs_dtype="uint8", threads=cores)
        e.reset()
        envs.append(e)
    total = sum(e.B for e in envs)
    acts = [O.discrete_to_buttons(O.philox_actions(total, s, RAGGED_SEED), 0.1) for s in range(16)]
    n, t0 = 0, time.perf_counter()
    while True:
        btn, look = acts[n % 16]
        o = 0
        for e in envs:
            e.step(btn[o:o + e.B], look[o:o + e.B])
            o += e.B
        n += 1
        el = time.perf_counter() - t0
        if el >= seconds or n >= 200:
            break
    return {"value": total * n / el, "unit": "env-steps/s", "cores": cores, "kind": "port",
            "sample": f"the 6 groups at 1/{scale} of their batch ({total} envs) x {n} steps ({el:.1f} s), "
                      f"oracle/mc_oracle.c with {cores} OpenMP threads"}


def run_mine_ragged(args):
    import torch
    from minecu import MineEnv, _C
    from minecu.ragged import RaggedBatch
    from minecu import autotune

    rank, world, local = dist_setup(args.gpus)
    dev = torch.device("cuda", local)
    K, Wm = args.steps, args.warmup

    def make(form):
        return [MineEnv(batch_size=b, world_size=w, render_width=r, render_height=r, device=str(dev),
                        ground_height=ragged_ground(w), obs_dtype="uint8", numerics="ref_fast", form=form)
                for b, w, r in RAGGED_GROUPS]

    envs = make("fused")
    batch = RaggedBatch(envs)
    total = batch.total
    t_tune = time.perf_counter()
    if args.no_tune:
        tuned = {"config": {k: v for k, v in batch.launch_config().items() if k != "smem_bytes"}, "trials": 0}
    else:
        tuned = autotune.tune_ragged(batch, use_cache=False)
    t_tune = time.perf_counter() - t_tune
    acts_w = torch.empty((Wm, total), dtype=torch.uint8, device=dev)
    acts_t = torch.empty((K, total), dtype=torch.uint8, device=dev)
    _C.philox_actions(acts_w, rank * total, 0, RAGGED_SEED)
    _C.philox_actions(acts_t, rank * total, Wm, RAGGED_SEED)
    batch.prepare_rollout(acts_w)
    batch.prepare_rollout(acts_t)
    stream = torch.cuda.current_stream()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn):
        torch.cuda.synchronize()
        barrier(world)
        ev0.record(stream)
        fn()
        ev1.record(stream)
        torch.cuda.synchronize()
        barrier(world)
        return max_over_ranks(ev0.elapsed_time(ev1) / 1e3, world)

    # ---- ragged: one persistent launch per step, K steps in one graph -------
    batch.reset()
    batch.rollout(acts_w)
    with ClockSampler(local) as clk:
        t_ragged = timed(lambda: batch.rollout(acts_t))
    batch.check_error()
    value = total * K * world / t_ragged

    # ---- the groups as separate fused launches (6 graphs per K steps) -------
    sl = [batch.group_slice(g) for g in range(len(envs))]
    gw = [acts_w[:, x].contiguous() for x in sl]
    gt = [acts_t[:, x].contiguous() for x in sl]
    for g, e in enumerate(envs):
        c = tuned["config"]
        team = c["team_warps"] if c["coop"][g] else 1
        e.set_launch_config(c["stage"][g], 8, 4, c["tile_w"][g], team_warps=team, coop=c["coop"][g])
        e.prepare_rollout(gw[g])
        e.prepare_rollout(gt[g])
        e.reset()
        e.rollout(gw[g])
    t_sep_fused = timed(lambda: [e.rollout(gt[g]) for g, e in enumerate(envs)])

    # ---- the groups as separate plain launches (the reference's sequence) ---
    for e in envs:
        e.form = "plain"
        e.reset()
    for s in range(Wm):
        for g, e in enumerate(envs):
            e.step(gw[g][s])
    t_plain = timed(lambda: [e.step(gt[g][s]) for s in range(K) for g, e in enumerate(envs)])
    for e in envs:
        e.form = "fused"

    # ---- e2e: RaggedBatch.step with host buffers ----------------------------
    h_acts = torch.cat([acts_w, acts_t]).cpu().pin_memory()
    h_rew = torch.empty((K, total), dtype=torch.float32).pin_memory()
    h_done = torch.empty((K, total), dtype=torch.bool).pin_memory()
    d_act = torch.empty((total,), dtype=torch.uint8, device=dev)
    batch.reset()
    for s in range(Wm):
        d_act.copy_(h_acts[s], non_blocking=True)
        batch.step(d_act)

    def e2e_loop():
        for s in range(K):
            d_act.copy_(h_acts[Wm + s], non_blocking=True)
            res = batch.step(d_act)
            for g, (obs, rew, done) in enumerate(res):
                h_rew[s, sl[g]].copy_(rew, non_blocking=True)
                h_done[s, sl[g]].copy_(done, non_blocking=True)

    t_e2e_step = timed(e2e_loop)
    _ = float(h_rew.sum())

    # the same through RaggedBatch.step_host (uploads and read-backs overlap
    # the neighbouring steps; the launch writes rewards and dones in batch order)
    batch.reset()
    for s in range(Wm):
        batch.step_host(h_acts[s], h_rew[s % K], h_done[s % K])
    batch.join_host()
    torch.cuda.synchronize()
    h_rew.zero_()

    def e2e_host_loop():
        for s in range(K):
            batch.step_host(h_acts[Wm + s], h_rew[s], h_done[s])
        batch.join_host()

    t_e2e = timed(e2e_host_loop)
    _ = float(h_rew.sum())

    peak, peak_kind = load_peaks()
    bps = ragged_bytes_per_step()
    achieved = bps / (t_ragged / K) / 1e9
    line = {
        "metric": RAGGED_METRIC, "value": value, "unit": "env-steps/s", "n_gpus": world, "steps": K, "warmup": Wm,
        "ms_per_step": t_ragged / K * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (reference world generator, Philox actions seed 3)",
        "config": {"workload": "ragged: groups (batch, world, res) " + ", ".join(
            f"({b}, {w}^3, {r}x{r})" for b, w, r in RAGGED_GROUPS) + "; uint8 shaded obs; 8^3 ground height 4",
                   "global_batch": total * world, "numerics": "ref_fast", "launch": tuned["config"],
                   "autotune": {"trials": tuned["trials"], "seconds": round(t_tune, 1)},
                   "parallelism": f"env-sharded x{world} (no collective)",
                   "trajectory": f"steps {Wm}..{Wm + K - 1} after reset(), every arm",
                   "l2": f"per-step working set {bps / 1e6:.0f} MB > 126 MB L2; no flush"},
        "separate_fused": {"value": total * K * world / t_sep_fused, "unit": "env-steps/s",
                           "ms_per_step": t_sep_fused / K * 1e3,
                           "form": "6 fused launches per step (one graph per group, each with the group's "
                                   "tuned tile/staging/team choice)"},
        "separate_plain": {"value": total * K * world / t_plain, "unit": "env-steps/s",
                           "ms_per_step": t_plain / K * 1e3, "ragged_speedup": t_plain / t_ragged,
                           "form": "6 groups x the reference's kernel sequence per step (eager)"},
        "e2e": {"value": total * K * world / t_e2e, "unit": "env-steps/s", "h2d_bytes_per_step": total,
                "d2h_bytes_per_step": total * 5,
                "path": "RaggedBatch.step_host per step: pinned host actions in, pinned host rewards+dones out; "
                        "uploads and read-backs overlap the neighbouring steps",
                "step_with_copies": {"value": total * K * world / t_e2e_step, "unit": "env-steps/s",
                                     "path": "RaggedBatch.step(actions); H2D actions, D2H rewards+dones per group, "
                                             "one stream"}},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": TRAFFIC["ragged"][0], "traffic_source": TRAFFIC["ragged"][1], "peak_kind": peak_kind,
                     "algorithmic_bytes_per_step": bps,
                     "kernel": "k_step_team (avg over the timed region)"},
        "gpu_launches": K * (1 + sum(1 for e in envs if e.episode_length)),
        "clocks": clk.summary(),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = ragged_cpu_baseline(args.cpu_seconds)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


# ---------------------------------------------------------------------------
# Workload legs of the default run: the late trajectory window of the peak
# shape, and the render-dominated, ragged and serving workloads, so that one
# `python bench.py` (and one `--impl reference`) measures all of them.
# ---------------------------------------------------------------------------
LATE_START = 700  # first timed step of the late window (most cameras have dug in by then)
LEG_STEPS = 50    # timed steps of the render and ragged legs
SERVE_LEG_LOADS = (0.8, 0.85)
SERVE_LEG_SECONDS = 3.0  # per level (at 85% load about 17,000 requests a second, p99 = the slowest 1%)


def _event_time(fn):
    import torch
    stream = torch.cuda.current_stream()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / 1e3


def _roof(bytes_per_step, seconds_per_step):
    peak, kind = load_peaks()
    a = bytes_per_step / seconds_per_step / 1e9
    return {"bound": "hbm", "achieved": a, "peak": peak, "unit": "GB/s", "frac": a / peak, "peak_kind": kind}


def mine_legs(args, dev, env, W):
    """This build's legs (see above); `env` is the peak-shape env."""
    import torch
    from minecu import MineEnv, _C, autotune
    from minecu.ragged import RaggedBatch
    from minecu.server import EnvServer
    K, B = args.steps, W["batch_size"]
    legs = {}
    # late window of the peak shape: steps LATE_START.. after reset(), fused graph
    a0 = torch.empty((LATE_START, B), dtype=torch.uint8, device=dev)
    a1 = torch.empty((K, B), dtype=torch.uint8, device=dev)
    _C.philox_actions(a0, 0, 0, W["seed"], W["break_half"])
    _C.philox_actions(a1, 0, LATE_START, W["seed"], W["break_half"])
    env.reset()
    env.rollout(a0)
    env.prepare_rollout(a1)
    t = _event_time(lambda: env.rollout(a1))
    env.check_error()
    bpe = W["world"] ** 3 + W["res"] ** 2 * 3
    legs["late_window"] = {"value": B * K / t, "unit": "env-steps/s", "ms_per_step": t / K * 1e3,
                           "trajectory": f"steps {LATE_START}..{LATE_START + K - 1} after reset()",
                           "roofline": _roof(bpe * B, t / K)}
    del a0, a1
    # render-dominated: B=4096, 32^3, 64x64, half break actions
    R = RENDER_WORKLOAD
    Wm = args.warmup
    er = MineEnv(batch_size=R["batch_size"], world_size=R["world"], render_width=R["res"], render_height=R["res"],
                 device=str(dev), max_steps=R["max_steps"], obs_dtype="uint8", look_delta=R["look_delta"])
    aw = torch.empty((Wm, R["batch_size"]), dtype=torch.uint8, device=dev)
    at = torch.empty((LEG_STEPS, R["batch_size"]), dtype=torch.uint8, device=dev)
    _C.philox_actions(aw, 0, 0, R["seed"], True)
    _C.philox_actions(at, 0, Wm, R["seed"], True)
    er.reset()
    er.rollout(aw)
    er.prepare_rollout(at)
    t = _event_time(lambda: er.rollout(at))
    er.check_error()
    er.form = "plain"
    er.reset()
    for s_ in range(Wm):
        er.step(aw[s_])
    tp = _event_time(lambda: [er.step(at[s_]) for s_ in range(LEG_STEPS)])
    bpr = R["world"] ** 3 + R["res"] ** 2 * 3
    legs["render"] = {"workload": R["workload"], "value": R["batch_size"] * LEG_STEPS / t, "unit": "env-steps/s",
                      "ms_per_step": t / LEG_STEPS * 1e3, "plain_ms_per_step": tp / LEG_STEPS * 1e3,
                      "launch": er.launch_config(), "trajectory": f"steps {Wm}..{Wm + LEG_STEPS - 1} after reset()",
                      "roofline": _roof(bpr * R["batch_size"], t / LEG_STEPS)}
    del er, aw, at
    # ragged: 24,576 envs in 6 groups, autotuned (a short search), one launch per step
    envs = [MineEnv(batch_size=b, world_size=w, render_width=r, render_height=r, device=str(dev),
                    ground_height=ragged_ground(w), obs_dtype="uint8") for b, w, r in RAGGED_GROUPS]
    batch = RaggedBatch(envs)
    t_tune = time.perf_counter()
    tuned = autotune.tune_ragged(batch, steps=10, warm_steps=20, rounds=1, use_cache=False)
    t_tune = time.perf_counter() - t_tune
    total = batch.total
    aw = torch.empty((Wm, total), dtype=torch.uint8, device=dev)
    at = torch.empty((LEG_STEPS, total), dtype=torch.uint8, device=dev)
    _C.philox_actions(aw, 0, 0, RAGGED_SEED)
    _C.philox_actions(at, 0, Wm, RAGGED_SEED)
    batch.reset()
    batch.rollout(aw)
    batch.prepare_rollout(at)
    t = _event_time(lambda: batch.rollout(at))
    batch.check_error()
    legs["ragged"] = {"workload": "ragged: 6 groups " + ", ".join(f"({b}, {w}^3, {r}x{r})" for b, w, r in
                                                                 RAGGED_GROUPS),
                      "value": total * LEG_STEPS / t, "unit": "env-steps/s", "ms_per_step": t / LEG_STEPS * 1e3,
                      "launch": tuned["config"], "autotune": {"trials": tuned["trials"], "seconds": round(t_tune, 1)},
                      "trajectory": f"steps {Wm}..{Wm + LEG_STEPS - 1} after reset()",
                      "roofline": _roof(ragged_bytes_per_step(), t / LEG_STEPS)}
    del batch, envs, aw, at
    # serving: closed-loop peak, then Poisson arrivals at 80% and 85% of it
    jobs = serve_jobs()
    srv = EnvServer(hbm_budget_bytes=150e9, batching=True, max_inflight=2, max_envs_per_launch=16384, device=dev)
    ids = [srv.admit(j["batch"], world_size=j["world"], render_width=j["res"], render_height=j["res"]) for j in jobs]
    srv.drive([(i, 0.0, 0, k + 1) for k, i in enumerate(ids)], seconds=0.3, closed_loop=True)  # warm-up
    pk = srv.drive([(i, 0.0, j["episode"], k + 1) for k, (i, j) in enumerate(zip(ids, jobs))],
                   seconds=SERVE_LEG_SECONDS, closed_loop=True)
    ntot = sum(j["batch"] for j in jobs)
    loads = []
    for frac in SERVE_LEG_LOADS:
        st = srv.drive([(i, frac * pk["env_steps_per_s"] / ntot, j["episode"], k + 1)
                        for k, (i, j) in enumerate(zip(ids, jobs))], seconds=SERVE_LEG_SECONDS)
        loads.append({"offered_frac": frac, "env_steps_per_s": st["env_steps_per_s"], "p50_us": st["p50_us"],
                      "p99_us": st["p99_us"], "max_us": st["max_us"]})
    srv.close()
    mean_bytes = sum(j["batch"] * (j["world"] ** 3 + j["res"] ** 2 * 3) for j in jobs) / ntot
    legs["serve"] = {"workload": "16 jobs (batch 256..8192 log-uniform, 16^3 or 32^3, 32x32 or 64x64), Poisson "
                                 "arrivals, HBM budget 150 GB",
                     "closed_loop_env_steps_per_s": pk["env_steps_per_s"], "closed_loop_p99_us": pk["p99_us"],
                     "loads": loads, "seconds_per_level": SERVE_LEG_SECONDS,
                     "roofline_at_closed_loop": _roof(mean_bytes * pk["env_steps_per_s"], 1.0)}
    return legs


def reference_legs(args, dev, W):
    """The reference build's legs: the late window of the peak shape and
    the render-dominated and ragged workloads (it has no server)."""
    import torch
    import oracle as O
    import ref_driver
    K, B = args.steps, W["batch_size"]

    def buttons(n, s0, steps, seed, break_half):
        bt = torch.empty((steps, n, 8), dtype=torch.int8)
        lk = torch.empty((steps, n, 2), dtype=torch.float32)
        for s_ in range(steps):
            b_, l_ = O.discrete_to_buttons(O.philox_actions(n, s0 + s_, seed, break_half=break_half), 0.1)
            bt[s_] = torch.from_numpy(b_)
            lk[s_] = torch.from_numpy(l_)
        return bt.to(dev), lk.to(dev)

    legs = {}
    env = ref_driver.RefEnv(batch_size=B, world_size=W["world"], render_width=W["res"], render_height=W["res"],
                            device=str(dev), max_steps=W["max_steps"], obs_dtype=W["obs_dtype"], target_block=3)
    bw, lw = buttons(B, 0, LATE_START, W["seed"], W["break_half"])
    bt, lt = buttons(B, LATE_START, K, W["seed"], W["break_half"])
    env.reset()
    for s_ in range(LATE_START):
        env.step(bw[s_], lw[s_])
    t = _event_time(lambda: [env.step(bt[s_], lt[s_]) for s_ in range(K)])
    legs["late_window"] = {"value": B * K / t, "unit": "env-steps/s", "ms_per_step": t / K * 1e3,
                           "trajectory": f"steps {LATE_START}..{LATE_START + K - 1} after reset()"}
    del env, bw, lw, bt, lt
    R = RENDER_WORKLOAD
    Wm = args.warmup
    env = ref_driver.RefEnv(batch_size=R["batch_size"], world_size=R["world"], render_width=R["res"],
                            render_height=R["res"], device=str(dev), max_steps=R["max_steps"], obs_dtype="uint8",
                            target_block=3)
    bw, lw = buttons(R["batch_size"], 0, Wm, R["seed"], True)
    bt, lt = buttons(R["batch_size"], Wm, LEG_STEPS, R["seed"], True)
    env.reset()
    for s_ in range(Wm):
        env.step(bw[s_], lw[s_])
    t = _event_time(lambda: [env.step(bt[s_], lt[s_]) for s_ in range(LEG_STEPS)])
    legs["render"] = {"workload": R["workload"], "value": R["batch_size"] * LEG_STEPS / t, "unit": "env-steps/s",
                      "ms_per_step": t / LEG_STEPS * 1e3,
                      "trajectory": f"steps {Wm}..{Wm + LEG_STEPS - 1} after reset()"}
    del env, bw, lw, bt, lt
    envs = [ref_driver.RefEnv(batch_size=b, world_size=w, render_width=r, render_height=r, device=str(dev),
                              ground_height=ragged_ground(w), obs_dtype="uint8", target_block=3)
            for b, w, r in RAGGED_GROUPS]
    total = sum(b for b, _, _ in RAGGED_GROUPS)
    offs = [0]
    for b, _, _ in RAGGED_GROUPS:
        offs.append(offs[-1] + b)
    bw, lw = buttons(total, 0, Wm, RAGGED_SEED, False)
    bt, lt = buttons(total, Wm, LEG_STEPS, RAGGED_SEED, False)
    gb = [(bw[:, offs[g]:offs[g + 1]].contiguous(), lw[:, offs[g]:offs[g + 1]].contiguous(),
           bt[:, offs[g]:offs[g + 1]].contiguous(), lt[:, offs[g]:offs[g + 1]].contiguous())
          for g in range(len(envs))]
    for e in envs:
        e.reset()
    for s_ in range(Wm):
        for g, e in enumerate(envs):
            e.step(gb[g][0][s_], gb[g][1][s_])
    t = _event_time(lambda: [e.step(gb[g][2][s_], gb[g][3][s_]) for s_ in range(LEG_STEPS)
                             for g, e in enumerate(envs)])
    legs["ragged"] = {"workload": "ragged: the same 6 groups, one reference MineEnv each, stepped in turn",
                      "value": total * LEG_STEPS / t, "unit": "env-steps/s", "ms_per_step": t / LEG_STEPS * 1e3,
                      "trajectory": f"steps {Wm}..{Wm + LEG_STEPS - 1} after reset()"}
    legs["serve"] = {"unavailable": "the reference has no env server"}
    return legs


REF_PKG = os.path.join(ROOT, "baseline", "_ref")
STATE_KEYS = ("voxels", "positions", "velocities", "yaws", "pitches", "on_ground", "step_count", "do_reset",
              "cameras", "rewards", "obs_buffer")


def run_stock_leg(args):
    """--stock-leg (run by the reference arm in a child process): the
    headline window through the reference package itself, built by its own
    setup.py into baseline/_ref: minecu.MineEnv(...).step(buttons, look)
    with persistent action buffers (its graphs keep the action pointers,
    src/kernels.cu:2526-2542).  After the window, every state tensor is
    compared bit for bit with the restated driver (oracle/ref_driver.py)
    stepped with the same actions: that is the check that the reference
    arm's driver runs the reference's own step."""
    import torch
    sys.path[:] = [q for q in sys.path if os.path.abspath(q) != os.path.join(ROOT, "mine.cu_b200")]
    sys.path.insert(0, REF_PKG)
    sys.path.insert(1, os.path.join(ROOT, "oracle"))
    import minecu as stock
    if not os.path.abspath(stock.__file__).startswith(REF_PKG):
        raise RuntimeError(f"expected the reference package from {REF_PKG}, got {stock.__file__}")
    import oracle as O
    import ref_driver
    W = workload(args)
    B, K, Wm = W["batch_size"], args.steps, args.warmup
    dev = torch.device("cuda", 0)
    btns = torch.empty((K + Wm, B, 8), dtype=torch.int8)
    looks = torch.empty((K + Wm, B, 2), dtype=torch.float32)
    for s in range(K + Wm):
        b, l = O.discrete_to_buttons(O.philox_actions(B, s, W["seed"], break_half=W["break_half"]), W["look_delta"])
        btns[s] = torch.from_numpy(b)
        looks[s] = torch.from_numpy(l)
    d_btn, d_look = btns.to(dev), looks.to(dev)
    kw = dict(batch_size=B, world_size=W["world"], render_width=W["res"], render_height=W["res"], device=str(dev),
              max_steps=W["max_steps"], obs_dtype=W["obs_dtype"], target_block=3)
    env = stock.MineEnv(**kw)
    pb = torch.zeros((B, 8), dtype=torch.int8, device=dev)
    pl = torch.zeros((B, 2), dtype=torch.float32, device=dev)

    def step(s):
        pb.copy_(d_btn[s])
        pl.copy_(d_look[s])
        env.step(pb, pl)
    env.reset()
    for s in range(Wm):
        step(s)
    t = _event_time(lambda: [step(Wm + s) for s in range(K)])
    ref = ref_driver.RefEnv(**kw)
    ref.reset()
    for s in range(Wm + K):
        ref.step(d_btn[s], d_look[s])
    torch.cuda.synchronize()

    def bits(x):
        return x.view(torch.int32) if x.dtype == torch.float32 else x
    differ = [k for k in STATE_KEYS if not torch.equal(bits(getattr(env, k)), bits(getattr(ref, k)))]
    print("STOCK " + json.dumps({
        "path": "baseline/_ref: the reference package built by its own setup.py (pip install --target, "
                "TORCH_CUDA_ARCH_LIST=10.0a), minecu.MineEnv.step(buttons, look), default stream",
        "value": B * K / t, "unit": "env-steps/s", "ms_per_step": t / K * 1e3,
        "trajectory": f"steps {Wm}..{Wm + K - 1} after reset()",
        "state_equal_to_restated_driver": not differ, "differing": differ}), flush=True)


def stock_leg(args):
    """The stock package's line for the reference arm (None when baseline/_ref is not installed)."""
    if not os.path.exists(os.path.join(REF_PKG, "minecu", "__init__.py")):
        return {"unavailable": "baseline/_ref is not installed"}
    r = subprocess.run([sys.executable, os.path.abspath(__file__), "--stock-leg", "--steps", str(args.steps),
                        "--warmup", str(args.warmup)], capture_output=True, text=True, timeout=900)
    for ln in r.stdout.splitlines():
        if ln.startswith("STOCK "):
            return json.loads(ln[6:])
    return {"unavailable": f"stock-package leg failed (rc {r.returncode}): {r.stderr.strip()[-300:]}"}


def run_reference(args):
    """The reference's own CUDA build (oracle/_ref/libminecu_ref.so, its
    src/kernels.cu compiled unmodified) driven in its MineEnv.step order, on
    the same workload.  The reference has no CPU implementation; its stock
    implementation of this path is these kernels."""
    import torch
    rank, world, local = dist_setup(args.gpus)
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    import ref_driver
    W = workload(args)
    if not ref_driver.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libminecu_ref.so not built"}))
        return
    B, K, Wm = W["batch_size"], args.steps, args.warmup
    dev = torch.device("cuda", local)
    env = ref_driver.RefEnv(batch_size=B, world_size=W["world"], render_width=W["res"], render_height=W["res"],
                            device=str(dev), max_steps=W["max_steps"], obs_dtype=W["obs_dtype"], target_block=3)
    Kr = K
    btns = torch.empty((Kr + Wm, B, 8), dtype=torch.int8)
    looks = torch.empty((Kr + Wm, B, 2), dtype=torch.float32)
    for s in range(Kr + Wm):
        b, l = O.discrete_to_buttons(O.philox_actions(B, s, W["seed"], break_half=W["break_half"]),
                                     W["look_delta"])
        btns[s] = torch.from_numpy(b)
        looks[s] = torch.from_numpy(l)
    d_btn, d_look = btns.to(dev), looks.to(dev)
    env.reset()
    for s in range(Wm):
        env.step(d_btn[s], d_look[s])
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for s in range(Kr):
        env.step(d_btn[Wm + s], d_look[Wm + s])
    ev1.record(stream)
    torch.cuda.synchronize()
    t = ev0.elapsed_time(ev1) / 1e3
    value = B * Kr / t
    # e2e: actions from pinned host memory, rewards + dones back, every step
    h_btn, h_look = btns.pin_memory(), looks.pin_memory()
    h_rew = torch.empty((Kr, B), dtype=torch.float32).pin_memory()
    h_done = torch.empty((Kr, B), dtype=torch.bool).pin_memory()
    env.reset()
    for s in range(Wm):
        env.step(d_btn[s], d_look[s])
    torch.cuda.synchronize()
    ev0.record(stream)
    for s in range(Kr):
        obs, rew, done = env.step(h_btn[Wm + s].to(dev, non_blocking=True), h_look[Wm + s].to(dev, non_blocking=True))
        h_rew[s].copy_(rew, non_blocking=True)
        h_done[s].copy_(done, non_blocking=True)
    ev1.record(stream)
    torch.cuda.synchronize()
    te = ev0.elapsed_time(ev1) / 1e3
    e2e = B * Kr / te
    # the other observation modes, same shape and window
    modes = {}
    if args.workload == "peak" and not args.shape:
        for mode in ("float32", "uint8_minimal", "uint8_prebasis_full"):
            env_m = ref_driver.RefEnv(batch_size=B, world_size=W["world"], render_width=W["res"],
                                      render_height=W["res"], device=str(dev), max_steps=W["max_steps"],
                                      obs_dtype=mode, target_block=3)
            env_m.reset()
            for s in range(Wm):
                env_m.step(d_btn[s], d_look[s])
            torch.cuda.synchronize()
            ev0.record(stream)
            for s in range(Kr):
                env_m.step(d_btn[Wm + s], d_look[Wm + s])
            ev1.record(stream)
            torch.cuda.synchronize()
            t_m = ev0.elapsed_time(ev1) / 1e3
            modes[mode] = {"value": B * Kr / t_m, "ms_per_step": t_m / Kr * 1e3}
            del env_m
    line = {
        "impl": "reference", "metric": RENDER_METRIC if args.workload == "render" else METRIC, "value": value,
        "unit": "env-steps/s", "n_gpus": 1, "steps": Kr,
        "warmup": Wm, "ms_per_step": t / Kr * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (reference world generator, Philox actions)",
        "config": {"workload": W["workload"], "global_batch": B, "world": "{0}x{0}x{0}".format(W["world"]),
                   "render": "{0}x{0}x3 uint8".format(W["res"]), "obs_dtype": W["obs_dtype"],
                   "trajectory": f"steps {Wm}..{Wm + Kr - 1} after reset()",
                   "path": "reference src/kernels.cu launch_step_uint8 + MineEnv.step glue (eager, default stream)"},
        "e2e": {"value": e2e, "unit": "env-steps/s", "h2d_bytes_per_step": B * 16, "d2h_bytes_per_step": B * 5},
        "cpu_baseline": {"value": value, "unit": "env-steps/s", "cores": None, "kind": "reference",
                         "sample": f"{Kr} steps of B={B}; the reference implementation is CUDA-only, so this arm "
                                   "runs its own kernels on the same B200"},
    }
    if modes:
        line["modes"] = modes
    if args.workload == "peak" and not args.shape:
        # the same window through the stock package, as a cross-check of this arm's driver
        line["stock_package"] = stock_leg(args)
    if args.workload == "peak" and not args.shape and not args.no_legs:
        del env
        legs = reference_legs(args, dev, W)
        line["workloads"] = legs
        line["late_window"] = legs["late_window"]
    print(json.dumps(line), flush=True)


# Serving: 16 client jobs, batch log-uniform in [256, 8192], world 16^3 or
# 32^3, 32x32 or 64x64 uint8 observations, episodes of 200..2000 steps (a
# reset request between episodes), Poisson arrivals at the same request rate
# for every job (offered env-steps/s = rate x total envs), HBM budget 150 GB.
# The server queues up to 2 launches on the device and caps one launch at
# 16,384 envs.
SERVE_SEED = 5
SERVE_LOADS = (0.2, 0.4, 0.6, 0.8, 0.85, 0.9, 0.95, 1.0, 1.2)
SERVE_METRIC = "served env-steps/s at p99 step latency < 2 ms (16 jobs, mixed sizes, Poisson arrivals)"


def serve_jobs(n=16, seed=SERVE_SEED):
    import numpy as np
    rng = np.random.default_rng(seed)
    jobs = []
    for _ in range(n):
        b = int(round(float(np.exp(rng.uniform(np.log(256), np.log(8192))))))
        jobs.append(dict(batch=b, world=int(rng.choice([16, 32])), res=int(rng.choice([32, 64])),
                         episode=int(rng.integers(200, 2001))))
    return jobs


def run_mine_serve(args):
    import torch
    from minecu.server import EnvServer

    rank, world, local = dist_setup(args.gpus)
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    jobs = serve_jobs()
    secs = args.serve_seconds

    def make(batching):
        srv = EnvServer(hbm_budget_bytes=150e9, batching=batching, max_inflight=2, max_envs_per_launch=16384,
                        device=dev)
        ids = [srv.admit(j["batch"], world_size=j["world"], render_width=j["res"], render_height=j["res"])
               for j in jobs]
        return srv, ids

    def sweep(srv, ids, peak):
        out = []
        total = sum(j["batch"] for j in jobs)
        for frac in SERVE_LOADS:
            rates = [frac * peak / total for _ in jobs]
            st = srv.drive([(i, r, j["episode"], k + 1) for k, (i, r, j) in enumerate(zip(ids, rates, jobs))],
                           seconds=secs)
            out.append({"offered_frac": frac, "offered_env_steps_per_s": frac * peak,
                        "env_steps_per_s": st["env_steps_per_s"], "p50_us": st["p50_us"], "p99_us": st["p99_us"],
                        "max_us": st["max_us"], "step_requests": st["step_requests"],
                        "reset_requests": st["reset_requests"], "mean_jobs_per_launch": st["mean_jobs_per_launch"]})
        return out

    results = {}
    with ClockSampler(local) as clk:
        for name, batching in (("batched", True), ("plain", False)):
            srv, ids = make(batching)
            srv.drive([(i, 0.0, 0, k + 1) for k, i in enumerate(ids)], seconds=0.5, closed_loop=True)  # warm-up
            peak = srv.drive([(i, 0.0, j["episode"], k + 1) for k, (i, j) in enumerate(zip(ids, jobs))],
                             seconds=secs, closed_loop=True)
            results[name] = {"closed_loop_env_steps_per_s": peak["env_steps_per_s"],
                             "closed_loop_p50_us": peak["p50_us"], "closed_loop_p99_us": peak["p99_us"]}
            if name == "batched":
                ref_peak = peak["env_steps_per_s"]
            results[name]["sweep"] = sweep(srv, ids, ref_peak)
            srv.close()
    ok = [r for r in results["batched"]["sweep"] if r["p99_us"] < 2000.0]
    value = max((r["env_steps_per_s"] for r in ok), default=0.0)
    plain_ok = [r for r in results["plain"]["sweep"] if r["p99_us"] < 2000.0]
    peak, peak_kind = load_peaks()
    mean_bytes = sum(j["batch"] * (j["world"] ** 3 + j["res"] ** 2 * 3) for j in jobs) / sum(j["batch"] for j in jobs)
    achieved = value * mean_bytes / 1e9
    line = {
        "metric": SERVE_METRIC, "value": value, "unit": "env-steps/s", "n_gpus": world, "steps": None,
        "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (reference world generator, Philox actions)",
        "config": {"workload": "serving: 16 jobs " + ", ".join(f"({j['batch']}, {j['world']}^3, {j['res']}^2, "
                                                               f"ep {j['episode']})" for j in jobs),
                   "hbm_budget_bytes": 150e9, "arrivals": "Poisson per job, the same request rate for every job",
                   "server": {"max_inflight": 2, "max_envs_per_launch": 16384},
                   "offered_loads": list(SERVE_LOADS), "seconds_per_level": secs, "numerics": "ref_fast",
                   "latency": "request submission to rewards/dones in host memory"},
        "batched": results["batched"], "plain_one_job_at_a_time": results["plain"],
        "sustained_vs_closed_loop_peak": value / results["batched"]["closed_loop_env_steps_per_s"]
        if results["batched"]["closed_loop_env_steps_per_s"] else None,
        "plain_value": max((r["env_steps_per_s"] for r in plain_ok), default=0.0),
        "e2e": {"value": value, "unit": "env-steps/s", "h2d_bytes_per_step": None, "d2h_bytes_per_step": None,
                "path": "EnvServer requests: host actions in, host rewards+dones out (every request)"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": None, "peak_kind": peak_kind, "algorithmic_bytes_per_env_step": mean_bytes,
                     "kernel": "k_step_team (served launches)"},
        "clocks": clk.summary(),
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def run_reference_ragged(args):
    """The ragged workload on the reference's own CUDA build: the reference
    runs one world size and resolution per MineEnv, so the 6 groups are 6
    envs stepped one after another each step (its plain per-group form)."""
    import torch
    rank, world, local = dist_setup(args.gpus)
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    import ref_driver
    if not ref_driver.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libminecu_ref.so not built"}))
        return
    K, Wm = args.steps, args.warmup
    dev = torch.device("cuda", local)
    envs = [ref_driver.RefEnv(batch_size=b, world_size=w, render_width=r, render_height=r, device=str(dev),
                              ground_height=ragged_ground(w), obs_dtype="uint8", target_block=3)
            for b, w, r in RAGGED_GROUPS]
    total = sum(b for b, _, _ in RAGGED_GROUPS)
    btns = torch.empty((K + Wm, total, 8), dtype=torch.int8)
    looks = torch.empty((K + Wm, total, 2), dtype=torch.float32)
    for s in range(K + Wm):
        b, l = O.discrete_to_buttons(O.philox_actions(total, s, RAGGED_SEED), 0.1)
        btns[s] = torch.from_numpy(b)
        looks[s] = torch.from_numpy(l)
    offs = [0]
    for b, _, _ in RAGGED_GROUPS:
        offs.append(offs[-1] + b)
    d_btn = [btns[:, offs[g]:offs[g + 1]].contiguous().to(dev) for g in range(len(envs))]
    d_look = [looks[:, offs[g]:offs[g + 1]].contiguous().to(dev) for g in range(len(envs))]

    def run(s0, n):
        for s in range(s0, s0 + n):
            for g, e in enumerate(envs):
                e.step(d_btn[g][s], d_look[g][s])

    for e in envs:
        e.reset()
    run(0, Wm)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    run(Wm, K)
    ev1.record(stream)
    torch.cuda.synchronize()
    t = ev0.elapsed_time(ev1) / 1e3
    value = total * K / t
    # e2e: actions from pinned host memory, rewards + dones back, every step
    h_btn, h_look = btns.pin_memory(), looks.pin_memory()
    h_rew = torch.empty((K, total), dtype=torch.float32).pin_memory()
    h_done = torch.empty((K, total), dtype=torch.bool).pin_memory()
    for e in envs:
        e.reset()
    run(0, Wm)
    torch.cuda.synchronize()
    ev0.record(stream)
    for s in range(K):
        for g, e in enumerate(envs):
            sl = slice(offs[g], offs[g + 1])
            obs, rew, done = e.step(h_btn[Wm + s, sl].to(dev, non_blocking=True),
                                    h_look[Wm + s, sl].to(dev, non_blocking=True))
            h_rew[s, sl].copy_(rew, non_blocking=True)
            h_done[s, sl].copy_(done, non_blocking=True)
    ev1.record(stream)
    torch.cuda.synchronize()
    te = ev0.elapsed_time(ev1) / 1e3
    line = {
        "impl": "reference", "metric": RAGGED_METRIC, "value": value, "unit": "env-steps/s", "n_gpus": 1,
        "steps": K, "warmup": Wm, "ms_per_step": t / K * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (reference world generator, Philox actions seed 3)",
        "config": {"workload": "ragged: the same 6 groups, one reference MineEnv each, stepped in turn",
                   "global_batch": total, "trajectory": f"steps {Wm}..{Wm + K - 1} after reset()",
                   "path": "reference src/kernels.cu launch_step_uint8 + MineEnv.step glue per group (eager)"},
        "e2e": {"value": total * K / te, "unit": "env-steps/s", "h2d_bytes_per_step": total * 16,
                "d2h_bytes_per_step": total * 5},
        "cpu_baseline": {"value": value, "unit": "env-steps/s", "cores": None, "kind": "reference",
                         "sample": f"{K} steps of all 6 groups; the reference implementation is CUDA-only, so "
                                   "this arm runs its own kernels on the same B200"},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="mine", choices=["mine", "reference"])
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--launch", default="", help="stage,warps_per_cta,ctas_per_sm,tile_w[,team_warps,coop]")
    ap.add_argument("--start-state", default="", help="peak: start every arm from this saved state (written "
                                                      "after the warm-up if it does not exist)")
    ap.add_argument("--traffic-bytes", type=float, default=0.0,
                    help="DRAM bytes per fused launch from an ncu capture (reported as roofline.traffic)")
    ap.add_argument("--workload", default="peak", choices=["peak", "render", "ragged", "serve"],
                    help="peak: B=32768, 16^3, 32x32 (default); render: B=4096, 32^3, 64x64, half break "
                         "actions; ragged: 24,576 envs in 6 groups; serve: the env server under Poisson load")
    ap.add_argument("--serve-seconds", type=float, default=2.0, help="seconds per offered-load level (serve)")
    ap.add_argument("--shape", default="", help="peak workload override B,W,R (batch, world edge, resolution)")
    ap.add_argument("--no-tune", action="store_true", help="ragged: keep the default launch configuration")
    ap.add_argument("--no-legs", action="store_true",
                    help="peak: skip the late-window, render, ragged and serve legs of the default run")
    ap.add_argument("--stock-leg", action="store_true", help=argparse.SUPPRESS)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.stock_leg:
        run_stock_leg(args)
    elif args.impl == "reference":
        if args.workload == "serve":
            print(json.dumps({"impl": "reference", "unavailable": "the reference has no env server; the "
                              "one-job-at-a-time loop is the serve line's plain_one_job_at_a_time arm"}))
        elif args.workload == "ragged":
            run_reference_ragged(args)
        else:
            run_reference(args)
    else:
        {"peak": run_mine, "render": run_mine, "ragged": run_mine_ragged, "serve": run_mine_serve}[args.workload](args)


if __name__ == "__main__":
    main()
