"""Launch-shape autotuner for the fused step kernel.

The reference has no tuner: its launch shapes are constants (16x16 blocks
for the render kernels, 256 threads elsewhere; src/kernels.cu:2087-2260).
Here the fused step has six knobs, searched on the device with the caller's
own envs:

* ``tile_w``        pixel tile a warp marches per iteration, tile_w x
                    (32 / tile_w) rays (one ray per lane: rays per warp
                    iteration = 32, in rows of tile_w; 4, 8, 16 or 32);
* ``stage``         staging depth of the worlds in shared memory: 0 none, 1
                    one world buffer per stepping warp, 2 one more env in
                    flight (team launches: the next unit's world is copied
                    into a second buffer while the current one renders; one
                    warp per env: the next env is claimed ahead and its world
                    prefetched into L2);
* ``team_warps``    warps per team (1, 2, 4, 8);
* ``coop``          1: a team renders each env together (envs per CTA =
                    teams per CTA); 0: each warp its own env (envs per CTA =
                    warps per CTA);
* ``warps_per_cta`` warps per CTA;
* ``ctas_per_sm``   persistent grid = SMs x ctas_per_sm.

For a `RaggedBatch` ``tile_w``, ``stage`` and ``coop`` are chosen per group.  Every
trial restores the same snapshot of the env state, replays the same K-step
action window through a CUDA graph and is timed with CUDA events, so trials
see identical work; the winner is set on the env and cached in a JSON file
keyed by device name and workload signature (``$MINECU_TUNE_CACHE`` or
``~/.cache/minecu_b200/autotune.json``).
"""
from __future__ import annotations

import json
import os
import time
from typing import Dict, Iterable, List, Optional, Sequence, Tuple

import torch

from minecu import MineEnv, _C

TILE_WIDTHS = (4, 8, 16)
MAX_SMEM = 227 * 1024


def cache_path() -> str:
    p = os.environ.get("MINECU_TUNE_CACHE")
    if p:
        return p
    return os.path.join(os.path.expanduser("~"), ".cache", "minecu_b200", "autotune.json")


def _load_cache() -> dict:
    try:
        with open(cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store_cache(key: str, value: dict) -> None:
    c = _load_cache()
    c[key] = value
    p = cache_path()
    try:
        os.makedirs(os.path.dirname(p), exist_ok=True)
        tmp = p + f".{os.getpid()}.tmp"
        with open(tmp, "w") as f:
            json.dump(c, f, indent=1, sort_keys=True)
        os.replace(tmp, p)
    except OSError:
        pass  # a read-only home: the result still applies to this process


def env_signature(e: MineEnv) -> str:
    return (f"B{e.batch_size}_w{e.world_x}x{e.world_y}x{e.world_z}_r{e.render_width}x{e.render_height}"
            f"_{e.obs_dtype}_{e.numerics}_ms{e.max_steps}_vd{e.view_distance}")


def _device_key(dev: torch.device) -> str:
    return torch.cuda.get_device_name(dev).replace(" ", "_")


def _time_window(run, restore, reps: int = 2) -> float:
    """Milliseconds of one call of `run` (best of `reps`), each from the same restored state."""
    best = float("inf")
    for _ in range(reps):
        restore()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        run()
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    return best


def _actions(n_envs: int, steps: int, seed: int, device) -> torch.Tensor:
    a = torch.empty((steps, n_envs), dtype=torch.uint8, device=device)
    _C.philox_actions(a, 0, 0, seed)
    return a


# ---------------------------------------------------------------------------
# one MineEnv
# ---------------------------------------------------------------------------
def env_candidates() -> List[Tuple[int, int, int, int, int, int]]:
    """(stage, warps_per_cta, ctas_per_sm, tile_w, team_warps, coop) tried by tune_env."""
    per_warp = [(st, wpc, cps, tw, 1, 0) for st in (0, 1, 2) for wpc in (4, 8) for cps in (2, 4, 8)
                for tw in TILE_WIDTHS]
    teams = [(st, 8, cps, tw, team, 1) for st in (0, 1, 2) for cps in (2, 3, 4) for tw in TILE_WIDTHS
             for team in (2, 4, 8)]
    return per_warp + teams


def tune_env(env: MineEnv, steps: int = 40, warm_steps: int = 50, seed: int = 1, use_cache: bool = True,
             candidates: Optional[Iterable[Tuple[int, ...]]] = None, verbose: bool = False) -> dict:
    """Choose (stage, warps_per_cta, ctas_per_sm, tile_w, team_warps, coop)
    for `env`'s fused step, set it on the env and return {"config": ...,
    "ms_per_step": ...}.  The env's state is restored afterwards."""
    key = f"env|{_device_key(env.device)}|{env_signature(env)}"
    if use_cache:
        hit = _load_cache().get(key)
        if hit:
            env.set_launch_config(*hit["config"])
            return hit
    with torch.cuda.device(env.device):
        saved = env.state_dict()
        acts = _actions(env.batch_size, warm_steps + steps, seed, env.device)
        env.reset()
        if warm_steps:
            env.rollout(acts[:warm_steps])
        snap = env.state_dict()
        window = acts[warm_steps:]
        if candidates is None:
            candidates = env_candidates()
        results: List[Tuple[float, tuple]] = []
        for cfg in candidates:
            try:
                env.set_launch_config(*cfg)
            except RuntimeError:
                continue  # not valid for this env (alignment, shared memory)
            env.prepare_rollout(window)
            ms = _time_window(lambda: env.rollout(window), lambda: env.load_state_dict(snap)) / steps
            results.append((ms, tuple(cfg)))
            if verbose:
                print(f"  {cfg}: {ms:.4f} ms/step")
        results.sort()
        best_ms, best = results[0]
        env.set_launch_config(*best)
        env.load_state_dict(saved)
        env.check_error()
    out = {"config": list(best), "ms_per_step": best_ms, "trials": len(results), "time": time.time()}
    _store_cache(key, out)
    return out


# ---------------------------------------------------------------------------
# a RaggedBatch
# ---------------------------------------------------------------------------
def _ragged_key(batch) -> str:
    return "ragged|" + _device_key(batch.device) + "|" + "+".join(env_signature(e) for e in batch.envs)


def tune_ragged(batch, steps: int = 30, warm_steps: int = 50, seed: int = 3, use_cache: bool = True,
                rounds: int = 2, verbose: bool = False) -> dict:
    """Coordinate search over a RaggedBatch's team size, launch shape and
    per-group (coop, stage, tile_w); sets the winner and returns
    {"config": ..., "ms_per_step": ...}.  The groups' state is restored
    afterwards."""
    key = _ragged_key(batch)
    G = len(batch.envs)
    if use_cache:
        hit = _load_cache().get(key)
        if hit:
            c = hit["config"]
            batch.set_launch_config(c["warps_per_cta"], c["ctas_per_sm"], c["stage"], c["tile_w"], c["team_warps"],
                                    c["coop"])
            return hit
    with torch.cuda.device(batch.device):
        saved = batch.state_dict()
        acts = _actions(batch.total, warm_steps + steps, seed, batch.device)
        batch.reset()
        if warm_steps:
            batch.rollout(acts[:warm_steps])
        snap = batch.state_dict()
        window = acts[warm_steps:]
        trials: Dict[tuple, float] = {}

        def measure(c: dict) -> float:
            k = (c["warps_per_cta"], c["ctas_per_sm"], c["team_warps"], tuple(c["stage"]), tuple(c["tile_w"]),
                 tuple(c["coop"]))
            if k in trials:
                return trials[k]
            try:
                batch.set_launch_config(c["warps_per_cta"], c["ctas_per_sm"], c["stage"], c["tile_w"],
                                        c["team_warps"], c["coop"])
            except RuntimeError:
                trials[k] = float("inf")
                return trials[k]
            if batch.launch_config()["smem_bytes"] * c["ctas_per_sm"] > 228 * 1024 * 2:
                trials[k] = float("inf")  # far more CTAs than fit: not worth timing
                return trials[k]
            batch.prepare_rollout(window)
            ms = _time_window(lambda: batch.rollout(window), lambda: batch.load_state_dict(snap)) / steps
            trials[k] = ms
            if verbose:
                print(f"  {c}: {ms:.4f} ms/step")
            return ms

        cur = batch.launch_config()
        best_cfg = {k: (list(v) if isinstance(v, list) else v) for k, v in cur.items() if k != "smem_bytes"}
        best = measure(best_cfg)

        def consider(c: dict) -> bool:
            nonlocal best, best_cfg
            ms = measure(c)
            if ms < best * 0.995:
                best, best_cfg = ms, c
                return True
            return False

        def with_(**kw) -> dict:
            c = {k: (list(v) if isinstance(v, list) else v) for k, v in best_cfg.items()}
            c.update(kw)
            return c

        for _ in range(rounds):
            improved = False
            # team size with the launch shape that fits it
            for team in (1, 2, 4, 8):
                improved |= consider(with_(team_warps=team, warps_per_cta=8))
            # per group: team rendering, tile shape and staging, the others fixed
            for g in range(G):
                for co in (0, 1):
                    for st in (0, 1):
                        for tw in TILE_WIDTHS:
                            c = with_()
                            c["coop"][g], c["stage"][g], c["tile_w"][g] = co, st, tw
                            improved |= consider(c)
            # staging depth of every staged group (the launch uses the largest)
            staged = [1 if x else 0 for x in best_cfg["stage"]]
            for depth in (1, 2):
                improved |= consider(with_(stage=[depth * x for x in staged]))
            # launch shape
            for w2 in (4, 8):
                if w2 % best_cfg["team_warps"]:
                    continue
                for c2 in (1, 2, 3, 4, 6, 8):
                    improved |= consider(with_(warps_per_cta=w2, ctas_per_sm=c2))
            if not improved:
                break
        c = best_cfg
        batch.set_launch_config(c["warps_per_cta"], c["ctas_per_sm"], c["stage"], c["tile_w"], c["team_warps"],
                                c["coop"])
        batch.load_state_dict(saved)
        batch.check_error()
    out = {"config": best_cfg, "ms_per_step": best, "trials": len(trials), "time": time.time()}
    _store_cache(key, out)
    return out
