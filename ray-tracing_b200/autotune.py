"""Launch-shape autotuner for batched rendering, with results cached per scene size.

Three knobs change only the speed of lrt_render_batch, never its images:
  wave_capacity   paths per wave (the queue capacity of every wavefront stage)
  blocks_per_sm   resident blocks per SM of every grid (0: the occupancy maximum)
  pixel_tile      path order inside a job: bands of this many rows walked column by column, so that a
                  warp's camera rays (and their first bounces) cover a compact patch of pixels
The traversal stack depth is not a knob: it must hold the deepest kd-tree path (the reference's
depth limit), and the kernels' block size is fixed at compile time.

tune() runs a coordinate descent over the candidates, timing the caller's jobs with their spp scaled
down so that one timing covers about `paths_per_trial` paths. Results are cached in a JSON file keyed
by the scene's size class (triangle count rounded up to a power of two, material and emitter
counts) and the job mix's size class.
"""
from __future__ import annotations

import json
import math
import os
import time

import lrt_abi as abi

HERE = os.path.dirname(os.path.abspath(__file__))
CACHE_PATH = os.path.join(HERE, "data", "autotune_cache.json")
DEFAULTS = {"wave_capacity": 1 << 24, "blocks_per_sm": 0, "pixel_tile": 1}  # the library's forward defaults
CANDIDATES = {
    "wave_capacity": [1 << 19, 1 << 20, 1 << 21, 1 << 22, 1 << 23, 1 << 24],
    "blocks_per_sm": [0, 2, 3],
    "pixel_tile": [1, 4, 8, 16],
}
ORDER = ["wave_capacity", "pixel_tile", "blocks_per_sm"]


def scene_key(scene, jobs) -> str:
    tris = max(1, scene.triangle_count())
    paths = sum(j.width * j.height * j.spp for j in jobs)
    return "tris2^%d_mats%d_emitters%d_paths2^%d" % (math.ceil(math.log2(tris)), len(scene.materials),
                                                     len(scene.emitters), math.ceil(math.log2(max(1, paths))))


def load_cache(path: str = CACHE_PATH) -> dict:
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f)
    return {}


def save_cache(cache: dict, path: str = CACHE_PATH) -> None:
    os.makedirs(os.path.dirname(path), exist_ok=True)
    with open(path, "w") as f:
        json.dump(cache, f, indent=1, sort_keys=True)


def apply(ctx, cfg: dict) -> None:
    for k in ORDER:
        ctx.set_option(k, int(cfg.get(k, DEFAULTS[k])))


def scaled_jobs(jobs, paths_per_trial: int):
    """the jobs with spp scaled so that they hold about paths_per_trial paths (at least 1 spp each)"""
    total = sum(j.width * j.height * j.spp for j in jobs)
    f = min(1.0, paths_per_trial / max(1, total))
    out = []
    for j in jobs:
        out.append(abi.JobDesc(j.camera, j.width, j.height, max(1, int(round(j.spp * f))), j.sample_offset,
                               j.override_object, j.override_material, j.output_offset))
    return out


def coordinate_descent(measure, candidates=CANDIDATES, order=ORDER, start=None, rounds: int = 1):
    """minimise measure(cfg) -> seconds over one knob at a time; returns (best cfg, best time, trials)"""
    best = dict(DEFAULTS if start is None else start)
    best_t = measure(best)
    trials = [(dict(best), best_t)]
    for _ in range(rounds):
        for knob in order:
            for v in candidates[knob]:
                if v == best[knob]:
                    continue
                cfg = dict(best, **{knob: v})
                t = measure(cfg)
                trials.append((dict(cfg), t))
                if t < best_t:
                    best, best_t = cfg, t
    return best, best_t, trials


def tune(ctx, jobs, max_depth: int, rr_depth: int, out_ptr: int, sync, paths_per_trial: int = 150_000_000,
         repeats: int = 2):
    """times lrt_render_batch_dev on scaled-down jobs; `sync` waits for the device"""
    trial_jobs = scaled_jobs(jobs, paths_per_trial)

    def measure(cfg):
        apply(ctx, cfg)
        ctx.render_batch_dev(trial_jobs, max_depth, rr_depth, out_ptr)  # warm (allocations, graph)
        sync()
        times = []
        for _ in range(repeats):
            t0 = time.perf_counter()
            ctx.render_batch_dev(trial_jobs, max_depth, rr_depth, out_ptr)
            sync()
            times.append(time.perf_counter() - t0)
        return min(times)

    best, best_t, trials = coordinate_descent(measure)
    apply(ctx, best)
    return best, best_t, trials


def tuned(ctx, scene, jobs, max_depth: int, rr_depth: int, out_ptr: int, sync, cache_path: str = CACHE_PATH,
          retune: bool = False):
    """the cached configuration for this scene/job size class, tuned now (and cached) if missing"""
    key = scene_key(scene, jobs)
    cache = load_cache(cache_path)
    if key in cache and not retune:
        cfg = {k: cache[key][k] for k in ORDER}
        apply(ctx, cfg)
        return cfg, key, True
    best, best_t, trials = tune(ctx, jobs, max_depth, rr_depth, out_ptr, sync)
    cache[key] = dict(best, seconds=best_t, trials=len(trials))
    save_cache(cache, cache_path)
    return best, key, False
