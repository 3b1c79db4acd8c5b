"""Launch-shape autotuner for batched rendering, with results cached per scene size.

Three knobs change only the speed of lrt_render_batch, never its images:
  wave_capacity   paths per wave (the queue capacity of every wavefront stage)
  blocks_per_sm   resident blocks per SM of every grid (0: the occupancy maximum)
  pixel_tile      path order inside a job: bands of this many rows walked column by column, so that a
                  warp's camera rays (and their first bounces) cover a compact patch of pixels
The traversal stack depth is not a knob: it must hold the deepest kd-tree path (the reference's
depth limit), and the kernels' block size is fixed at compile time.

The timing and the coordinate descent over the candidates are the library's (lrt_autotune: the
caller's jobs with spp scaled to about 150M paths per trial, one knob at a time from the defaults).
This module keeps the chosen configurations in a JSON file keyed by the scene's size class (triangle
count rounded up to a power of two, material and emitter counts) and the job mix's size class, the
same key the library's own text cache uses.
"""
from __future__ import annotations

import json
import math
import os


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


def tune(ctx, jobs, max_depth: int, rr_depth: int, out_ptr: int):
    """lrt_autotune without a cache file: (best configuration, its trial seconds, configurations timed)"""
    r = ctx.autotune(jobs, max_depth, rr_depth, out_ptr)
    return {k: r[k] for k in ORDER}, r["seconds"], r["trials"]


def tuned(ctx, scene, jobs, max_depth: int, rr_depth: int, out_ptr: int, cache_path: str = CACHE_PATH,
          retune: bool = False):
    """the cached configuration for this scene/job size class, tuned now (and cached) if missing"""
    key = scene_key(scene, jobs)
    cache = load_cache(cache_path)
    if key in cache and not retune:
        cfg = {k: cache[key][k] for k in ORDER}
        apply(ctx, cfg)
        return cfg, key, True
    best, best_t, trials = tune(ctx, jobs, max_depth, rr_depth, out_ptr)
    cache[key] = dict(best, seconds=best_t, trials=trials)
    save_cache(cache, cache_path)
    return best, key, False
