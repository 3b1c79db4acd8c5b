"""Small, fixed render case for profiler captures (ncu) of the wavefront kernels.

    python ray-tracing_b200/profile_case.py [--material rough_plastic] [--size 512] [--spp 4] [--frames 2]

Renders `frames` frames of one open-box scene (the benchmark geometry) on cuda:0, then re-renders the
last frame with work counting on and prints the extension rays of every bounce of that frame, so that
DRAM bytes an ncu capture reports for one k_extend launch of the last frame can be divided by the rays
that launch traced. One frame at 512x512x4 spp is one wave of 1M paths: max_depth x 3 + 2 launches,
about 0.5 GB of device memory. With the defaults, k_extend launch number 9 (0-based, `ncu -k
regex:k_extend -s 9 -c 1`) is bounce 1 of the last frame.
"""
import argparse
import json
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

import numpy as np  # noqa: E402

import lrt  # noqa: E402
import scenes  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--material", default="rough_plastic", choices=scenes.MATERIAL_NAMES)
    ap.add_argument("--size", type=int, default=512)
    ap.add_argument("--spp", type=int, default=4)
    ap.add_argument("--frames", type=int, default=2)
    ap.add_argument("--depth", type=int, default=8)
    args = ap.parse_args()
    with lrt.Context(0) as ctx:
        ctx.upload(scenes.open_box(args.material))
        img = np.zeros((args.size, args.size, 3), np.float32)

        def params(f):
            return scenes.render_params(args.size, args.size, args.spp, args.depth, 3, sample_offset=f * args.spp)

        ctx.set_option("stage_timing", 1)
        for f in range(args.frames):
            ctx.render(params(f), img)
        timed = ctx.stats()
        ctx.set_option("stage_timing", 0)
        ctx.reset_stats()
        ctx.set_option("count_work", 1)
        ctx.render(params(args.frames - 1), img)
        counted = ctx.stats()
        print(json.dumps({"paths": timed["paths"], "stage_ms": timed["stage_ms"], "launches": timed["kernel_launches"],
                          "last_frame_rays_at_depth": counted["rays_at_depth"][: args.depth],
                          "last_frame_nodes_per_ray": counted["nodes_visited"] / max(1, counted["extension_rays"]),
                          "last_frame_triangles_per_ray": counted["triangles_tested"] / max(1, counted["extension_rays"]),
                          "mean": float(img.mean())}))


if __name__ == "__main__":
    main()
