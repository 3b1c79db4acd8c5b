"""Small, fixed render case for profiler captures (ncu) of the wavefront kernels.

    python ray-tracing_b200/profile_case.py [--material rough_plastic] [--size 512] [--spp 4] [--frames 2]

Renders `frames` frames of one open-box scene (the benchmark geometry) on cuda:0 and prints the
per-stage device time. One frame at 512x512x4 spp is one wave of 1M paths: a few dozen launches,
about 0.5 GB of device memory.
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
        ctx.set_option("stage_timing", 1)
        img = np.zeros((args.size, args.size, 3), np.float32)
        for f in range(args.frames):
            ctx.render(scenes.render_params(args.size, args.size, args.spp, args.depth, 3, sample_offset=f * args.spp),
                       img)
        st = ctx.stats()
        print(json.dumps({"paths": st["paths"], "stage_ms": st["stage_ms"], "launches": st["kernel_launches"],
                          "mean": float(img.mean())}))


if __name__ == "__main__":
    main()
