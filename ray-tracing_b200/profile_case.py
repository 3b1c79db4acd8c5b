"""Small, fixed cases for profiler captures (ncu) of the library's kernels.

    python ray-tracing_b200/profile_case.py [--case render|eye|adjoint|batch|kdbuild] [options]

render (default): `frames` frames of one open-box scene (the benchmark geometry), then the last frame
  again with work counting on, printing the extension rays of every bounce of that frame, so that DRAM
  bytes an ncu capture reports for one k_extend launch can be divided by the rays it traced. One frame
  at 512x512x4 spp is one wave of 1M paths: raygen and accumulate, and per bounce extend, hit records,
  shadow and one shading kernel per shading key present (three here: misses, the diffuse walls, the
  sphere's material); about 0.5 GB of device memory.
  With the defaults, k_extend launch number 9 (0-based, `ncu -k regex:k_extend -s 9 -c 1`) is bounce 1
  of the last frame.
eye: the large photon-mapping scene (256 level-5 spheres, 5.24M triangles), `photons` photons, one
  photon-mapper image of size x size x 1 with the wavefront eye pass (k_eye_shade / k_eye_trace), about
  2 GB of device memory with the defaults.
adjoint: the seven-material scene at size x size x spp per material (7 jobs), one render and one
  path-replay adjoint (k_shade_adj, k_adj_nee, k_adj_suffix).
batch: 16 seeded jobs of the batched workload with spp scaled down (one graph-replayed wave sequence).
kdbuild: the SAH kd-trees of the large scene's 257 meshes (5.24M triangle boxes) built on the GPU in one
  lrt_kdtree_build_device call (radix sort, then 25 levels of scans, costs, decisions and partitions).
"""
import argparse
import json
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

import numpy as np  # noqa: E402

import lrt  # noqa: E402
import scenes  # noqa: E402


def eye_case(args):
    with lrt.Context(0) as ctx:
        ctx.upload(scenes.large_scene())
        pp, shots = ctx.photon_preprocess(args.photons, 0, max_depth=8, rr_depth=5, radius_cap=0.05, lookup_size=100)
        img = ctx.render_photon(scenes.render_params(args.size, args.size, 1, 8, 3), pp)
        print(json.dumps({"photons": args.photons, "shot": shots[0], "launches": ctx.stats()["kernel_launches"],
                          "mean": float(img.mean())}))


def adjoint_case(args):
    import diff
    scene, sphere, index = scenes.open_box_library()
    with lrt.Context(0) as ctx:
        ctx.upload(scene)
        dm = diff.Differentiable(ctx, scene)
        jobs, off = [], 0
        for name in scenes.MATERIAL_NAMES:
            jobs.append(scenes.job_desc(scene.camera, args.size, args.size, args.spp, 0, sphere, index[name], off))
            off += 3 * args.size * args.size
        img = ctx.render_batch(jobs, 6, 3)
        g = dm.adjoint(jobs, 6, 3, np.ones(off, np.float32) / off)
        print(json.dumps({"mean": float(img.mean()), "grad_norm": float(np.linalg.norm(g))}))


def batch_case(args):
    scene, sphere, index = scenes.open_box_library()
    jobs, specs = scenes.batch_jobs(index, sphere, n_jobs=16, spp_range=(1, 16))
    with lrt.Context(0) as ctx:
        ctx.upload(scene)
        out = ctx.render_batch(jobs, 8, 3)
        print(json.dumps({"jobs": len(jobs), "launches": ctx.stats()["kernel_launches"], "mean": float(np.nanmean(out))}))


def kdbuild_case(args):
    import time
    import lrt_abi as abi
    meshes = []
    for o in scenes.large_scene().objects:
        if o["kind"] == abi.OBJ_MESH:
            tri = o["positions"][o["indices"].reshape(-1, 3)]
            meshes.append((tri.min(axis=1).astype(np.float32), tri.max(axis=1).astype(np.float32)))
    with lrt.Context(0) as ctx:
        t0 = time.perf_counter()
        trees = ctx.kdtree_build_device(meshes)
        seconds = time.perf_counter() - t0
        print(json.dumps({"meshes": len(meshes), "boxes": int(sum(len(b) for b, _ in meshes)),
                          "nodes": int(sum(len(t[0]) for t in trees)), "refs": int(sum(len(t[1]) for t in trees)),
                          "seconds_with_python": seconds}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--case", default="render", choices=["render", "eye", "adjoint", "batch", "kdbuild"])
    ap.add_argument("--material", default="rough_plastic", choices=scenes.MATERIAL_NAMES)
    ap.add_argument("--size", type=int, default=512)
    ap.add_argument("--spp", type=int, default=4)
    ap.add_argument("--frames", type=int, default=2)
    ap.add_argument("--depth", type=int, default=8)
    ap.add_argument("--photons", type=int, default=2_000_000)
    args = ap.parse_args()
    if args.case == "eye":
        return eye_case(args)
    if args.case == "adjoint":
        return adjoint_case(args)
    if args.case == "batch":
        return batch_case(args)
    if args.case == "kdbuild":
        return kdbuild_case(args)
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
