#!/usr/bin/env python
"""Benchmark of the LinRT rendering hot path on B200: Mpaths/s of the wavefront path tracer.

Workload (one step): the seven-material open-box scene set (Cornell-style box open to a Hosek sky, a
displaced level-6 icosphere of 81,920 triangles carrying each of the seven BSDFs in turn), 512x512
pixels, 64 samples per pixel, max depth 8, Russian roulette from depth 3 -- 7 x 16.8M = 117.4M camera
paths per step. Inputs are synthetic and seeded (scenes.py).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl lrt|reference]
    python bench.py --workload batch|adjoint|large     (one GPU; see run_batch, run_adjoint, run_large)

N > 1 runs as one process per GPU under torch.distributed (NCCL): every rank renders its own replica
with a disjoint sample range (no data-path collective), the timed region is bracketed by barriers and
the max over ranks is reported. --impl reference times the reference's own CPU renderer (the unmodified
sources built in oracle/_ref) on this host's cores.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "ray-tracing_b200"))

import scenes  # noqa: E402

W, H = scenes.CONFIG1["width"], scenes.CONFIG1["height"]
SPP, DEPTH, RR = scenes.CONFIG1["spp"], scenes.CONFIG1["max_depth"], scenes.CONFIG1["rr_depth"]
MATERIALS = scenes.MATERIAL_NAMES
METRIC = "Mpaths/s (path tracer, 7 materials x 512x512 x 64 spp, depth 8, Hosek sky)"
WORKLOAD = "open_box_7_materials_512x512_64spp_depth8"
PATHS_PER_STEP = len(MATERIALS) * W * H * SPP
ARGS_WAVE_CAPACITY = [0]


def config(extra=None):
    c = {"workload": WORKLOAD, "width": W, "height": H, "spp": SPP, "max_depth": DEPTH, "rr_depth": RR,
         "materials": MATERIALS, "triangles": 81920 + 12, "paths_per_step": PATHS_PER_STEP,
         "l2": "flushed (256 MB write) between timed steps", "parallelism": "replicas",
         "wave_capacity": ARGS_WAVE_CAPACITY[0] or "library default (2^24: one wave per frame)"}
    if extra:
        c.update(extra)
    return c


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle-reason samples every 200 ms while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu_index = gpu_index
        self.proc = None
        self.file = None

    def start(self):
        try:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(["nvidia-smi", "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                                          "-i", str(self.gpu_index), "-lms", "200"], stdout=self.file,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.file.flush()
        self.file.seek(0)
        rows = [r.split(",") for r in self.file.read().strip().splitlines() if r.count(",") >= 8]
        os.unlink(self.file.name)
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if "Active" in r[5 + i] and "Not" not in r[5 + i]})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ------------------------------------------------------------------------------------------------
# CPU reference (oracle/_ref: the unmodified reference sources); used by --impl reference and by the
# cpu_baseline field

def reference_worlds():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    if not oracle.reference_available():
        return None, None
    return oracle, [oracle.RefWorld(scenes.open_box(m)) for m in MATERIALS]


def reference_pass(oracle, worlds, spp, sample_offset=0):
    """one pass over the seven scenes at 512x512 x `spp` on all host cores; returns (paths, seconds)"""
    secs = 0.0
    for w in worlds:
        _, _, s = w.render(scenes.render_params(W, H, spp, DEPTH, RR, sample_offset=sample_offset), 0)
        secs += s
    return len(worlds) * W * H * spp, secs


def cpu_baseline(budget_s=15.0):
    oracle, worlds = reference_worlds()
    if worlds is None:
        return None
    spp, paths, secs = 1, 0, 0.0
    while secs < budget_s:
        p, s = reference_pass(oracle, worlds, spp, sample_offset=paths)
        paths += p
        secs += s
        if secs < budget_s / 4:
            spp *= 2
    return {"value": paths / secs / 1e6, "unit": "Mpaths/s", "cores": oracle.hardware_concurrency(),
            "kind": "reference",
            "sample": "%d paths: the 7 scenes at 512x512 with %d..%d spp per pass (same scenes, depth, roulette), "
                      "32x32 tiles on a thread pool of hardware_concurrency workers, built -O3 without -march"
                      % (paths, 1, spp)}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    oracle, worlds = reference_worlds()
    if worlds is None:
        print(json.dumps({"impl": "reference", "unavailable": "reference sources not built (oracle/_ref missing)"}))
        return 0
    spp = 1
    for i in range(args.warmup):
        reference_pass(oracle, worlds, spp, sample_offset=1000 + 8 * i)
    times, paths = [], 0
    for i in range(args.steps):
        p, s = reference_pass(oracle, worlds, spp, sample_offset=8 * i)
        times.append(s)
        paths += p
    total = sum(times)
    value = paths / total / 1e6
    cores = oracle.hardware_concurrency()
    line = {"metric": METRIC, "value": value, "unit": "Mpaths/s", "impl": "reference", "n_gpus": 0,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * total / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": config({"reference_spp_per_step": spp}),
            "cpu_baseline": {"value": value, "unit": "Mpaths/s", "cores": cores, "kind": "reference",
                             "sample": "each step: the 7 scenes at 512x512 x %d spp (%d paths) on %d threads"
                                       % (spp, len(worlds) * W * H * spp, cores)},
            "e2e": {"value": value, "unit": "Mpaths/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ------------------------------------------------------------------------------------------------
# replicas (N > 1): one process per GPU, disjoint sample ranges, the slowest rank's time

def replica_sample_offset(rank: int, spp: int) -> int:
    """rank r renders samples [r * spp, (r + 1) * spp) of every pixel: replicas never repeat a sample"""
    return rank * spp


def max_over_ranks(dist, value: float, device) -> float:
    """the slowest rank's value (every rank takes this collective at the same point of the run)"""
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_mpaths(world: int, paths_per_step: int, steps: int, seconds: float) -> float:
    """paths of all ranks over the slowest rank's time"""
    return world * paths_per_step * steps / seconds / 1e6


def run_lrt(args):
    import torch
    import lrt

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(dev)  # the library's stream; flushes and timing events go on it too
    torch.cuda.set_stream(stream)

    ctxs = []
    for m in MATERIALS:
        c = lrt.Context(local, stream.cuda_stream)
        c.upload(scenes.open_box(m))
        if args.wave_capacity:
            c.set_option("wave_capacity", args.wave_capacity)
        ctxs.append(c)
    out = torch.empty((H, W, 3), dtype=torch.float32, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    offset = replica_sample_offset(rank, SPP)
    params = scenes.render_params(W, H, SPP, DEPTH, RR, sample_offset=offset)

    # algorithmic work per path (exact traversal counts; untimed pass at 8 spp)
    for c in ctxs:
        c.set_option("count_work", 1)
        c.reset_stats()
        c.render_dev(scenes.render_params(W, H, 8, DEPTH, RR, sample_offset=offset + 1 << 20), out.data_ptr())
        c.set_option("count_work", 0)
    st = [c.stats() for c in ctxs]
    paths_c = sum(s["paths"] for s in st)
    ext_rays = sum(s["extension_rays"] for s in st)
    ext_bytes = sum(8 * s["nodes_visited"] + 48 * s["triangles_tested"] for s in st) + (32 + 16) * ext_rays
    sh_rays = sum(s["shadow_rays"] for s in st)
    sh_bytes = sum(8 * s["shadow_nodes_visited"] + 48 * s["shadow_triangles_tested"] for s in st) + 32 * sh_rays
    work = {"extension_rays_per_path": ext_rays / paths_c, "shadow_rays_per_path": sh_rays / paths_c,
            "extend_bytes_per_path": ext_bytes / paths_c, "shadow_bytes_per_path": sh_bytes / paths_c,
            "nodes_per_extension_ray": sum(s["nodes_visited"] for s in st) / max(1, ext_rays),
            "triangles_per_extension_ray": sum(s["triangles_tested"] for s in st) / max(1, ext_rays)}

    def step():
        for c in ctxs:
            c.render_dev(params, out.data_ptr())

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    for c in ctxs:
        c.reset_stats()
        c.set_option("stage_timing", 1)

    clocks = ClockSampler(os.environ.get("CUDA_VISIBLE_DEVICES", str(local)).split(",")[0] if world == 1 else local)
    if dist:
        dist.barrier()
    torch.cuda.synchronize(dev)
    clocks.start()
    step_ms = []
    for _ in range(args.steps):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        step()
        e1.record(stream)
        e1.synchronize()
        step_ms.append(e0.elapsed_time(e1))
    torch.cuda.synchronize(dev)
    if dist:
        dist.barrier()
    clock_info = clocks.stop()
    total_ms = float(sum(step_ms))
    st = [c.stats() for c in ctxs]
    launches = int(sum(s["kernel_launches"] for s in st))
    extend_ms = sum(s["stage_ms"]["extend"] for s in st)
    extend_launches = sum(s["stage_launches"]["extend"] for s in st)
    stage_ms = {k: sum(s["stage_ms"][k] for s in st) for k in abi_stage_names()}
    for c in ctxs:
        c.set_option("stage_timing", 0)
    total_ms = max_over_ranks(dist, total_ms, dev)

    # end to end: the public host-buffer call (lrt_render: render + device->host copy of the image)
    host_img = np.zeros((H, W, 3), dtype=np.float32)
    e2e_times = []
    if dist:
        dist.barrier()
    for i in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        for c in ctxs:
            c.render(params, host_img)
        e2e_times.append(time.perf_counter() - t0)
    e2e_total = max_over_ranks(dist, sum(e2e_times), dev)

    value = whole_job_mpaths(world, PATHS_PER_STEP, args.steps, total_ms / 1000.0)
    e2e_value = whole_job_mpaths(world, PATHS_PER_STEP, args.steps, e2e_total)
    peak, peak_kind = measured_peaks()
    timed_paths = PATHS_PER_STEP * args.steps
    achieved = (work["extend_bytes_per_path"] * timed_paths / 1e9) / (extend_ms / 1000.0) if extend_ms > 0 else None
    traffic = None
    issue = None
    tpath = os.path.join(ROOT, "profiles", "extend_traffic.json")
    if os.path.exists(tpath) and extend_launches:
        with open(tpath) as f:
            tr = json.load(f)
        issue = {"issue_active_frac": tr.get("issue_active_frac"),
                 "simt_lane_efficiency": tr.get("lanes_per_warp_instruction", 0) / 32.0 or None,
                 "source": "ncu capture summarised in profiles/k_extend_persistent_open_box_bounce1.md"}
        # DRAM bytes per extension ray from an ncu capture, scaled to this run's average launch
        traffic = tr["dram_bytes_per_extension_ray"] * work["extension_rays_per_path"] * timed_paths / extend_launches
    cpu = cpu_baseline() if (rank == 0 and world == 1 and not args.no_cpu_baseline) else None

    # the plain GPU path tracer (one launch per frame, one thread per pixel, whole path in registers) on
    # the same frames and samples: same images, its time beside the wavefront's
    plain = None
    if rank == 0 and world == 1:
        cam = scenes.open_box(MATERIALS[0], attach=False).camera
        job = scenes.job_desc(cam, W, H, SPP, offset)
        for c in ctxs:
            c.render_plain_dev([job], DEPTH, RR, out.data_ptr())  # warm
        flush.zero_()
        torch.cuda.synchronize(dev)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for c in ctxs:
            c.render_plain_dev([job], DEPTH, RR, out.data_ptr())
        e1.record(stream)
        e1.synchronize()
        plain_s = e0.elapsed_time(e1) / 1000.0
        plain = {"value": PATHS_PER_STEP / plain_s / 1e6, "unit": "Mpaths/s", "steps": 1,
                 "kernel": "k_pt_plain (lrt_render_plain): one launch per frame, one thread per pixel",
                 "wavefront_speedup": value * plain_s * 1e6 / PATHS_PER_STEP}

    # equal RMSE: the same samples give the reference's image, so the error against a converged render
    # is the reference's (the cornell box fixture: 32x32, 64 spp vs the reference's 4096 spp)
    rmse = None
    gpath = os.path.join(ROOT, "tests", "golden", "image_kat.npz")
    if rank == 0 and os.path.exists(gpath):
        g = np.load(gpath)
        c = lrt.Context(local, stream.cuda_stream)
        c.upload(scenes.cornell_box())
        img = c.render(scenes.render_params(32, 32, 64, 6, 3))
        c.close()
        ref4096 = g["cornell_4096"].astype(np.float64)
        rmse = {"gpu_64spp": float(np.sqrt(np.mean((img - ref4096) ** 2))),
                "reference_64spp": float(np.sqrt(np.mean((g["cornell_64"] - ref4096) ** 2))),
                "against": "the reference renderer's 4096-spp cornell box (32x32, depth 6, tests/golden)"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "Mpaths/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scenes.py)",
            "config": config({"work_per_path": work, "stage_ms_per_step": {k: v / args.steps for k, v in stage_ms.items()}}),
            "e2e": {"value": e2e_value, "unit": "Mpaths/s", "h2d_bytes_per_step": len(MATERIALS) * 32,
                    "d2h_bytes_per_step": len(MATERIALS) * W * H * 3 * 4,
                    "path": "lrt_render (host output buffer; scene resident after lrt_scene_upload)"},
            "roofline": {"kernel": "k_extend (closest-hit kd-tree traversal)", "bound": "hbm",
                         "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": (achieved / peak) if achieved else None, "peak_kind": peak_kind,
                         "traffic": traffic,
                         "algorithmic_bytes": "per extension ray 8*nodes + 48*triangles + 32 ray + 16 hit",
                         "avg_launch_ms": extend_ms / max(1, extend_launches),
                         "issue": issue},
            "cpu_baseline": cpu,
            "rmse": rmse,
            "plain_gpu_pt": plain,
            "clocks": clock_info,
            "gpu_launches": launches,
        }
        print(json.dumps(line))
    for c in ctxs:
        c.close()
    if dist:
        dist.destroy_process_group()
    return 0


# ------------------------------------------------------------------------------------------------
# batched workload: 64 seeded jobs (resolution, spp 4-256, camera, sphere material) on the open box

BATCH_METRIC = "jobs/s (64 seeded jobs: 128^2..1024x768, 4-256 spp, 7 materials, depth 8)"


def run_batch(args):
    import torch
    import autotune
    import lrt

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(dev)  # the library's stream; flushes and timing events go on it too
    torch.cuda.set_stream(stream)
    scene, sphere, index = scenes.open_box_library()
    jobs, specs = scenes.batch_jobs(index, sphere, n_jobs=args.jobs)
    n_paths = sum(j["width"] * j["height"] * j["spp"] for j in specs)
    floats = max(j["output_offset"] + 3 * j["width"] * j["height"] for j in specs)
    ctx = lrt.Context(local, stream.cuda_stream)
    ctx.upload(scene)
    out = torch.zeros(floats, dtype=torch.float32, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    tuned = {"launch_config": dict(autotune.DEFAULTS), "autotune": "off"}
    if not args.no_autotune:
        cfg, key, hit = autotune.tuned(ctx, scene, jobs, DEPTH, RR, out.data_ptr())
        tuned = {"launch_config": cfg, "autotune": "cache hit" if hit else "tuned now", "autotune_key": key}

    def batched():
        ctx.render_batch_dev(jobs, DEPTH, RR, out.data_ptr())

    def per_job_plain():
        for j in jobs:
            ctx.render_plain_dev([j], DEPTH, RR, out.data_ptr())

    def per_job_wavefront():
        for j in jobs:
            ctx.render_batch_dev([j], DEPTH, RR, out.data_ptr())

    arms = {"batched": batched, "per_job_plain": per_job_plain, "per_job_wavefront": per_job_wavefront}
    results, images = {}, {}
    clocks = ClockSampler(os.environ.get("CUDA_VISIBLE_DEVICES", str(local)).split(",")[0])
    clocks.start()
    for name, fn in arms.items():
        if name == "per_job_wavefront":
            ctx.set_option("batch_graph", 0)
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize(dev)
        ctx.reset_stats()
        ms = []
        for _ in range(args.steps):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
        ctx.set_option("batch_graph", 1)
        total = sum(ms) / 1000.0
        results[name] = {"jobs_per_s": len(jobs) * args.steps / total, "ms_per_step": 1000 * total / args.steps,
                         "mpaths_per_s": n_paths * args.steps / total / 1e6,
                         "gpu_launches": int(ctx.stats()["kernel_launches"])}
        images[name] = out.cpu().numpy()
    clock_info = clocks.stop()
    same = all(np.array_equal(images["batched"], images[k], equal_nan=True) for k in images)
    nonfinite = {k: int((~np.isfinite(v)).sum()) for k, v in images.items()}
    max_diff = {k: float(np.nanmax(np.abs(images["batched"] - v))) for k, v in images.items()}

    # end to end: lrt_render_batch with the host output buffer
    host = np.zeros(floats, dtype=np.float32)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        ctx.render_batch(jobs, DEPTH, RR, host)
    e2e = len(jobs) * args.steps / (time.perf_counter() - t0)
    b = results["batched"]
    line = {"metric": BATCH_METRIC, "value": b["jobs_per_s"], "unit": "jobs/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": b["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scenes.batch_jobs)",
            "config": {"workload": "batch_%d_jobs_seed_%d" % (len(jobs), scenes.BATCH_SEED), "jobs": len(jobs),
                       "paths_per_step": n_paths, "max_depth": DEPTH, "rr_depth": RR,
                       "l2": "flushed (256 MB write) between timed steps", "arms": results,
                       "images_identical_across_arms": same, "nonfinite_floats": nonfinite,
                       "max_abs_diff_to_batched": max_diff, **tuned},
            "e2e": {"value": e2e, "unit": "jobs/s", "h2d_bytes_per_step": 80 * len(jobs),
                    "d2h_bytes_per_step": 4 * floats, "path": "lrt_render_batch (host output buffer)"},
            "clocks": clock_info, "gpu_launches": b["gpu_launches"]}
    print(json.dumps(line))
    ctx.close()
    return 0


# ------------------------------------------------------------------------------------------------
# differentiation workload: L2 image loss of the seven-material scene against a target at alpha 0.3,
# sphere albedo (0.7, 0.5, 0.3); Adam (lr 0.01) from alpha 0.6 on the 32 material parameters

ADJ_METRIC = "grad-steps/s (7 materials x 256x256 x 32 spp, depth 6, 32 material parameters, Adam)"


def run_adjoint(args):
    import torch
    import diff
    import lrt

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    w = h = 256
    spp, depth, rr = 32, 6, 3
    scene, sphere, index = scenes.open_box_library()
    ctx = lrt.Context(local, stream.cuda_stream)
    ctx.upload(scene)
    dm = diff.Differentiable(ctx, scene)
    params = dm.params
    names = dm.names()

    def jobs_at(spp_, offset):
        out, off = [], 0
        for name in MATERIALS:
            out.append(scenes.job_desc(scene.camera, w, h, spp_, offset, sphere, index[name], off))
            off += 3 * w * h
        return out, off

    _, floats = jobs_at(spp, 0)
    n_paths = len(MATERIALS) * w * h * spp
    # target: every roughness 0.3, the diffuse sphere's albedo (0.7, 0.5, 0.3), copper as in the scene
    target_values = dm.values()
    start_values = dm.values()
    for j, (m, field, c) in enumerate(params):
        if field == "alpha":
            target_values[j], start_values[j] = 0.3, 0.6
        if m == index["diffuse"] and field == "diffuse_reflectance":
            target_values[j] = (0.7, 0.5, 0.3)[c]
    img = torch.empty(floats, dtype=torch.float32, device=dev)
    target = torch.empty(floats, dtype=torch.float32, device=dev)
    dm.set_values(target_values, setup=False)
    ctx.render_batch_dev(jobs_at(256, 1 << 24)[0], depth, rr, target.data_ptr())
    grad = torch.zeros(len(params), dtype=torch.float64, device=dev)

    def clean_loss(values):
        dm.set_values(values, setup=False)
        ctx.render_batch_dev(jobs_at(128, 1 << 26)[0], depth, rr, img.data_ptr())
        return float(((img - target) ** 2).mean())

    loss_start = clean_loss(start_values)
    dm.set_values(start_values)
    m1 = np.zeros(len(params))
    m2 = np.zeros(len(params))
    lr, b1, b2, eps = 0.01, 0.9, 0.999, 1e-8
    values = start_values.copy()
    fwd_ms, adj_ms, step_s, losses = [], [], [], []
    steps = args.adjoint_steps
    clocks = ClockSampler(os.environ.get("CUDA_VISIBLE_DEVICES", str(local)).split(",")[0])
    clocks.start()
    ctx.reset_stats()
    for it in range(steps):
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        e[0].record(stream)
        ctx.render_batch_dev(jobs_at(spp, 2 * spp * it)[0], depth, rr, img.data_ptr())
        e[1].record(stream)
        adjoint = (2.0 / floats) * (img - target)
        grad.zero_()
        dm.adjoint_dev(jobs_at(spp, 2 * spp * it + spp)[0], depth, rr, adjoint.data_ptr(), grad.data_ptr())
        e[2].record(stream)
        g = grad.cpu().numpy()
        losses.append(float(((img - target) ** 2).mean()))
        m1 = b1 * m1 + (1 - b1) * g
        m2 = b2 * m2 + (1 - b2) * g * g
        values = values - lr * (m1 / (1 - b1 ** (it + 1))) / (np.sqrt(m2 / (1 - b2 ** (it + 1))) + eps)
        for j, (m, field, c) in enumerate(params):
            values[j] = np.clip(values[j], 0.05, 1.0) if field == "alpha" else max(values[j], 1e-3)
        dm.set_values(values)
        torch.cuda.synchronize(dev)
        step_s.append(time.perf_counter() - t0)
        fwd_ms.append(e[0].elapsed_time(e[1]))
        adj_ms.append(e[1].elapsed_time(e[2]))
    clock_info = clocks.stop()
    launches = int(ctx.stats()["kernel_launches"])
    loss_end = clean_loss(values)
    timed = slice(min(3, steps - 1), steps)  # the first steps include one-time set-up
    total = float(sum(step_s[timed]))
    n_timed = len(step_s[timed])
    alpha_idx = [j for j, p in enumerate(params) if p[1] == "alpha"]
    line = {"metric": ADJ_METRIC, "value": n_timed / total, "unit": "grad-steps/s", "n_gpus": 1,
            "steps": n_timed, "warmup": steps - n_timed, "ms_per_step": 1000 * total / n_timed,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded scenes.open_box_library)",
            "config": {"workload": "adjoint_7x256x256x32spp_depth6_adam200", "paths_per_render": n_paths,
                       "parameters": len(params), "adam_steps": steps, "lr": lr,
                       "forward_ms": statistics.median(fwd_ms[timed]), "adjoint_ms": statistics.median(adj_ms[timed]),
                       "adjoint_over_forward": statistics.median(adj_ms[timed]) / statistics.median(fwd_ms[timed]),
                       "forward_mpaths_s": n_paths / statistics.median(fwd_ms[timed]) / 1e3,
                       "adjoint_mpaths_s": n_paths / statistics.median(adj_ms[timed]) / 1e3,
                       "clean_loss_start": loss_start, "clean_loss_end": loss_end,
                       "loss_first": losses[0], "loss_last": losses[-1],
                       "alphas_end": {names[j]: float(values[j]) for j in alpha_idx},
                       "sphere_albedo_end": [float(values[j]) for j, p in enumerate(params)
                                             if p[0] == index["diffuse"]],
                       "l2": "inputs (scene, 7 x 256x256 images) are L2-resident; not flushed"},
            "e2e": {"value": n_timed / total, "unit": "grad-steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 8 * len(params),
                    "path": "render_batch_dev + adjoint_dev + host Adam + lrt_scene_update_materials + lrt_diff_setup"},
            "clocks": clock_info, "gpu_launches": launches}
    print(json.dumps(line))
    ctx.close()
    return 0


# ------------------------------------------------------------------------------------------------
# large photon-mapping scene: 256 displaced level-5 icospheres (5.24M triangles) on a ground quad, sky
# + 4 quad lights; 16M photons (depth 8), k = 100, radius cap 0.05; 1024x1024 x 32 spp

LARGE_METRIC = "Mpaths/s (photon mapper eye pass, 1024x1024 x 32 spp, 5.24M-triangle 256-sphere scene, 16M photons, k=100)"


def run_large(args):
    import torch
    import lrt

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    c3 = scenes.CONFIG3
    w, h, spp = c3["width"], c3["height"], args.large_spp or c3["spp"]
    t0 = time.perf_counter()
    scene = scenes.large_scene()
    t_gen = time.perf_counter() - t0
    # the same upload with the kd-trees built on the host cores, for comparison (the default builds them on
    # the GPU at this size; the trees are identical)
    with lrt.Context(local, stream.cuda_stream) as ch:
        ch.set_option("kd_build_device", 0)
        t0 = time.perf_counter()
        ch.upload(scene)
        t_upload_host = time.perf_counter() - t0
    ctx = lrt.Context(local, stream.cuda_stream)
    t0 = time.perf_counter()
    ctx.upload(scene)
    t_upload = time.perf_counter() - t0
    out = torch.zeros(w * h * 3, dtype=torch.float32, device=dev)

    def timed(fn):
        torch.cuda.synchronize(dev)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / 1000.0

    clocks = ClockSampler(os.environ.get("CUDA_VISIBLE_DEVICES", str(local)).split(",")[0])
    clocks.start()
    t0 = time.perf_counter()
    pp, shots = ctx.photon_preprocess(c3["photons"], 0, max_depth=c3["photon_depth"], rr_depth=5,
                                      radius_cap=c3["radius_cap"], lookup_size=c3["k"])
    torch.cuda.synchronize(dev)
    t_photons = time.perf_counter() - t0
    pt_params = scenes.render_params(w, h, spp, 8, 3)
    ctx.render_dev(pt_params, out.data_ptr())  # warm: the wave buffers at the timed frame's size
    t_pt = timed(lambda: ctx.render_dev(pt_params, out.data_ptr()))
    ctx.reset_stats()
    t_eye = timed(lambda: ctx.render_photon_dev(pt_params, pp, out.data_ptr()))
    launches = int(ctx.stats()["kernel_launches"])
    clock_info = clocks.stop()
    img = out.view(h, w, 3).cpu().numpy()
    paths = w * h * spp
    line = {"metric": LARGE_METRIC, "value": paths / t_eye / 1e6, "unit": "Mpaths/s", "n_gpus": 1, "steps": 1,
            "warmup": 1, "ms_per_step": 1000 * t_eye, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scenes.large_scene)",
            "config": {"workload": "large_grid_8x8x4_level5_photon_1024x1024x%dspp" % spp,
                       "triangles": scene.triangle_count(), "objects": len(scene.objects),
                       "scene_gen_s": t_gen, "upload_s (kd-trees + object hierarchy + copy)": t_upload,
                       "upload_host_trees_s": t_upload_host,
                       "device_scene_mb": ctx.scene_bytes() / 1e6,
                       "photons": c3["photons"], "photon_particles_shot": shots[0],
                       "photon_preprocess_s (trace + map build)": t_photons, "k": c3["k"],
                       "radius": pp.global_radius, "photon_depth": c3["photon_depth"],
                       "path_tracer_mpaths_s (same scene, 1024x1024, depth 8)": paths / t_pt / 1e6,
                       "image_mean": [float(x) for x in img.reshape(-1, 3).mean(axis=0)],
                       "nonfinite": int((~np.isfinite(img)).sum())},
            "clocks": clock_info, "gpu_launches": launches}
    print(json.dumps(line))
    ctx.close()
    return 0


def abi_stage_names():
    import lrt_abi
    return lrt_abi.STAGE_NAMES


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="lrt", choices=["lrt", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--wave-capacity", type=int, default=0, help="paths per wave (0: the library's default)")
    ap.add_argument("--workload", default="paths", choices=["paths", "batch", "adjoint", "large"],
                    help="paths: the seven-material Mpaths/s workload; batch: the 64-job jobs/s comparison; "
                         "adjoint: gradient steps of the material optimisation")
    ap.add_argument("--jobs", type=int, default=64)
    ap.add_argument("--no-autotune", action="store_true", help="batch workload: default launch shapes")
    ap.add_argument("--adjoint-steps", type=int, default=200)
    ap.add_argument("--large-spp", type=int, default=0, help="large workload: spp (0: the configuration's 32)")
    args = ap.parse_args()
    ARGS_WAVE_CAPACITY[0] = args.wave_capacity
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "batch":
        return run_batch(args)
    if args.workload == "adjoint":
        return run_adjoint(args)
    if args.workload == "large":
        return run_large(args)
    return run_lrt(args)


if __name__ == "__main__":
    sys.exit(main())
