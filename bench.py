#!/usr/bin/env python
"""Benchmark of the LinRT rendering hot path on B200: Mpaths/s of the wavefront path tracer.

Headline workload (one step): the seven-material open-box scene set (Cornell-style box open to a Hosek
sky, a displaced level-6 icosphere of 81,920 triangles carrying each of the seven BSDFs in turn),
512x512 pixels, 64 samples per pixel, max depth 8, Russian roulette from depth 3 -- 7 x 16.8M = 117.4M
camera paths per step. Inputs are synthetic and seeded (scenes.py).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl lrt|reference] [--no-extras]
    python bench.py --workload batch|adjoint|large     (one GPU; one JSON line each)
    python bench.py --workload profile --case render|eye|adjoint|batch|kdbuild|knn   (small fixed cases
                                                        for ncu captures; prints a JSON summary)

The headline line also carries, measured in the same run on rank 0 at N = 1 (skipped with --no-extras),
the other configurations of the workload set, each with its own cpu_baseline:
  closed_box     the closed box under the ceiling light, 256x256 x 16 spp, depth 6 (Mpaths/s);
  photon_mapper  the photon mapper on the seven materials, 1M photons per map, k = 64 (photon trace and
                 map build, eye pass Mpaths/s, and the k-nearest-photon query's roofline);
  batch          64 seeded jobs in shared waves against per-job launches (jobs/s);
  adjoint        gradient steps of the 38-parameter material optimisation (grad-steps/s, adjoint cost
                 over forward cost).

N > 1 runs as one process per GPU under torch.distributed (NCCL): every rank renders its own replica
with a disjoint sample range (no data-path collective), the timed region is bracketed by barriers and
the max over ranks is reported. --impl reference times the reference's own CPU renderer (the
unmodified sources built in oracle/_ref, timing build) on this host's cores, on the headline
workload's configuration, each step a bounded sample of it.
"""
import argparse
import hashlib
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
GOLDEN = os.path.join(ROOT, "tests", "golden")


def config():
    """the headline workload (identical in both arms)"""
    return {"workload": WORKLOAD, "width": W, "height": H, "spp": SPP, "max_depth": DEPTH, "rr_depth": RR,
            "materials": MATERIALS, "triangles": 81920 + 12, "paths_per_step": PATHS_PER_STEP,
            "l2": "flushed (256 MB write) between timed steps", "parallelism": "replicas",
            "wave_capacity": ARGS_WAVE_CAPACITY[0] or "library default (2^24: one wave per frame)"}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def source_digest(names):
    """first 16 hex digits of the SHA-256 of the named library sources (ties a capture to its kernel). A
    name "file:marker" takes only the text of file from the line holding marker to the next line that is
    a lone closing brace (one function), so that edits elsewhere in a large file leave the digest alone;
    "file@marker" takes the text of file up to marker (its leading part)."""
    h = hashlib.sha256()
    for n in names:
        path, _, marker = n.partition(":")
        path, _, until = path.partition("@")
        with open(os.path.join(ROOT, "ray-tracing_b200", "csrc", path), "rb") as f:
            text = f.read()
        if marker:
            i = text.index(marker.encode())
            i = text.rindex(b"\n", 0, i) + 1
            text = text[i:text.index(b"\n}\n", i) + 3]
        if until:
            text = text[:text.index(until.encode())]
        h.update(text)
    return h.hexdigest()[:16]


# the closest-hit kernel: the traversal part of lrt_scene.cuh (everything before the hit-record and
# emitter code), its other headers and its own function in lrt_api.cu
EXTEND_SOURCES = ["lrt_scene.cuh@// The hit record of a finished closest-hit traversal", "lrt_math.cuh", "lrt_types.h",
                  "lrt_api.cu:__global__ void __launch_bounds__(kBlock, 8) k_extend_persistent(",
                  "lrt_api.cu:constexpr int kRefillLanes"]


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
            return self
        # nvidia-smi takes a second or more to start: wait (at most 10 s) for its first sample, so that the
        # samples cover the whole timed region that follows
        deadline = time.monotonic() + 10.0
        while time.monotonic() < deadline and self.proc.poll() is None and os.path.getsize(self.file.name) == 0:
            time.sleep(0.05)
        return self

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


def gpu_index(local):
    return os.environ.get("CUDA_VISIBLE_DEVICES", str(local)).split(",")[0]


class Gpu:
    """torch device, the library's stream (flushes and timing events go on it too) and an L2 flush"""

    def __init__(self, local):
        import torch
        self.torch = torch
        torch.cuda.set_device(local)
        self.local = local
        self.dev = torch.device("cuda", local)
        self.stream = torch.cuda.Stream(self.dev)
        torch.cuda.set_stream(self.stream)
        self.flush_buf = torch.empty(256 << 20, dtype=torch.uint8, device=self.dev)

    def flush(self):
        self.flush_buf.zero_()

    def sync(self):
        self.torch.cuda.synchronize(self.dev)

    def time(self, fn):
        """seconds of fn's work on the library's stream (CUDA events)"""
        e0 = self.torch.cuda.Event(enable_timing=True)
        e1 = self.torch.cuda.Event(enable_timing=True)
        e0.record(self.stream)
        fn()
        e1.record(self.stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / 1000.0

    def context(self):
        import lrt
        return lrt.Context(self.local, self.stream.cuda_stream)


# ------------------------------------------------------------------------------------------------
# CPU reference (oracle/_ref: the unmodified reference sources); only the cpu_baseline legs and
# --impl reference use it

def load_oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    return oracle if oracle.reference_available() else None


def ref_world(oracle, scene):
    return oracle.RefWorld(scene, timing=True)


def timing_note(oracle):
    return "reference sources built %s, %d threads (hardware_concurrency)" % (
        oracle.timing_build_flags(), oracle.hardware_concurrency())


def headline_worlds(oracle):
    """the seven open-box scenes as the reference builds them (its own materials, tables and sky)"""
    return [ref_world(oracle, scenes.open_box(m, attach=False)) for m in MATERIALS]


def reference_pass(worlds, spp, sample_offset=0):
    """one pass over the seven scenes at 512x512 x `spp` on all host cores; returns (paths, seconds)"""
    secs = 0.0
    for w in worlds:
        _, _, s = w.render(scenes.render_params(W, H, spp, DEPTH, RR, sample_offset=sample_offset), 0)
        secs += s
    return len(worlds) * W * H * spp, secs


def cpu_baseline(oracle, budget_s=15.0):
    worlds = headline_worlds(oracle)
    spp, paths, secs = 1, 0, 0.0
    while secs < budget_s:
        p, s = reference_pass(worlds, spp, sample_offset=paths)
        paths += p
        secs += s
        if secs < budget_s / 4:
            spp *= 2
    for w in worlds:
        w.close()
    return {"value": paths / secs / 1e6, "unit": "Mpaths/s", "cores": oracle.hardware_concurrency(),
            "kind": "reference",
            "sample": "%d paths: the 7 scenes at 512x512 with %d..%d spp per pass (same scenes, depth, roulette), "
                      "32x32 tiles as main.cpp; %s" % (paths, 1, spp, timing_note(oracle))}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    oracle = load_oracle()
    if oracle is None:
        print(json.dumps({"impl": "reference", "unavailable": "reference sources not built (oracle/_ref missing)"}))
        return 0
    worlds = headline_worlds(oracle)
    spp = 1
    for i in range(args.warmup):
        reference_pass(worlds, spp, sample_offset=1000 + 8 * i)
    times, paths = [], 0
    for i in range(args.steps):
        p, s = reference_pass(worlds, spp, sample_offset=8 * i)
        times.append(s)
        paths += p
    for w in worlds:
        w.close()
    total = sum(times)
    value = paths / total / 1e6
    cores = oracle.hardware_concurrency()
    line = {"metric": METRIC, "value": value, "unit": "Mpaths/s", "impl": "reference", "n_gpus": 0,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * total / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": config(),
            "cpu_baseline": {"value": value, "unit": "Mpaths/s", "cores": cores, "kind": "reference",
                             "sample": "each step: the 7 scenes at 512x512 x %d spp (%d paths, a bounded sample of "
                                       "the 64-spp workload); %s" % (spp, len(MATERIALS) * W * H * spp,
                                                                    timing_note(oracle))},
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


def abi_stage_names():
    import lrt_abi
    return lrt_abi.STAGE_NAMES


def extend_traffic(work, timed_paths, extend_launches):
    """DRAM bytes per k_extend launch from the committed ncu capture, scaled to this run's average launch
    by its extension rays; null when the kernel's sources changed since that capture"""
    tpath = os.path.join(ROOT, "profiles", "extend_traffic.json")
    if not os.path.exists(tpath) or not extend_launches:
        return None, None, "no capture"
    with open(tpath) as f:
        tr = json.load(f)
    issue = {"issue_active_frac": tr.get("issue_active_frac"),
             "simt_lane_efficiency": (tr.get("lanes_per_warp_instruction") or 0) / 32.0 or None,
             "source": tr.get("source")}
    digest = source_digest(EXTEND_SOURCES)
    if tr.get("source_sha16") != digest:
        return None, issue, "stale: the kernel's sources changed since the capture (%s, now %s)" % (
            tr.get("source_sha16"), digest)
    traffic = tr["dram_bytes_per_extension_ray"] * work["extension_rays_per_path"] * timed_paths / extend_launches
    return traffic, issue, "ncu capture %s scaled by extension rays" % tr.get("source")


def crop_rmse(gpu, ctxs, oracle):
    """Error at equal spp: each material's frame at 64 spp (the timed frames' samples) over the crop the
    4096-spp reference fixture holds, against that fixture; beside it the error the fixture's per-pixel
    variance predicts for 64 spp, and (CPU) the reference renderer's own 64-spp crop on the same samples."""
    path = os.path.join(GOLDEN, "converged_kat.npz")
    if not os.path.exists(path):
        return None
    g = np.load(path)
    r0, r1, x0, x1 = (int(v) for v in g["crop"])
    n_ref = int(g["spp"])
    out = {}
    for name, c in zip(MATERIALS, ctxs):
        img = c.render(scenes.render_params(W, H, SPP, DEPTH, RR, row_begin=r0, row_end=r1))[r0:r1, x0:x1]
        mean, sq = g["open_%s_mean" % name].astype(np.float64), g["open_%s_sq" % name].astype(np.float64)
        var = np.maximum(sq - mean * mean, 0.0)
        entry = {"gpu_64spp": float(np.sqrt(np.mean((img - mean) ** 2))),
                 "predicted_64spp": float(np.sqrt(np.mean(var / SPP + var / n_ref)))}
        if oracle is not None:
            w = oracle.RefWorld(scenes.open_box(name, attach=False))
            ref, _, _ = w.render_window(scenes.render_params(W, H, SPP, DEPTH, RR, row_begin=r0, row_end=r1), x0, x1)
            w.close()
            entry["reference_64spp"] = float(np.sqrt(np.mean((ref[r0:r1, x0:x1] - mean) ** 2)))
        out[name] = entry
    return {"per_material": out,
            "against": "the reference renderer's 4096-spp render of each 512x512 frame over rows %d-%d, columns "
                       "%d-%d (tests/golden/converged_kat.npz)" % (r0, r1 - 1, x0, x1 - 1)}


# ------------------------------------------------------------------------------------------------
# headline workload

def run_lrt(args):
    import lrt

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    gpu = Gpu(local)
    torch = gpu.torch

    ctxs = []
    for m in MATERIALS:
        c = gpu.context()
        c.upload(scenes.open_box(m))
        if args.wave_capacity:
            c.set_option("wave_capacity", args.wave_capacity)
        ctxs.append(c)
    out = torch.empty((H, W, 3), dtype=torch.float32, device=gpu.dev)
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
    gpu.sync()
    for c in ctxs:
        c.reset_stats()
        c.set_option("stage_timing", 1)

    clocks = ClockSampler(gpu_index(local) if world == 1 else local)
    if dist:
        dist.barrier()
    gpu.sync()
    clocks.start()
    step_ms = []
    for _ in range(args.steps):
        gpu.flush()
        step_ms.append(1000.0 * gpu.time(step))
    gpu.sync()
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
    total_ms = max_over_ranks(dist, total_ms, gpu.dev)

    # end to end: the public host-buffer call (lrt_render: render + device->host copy of the image)
    host_img = np.zeros((H, W, 3), dtype=np.float32)
    e2e_times = []
    if dist:
        dist.barrier()
    for i in range(args.steps):
        gpu.flush()
        gpu.sync()
        t0 = time.perf_counter()
        for c in ctxs:
            c.render(params, host_img)
        e2e_times.append(time.perf_counter() - t0)
    e2e_total = max_over_ranks(dist, sum(e2e_times), gpu.dev)

    value = whole_job_mpaths(world, PATHS_PER_STEP, args.steps, total_ms / 1000.0)
    e2e_value = whole_job_mpaths(world, PATHS_PER_STEP, args.steps, e2e_total)
    peak, peak_kind = measured_peaks()
    timed_paths = PATHS_PER_STEP * args.steps
    achieved = (work["extend_bytes_per_path"] * timed_paths / 1e9) / (extend_ms / 1000.0) if extend_ms > 0 else None
    traffic, issue, traffic_note = extend_traffic(work, timed_paths, extend_launches)

    solo = rank == 0 and world == 1
    oracle = load_oracle() if solo else None
    cpu = cpu_baseline(oracle) if (oracle is not None and not args.no_cpu_baseline) else None

    # the plain GPU path tracer (one launch per frame, one thread per pixel, whole path in registers) on
    # the same frames and samples: same images, its time beside the wavefront's
    plain = None
    if solo:
        cam = scenes.open_box(MATERIALS[0], attach=False).camera
        job = scenes.job_desc(cam, W, H, SPP, offset)

        def plain_step():
            for c in ctxs:
                c.render_plain_dev([job], DEPTH, RR, out.data_ptr())

        plain_step()  # warm
        gpu.flush()
        gpu.sync()
        plain_s = gpu.time(plain_step)
        plain = {"value": PATHS_PER_STEP / plain_s / 1e6, "unit": "Mpaths/s", "steps": 1,
                 "kernel": "k_pt_plain (lrt_render_plain): one launch per frame, one thread per pixel",
                 "wavefront_speedup": value * plain_s * 1e6 / PATHS_PER_STEP}
    rmse = crop_rmse(gpu, ctxs, oracle if not args.no_cpu_baseline else None) if solo else None
    for c in ctxs:
        c.close()

    extras = {}
    if solo and not args.no_extras:
        extras["closed_box"] = measure_closed_box(gpu, oracle, args)
        extras["photon_mapper"] = measure_photon_mapper(gpu, oracle, args)
        extras["batch"] = measure_batch(gpu, oracle, args, steps=2, warmup=1)
        extras["adjoint"] = measure_adjoint(gpu, oracle, args, adam_steps=args.adjoint_steps)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "Mpaths/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scenes.py)",
            "config": config(),
            "e2e": {"value": e2e_value, "unit": "Mpaths/s", "h2d_bytes_per_step": len(MATERIALS) * 32,
                    "d2h_bytes_per_step": len(MATERIALS) * W * H * 3 * 4,
                    "path": "lrt_render (host output buffer; scene resident after lrt_scene_upload)"},
            "roofline": {"kernel": "k_extend (closest-hit kd-tree traversal)", "bound": "hbm",
                         "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": (achieved / peak) if achieved else None, "peak_kind": peak_kind,
                         "traffic": traffic, "traffic_source": traffic_note,
                         "algorithmic_bytes": "per extension ray 8*nodes + 48*triangles + 32 ray + 16 hit",
                         "avg_launch_ms": extend_ms / max(1, extend_launches),
                         "issue": issue},
            "cpu_baseline": cpu,
            "work_per_path": work,
            "stage_ms_per_step": {k: v / args.steps for k, v in stage_ms.items()},
            "rmse": rmse,
            "plain_gpu_pt": plain,
            "clocks": clock_info,
            "gpu_launches": launches,
        }
        line.update(extras)
        print(json.dumps(line))
    if dist:
        dist.destroy_process_group()
    return 0


# ------------------------------------------------------------------------------------------------
# closed box (the reference's CPU-runnable configuration): 256x256 x 16 spp, depth 6, RR from 3

def measure_closed_box(gpu, oracle, args, steps=20, warmup=3):
    c0 = scenes.CONFIG0
    w, h, spp = c0["width"], c0["height"], c0["spp"]
    ctx = gpu.context()
    ctx.upload(scenes.cornell_box())
    out = gpu.torch.empty((h, w, 3), dtype=gpu.torch.float32, device=gpu.dev)
    params = scenes.render_params(w, h, spp, c0["max_depth"], c0["rr_depth"])
    for _ in range(warmup):
        ctx.render_dev(params, out.data_ptr())
    gpu.sync()
    ctx.reset_stats()
    secs = []
    for _ in range(steps):
        gpu.flush()
        secs.append(gpu.time(lambda: ctx.render_dev(params, out.data_ptr())))
    launches = int(ctx.stats()["kernel_launches"])
    host = np.zeros((h, w, 3), dtype=np.float32)
    gpu.sync()
    t0 = time.perf_counter()
    for _ in range(steps):
        ctx.render(params, host)
    e2e = w * h * spp * steps / (time.perf_counter() - t0) / 1e6
    paths = w * h * spp
    res = {"metric": "Mpaths/s (closed box, 256x256 x 16 spp, depth 6)", "value": paths * steps / sum(secs) / 1e6,
           "unit": "Mpaths/s", "steps": steps, "ms_per_step": 1000 * sum(secs) / steps,
           "config": {"workload": "closed_box_256x256_16spp_depth6", "paths_per_step": paths,
                      "l2": "flushed between timed steps"},
           "e2e": {"value": e2e, "unit": "Mpaths/s", "h2d_bytes_per_step": 32, "d2h_bytes_per_step": 4 * 3 * w * h},
           "gpu_launches": launches}
    path = os.path.join(GOLDEN, "converged_kat.npz")
    if os.path.exists(path):
        g = np.load(path)
        mean, sq = g["closed_box_mean"].astype(np.float64), g["closed_box_sq"].astype(np.float64)
        var = np.maximum(sq - mean * mean, 0.0)
        res["rmse"] = {"gpu_16spp": float(np.sqrt(np.mean((host - mean) ** 2))),
                       "predicted_16spp": float(np.sqrt(np.mean(var / spp + var / int(g["spp"])))),
                       "against": "the reference renderer's 4096-spp 256x256 render (tests/golden/converged_kat.npz)"}
    ctx.close()
    if oracle is not None and not args.no_cpu_baseline:
        wld = ref_world(oracle, scenes.cornell_box(attach=False))
        rows, n, secs_cpu = 32, 0, 0.0
        while secs_cpu < 4.0:
            p = scenes.render_params(w, h, spp, c0["max_depth"], c0["rr_depth"], sample_offset=n * spp,
                                     row_begin=(n * rows) % h, row_end=(n * rows) % h + rows)
            secs_cpu += wld.render(p, 0)[2]
            n += 1
        wld.close()
        res["cpu_baseline"] = {"value": n * rows * w * spp / secs_cpu / 1e6, "unit": "Mpaths/s",
                               "cores": oracle.hardware_concurrency(), "kind": "reference",
                               "sample": "%d bands of %d rows x 256 x 16 spp; %s" % (n, rows, timing_note(oracle))}
    return res


# ------------------------------------------------------------------------------------------------
# photon mapper on the seven materials: 1M photons per map (global and caustic), k = 64

PHOTONS = scenes.CONFIG1["photons"]
KNN_K = scenes.CONFIG1["k"]


def diffuse_query_points(ctx, scene, w, h):
    """first hits of one camera ray per pixel on diffuse surfaces (where the eye pass looks photons up):
    points and shading normals, float32"""
    import lrt_abi as abi
    ps = np.zeros((w * h, 2), dtype=np.uint32)
    ps[:, 0] = np.arange(w * h)
    rays = ctx.camera_rays(w, h, ps)
    hits = ctx.trace(rays)
    diffuse = {i for i, o in enumerate(scene.objects)
               if o.get("material", -1) >= 0 and scene.materials[o["material"]]["type"] == abi.MAT_DIFFUSE}
    keep = np.array([o in diffuse for o in hits["object"]])
    return (np.ascontiguousarray(hits["p"][keep], dtype=np.float32),
            np.ascontiguousarray(hits["normal"][keep], dtype=np.float32))


def reference_eye_rate(ctx, oracle, material, pp, w, h, budget_s):
    """The reference's photon-mapper eye pass on the host cores over bands of rows of one material's scene,
    with the photon maps this context's preprocess built (traced again here as photon arrays): Mpaths/s
    and the number of 8-row bands rendered."""
    import lrt_abi as abi
    g, shot_g = ctx.photon_trace(abi.GATHER_SURFACE, PHOTONS, 128, 5)
    c, shot_c = np.zeros(0, dtype=abi.PHOTON_DTYPE), 1
    if pp.caustic_map >= 0:
        c, shot_c = ctx.photon_trace(abi.GATHER_CAUSTIC, PHOTONS, 128, 5)
    wld = ref_world(oracle, scenes.cornell_box(material=material, attach=False))
    rows, n, secs = 8, 0, 0.0
    while secs < budget_s and n < 64:
        p = scenes.render_params(w, h, 1, DEPTH, RR, sample_offset=n, row_begin=(n * 37 * rows) % h,
                                 row_end=(n * 37 * rows) % h + rows)
        pq = abi.PhotonRenderParams.reference_defaults(lookup_size=KNN_K)
        pq.global_radius, pq.caustic_radius = pp.global_radius, pp.caustic_radius
        _, _, t = wld.render_photon(p, pq, g, np.float32(1.0 / max(1, shot_g)), c,
                                    np.float32(1.0 / max(1, shot_c)), want_sq=False)
        secs += t
        n += 1
    wld.close()
    return n * rows * w / secs / 1e6, n


def measure_photon_mapper(gpu, oracle, args, spp=4, knn_steps=10):
    import lrt_abi as abi
    torch = gpu.torch
    c1 = scenes.CONFIG1
    w, h = c1["width"], c1["height"]
    params = scenes.render_params(w, h, spp, DEPTH, RR)
    out = torch.empty((h, w, 3), dtype=torch.float32, device=gpu.dev)
    per, knn_bytes, knn_s, knn_q = {}, 0.0, 0.0, 0
    pre_s, eye_s, launches = 0.0, 0.0, 0
    cpu_rates = {}
    for m in MATERIALS:
        scene = scenes.cornell_box(material=m)
        ctx = gpu.context()
        ctx.upload(scene)
        gpu.sync()
        t0 = time.perf_counter()
        pp, shots = ctx.photon_preprocess(PHOTONS, PHOTONS, max_depth=128, rr_depth=5, lookup_size=KNN_K)
        gpu.sync()
        t_pre = time.perf_counter() - t0
        ctx.render_photon_dev(params, pp, out.data_ptr())  # warm: the eye pass's slots sized for this image
        gpu.flush()
        gpu.sync()
        ctx.reset_stats()
        t_eye = gpu.time(lambda: ctx.render_photon_dev(params, pp, out.data_ptr()))
        launches += int(ctx.stats()["kernel_launches"])
        # the k-nearest-photon query alone: the global map at the eye pass's first diffuse hits
        pts, nrm = diffuse_query_points(ctx, scene, w, h)
        dp = torch.from_numpy(pts).to(gpu.dev)
        dn = torch.from_numpy(nrm).to(gpu.dev)
        rgb = torch.empty_like(dp)
        n = len(pts)

        def knn():
            ctx.photon_irradiance_dev(pp.global_map, dp.data_ptr(), dn.data_ptr(), n, pp.global_radius, 128, KNN_K,
                                      rgb.data_ptr())

        ctx.set_option("count_work", 1)
        ctx.reset_stats()
        knn()
        s = ctx.stats()
        ctx.set_option("count_work", 0)
        bytes_q = (16 * s["knn_nodes_visited"] + 16 * s["knn_photons_tested"] + 48 * s["knn_photons_found"])
        knn()
        gpu.flush()
        gpu.sync()
        ks = sum(gpu.time(knn) for _ in range(knn_steps))
        knn_bytes += bytes_q * knn_steps
        knn_s += ks
        knn_q += n * knn_steps
        per[m] = {"photon_preprocess_s": t_pre, "eye_ms": 1000 * t_eye, "particles_shot": list(shots),
                  "radius": pp.global_radius, "knn_queries": n,
                  "knn_nodes_per_query": s["knn_nodes_visited"] / max(1, n),
                  "knn_photons_tested_per_query": s["knn_photons_tested"] / max(1, n),
                  "knn_photons_found_per_query": s["knn_photons_found"] / max(1, n)}
        pre_s += t_pre
        eye_s += t_eye
        if oracle is not None and not args.no_cpu_baseline:
            cpu_rates[m] = reference_eye_rate(ctx, oracle, m, pp, w, h, budget_s=2.5)
            per[m]["cpu_mpaths_s"] = cpu_rates[m][0]
        del dp, dn, rgb
        ctx.close()
    paths = len(MATERIALS) * w * h * spp
    peak, peak_kind = measured_peaks()
    achieved = knn_bytes / knn_s / 1e9
    res = {"metric": "Mpaths/s (photon-mapper eye pass, 7 materials x 512x512 x %d spp, 1M photons per map, k=64)"
                     % spp, "value": paths / eye_s / 1e6, "unit": "Mpaths/s",
           "config": {"workload": "closed_box_7_materials_photon_mapper_512x512_%dspp" % spp,
                      "scenes": "the closed box (ceiling light) with each material on the sphere: the open box's sky "
                                "emits no photons (env_emitter.h:96-98), so photon mapping needs the area light",
                      "photons_per_map": PHOTONS, "maps": "global + caustic", "k": KNN_K, "photon_depth": 128,
                      "eye_max_depth": DEPTH},
           "photon_preprocess_s_total": pre_s,
           "photon_preprocess_mphotons_s": 2 * PHOTONS * len(MATERIALS) / pre_s / 1e6,
           "per_material": per, "gpu_launches": launches,
           "knn_roofline": {"kernel": "k_irradiance (k-nearest photons + irradiance estimate, one query per thread)",
                            "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                            "frac": achieved / peak, "peak_kind": peak_kind,
                            "queries_per_s": knn_q / knn_s,
                            "algorithmic_bytes": "per query 16*nodes + 16*photon positions tested + 48*photons found "
                                                 "(16-byte nodes; direction, normal, power of each photon found)",
                            "note": "1M-photon maps (~80 MB with nodes) are L2-resident"}}
    if cpu_rates:
        # equal paths per material, as the GPU figure: the harmonic combination of the per-material rates
        value = len(cpu_rates) / sum(1.0 / r for r, _ in cpu_rates.values())
        res["cpu_baseline"] = {"value": value, "unit": "Mpaths/s", "cores": oracle.hardware_concurrency(),
                               "kind": "reference",
                               "sample": "each material's eye pass (photon_integrator::radiance) over bands of 8 rows x "
                                         "512 x 1 spp (%s bands), with the GPU's 1M-photon global and caustic maps, "
                                         "rates combined for equal paths per material; %s"
                                         % (", ".join("%s %d" % (m, n) for m, (_, n) in cpu_rates.items()),
                                            timing_note(oracle))}
    return res


# ------------------------------------------------------------------------------------------------
# batched workload: 64 seeded jobs (resolution, spp 4-256, camera, sphere material) on the open box

BATCH_METRIC = "jobs/s (64 seeded jobs: 128^2..1024x768, 4-256 spp, 7 materials, depth 8)"


def measure_batch(gpu, oracle, args, steps, warmup):
    import autotune
    torch = gpu.torch
    scene, sphere, index = scenes.open_box_library()
    jobs, specs = scenes.batch_jobs(index, sphere, n_jobs=args.jobs)
    n_paths = sum(j["width"] * j["height"] * j["spp"] for j in specs)
    floats = max(j["output_offset"] + 3 * j["width"] * j["height"] for j in specs)
    ctx = gpu.context()
    ctx.upload(scene)
    out = torch.zeros(floats, dtype=torch.float32, device=gpu.dev)
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

    arms = {"batched": batched, "per_job_plain": per_job_plain, "per_job_wavefront": per_job_wavefront,
            "persistent_queue": batched}
    results, images = {}, {}
    for name, fn in arms.items():
        if name == "per_job_wavefront":
            ctx.set_option("batch_graph", 0)
        # one persistent megakernel launch pulling (job, 32-pixel tile) items from a device queue
        ctx.set_option("batch_queue", 1 if name == "persistent_queue" else 0)
        for _ in range(warmup):
            fn()
        gpu.sync()
        ctx.reset_stats()
        secs = []
        for _ in range(steps):
            gpu.flush()
            secs.append(gpu.time(fn))
        ctx.set_option("batch_graph", 1)
        ctx.set_option("batch_queue", 0)
        total = sum(secs)
        results[name] = {"jobs_per_s": len(jobs) * steps / total, "ms_per_step": 1000 * total / steps,
                         "mpaths_per_s": n_paths * steps / total / 1e6,
                         "gpu_launches": int(ctx.stats()["kernel_launches"])}
        images[name] = out.cpu().numpy()
    same = all(np.array_equal(images["batched"], images[k], equal_nan=True) for k in images)
    nonfinite = {k: int((~np.isfinite(v)).sum()) for k, v in images.items()}

    # end to end: lrt_render_batch with the host output buffer
    host = np.zeros(floats, dtype=np.float32)
    gpu.sync()
    t0 = time.perf_counter()
    for _ in range(steps):
        ctx.render_batch(jobs, DEPTH, RR, host)
    e2e = len(jobs) * steps / (time.perf_counter() - t0)
    ctx.close()
    b = results["batched"]
    res = {"metric": BATCH_METRIC, "value": b["jobs_per_s"], "unit": "jobs/s", "steps": steps, "warmup": warmup,
           "ms_per_step": b["ms_per_step"],
           "config": {"workload": "batch_%d_jobs_seed_%d" % (len(jobs), scenes.BATCH_SEED), "jobs": len(jobs),
                      "paths_per_step": n_paths, "max_depth": DEPTH, "rr_depth": RR,
                      "l2": "flushed (256 MB write) between timed steps"},
           "arms": results, "batched_over_per_job_plain": b["jobs_per_s"] / results["per_job_plain"]["jobs_per_s"],
           "batched_over_per_job_wavefront": b["jobs_per_s"] / results["per_job_wavefront"]["jobs_per_s"],
           "batched_over_persistent_queue": b["jobs_per_s"] / results["persistent_queue"]["jobs_per_s"],
           "images_identical_across_arms": same, "nonfinite_floats": nonfinite, **tuned,
           "e2e": {"value": e2e, "unit": "jobs/s", "h2d_bytes_per_step": 80 * len(jobs),
                   "d2h_bytes_per_step": 4 * floats, "path": "lrt_render_batch (host output buffer)"},
           "gpu_launches": b["gpu_launches"]}
    if oracle is not None and not args.no_cpu_baseline:
        # the reference renders jobs one after another; its jobs/s follows from its path throughput on the
        # jobs' scenes and cameras (a band of rows of every job at 1 spp) and the batch's paths per job
        worlds = {}
        secs_cpu, paths_cpu = 0.0, 0
        for k, (j, spec) in enumerate(zip(jobs, specs)):
            name = spec["material"]
            sc = scenes.open_box(name, attach=False)
            sc.camera = spec["camera"]
            wld = ref_world(oracle, sc)
            rows = max(1, 4096 // spec["width"])
            p = scenes.render_params(spec["width"], spec["height"], 1, DEPTH, RR, sample_offset=k,
                                     row_begin=0, row_end=rows)
            secs_cpu += wld.render(p, 0)[2]
            paths_cpu += rows * spec["width"]
            wld.close()
        mpaths = paths_cpu / secs_cpu / 1e6
        res["cpu_baseline"] = {"value": mpaths * 1e6 / (n_paths / len(jobs)), "unit": "jobs/s",
                               "cores": oracle.hardware_concurrency(), "kind": "reference",
                               "mpaths_per_s": mpaths,
                               "sample": "%d paths: a band of rows of each of the 64 jobs (its scene, material and "
                                         "camera) at 1 spp, jobs/s = path rate / the batch's mean paths per job; %s"
                                         % (paths_cpu, timing_note(oracle))}
    return res


def run_batch(args):
    gpu = Gpu(int(os.environ.get("LOCAL_RANK", "0")))
    oracle = None if args.no_cpu_baseline else load_oracle()
    clocks = ClockSampler(gpu_index(gpu.local)).start()
    res = measure_batch(gpu, oracle, args, steps=args.steps, warmup=args.warmup)
    line = {"metric": res.pop("metric"), "value": res.pop("value"), "unit": res.pop("unit"), "n_gpus": 1,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded scenes.batch_jobs)", **res, "clocks": clocks.stop()}
    print(json.dumps(line))
    return 0


# ------------------------------------------------------------------------------------------------
# differentiation workload: L2 image loss of the seven-material scene against a target at alpha 0.3,
# sphere albedo (0.7, 0.5, 0.3); Adam (lr 0.01) from alpha 0.6 on the 38 material parameters

ADJ_METRIC = "grad-steps/s (7 materials x 256x256 x 32 spp, depth 6, 38 material parameters, Adam)"


def measure_adjoint(gpu, oracle, args, adam_steps):
    import diff
    torch = gpu.torch
    w = h = 256
    spp, depth, rr = 32, 6, 3
    scene, sphere, index = scenes.open_box_library()
    ctx = gpu.context()
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
    img = torch.empty(floats, dtype=torch.float32, device=gpu.dev)
    target = torch.empty(floats, dtype=torch.float32, device=gpu.dev)
    dm.set_values(target_values, setup=False)
    ctx.render_batch_dev(jobs_at(256, 1 << 24)[0], depth, rr, target.data_ptr())
    grad = torch.zeros(len(params), dtype=torch.float64, device=gpu.dev)

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
    ctx.reset_stats()
    for it in range(adam_steps):
        gpu.sync()
        t0 = time.perf_counter()
        e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        e[0].record(gpu.stream)
        ctx.render_batch_dev(jobs_at(spp, 2 * spp * it)[0], depth, rr, img.data_ptr())
        e[1].record(gpu.stream)
        adjoint = (2.0 / floats) * (img - target)
        grad.zero_()
        dm.adjoint_dev(jobs_at(spp, 2 * spp * it + spp)[0], depth, rr, adjoint.data_ptr(), grad.data_ptr())
        e[2].record(gpu.stream)
        g = grad.cpu().numpy()
        losses.append(float(((img - target) ** 2).mean()))
        m1 = b1 * m1 + (1 - b1) * g
        m2 = b2 * m2 + (1 - b2) * g * g
        values = values - lr * (m1 / (1 - b1 ** (it + 1))) / (np.sqrt(m2 / (1 - b2 ** (it + 1))) + eps)
        for j, (m, field, c) in enumerate(params):
            values[j] = np.clip(values[j], 0.05, 1.0) if field == "alpha" else max(values[j], 1e-3)
        dm.set_values(values)
        gpu.sync()
        step_s.append(time.perf_counter() - t0)
        fwd_ms.append(e[0].elapsed_time(e[1]))
        adj_ms.append(e[1].elapsed_time(e[2]))
    launches = int(ctx.stats()["kernel_launches"])
    loss_end = clean_loss(values)
    ctx.close()
    timed = slice(min(3, adam_steps - 1), adam_steps)  # the first steps include one-time set-up
    total = float(sum(step_s[timed]))
    n_timed = len(step_s[timed])
    alpha_idx = [j for j, p in enumerate(params) if p[1] == "alpha"]
    fwd, adj = statistics.median(fwd_ms[timed]), statistics.median(adj_ms[timed])
    res = {"metric": ADJ_METRIC, "value": n_timed / total, "unit": "grad-steps/s", "steps": n_timed,
           "warmup": adam_steps - n_timed, "ms_per_step": 1000 * total / n_timed,
           "config": {"workload": "adjoint_7x256x256x32spp_depth6_adam%d" % adam_steps, "paths_per_render": n_paths,
                      "parameters": len(params), "adam_steps": adam_steps, "lr": lr,
                      "l2": "inputs (scene, 7 x 256x256 images) are L2-resident; not flushed"},
           "forward_ms": fwd, "adjoint_ms": adj, "adjoint_over_forward": adj / fwd,
           "forward_mpaths_s": n_paths / fwd / 1e3, "adjoint_mpaths_s": n_paths / adj / 1e3,
           "clean_loss_start": loss_start, "clean_loss_end": loss_end,
           "loss_first": losses[0], "loss_last": losses[-1],
           "alphas_end": {names[j]: float(values[j]) for j in alpha_idx},
           "sphere_albedo_end": [float(values[j]) for j, p in enumerate(params) if p[0] == index["diffuse"]],
           "e2e": {"value": n_timed / total, "unit": "grad-steps/s", "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 8 * len(params),
                   "path": "render_batch_dev + adjoint_dev + host Adam + lrt_scene_update_materials + lrt_diff_setup"},
           "gpu_launches": launches}
    if oracle is not None and not args.no_cpu_baseline:
        # the reference has no adjoint: its gradient is a central difference per parameter, 2 renders of the
        # seven frames per parameter plus the loss render; grad-steps/s follows from its path rate here
        secs_cpu, paths_cpu = 0.0, 0
        for name in MATERIALS:
            wld = ref_world(oracle, scenes.open_box(name, attach=False))
            p = scenes.render_params(w, h, 1, depth, rr, row_begin=0, row_end=64)
            secs_cpu += wld.render(p, 0)[2]
            paths_cpu += 64 * w
            wld.close()
        mpaths = paths_cpu / secs_cpu / 1e6
        renders = 2 * len(params) + 1
        res["cpu_baseline"] = {"value": 1.0 / (renders * n_paths / (mpaths * 1e6)), "unit": "grad-steps/s",
                               "cores": oracle.hardware_concurrency(), "kind": "reference", "mpaths_per_s": mpaths,
                               "sample": "%d paths (64 rows of each of the 7 frames at 1 spp, depth 6); a gradient "
                                         "by central differences = %d renders of 7 x 256x256 x 32 spp; %s"
                                         % (paths_cpu, renders, timing_note(oracle))}
    return res


def run_adjoint(args):
    gpu = Gpu(int(os.environ.get("LOCAL_RANK", "0")))
    oracle = None if args.no_cpu_baseline else load_oracle()
    clocks = ClockSampler(gpu_index(gpu.local)).start()
    res = measure_adjoint(gpu, oracle, args, adam_steps=args.adjoint_steps)
    line = {"metric": res.pop("metric"), "value": res.pop("value"), "unit": res.pop("unit"), "n_gpus": 1,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded scenes.open_box_library)", **res, "clocks": clocks.stop()}
    print(json.dumps(line))
    return 0


# ------------------------------------------------------------------------------------------------
# large photon-mapping scene: 256 displaced level-5 icospheres (5.24M triangles) on a ground quad, sky
# + 4 quad lights; 16M photons (depth 8), k = 100, radius cap 0.05; 1024x1024 x 32 spp

LARGE_METRIC = "Mpaths/s (photon mapper eye pass, 1024x1024 x 32 spp, 5.24M-triangle 256-sphere scene, 16M photons, k=100)"


def run_large(args):
    gpu = Gpu(int(os.environ.get("LOCAL_RANK", "0")))
    torch = gpu.torch
    c3 = scenes.CONFIG3
    w, h, spp = c3["width"], c3["height"], args.large_spp or c3["spp"]
    t0 = time.perf_counter()
    scene = scenes.large_scene()
    t_gen = time.perf_counter() - t0
    # the same upload with the kd-trees built on the host cores, for comparison (the default builds them on
    # the GPU at this size; the trees are identical)
    with gpu.context() as ch:
        ch.set_option("kd_build_device", 0)
        t0 = time.perf_counter()
        ch.upload(scene)
        t_upload_host = time.perf_counter() - t0
    ctx = gpu.context()
    t0 = time.perf_counter()
    ctx.upload(scene)
    t_upload = time.perf_counter() - t0
    out = torch.zeros(w * h * 3, dtype=torch.float32, device=gpu.dev)
    clocks = ClockSampler(gpu_index(gpu.local)).start()
    t0 = time.perf_counter()
    pp, shots = ctx.photon_preprocess(c3["photons"], 0, max_depth=c3["photon_depth"], rr_depth=5,
                                      radius_cap=c3["radius_cap"], lookup_size=c3["k"])
    gpu.sync()
    t_photons = time.perf_counter() - t0
    pt_params = scenes.render_params(w, h, spp, 8, 3)
    ctx.render_dev(pt_params, out.data_ptr())  # warm: the wave buffers at the timed frame's size
    gpu.sync()
    t_pt = gpu.time(lambda: ctx.render_dev(pt_params, out.data_ptr()))
    ctx.reset_stats()
    gpu.sync()
    t_eye = gpu.time(lambda: ctx.render_photon_dev(pt_params, pp, out.data_ptr()))
    launches = int(ctx.stats()["kernel_launches"])
    clock_info = clocks.stop()
    img = out.view(h, w, 3).cpu().numpy()
    paths = w * h * spp
    line = {"metric": LARGE_METRIC, "value": paths / t_eye / 1e6, "unit": "Mpaths/s", "n_gpus": 1, "steps": 1,
            "warmup": 1, "ms_per_step": 1000 * t_eye, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scenes.large_scene)",
            "config": {"workload": "large_grid_8x8x4_level5_photon_1024x1024x%dspp" % spp,
                       "triangles": scene.triangle_count(), "objects": len(scene.objects),
                       "photons": c3["photons"], "k": c3["k"], "photon_depth": c3["photon_depth"]},
            "scene_gen_s": t_gen, "upload_s": t_upload, "upload_host_trees_s": t_upload_host,
            "device_scene_mb": ctx.scene_bytes() / 1e6, "photon_particles_shot": shots[0],
            "photon_preprocess_s": t_photons, "radius": pp.global_radius,
            "path_tracer_mpaths_s": paths / t_pt / 1e6,
            "image_mean": [float(x) for x in img.reshape(-1, 3).mean(axis=0)],
            "nonfinite": int((~np.isfinite(img)).sum()), "clocks": clock_info, "gpu_launches": launches}
    oracle = None if args.no_cpu_baseline else load_oracle()
    if oracle is not None:
        # the reference's eye pass over a few rows of the frame with the GPU's photon map (its own photon
        # trace and tree build of 16M photons would take minutes on its own)
        import lrt_abi as abi
        g, shot_g = ctx.photon_trace(abi.GATHER_SURFACE, c3["photons"], c3["photon_depth"], 5)
        wld = ref_world(oracle, scenes.large_scene(attach=False))
        pq = abi.PhotonRenderParams.reference_defaults(lookup_size=c3["k"])
        pq.global_radius, pq.caustic_radius = pp.global_radius, pp.caustic_radius
        rows, n, secs_cpu = 2, 0, 0.0
        empty = np.zeros(0, dtype=abi.PHOTON_DTYPE)
        while secs_cpu < 10.0 and n < 32:
            p = scenes.render_params(w, h, 1, 8, 3, sample_offset=n, row_begin=400 + n * rows,
                                     row_end=400 + (n + 1) * rows)
            secs_cpu += wld.render_photon(p, pq, g, np.float32(1.0 / shot_g), empty, np.float32(1.0),
                                          want_sq=False)[2]
            n += 1
        wld.close()
        line["cpu_baseline"] = {"value": n * rows * w / secs_cpu / 1e6, "unit": "Mpaths/s",
                                "cores": oracle.hardware_concurrency(), "kind": "reference",
                                "sample": "photon_integrator::radiance over %d rows x 1024 x 1 spp (rows 400..) with "
                                          "the GPU's 16M-photon map; %s" % (n * rows, timing_note(oracle))}
    ctx.close()
    print(json.dumps(line))
    return 0


# ------------------------------------------------------------------------------------------------
# small fixed cases for ncu captures of the library's kernels (never timed as bench values)

def run_profile_case(args):
    """render (default): `frames` frames of one open-box scene (the benchmark geometry) at size x size x spp,
    then the last frame again with work counting on, printing the extension rays of every bounce of
    that frame, so that DRAM bytes an ncu capture reports for one k_extend launch can be divided by the
    rays it traced. One frame at 512x512x4 spp is one wave of 1M paths: raygen and accumulate, and per
    bounce extend, hit records, shadow and one shading kernel per shading key present; about 0.5 GB.
    With the defaults, k_extend launch number 9 (0-based) is bounce 1 of the last frame.
    eye: the large photon-mapping scene, `photons` photons, one photon-mapper image of size x size x 1.
    eye_box: the closed box with `material` on the sphere, 1M photons per map (k = 64), one photon-mapper
    image of size x size x spp.
    adjoint: the seven-material scene at size x size x spp per material, one render and one adjoint.
    batch: 16 seeded jobs of the batched workload with spp scaled down.
    kdbuild: the SAH kd-trees of the large scene's 257 meshes built on the GPU in one call.
    knn: the closed box's 1M-photon global map, the irradiance estimate (k = 64) at the first diffuse hits
    of one camera ray per pixel (size x size)."""
    import lrt
    import lrt_abi as abi
    ctx = lrt.Context(0)
    for opt in args.option:  # library options, e.g. --option photon_eye_tail=0
        name, value = opt.split("=", 1)
        ctx.set_option(name, int(value))
    if args.case == "eye":
        ctx.upload(scenes.large_scene())
        pp, shots = ctx.photon_preprocess(args.photons, 0, max_depth=8, rr_depth=5, radius_cap=0.05, lookup_size=100)
        ctx.reset_stats()
        t0 = time.perf_counter()
        img = ctx.render_photon(scenes.render_params(args.size, args.size, 1, 8, 3), pp)
        out = {"photons": args.photons, "shot": shots[0], "seconds": time.perf_counter() - t0,
               "launches": ctx.stats()["kernel_launches"], "mean": float(img.mean())}
    elif args.case == "eye_box":
        ctx.upload(scenes.cornell_box(material=args.material))
        pp, shots = ctx.photon_preprocess(PHOTONS, PHOTONS, max_depth=128, rr_depth=5, lookup_size=KNN_K)
        ctx.reset_stats()
        t0 = time.perf_counter()
        img = ctx.render_photon(scenes.render_params(args.size, args.size, args.spp, DEPTH, RR), pp)
        out = {"material": args.material, "shots": list(shots), "seconds": time.perf_counter() - t0,
               "launches": ctx.stats()["kernel_launches"], "mean": float(img.mean())}
    elif args.case == "adjoint":
        import diff
        scene, sphere, index = scenes.open_box_library()
        ctx.upload(scene)
        dm = diff.Differentiable(ctx, scene)
        jobs, off = [], 0
        for name in MATERIALS:
            jobs.append(scenes.job_desc(scene.camera, args.size, args.size, args.spp, 0, sphere, index[name], off))
            off += 3 * args.size * args.size
        img = ctx.render_batch(jobs, 6, 3)
        g = dm.adjoint(jobs, 6, 3, np.ones(off, np.float32) / off)
        out = {"mean": float(img.mean()), "grad_norm": float(np.linalg.norm(g))}
    elif args.case == "batch":
        scene, sphere, index = scenes.open_box_library()
        jobs, specs = scenes.batch_jobs(index, sphere, n_jobs=16, spp_range=(1, 16))
        ctx.upload(scene)
        img = ctx.render_batch(jobs, 8, 3)
        out = {"jobs": len(jobs), "launches": ctx.stats()["kernel_launches"], "mean": float(np.nanmean(img))}
    elif args.case == "kdbuild":
        meshes = []
        for o in scenes.large_scene().objects:
            if o["kind"] == abi.OBJ_MESH:
                tri = o["positions"][o["indices"].reshape(-1, 3)]
                meshes.append((tri.min(axis=1).astype(np.float32), tri.max(axis=1).astype(np.float32)))
        t0 = time.perf_counter()
        trees = ctx.kdtree_build_device(meshes)
        out = {"meshes": len(meshes), "boxes": int(sum(len(b) for b, _ in meshes)),
               "nodes": int(sum(len(t[0]) for t in trees)), "refs": int(sum(len(t[1]) for t in trees)),
               "seconds_with_python": time.perf_counter() - t0}
    elif args.case == "knn":
        scene = scenes.cornell_box()
        ctx.upload(scene)
        pp, shots = ctx.photon_preprocess(PHOTONS, 0, max_depth=128, rr_depth=5, lookup_size=KNN_K)
        pts, nrm = diffuse_query_points(ctx, scene, args.size, args.size)
        rgb = ctx.photon_irradiance(pp.global_map, pts, nrm, pp.global_radius, 128, KNN_K)
        ctx.set_option("count_work", 1)
        ctx.reset_stats()
        ctx.photon_irradiance(pp.global_map, pts, nrm, pp.global_radius, 128, KNN_K)
        s = ctx.stats()
        out = {"queries": len(pts), "radius": pp.global_radius, "mean": float(rgb.mean()),
               "nodes_per_query": s["knn_nodes_visited"] / len(pts),
               "tested_per_query": s["knn_photons_tested"] / len(pts),
               "found_per_query": s["knn_photons_found"] / len(pts)}
    else:
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
        out = {"paths": timed["paths"], "stage_ms": timed["stage_ms"], "launches": timed["kernel_launches"],
               "last_frame_rays_at_depth": counted["rays_at_depth"][: args.depth],
               "last_frame_nodes_per_ray": counted["nodes_visited"] / max(1, counted["extension_rays"]),
               "last_frame_triangles_per_ray": counted["triangles_tested"] / max(1, counted["extension_rays"]),
               "extend_source_sha16": source_digest(EXTEND_SOURCES), "mean": float(img.mean())}
    ctx.close()
    print(json.dumps(out))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="lrt", choices=["lrt", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="headline line only (no closed box, photon mapper, "
                                                             "batch and adjoint keys)")
    ap.add_argument("--wave-capacity", type=int, default=0, help="paths per wave (0: the library's default)")
    ap.add_argument("--workload", default="paths", choices=["paths", "batch", "adjoint", "large", "profile"],
                    help="paths: the seven-material Mpaths/s workload; batch: the 64-job jobs/s comparison; "
                         "adjoint: gradient steps of the material optimisation; large: the large photon-mapping "
                         "scene; profile: a small fixed case for ncu (--case)")
    ap.add_argument("--jobs", type=int, default=64)
    ap.add_argument("--no-autotune", action="store_true", help="batch workload: default launch shapes")
    ap.add_argument("--adjoint-steps", type=int, default=200)
    ap.add_argument("--large-spp", type=int, default=0, help="large workload: spp (0: the configuration's 32)")
    ap.add_argument("--case", default="render", choices=["render", "eye", "eye_box", "adjoint", "batch", "kdbuild", "knn"])
    ap.add_argument("--material", default="rough_plastic", choices=scenes.MATERIAL_NAMES)
    ap.add_argument("--option", action="append", default=[], help="profile workload: a library option name=value")
    ap.add_argument("--size", type=int, default=512)
    ap.add_argument("--spp", type=int, default=4)
    ap.add_argument("--frames", type=int, default=2)
    ap.add_argument("--depth", type=int, default=8)
    ap.add_argument("--photons", type=int, default=2_000_000)
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
    if args.workload == "profile":
        return run_profile_case(args)
    return run_lrt(args)


if __name__ == "__main__":
    sys.exit(main())
