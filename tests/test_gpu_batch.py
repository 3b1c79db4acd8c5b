"""Batched rendering: many jobs (own camera, resolution, spp, sphere material) in shared waves.

Every path of a batch job draws the same samples as the same path of a single-image render, and a
job's pixel sums add its samples in sample order, so a job's image equals lrt_render's image of the
same camera, size and material bit for bit — whether a pixel's samples share a wave or span several,
and whether the wave sequence is replayed from a CUDA graph or launched directly.
"""
import numpy as np
import pytest

import lrt
import lrt_abi as abi
import scenes

pytestmark = pytest.mark.gpu

DEPTH, RR = 6, 3


@pytest.fixture(scope="module")
def library(ctx):
    scene, sphere, index = scenes.open_box_library(level=4)
    return scene, sphere, index


def single(ctx, scene, w, h, spp, offset=0):
    ctx.upload(scene)
    return ctx.render(scenes.render_params(w, h, spp, DEPTH, RR, sample_offset=offset)).reshape(-1)


def test_single_job_equals_render(ctx):
    scene = scenes.open_box("rough_plastic", level=4)
    ref = single(ctx, scene, 48, 40, 8)
    out = ctx.render_batch([scenes.job_desc(scene.camera, 48, 40, 8)], DEPTH, RR)
    assert np.array_equal(out, ref)


@pytest.mark.parametrize("name", ["rough_conductor", "coating", "rough_dielectric"])
def test_material_override_equals_scene(ctx, library, name):
    scene, sphere, index = library
    own = scenes.open_box(name, level=4)
    ref = single(ctx, own, 40, 32, 6)
    ctx.upload(scene)
    out = ctx.render_batch([scenes.job_desc(scene.camera, 40, 32, 6, 0, sphere, index[name])], DEPTH, RR)
    assert np.array_equal(out, ref)


def test_mixed_jobs_and_offsets(ctx, library):
    scene, sphere, index = library
    cam_b = dict(scene.camera, origin=(0.5, 1.2, 1.6), aspect=1.5)
    specs = [  # (camera, w, h, spp, sample_offset, material)
        (scene.camera, 32, 32, 5, 0, "diffuse"),
        (cam_b, 48, 32, 3, 7, "plastic"),
        (scene.camera, 24, 40, 9, 2, "rough_coating"),
        (cam_b, 30, 20, 1, 0, "rough_conductor"),
    ]
    jobs, off = [], 16  # leave a gap at the start: output offsets are honoured
    for cam, w, h, spp, so, mat in specs:
        jobs.append(scenes.job_desc(cam, w, h, spp, so, sphere, index[mat], off))
        off += 3 * w * h
    ctx.upload(scene)
    out = ctx.render_batch(jobs, DEPTH, RR)
    assert np.all(out[:16] == 0.0)
    for (cam, w, h, spp, so, mat), job in zip(specs, jobs):
        own = scenes.open_box(mat, level=4)
        own.camera = cam
        ref = single(ctx, own, w, h, spp, so)
        got = out[job.output_offset:job.output_offset + 3 * w * h]
        assert np.array_equal(got, ref), mat


def test_pixels_spanning_waves(ctx, library):
    scene, sphere, index = library
    jobs = [scenes.job_desc(scene.camera, 36, 28, 7, 0, sphere, index["rough_plastic"], 0),
            scenes.job_desc(scene.camera, 20, 20, 13, 3, sphere, index["coating"], 3 * 36 * 28)]
    ctx.upload(scene)
    whole = ctx.render_batch(jobs, DEPTH, RR)
    try:
        for cap in (1024, 4099):  # waves end in the middle of a pixel's samples
            ctx.set_option("wave_capacity", cap)
            split = ctx.render_batch(jobs, DEPTH, RR)
            assert np.array_equal(split, whole), cap
    finally:
        ctx.set_option("wave_capacity", 1 << 21)


def test_graph_replay_equals_direct_launches(ctx, library):
    scene, sphere, index = library
    jobs = [scenes.job_desc(scene.camera, 32, 24, 4, 0, sphere, index[n], 3 * 32 * 24 * i)
            for i, n in enumerate(scenes.MATERIAL_NAMES)]
    ctx.upload(scene)
    try:
        ctx.set_option("wave_capacity", 8192)
        ctx.set_option("batch_graph", 1)
        g = ctx.render_batch(jobs, DEPTH, RR)
        ctx.set_option("batch_graph", 0)
        d = ctx.render_batch(jobs, DEPTH, RR)
    finally:
        ctx.set_option("batch_graph", 1)
        ctx.set_option("wave_capacity", 1 << 21)
    assert np.array_equal(g, d)
    assert np.all(np.isfinite(g)) and g.max() > 0.0


def test_batch_stats_count_paths(ctx, library):
    scene, sphere, index = library
    ctx.upload(scene)
    ctx.reset_stats()
    jobs = [scenes.job_desc(scene.camera, 16, 16, 3), scenes.job_desc(scene.camera, 8, 12, 5, 0, -1, -1, 3 * 256)]
    ctx.render_batch(jobs, DEPTH, RR)
    st = ctx.stats()
    assert st["paths"] == 16 * 16 * 3 + 8 * 12 * 5
    # one wave: raygen, accumulate, advance; per bounce extend, hit records, shadow, the sky samples'
    # radiance (the scene has a sky) and one shading kernel per key the scene can produce (misses, hits
    # without a BSDF, each material type)
    keys = 2 + len({m["type"] for m in scene.materials})
    sky = int(any(e["kind"] == abi.EMITTER_ENV for e in scene.emitters))
    assert st["kernel_launches"] == 3 + (3 + sky + keys) * DEPTH
    ctx.set_option("shade_per_key", 0)
    try:
        ctx.reset_stats()
        ctx.render_batch(jobs, DEPTH, RR)
        assert ctx.stats()["kernel_launches"] == 3 + (4 + sky) * DEPTH
    finally:
        ctx.set_option("shade_per_key", 1)


def test_batch_rejects_bad_jobs(ctx, library):
    scene, sphere, index = library
    ctx.upload(scene)
    bad = [
        scenes.job_desc(scene.camera, 1, 16, 1),                            # width < 2
        scenes.job_desc(scene.camera, 16, 16, 0),                           # no samples
        scenes.job_desc(scene.camera, 16, 16, 1, 0, len(scene.objects), 0),  # object out of range
        scenes.job_desc(scene.camera, 16, 16, 1, 0, sphere, len(scene.materials)),
        scenes.job_desc(scene.camera, 16, 16, 1, 0, sphere, -1),            # override without material
    ]
    for job in bad:
        with pytest.raises(lrt.LrtError) as e:
            ctx.render_batch([job], DEPTH, RR)
        assert e.value.status == abi.LRT_ERR_INVALID_ARGUMENT
    with pytest.raises(lrt.LrtError):
        ctx.render_batch([scenes.job_desc(scene.camera, 16, 16, 1)], 0, RR)


def test_plain_path_tracer_equals_batch(ctx, library):
    scene, sphere, index = library
    cam_b = dict(scene.camera, origin=(-0.4, 1.1, 1.5), aspect=1.25)
    jobs = [scenes.job_desc(scene.camera, 32, 24, 5, 0, sphere, index["rough_plastic"], 0),
            scenes.job_desc(cam_b, 40, 32, 3, 11, sphere, index["rough_dielectric"], 3 * 32 * 24),
            scenes.job_desc(scene.camera, 16, 16, 7, 0, -1, -1, 3 * (32 * 24 + 40 * 32))]
    ctx.upload(scene)
    plain = ctx.render_plain(jobs, DEPTH, RR)
    batch = ctx.render_batch(jobs, DEPTH, RR)
    assert np.array_equal(plain, batch)
    # the persistent megakernel over the (job, tile) queue: the same images
    ctx.set_option("batch_queue", 1)
    try:
        queued = ctx.render_batch(jobs, DEPTH, RR)
    finally:
        ctx.set_option("batch_queue", 0)
    assert np.array_equal(plain, queued)


def test_launch_knobs_keep_images(ctx, library, tmp_path):
    """pixel_tile (a path-order bijection, here on sizes that are not multiples of the tile),
    blocks_per_sm and wave_capacity change speed only; the autotuner picks among them and caches"""
    import autotune
    scene, sphere, index = library
    jobs = [scenes.job_desc(scene.camera, 37, 29, 5, 0, sphere, index["rough_plastic"], 0),
            scenes.job_desc(scene.camera, 21, 34, 3, 4, sphere, index["coating"], 3 * 37 * 29)]
    ctx.upload(scene)
    ref = ctx.render_batch(jobs, DEPTH, RR)
    try:
        for knob, v in [("pixel_tile", 3), ("pixel_tile", 8), ("pixel_tile", 64), ("blocks_per_sm", 1),
                        ("blocks_per_sm", 2), ("wave_capacity", 2048)]:
            ctx.set_option(knob, v)
            assert np.array_equal(ctx.render_batch(jobs, DEPTH, RR), ref), (knob, v)
            autotune.apply(ctx, autotune.DEFAULTS)
        import torch
        out = torch.zeros(ref.size, dtype=torch.float32, device="cuda")
        cache = str(tmp_path / "cache.json")
        cfg, key, hit = autotune.tuned(ctx, scene, jobs, DEPTH, RR, out.data_ptr(), cache_path=cache)
        assert not hit and all(cfg[k] in autotune.CANDIDATES[k] for k in autotune.ORDER)
        cfg2, key2, hit2 = autotune.tuned(ctx, scene, jobs, DEPTH, RR, out.data_ptr(), cache_path=cache)
        assert hit2 and cfg2 == cfg and key2 == key
        assert np.array_equal(ctx.render_batch(jobs, DEPTH, RR), ref)
        # the library's own text cache: timed once (6 + 3 + 2 configurations at most), then read back
        native = str(tmp_path / "launch_cache.txt")
        r1 = ctx.autotune(jobs, DEPTH, RR, out.data_ptr(), native)
        assert not r1["from_cache"] and r1["trials"] == 11 and r1["seconds"] > 0
        assert all(r1[k] in autotune.CANDIDATES[k] for k in autotune.ORDER)
        r2 = ctx.autotune(jobs, DEPTH, RR, out.data_ptr(), native)
        assert r2["from_cache"] and all(r2[k] == r1[k] for k in autotune.ORDER)
        with open(native) as f:
            line = f.read().split()
        assert line[0] == key and [int(x) for x in line[1:4]] == [r1[k] for k in autotune.ORDER]
        assert np.array_equal(ctx.render_batch(jobs, DEPTH, RR), ref)
    finally:
        autotune.apply(ctx, autotune.DEFAULTS)
