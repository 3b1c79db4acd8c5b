"""Scenes of many objects: the object hierarchy (object_bvh) against the reference's in-order list walk.

The hierarchy visits every object whose box the ray may reach, front to back, and resolves equal t by
object index, so hits must equal the reference's hittable_list::hit bit for bit -- on a reduced large
scene (a 4 x 4 x 2 grid of level-2 spheres, ground, four quad lights, sky: 37 objects), on a scene of
20 coincident quads where every hit is a tie (the last object must win), and through whole renders
with the hierarchy on and off.
"""
import numpy as np
import pytest

import lrt_abi as abi
import oracle
import scenes
from test_gpu_parity import _check_hits

pytestmark = pytest.mark.gpu
needs_ref = pytest.mark.skipif(not oracle.reference_available(), reason="reference build (oracle/_ref) missing")


@pytest.fixture(scope="module")
def grid_scene():
    return scenes.large_scene(level=2, grid=(4, 4, 2))


def random_rays(rng, n, lo, hi):
    rays = np.zeros(n, dtype=abi.RAY_DTYPE)
    rays["origin"] = rng.uniform(lo, hi, (n, 3))
    d = rng.normal(size=(n, 3))
    d[: n // 20, rng.integers(0, 3)] = 0.0
    rays["direction"] = d / np.linalg.norm(d, axis=1, keepdims=True)
    rays["t_min"] = 0.001
    rays["t_max"] = np.where(rng.random(n) < 0.2, rng.uniform(0.01, 4.0, n), np.inf)
    return rays


def both_walks(ctx, fn):
    try:
        ctx.set_option("object_bvh", 1)
        a = fn()
        ctx.set_option("object_bvh", 0)
        b = fn()
    finally:
        ctx.set_option("object_bvh", 1)
    return a, b


@needs_ref
def test_grid_scene_trace_vs_reference(ctx, grid_scene):
    assert len(grid_scene.objects) > 16
    ctx.upload(grid_scene)
    rng = np.random.default_rng(5)
    rays = random_rays(rng, 30000, (-3.0, 0.0, -3.0), (3.0, 4.5, 3.0))
    world = oracle.RefWorld(grid_scene)
    ref, _ = world.trace(rays)
    world.close()
    bvh, linear = both_walks(ctx, lambda: ctx.trace(rays))
    _check_hits(bvh, ref)
    _check_hits(linear, ref)


def test_grid_scene_occlusion_walks_agree(ctx, grid_scene):
    ctx.upload(grid_scene)
    rng = np.random.default_rng(6)
    rays = random_rays(rng, 20000, (-3.0, 0.0, -3.0), (3.0, 4.5, 3.0))
    for light in range(len(grid_scene.emitters)):
        bvh, linear = both_walks(ctx, lambda: ctx.occluded(rays, light))
        assert np.array_equal(bvh, linear), light


@needs_ref
def test_ties_resolve_to_the_later_object(ctx):
    mats = [{"type": abi.MAT_DIFFUSE, "diffuse_reflectance": (0.5, 0.5, 0.5)}]
    objects = [scenes.quad_mesh((-1, 0, 1), (1, 0, 1), (1, 0, -1), (-1, 0, -1), 0) for _ in range(20)]
    objects.append({"kind": abi.OBJ_RECTANGLE, "material": -1, "corner": (-1, 0, -1), "edge_u": (2, 0, 0),
                    "edge_v": (0, 0, 2)})
    objects += [scenes.quad_mesh((-1, 0, 1), (1, 0, 1), (1, 0, -1), (-1, 0, -1), 0) for _ in range(3)]
    emitters = [{"kind": abi.EMITTER_AREA, "object": 20, "radiance": (1, 1, 1)}]
    sc = scenes.Scene(objects, mats, emitters, scenes.default_camera(), "ties")
    ctx.upload(sc)
    rng = np.random.default_rng(7)
    n = 4000
    rays = np.zeros(n, dtype=abi.RAY_DTYPE)
    rays["origin"] = np.stack([rng.uniform(-0.9, 0.9, n), np.full(n, 1.0), rng.uniform(-0.9, 0.9, n)], 1)
    d = np.stack([rng.uniform(-0.3, 0.3, n), -np.ones(n), rng.uniform(-0.3, 0.3, n)], 1)
    rays["direction"] = d / np.linalg.norm(d, axis=1, keepdims=True)
    rays["t_min"] = 0.001
    rays["t_max"] = np.inf
    world = oracle.RefWorld(sc)
    ref, _ = world.trace(rays)
    world.close()
    bvh, linear = both_walks(ctx, lambda: ctx.trace(rays))
    _check_hits(bvh, ref)
    _check_hits(linear, ref)
    assert np.all(ref["object"][ref["object"] >= 0] == len(objects) - 1)


def test_grid_scene_renders_identical_across_walks(ctx, grid_scene):
    ctx.upload(grid_scene)
    p = scenes.render_params(40, 32, 4, 8, 3)
    bvh, linear = both_walks(ctx, lambda: ctx.render(p))
    assert np.array_equal(bvh, linear, equal_nan=True)
    pp, _ = ctx.photon_preprocess(100_000, 0, max_depth=8, rr_depth=5, radius_cap=0.05, lookup_size=32)
    pq = scenes.render_params(24, 20, 1, 8, 3)
    bvh, linear = both_walks(ctx, lambda: ctx.render_photon(pq, pp))
    assert np.array_equal(bvh, linear, equal_nan=True)
    try:
        ctx.set_option("photon_eye_kernel", 0)
        per_thread = ctx.render_photon(pq, pp)
        ctx.set_option("photon_eye_kernel", 1)
        persistent = ctx.render_photon(pq, pp)
    finally:
        ctx.set_option("photon_eye_kernel", 2)
    assert np.array_equal(bvh, per_thread, equal_nan=True)
    assert np.array_equal(bvh, persistent, equal_nan=True)


@needs_ref
def test_grid_scene_image_vs_reference(ctx, grid_scene):
    """same samples as the reference renderer: every pixel within 3 MC standard errors"""
    ctx.upload(grid_scene)
    p = scenes.render_params(24, 24, 32, 8, 3)
    img = ctx.render(p)
    world = oracle.RefWorld(grid_scene)
    ref, sq, _ = world.render(p, want_sq=True)
    world.close()
    se = np.sqrt(np.maximum(sq - ref * ref, 0.0) / 32)
    diff = np.abs(img - ref)
    assert np.all(diff <= 3 * se + 1e-5), float(np.max(diff / (se + 1e-12)))
    assert np.median(diff / np.maximum(ref, 1e-6)) < 1e-3
