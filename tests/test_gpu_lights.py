"""Analytic spheres and area lights over every shape, on the reference's own demo scene.

* src/main.cpp:58-90's scene: the bunny, the ground as a sphere of radius 100 (sphere.h:21-49), the
  rectangle light, and the sphere light main.cpp:55-56 defines -- closest hits bit-exact against the
  reference on random rays, path-traced and photon-mapped images within 3 Monte Carlo standard errors
  of the reference renderer on the same samples.
* Area lights over triangle meshes (area_emitter.h:17-147 over triangle_mesh::sample_position,
  triangle_mesh.h:109-138): emitter sampling and pdf against the reference (golden fixture and live),
  the occlusion rule, photon emission per particle and same-sample images.
"""
import os

import numpy as np
import pytest

from conftest import golden, rel_close

import lrt_abi as abi
import oracle
import scenes
from test_gpu_parity import _check_hits

pytestmark = pytest.mark.gpu
needs_ref = pytest.mark.skipif(not oracle.reference_available(), reason="reference oracle not built")
needs_bunny = pytest.mark.skipif(not oracle.reference_available() or not os.path.exists(oracle.BUNNY_PATH),
                                 reason="reference build with its bunny.obj (oracle/_ref) missing")


def _se(mean, sq, spp):
    return np.sqrt(np.maximum(sq - mean * mean, 0.0) / spp)


def _random_rays(rng, n, lo, hi):
    rays = np.zeros(n, dtype=abi.RAY_DTYPE)
    rays["origin"] = rng.uniform(lo, hi, (n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3))
    d[: n // 16, rng.integers(0, 3)] = 0.0
    rays["direction"] = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    rays["t_min"] = 0.001
    rays["t_max"] = np.where(rng.random(n) < 0.2, rng.uniform(0.05, 3.0, n), np.inf).astype(np.float32)
    return rays


@pytest.fixture(scope="module")
def demo():
    return scenes.demo_scene(oracle.BUNNY_PATH, sphere_light=True)


@needs_bunny
def test_demo_scene_trace_vs_reference(ctx, demo):
    ctx.upload(demo)
    rng = np.random.default_rng(31)
    rays = _random_rays(rng, 40000, (-1.6, -0.45, -1.6), (1.6, 1.9, 2.5))
    # rays from the camera's side towards the bunny and the ground
    cam = np.zeros(8000, dtype=abi.RAY_DTYPE)
    cam["origin"] = (0.0, 0.5, 3.0)
    tgt = rng.normal(scale=0.6, size=(8000, 3)) + (0.0, 0.0, 0.0)
    d = tgt - np.array([0.0, 0.5, 3.0])
    cam["direction"] = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    cam["t_min"], cam["t_max"] = 0.001, np.inf
    rays = np.concatenate([rays, cam])
    world = oracle.RefWorld(demo)
    ref, _ = world.trace(rays)
    world.close()
    _check_hits(ctx.trace(rays), ref)
    for obj in range(4):  # bunny, ground sphere, rectangle light, sphere light
        assert (ref["object"] == obj).sum() > 200, obj


@needs_bunny
def test_demo_scene_occlusion_rule(ctx, demo):
    """blocked == (closest hit exists and is not the light) for the rectangle light and the sphere light"""
    ctx.upload(demo)
    rng = np.random.default_rng(32)
    rays = _random_rays(rng, 20000, (-1.2, -0.3, -1.2), (1.6, 1.4, 1.5))
    world = oracle.RefWorld(demo)
    ref, _ = world.trace(rays)
    world.close()
    for light in (0, 1):
        obj = demo.emitters[light]["object"]
        expected = (ref["object"] >= 0) & (ref["object"] != obj)
        assert np.array_equal(ctx.occluded(rays, light).astype(bool), expected)


@needs_bunny
@pytest.mark.parametrize("sphere_light", [False, True])
def test_demo_scene_image_same_samples(ctx, sphere_light):
    sc = scenes.demo_scene(oracle.BUNNY_PATH, sphere_light=sphere_light)
    ctx.upload(sc)
    p = scenes.render_params(32, 32, 16, 8, 3)
    img = ctx.render(p)
    world = oracle.RefWorld(sc)
    ref, sq, _ = world.render(p, 0, True)
    world.close()
    z = np.abs(img - ref) / (_se(ref, sq, 16) + 1e-6)
    assert (z > 3).mean() <= 0.01, "fraction beyond 3 sigma %g (max z %g)" % ((z > 3).mean(), z.max())
    assert np.median(np.abs(img - ref) / np.maximum(ref, 1e-6)) < 1e-3


@needs_bunny
def test_demo_scene_photon_mapper(ctx):
    """main.cpp's default integrator (photon_integrator) on its own scene, with photon maps both sides
    build from the same photon arrays"""
    sc = scenes.demo_scene(oracle.BUNNY_PATH)
    ctx.upload(sc)
    g, shot_g = ctx.photon_trace(abi.GATHER_SURFACE, 30000, 127, 5)
    c, shot_c = ctx.photon_trace(abi.GATHER_CAUSTIC, 30000, 127, 5)
    if len(c) < 30000:
        c = c[:0]
    pp = abi.PhotonRenderParams.reference_defaults(lookup_size=64)
    pp.global_radius, pp.caustic_radius = 0.1, 0.025
    ctx.photon_map_build(0, g, 1.0 / shot_g)
    pp.global_map = 0
    if len(c):
        ctx.photon_map_build(1, c, 1.0 / shot_c)
        pp.caustic_map = 1
    params = scenes.render_params(24, 24, 4, 8, 3)
    img = ctx.render_photon(params, pp)
    world = oracle.RefWorld(sc)
    ref, sq, _ = world.render_photon(params, pp, g, np.float32(1.0 / shot_g), c,
                                     np.float32(1.0 / shot_c) if len(c) else np.float32(1.0))
    world.close()
    z = np.abs(img - ref) / (_se(ref, sq, 4) + 1e-6 * np.maximum(ref, 1e-3))
    assert (z > 3).mean() <= 0.01, "fraction beyond 3 sigma %g" % (z > 3).mean()
    assert abs(img.mean() - ref.mean()) <= 0.02 * ref.mean()


# ---- area lights over triangle meshes ----

def _emitter_compare(out, pdf, ref, ref_pdf):
    assert np.array_equal(out[:, 0], ref[:, 0])
    ok = ref[:, 0] > 0
    cols = [1, 2, 3, 4, 5, 6, 10, 11, 12, 13, 14, 15]
    assert rel_close(out[ok][:, cols], ref[ok][:, cols]).all()
    assert rel_close(pdf, ref_pdf).all()


def test_mesh_light_emitter_golden(ctx):
    g = golden("light_kat.npz")
    ctx.upload(scenes.mesh_light_box(level=1))
    out, pdf = ctx.emitter_query(g["mesh_points"], g["mesh_u2"], g["mesh_dirs"])
    _emitter_compare(out, pdf, g["mesh_sample"], g["mesh_pdf"])
    assert (g["mesh_sample"][:, 15] == 0).sum() > 100 and (g["mesh_pdf"] > 0).sum() > 100


@needs_ref
def test_mesh_light_emitter_random_vs_reference(ctx):
    sc = scenes.mesh_light_box(level=2)
    ctx.upload(sc)
    rng = np.random.default_rng(41)
    n = 20000
    p = np.stack([rng.uniform(-0.95, 0.95, n), rng.uniform(0.02, 1.95, n), rng.uniform(-0.95, 1.45, n)], 1)
    p = p.astype(np.float32)
    u2 = rng.random((n, 2), dtype=np.float32)
    u2[:64, 0] = [0.0, 1.0, 0.49999997, 0.5] * 16  # the light-pick and CDF ends
    world = oracle.RefWorld(sc)
    ds = world.emitter_sample(p, u2)
    d = rng.normal(size=(n, 3))
    dirs = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    ok = ds[:, 0] > 0
    half = ok & (rng.random(n) < 0.7)
    dirs[half] = ds[half, 1:4]  # most pdf queries along sampled directions (they reach the light)
    ref_pdf = world.emitter_pdf(p, dirs)
    world.close()
    out, pdf = ctx.emitter_query(p, u2, dirs)
    _emitter_compare(out, pdf, ds, ref_pdf)
    assert (ref_pdf > 0).mean() > 0.3


@needs_ref
def test_mesh_light_occlusion_rule(ctx):
    sc = scenes.mesh_light_box(level=2)
    ctx.upload(sc)
    rng = np.random.default_rng(42)
    rays = _random_rays(rng, 20000, (-0.9, 0.05, -0.9), (0.9, 1.9, 1.4))
    # rays aimed at the mesh light, bounded just past it and just before it
    light = sc.objects[sc.emitters[0]["object"]]
    tgt = light["positions"][rng.integers(0, len(light["positions"]), 4000)]
    o = rays["origin"][:4000].astype(np.float64)
    d = tgt - o
    dist = np.linalg.norm(d, axis=1)
    rays["direction"][:4000] = (d / dist[:, None]).astype(np.float32)
    rays["t_max"][:4000] = (dist * rng.choice([0.97, 1.03], 4000)).astype(np.float32)
    world = oracle.RefWorld(sc)
    ref, _ = world.trace(rays)
    world.close()
    for k in range(len(sc.emitters)):
        obj = sc.emitters[k]["object"]
        expected = (ref["object"] >= 0) & (ref["object"] != obj)
        assert np.array_equal(ctx.occluded(rays, k).astype(bool), expected), k


def test_mesh_light_photons_golden(ctx):
    g = golden("light_kat.npz")
    ctx.upload(scenes.mesh_light_box(level=3))
    ph, cnt = ctx.photon_trace_particles(abi.GATHER_SURFACE, 0, 2048, 8, 5, max_per=16)
    ref_ph, ref_cnt = g["mesh_photons"], g["mesh_photon_counts"]
    same = cnt == ref_cnt
    assert same.mean() >= 0.99, "photon counts differ for %.3f of particles" % (1 - same.mean())
    for i in np.nonzero(same)[0]:
        n = min(int(cnt[i]), 16)
        if n == 0:
            continue
        a, b = ph[i, :n], ref_ph[i, :n]
        assert np.array_equal(a["depth"], b["depth"])
        if not (rel_close(a["position"], b["position"], 1e-3, 1e-4).all()
                and rel_close(a["power"], b["power"], 1e-3, 1e-6).all()):
            same[i] = False
    assert same.mean() >= 0.98
    assert cnt.sum() > 1000


@needs_ref
@pytest.mark.parametrize("material", ["diffuse", "rough_conductor"])
def test_mesh_light_image_same_samples(ctx, material):
    sc = scenes.mesh_light_box(level=4, material=material)
    ctx.upload(sc)
    p = scenes.render_params(24, 24, 64, 6, 3)
    img = ctx.render(p)
    world = oracle.RefWorld(sc)
    ref, sq, _ = world.render(p, 0, True)
    world.close()
    z = np.abs(img - ref) / (_se(ref, sq, 64) + 1e-6)
    assert (z > 3).mean() <= 0.01, "fraction beyond 3 sigma %g (max z %g)" % ((z > 3).mean(), z.max())
    assert np.median(np.abs(img - ref) / np.maximum(ref, 1e-6)) < 1e-3
    assert img.mean() > 0


@needs_ref
def test_mesh_light_plain_and_batch_agree(ctx):
    """the plain one-thread-per-pixel path tracer and a batched job give the wavefront's image on a
    mesh-lit scene"""
    sc = scenes.mesh_light_box(level=3)
    ctx.upload(sc)
    p = scenes.render_params(20, 16, 8, 6, 3)
    img = ctx.render(p)
    job = scenes.job_desc(sc.camera, 20, 16, 8)
    plain = ctx.render_plain([job], 6, 3)
    batch = ctx.render_batch([job], 6, 3)
    assert np.array_equal(plain.reshape(img.shape), img, equal_nan=True)
    assert np.array_equal(batch.reshape(img.shape), img, equal_nan=True)
