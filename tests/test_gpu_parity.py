"""GPU parity of the per-function entry points against the reference: committed golden fixtures (made
by the unmodified reference, tests/golden/make_golden.py) and, where the oracle build is present, the
live reference on fresh random inputs.

Bars: the sampler, camera rays and kd-tree traversal (object, triangle, t, hit point, normal) are
bit-exact; BSDF eval/pdf, sky radiance and emitter sampling agree within 1e-5 relative (FP32) on every
query; BSDF sampling agrees within 1e-5 on all but a measured, bounded handful (_compare_bsdf)."""
import numpy as np
import pytest

from conftest import golden, rel_close

import lrt_abi as abi
import oracle
import scenes

pytestmark = pytest.mark.gpu
needs_ref = pytest.mark.skipif(not oracle.reference_available(), reason="reference oracle not built")


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


def test_sampler_bit_exact(ctx):
    g = golden("sampler_kat.npz")
    ctx.upload(scenes.cornell_box(level=1))
    v = ctx.sampler_values(g["pixel_sample"], g["values"].shape[1])
    assert np.array_equal(bits(v), bits(g["values"]))


def test_camera_rays_bit_exact(ctx):
    g = golden("camera_kat.npz")
    ctx.upload(scenes.cornell_box())
    rays = ctx.camera_rays(256, 256, g["pixel_sample"])
    assert np.array_equal(bits(rays["origin"]), bits(g["rays"]["origin"]))
    assert np.array_equal(bits(rays["direction"]), bits(g["rays"]["direction"]))


def _check_hits(hits, ref):
    assert np.array_equal(hits["object"], ref["object"])
    assert np.array_equal(hits["prim"], ref["prim"])
    m = ref["object"] >= 0
    assert np.array_equal(bits(hits["t"][m]), bits(ref["t"][m]))
    assert np.array_equal(hits["front_face"][m], ref["front_face"][m])
    assert np.array_equal(bits(hits["p"][m]), bits(ref["p"][m]))
    assert np.array_equal(bits(hits["normal"][m]), bits(ref["normal"][m]))


@pytest.mark.parametrize("name", ["cornell", "open"])
def test_trace_golden_bit_exact(ctx, name):
    g = golden("trace_kat.npz")
    ctx.upload(scenes.cornell_box() if name == "cornell" else scenes.open_box("rough_coating"))
    hits = ctx.trace(g[name + "_rays"])
    _check_hits(hits, g[name + "_hits"])


@needs_ref
def test_trace_random_vs_reference(ctx):
    rng = np.random.default_rng(99)
    sc = scenes.cornell_box()
    ctx.upload(sc)
    world = oracle.RefWorld(sc)
    n = 40000
    rays = np.zeros(n, dtype=abi.RAY_DTYPE)
    rays["origin"] = np.stack([rng.uniform(-1, 1, n), rng.uniform(0, 2, n), rng.uniform(-1, 1.5, n)], 1)
    d = rng.normal(size=(n, 3))
    d[: n // 10, rng.integers(0, 3)] = 0.0
    rays["direction"] = d / np.linalg.norm(d, axis=1, keepdims=True)
    rays["t_min"] = 0.001
    rays["t_max"] = np.where(rng.random(n) < 0.2, rng.uniform(0.01, 2.0, n), np.inf)
    ref, _ = world.trace(rays)
    _check_hits(ctx.trace(rays), ref)


@pytest.mark.parametrize("name", ["cornell", "open"])
def test_occlusion_matches_closest_hit_rule(ctx, name):
    """blocked == (closest hit exists and is not the light), path_integrator.h:113-115, on the golden rays
    (whose closest hits the reference computed) towards emitter 0 (area light / sky)"""
    g = golden("trace_kat.npz")
    sc = scenes.cornell_box() if name == "cornell" else scenes.open_box("rough_coating")
    ctx.upload(sc)
    rays, hits = g[name + "_rays"], g[name + "_hits"]
    light_obj = sc.emitters[0].get("object", -999)
    expected = (hits["object"] >= 0) & (hits["object"] != light_obj)
    assert np.array_equal(ctx.occluded(rays, 0).astype(bool), expected)


def test_trace_edge_cases(ctx):
    sc = scenes.cornell_box(level=2)
    ctx.upload(sc)
    rays = np.zeros(6, dtype=abi.RAY_DTYPE)
    rays["origin"] = [[0, 1, 0.5]] * 6
    rays["direction"] = [[0, -1, 0], [0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, -1], [0.0, -0.0, 1.0]]
    rays["t_min"] = 0.001
    rays["t_max"] = [np.inf, np.inf, 1e-4, np.inf, np.inf, np.inf]
    hits = ctx.trace(rays)
    assert hits["object"][0] >= 0          # floor
    assert hits["object"][2] == -1         # bounded before any surface
    assert hits["object"][3] >= 0          # roof or light
    if oracle.reference_available():
        ref, _ = oracle.RefWorld(sc).trace(rays)
        _check_hits(hits, ref)


def _max_rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    d = np.abs(a - b) / np.maximum(np.maximum(np.abs(a), np.abs(b)), 1e-30)
    d[(a == b) | (np.isnan(a) & np.isnan(b))] = 0.0
    return float(d.max()) if d.size else 0.0


def _compare_bsdf(res, ref, q, material):
    """BSDF parity bars, with the sizes measured on B200 against the reference built with glibc:

    * eval and pdf: every query within 1e-5 relative (+1e-7 absolute); measured worst 5.5e-7.
    * the sampled lobe and component: identical for all but 1 in 10,000 queries (measured: none differ
      in 13 x 20,768 queries).
    * the sampled weight, pdf, eta and direction: within 1e-5 for all but 1 in 5,000 queries, and those
      within 1e-3 (measured: at most 2 of 20,000 per material, worst 1.4e-4). The sampled directions
      pass through sin/cos, which the library evaluates in double and rounds once (the correctly
      rounded float), glibc's sinf/cosf being under 0.56 ulp but not always correctly rounded; a grazing
      reflection amplifies that last-bit difference.
    """
    n = len(q)
    type_ok = (res["sampled_type"] == ref["sampled_type"]) & (res["sampled_component"] == ref["sampled_component"])
    assert (~type_ok).sum() <= n // 10000, "material %d: %d samples chose another lobe" % (material, (~type_ok).sum())
    e_ok = rel_close(res["eval"], ref["eval"]).all(axis=1) & rel_close(res["pdf"], ref["pdf"])
    assert e_ok.all(), "material %d: %d eval/pdf beyond 1e-5 (worst %.3g / %.3g): %s vs %s" % (
        material, (~e_ok).sum(), _max_rel(res["eval"], ref["eval"]), _max_rel(res["pdf"], ref["pdf"]),
        res[~e_ok][:2], ref[~e_ok][:2])
    w_ok = rel_close(res["sample_weight"], ref["sample_weight"]).all(axis=1)
    pdf_ok = rel_close(res["sample_pdf"], ref["sample_pdf"])
    eta_ok = res["sample_eta"] == ref["sample_eta"]
    nonzero = np.any(ref["sample_weight"] != 0, axis=1)
    wo_ok = rel_close(res["sample_wo"], ref["sample_wo"], rtol=1e-5, atol=1e-6).all(axis=1) | ~nonzero
    bad = type_ok & ~(w_ok & pdf_ok & eta_ok & wo_ok)
    assert bad.sum() <= max(1, n // 5000), "material %d: %d sample mismatches, e.g. %s vs %s" % (
        material, bad.sum(), res[bad][:2], ref[bad][:2])
    loose = (rel_close(res["sample_weight"], ref["sample_weight"], 1e-3, 1e-6).all(axis=1)
             & rel_close(res["sample_pdf"], ref["sample_pdf"], 1e-3, 1e-6)
             & rel_close(res["sample_wo"], ref["sample_wo"], 1e-3, 1e-5).all(axis=1) & eta_ok)
    assert loose[bad].all(), "material %d: a sample differs by more than 1e-3: %s vs %s" % (
        material, res[bad & ~loose][:2], ref[bad & ~loose][:2])


def _zoo():
    import importlib.util
    import os
    from conftest import GOLDEN
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLDEN, "make_golden.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_bsdf_golden(ctx):
    g = golden("bsdf_kat.npz")
    mg = _zoo()
    sc = mg.material_zoo()
    ctx.upload(sc)
    for m in range(len(sc.materials)):
        q = g["q%d" % m]
        _compare_bsdf(ctx.bsdf(m, q), g["r%d" % m], q, m)


@needs_ref
def test_bsdf_random_vs_reference(ctx):
    mg = _zoo()
    sc = mg.material_zoo()
    ctx.upload(sc)
    world = oracle.RefWorld(sc)
    rng = np.random.default_rng(1234)
    for m in range(len(sc.materials)):
        q = mg.bsdf_queries(rng, 20000)
        _compare_bsdf(ctx.bsdf(m, q), world.bsdf(m, q), q, m)


def test_sky_golden(ctx):
    g = golden("sky_kat.npz")
    ctx.upload(scenes.open_box(level=1))
    rgb = ctx.sky(g["dirs"])
    assert rel_close(rgb, g["rgb"]).all()


@pytest.mark.parametrize("name", ["cornell", "open"])
def test_emitter_golden(ctx, name):
    g = golden("emitter_kat.npz")
    ctx.upload(scenes.cornell_box(level=1) if name == "cornell" else scenes.open_box(level=1))
    out, pdf = ctx.emitter_query(g[name + "_points"], g[name + "_u2"], g[name + "_dirs"])
    ref = g[name + "_sample"]
    assert np.array_equal(out[:, 0], ref[:, 0])
    ok = ref[:, 0] > 0
    cols = [1, 2, 3, 4, 5, 6, 10, 11, 12, 13, 14, 15]
    assert rel_close(out[ok][:, cols], ref[ok][:, cols]).all()
    assert rel_close(pdf, g[name + "_pdf"]).all()
