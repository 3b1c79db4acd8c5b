"""A mesh loaded from a Wavefront OBJ (lrt_load_obj, bit-identical to the reference's load_obj) rendered
through the GPU path: the reference's own demo mesh, the bunny of src/main.cpp:69, in the closed box
under the ceiling light, against the reference renderer on the same samples (every pixel within 3 MC
standard errors), plus bit-exact traversal on random rays."""
import os

import numpy as np
import pytest

import lrt_abi as abi
import oracle
import scenes
from test_gpu_parity import _check_hits

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not oracle.reference_available() or not os.path.exists(oracle.BUNNY_PATH),
                                 reason="reference build with its bunny.obj (oracle/_ref) missing")]


@pytest.fixture(scope="module")
def bunny_box():
    return scenes.mesh_box(oracle.BUNNY_PATH, "rough_plastic")


def test_bunny_trace_vs_reference(ctx, bunny_box):
    ctx.upload(bunny_box)
    rng = np.random.default_rng(12)
    n = 30000
    rays = np.zeros(n, dtype=abi.RAY_DTYPE)
    rays["origin"] = np.stack([rng.uniform(-0.9, 0.9, n), rng.uniform(0.05, 1.9, n), rng.uniform(-0.9, 1.4, n)], 1)
    d = rng.normal(size=(n, 3))
    rays["direction"] = d / np.linalg.norm(d, axis=1, keepdims=True)
    rays["t_min"] = 0.001
    rays["t_max"] = np.inf
    world = oracle.RefWorld(bunny_box)
    ref, _ = world.trace(rays)
    world.close()
    hits = ctx.trace(rays)
    _check_hits(hits, ref)
    assert (ref["object"] == len(bunny_box.objects) - 2).sum() > 1000  # the bunny is hit


def test_bunny_image_vs_reference(ctx, bunny_box):
    ctx.upload(bunny_box)
    p = scenes.render_params(24, 24, 16, 6, 3)
    img = ctx.render(p)
    world = oracle.RefWorld(bunny_box)
    ref, sq, _ = world.render(p, want_sq=True)
    world.close()
    se = np.sqrt(np.maximum(sq - ref * ref, 0.0) / 16)
    diff = np.abs(img - ref)
    assert (diff > 3 * se + 1e-5).mean() <= 0.01, float(np.max(diff / (se + 1e-12)))
    assert np.median(diff / np.maximum(ref, 1e-6)) < 1e-3
