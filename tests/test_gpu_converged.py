"""Converged-image parity on the two benchmarked path-tracing configurations, against 4096-spp renders
by the reference's own path integrator (tests/golden/converged_kat.npz, made by
tests/golden/make_converged.py with the reference's samples 65536.. of every pixel):

* the closed box at its full 256 x 256 frame, depth 6, Russian roulette from depth 3;
* each of the seven materials in the box open to the Hosek sky, 512 x 512, depth 8, Russian roulette
  from depth 3, over the 64 x 64 crop the fixture holds.

The GPU renders the same frames at 4096 spp on samples 0..4095, so the two images are independent
estimates of the same converged image: per pixel their difference has standard error
sqrt(2) * SE_reference (the same estimator, so the same per-pixel variance). The bar is the one a
3-sigma test admits: at most 1% of pixels beyond 3 standard errors (0.27% expected), and the frame means
within 3 standard errors of the mean.
"""
import numpy as np
import pytest

from conftest import golden

import scenes

pytestmark = pytest.mark.gpu


def _z(img, mean, sq, spp):
    se = np.sqrt(np.maximum(sq - mean * mean, 0.0) / spp) * np.sqrt(2.0)
    both = np.isfinite(img) & np.isfinite(mean)
    z = np.abs(img - mean) / (se + 1e-7)
    return z[both], se[both], both


def _check(img, mean, sq, spp, what):
    z, se, finite = _z(img, mean, sq, spp)
    assert finite.mean() >= 0.999, "%s: %d non-finite pixels" % (what, (~finite).sum())
    frac = (z > 3).mean()
    assert frac <= 0.01, "%s: fraction beyond 3 sigma %.4f (max z %.1f)" % (what, frac, z.max())
    a, b = img[finite], mean[finite]
    se_mean = np.sqrt((se ** 2).sum()) / se.size
    assert abs(a.mean() - b.mean()) <= 3 * se_mean + 1e-7, "%s: means %.6g vs %.6g (SE %.3g)" % (
        what, a.mean(), b.mean(), se_mean)


def test_closed_box_converged_full_frame(ctx):
    g = golden("converged_kat.npz")
    c0 = scenes.CONFIG0
    spp = int(g["spp"])
    ctx.upload(scenes.cornell_box())
    img = ctx.render(scenes.render_params(c0["width"], c0["height"], spp, c0["max_depth"], c0["rr_depth"]))
    _check(img, g["closed_box_mean"], g["closed_box_sq"], spp, "closed box 256x256")


@pytest.mark.parametrize("material", scenes.MATERIAL_NAMES)
def test_open_box_converged_crop(ctx, material):
    g = golden("converged_kat.npz")
    c1 = scenes.CONFIG1
    spp = int(g["spp"])
    r0, r1, x0, x1 = (int(v) for v in g["crop"])
    ctx.upload(scenes.open_box(material))
    img = ctx.render(scenes.render_params(c1["width"], c1["height"], spp, c1["max_depth"], c1["rr_depth"],
                                          row_begin=r0, row_end=r1))
    _check(img[r0:r1, x0:x1], g["open_%s_mean" % material], g["open_%s_sq" % material], spp,
           "open box %s crop" % material)
