"""The image writer's float-to-byte conversion on the device (lrt_tonemap / lrt_tonemap_dev) against the
reference's ImageWriter (io/image_write.cpp:10-20 and its vertical flip, image_write.cpp:60-69):
bit-exact on the golden fixture (special values and both sides of every byte boundary), on live
random images against the reference build, and on a rendered image left on the device."""
import numpy as np
import pytest

from conftest import golden

import oracle
import scenes

pytestmark = pytest.mark.gpu
needs_ref = pytest.mark.skipif(not oracle.reference_available(), reason="reference oracle not built")


def test_tonemap_golden(ctx):
    g = golden("image_out_kat.npz")
    rgb = g["rgb"]
    assert np.array_equal(ctx.tonemap(rgb), g["bytes"])
    assert np.array_equal(ctx.tonemap(rgb, flip=True), g["bytes_flipped"])


@needs_ref
@pytest.mark.parametrize("shape", [(1, 1), (2, 3), (37, 53), (480, 640)])
def test_tonemap_random_against_reference(ctx, shape):
    rng = np.random.default_rng(shape[0] * 1000 + shape[1])
    h, w = shape
    rgb = np.exp(rng.normal(-1.0, 2.0, (h, w, 3))).astype(np.float32)
    rgb[rng.random((h, w, 3)) < 0.01] = np.nan
    rgb[rng.random((h, w, 3)) < 0.01] *= -1.0
    for flip in (False, True):
        assert np.array_equal(ctx.tonemap(rgb, flip=flip), oracle.to_bytes(rgb, flip=flip))


@needs_ref
def test_tonemap_device_buffers_of_a_render(ctx):
    import torch
    import lrt
    sc = scenes.cornell_box()
    ctx.upload(sc)
    w, h = 64, 48
    p = scenes.render_params(w, h, 4, 6, 3)
    img = torch.zeros((h, w, 3), dtype=torch.float32, device="cuda:0")
    ctx.render_dev(p, img.data_ptr())
    out = torch.empty((h, w, 3), dtype=torch.uint8, device="cuda:0")
    torch.cuda.synchronize()
    ctx._check(lrt.lib().lrt_tonemap_dev(ctx.handle, img.data_ptr(), w, h, 1, out.data_ptr()))
    torch.cuda.synchronize()
    ref = oracle.to_bytes(img.cpu().numpy(), flip=True)
    assert np.array_equal(out.cpu().numpy(), ref)
