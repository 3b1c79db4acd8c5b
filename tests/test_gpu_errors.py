"""Error paths on a GPU that stay on the host side of the device: a device allocation the GPU cannot
satisfy is reported as LRT_ERR_OUT_OF_MEMORY with the failing call in the message, and the context
keeps working afterwards; calls without a scene report LRT_ERR_NO_SCENE. Nothing here faults the GPU:
cudaMalloc of more memory than the device has returns an error and allocates nothing."""
import ctypes as C

import numpy as np
import pytest

import lrt
import lrt_abi as abi
import scenes

pytestmark = pytest.mark.gpu


def test_out_of_memory_reported_and_context_usable(ctx):
    ctx.upload(scenes.cornell_box(level=2))
    L = lrt.lib()
    out = np.zeros(1, dtype=abi.PHOTON_DTYPE)
    n, shot = C.c_uint32(0), C.c_uint64(0)
    # 4e9 photons x 52 bytes: more device memory than a B200 has
    st = L.lrt_photon_trace(ctx.handle, abi.GATHER_SURFACE, 4_000_000_000, 8, 5, abi.ptr(out, abi.Photon),
                            C.byref(n), C.byref(shot))
    assert st == abi.LRT_ERR_OUT_OF_MEMORY, st
    assert b"cudaMalloc" in L.lrt_last_error(ctx.handle) or b"ensure" in L.lrt_last_error(ctx.handle)
    ph, shot = ctx.photon_trace(abi.GATHER_SURFACE, 1000, 8, 5)
    assert len(ph) == 1000 and shot > 0
    img = ctx.render(scenes.render_params(16, 16, 2, 4, 2))
    assert np.isfinite(img).all() and img.mean() > 0


def test_no_scene_reported():
    with lrt.Context(0) as fresh:
        L = lrt.lib()
        p = scenes.render_params(8, 8, 1, 2, 1)
        rgb = np.zeros((8, 8, 3), np.float32)
        assert L.lrt_render(fresh.handle, C.byref(p), abi.ptr(rgb, C.c_float)) == abi.LRT_ERR_NO_SCENE
