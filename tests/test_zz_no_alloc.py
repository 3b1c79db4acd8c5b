"""The allocation-free render entry point (lrt_render_dev_noalloc), called through the C ABI.

It exists for callers that cannot let the library allocate device memory (a cudaMalloc can synchronise
the device, and fails where memory is already committed to a caching allocator or a fixed budget). Its
state lives in a fixed 32 MiB device array, so with 160x120x16 spp = 307,200 paths it renders in three
waves where lrt_render_dev renders in one; per-pixel sums keep the sample order, so the images must
agree. Two calls in a row check that the shared array's leftover contents do not leak into the next
call. On a fresh context (no wave buffers yet) the entry point is called first and the library's
count of device allocations (lrt_device_allocations) must not move, while lrt_render_dev on the same
context allocates its wave. This file is named to be collected last."""
import ctypes as C

import numpy as np
import pytest

from conftest import gpu_available, rel_close

import lrt
import scenes

pytestmark = pytest.mark.gpu


def test_render_noalloc_matches_render_dev():
    if not gpu_available():
        pytest.skip("no CUDA device")
    import torch

    L = lrt.lib()
    with lrt.Context(0) as ctx:
        ctx.upload(scenes.cornell_box(level=4))
        params = scenes.render_params(160, 120, 16, 6, 3)
        ref = torch.zeros((120, 160, 3), dtype=torch.float32, device="cuda")
        ctx.render_dev(params, ref.data_ptr())
        torch.cuda.synchronize()
        expected = ref.cpu().numpy()
        assert expected.mean() > 0
        for call in range(2):
            out = torch.full((120, 160, 3), -1.0, dtype=torch.float32, device="cuda")
            st = L.lrt_render_dev_noalloc(ctx.handle, C.byref(params), C.c_void_p(out.data_ptr()))
            assert st == 0, L.lrt_last_error(ctx.handle).decode()
            torch.cuda.synchronize()
            got = out.cpu().numpy()
            assert rel_close(got, expected).all(), "call %d differs from lrt_render_dev" % call
        too_deep = scenes.render_params(8, 8, 1, 65, 3)
        assert L.lrt_render_dev_noalloc(ctx.handle, C.byref(too_deep), C.c_void_p(out.data_ptr())) == -5
        assert b"max_depth" in L.lrt_last_error(ctx.handle)


def test_render_noalloc_first_on_fresh_context_allocates_nothing():
    if not gpu_available():
        pytest.skip("no CUDA device")
    import torch

    L = lrt.lib()
    with lrt.Context(0) as ctx:
        ctx.upload(scenes.cornell_box(level=3))
        params = scenes.render_params(96, 64, 8, 6, 3)
        out = torch.full((64, 96, 3), -1.0, dtype=torch.float32, device="cuda")
        ref = torch.zeros((64, 96, 3), dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        before = L.lrt_device_allocations()
        for call in range(2):
            st = L.lrt_render_dev_noalloc(ctx.handle, C.byref(params), C.c_void_p(out.data_ptr()))
            assert st == 0, L.lrt_last_error(ctx.handle).decode()
        torch.cuda.synchronize()
        assert L.lrt_device_allocations() == before, "the allocation-free entry point allocated device memory"
        got = out.cpu().numpy()
        ctx.render_dev(params, ref.data_ptr())
        torch.cuda.synchronize()
        assert L.lrt_device_allocations() > before  # the counter sees lrt_render_dev's wave buffers
        assert rel_close(got, ref.cpu().numpy()).all()
        assert got.mean() > 0
