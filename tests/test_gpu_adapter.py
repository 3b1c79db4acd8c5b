"""The reference-side adapter (include/lrt_linrt.hpp) compiled against the reference's own headers
(oracle/_ref/adapter_test, built by oracle/Makefile from tests/adapter_test.cpp): the reference's demo
scene (src/main.cpp:38-90 plus its sphere light) built from the reference's classes, translated by the
adapter's scene walk (hittable_list::for_each), rendered on the GPU by gpu_path_integrator /
gpu_photon_integrator and on the CPU by the reference's own integrators with their own constants; every
pixel within 3 Monte Carlo standard errors of the reference's per-pixel spread (at most 1% beyond, the
3-sigma tail plus paths that diverge after a last-bit difference)."""
import json
import os
import subprocess

import pytest

import oracle

pytestmark = pytest.mark.gpu

ADAPTER_TEST = os.path.join(oracle.REF_DIR, "adapter_test")
needs_adapter = pytest.mark.skipif(not os.path.exists(ADAPTER_TEST) or not os.path.exists(oracle.BUNNY_PATH),
                                   reason="adapter test program (oracle/_ref/adapter_test) not built")


def run(mode, w, h, spp):
    # the reference's rough_transmittance reads third_party/data/ggx.dat relative to the working directory
    out = subprocess.run([ADAPTER_TEST, oracle.BUNNY_PATH, mode, str(w), str(h), str(spp)], capture_output=True,
                         text=True, timeout=600, cwd=oracle.REF_DIR)
    assert out.returncode == 0, out.stdout + out.stderr
    return json.loads(out.stdout.strip().splitlines()[-1])


@needs_adapter
def test_adapter_path_integrator_matches_reference(ctx):
    r = run("path", 48, 48, 16)
    assert r["pixels"] == 48 * 48 and r["nonfinite"] == 0
    assert r["beyond_3se"] <= 0.01, r
    assert abs(r["gpu_mean"] - r["reference_mean"]) <= 0.01 * r["reference_mean"], r


@needs_adapter
def test_adapter_photon_integrator_matches_reference(ctx):
    r = run("photon", 32, 32, 4)
    assert r["pixels"] == 32 * 32 and r["nonfinite"] == 0
    assert r["beyond_3se"] <= 0.01, r
    assert abs(r["gpu_mean"] - r["reference_mean"]) <= 0.02 * r["reference_mean"], r
