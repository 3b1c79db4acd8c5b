"""The photon map's kd-tree built on the GPU (lrt_photon_tree.cu) against the reference's own
photon_map::build (photon_map.h:83-114, oracle/_ref): the photon order, every node and every split
value identical -- for uniform, clustered and tie-heavy positions, for photons traced in a scene, and
with a small partition budget that drives std::nth_element's heap-selection path (compared with
libstdc++'s introselect given the same budget). The host build (option photon_tree_device = 0) gives
the same tree."""
import numpy as np
import pytest

import lrt_abi as abi
import oracle
import scenes

pytestmark = pytest.mark.gpu
needs_ref = pytest.mark.skipif(not oracle.reference_available(), reason="reference oracle not built")


def _photons(rng, n, kind):
    ph = np.zeros(n, dtype=abi.PHOTON_DTYPE)
    if kind == "uniform":
        p = rng.random((n, 3)) * np.array([3.0, 1.0, 2.0])
    elif kind == "clustered":
        centers = rng.random((16, 3)) * 4.0
        p = centers[rng.integers(0, 16, n)] + rng.normal(0.0, 0.02, (n, 3))
    elif kind == "ties":  # coarse grid: many equal keys on every axis
        p = rng.integers(0, 7, (n, 3)) * 0.25
    else:  # "planes": photons on the faces of a box, one coordinate exactly constant per face
        p = rng.random((n, 3)) * 2.0 - 1.0
        face = rng.integers(0, 6, n)
        p[np.arange(n), face % 3] = np.where(face < 3, -1.0, 1.0)
    ph["position"] = p.astype(np.float32)
    ph["direction"] = rng.normal(size=(n, 3)).astype(np.float32)
    ph["power"] = rng.random((n, 3)).astype(np.float32)
    ph["depth"] = rng.integers(1, 8, n)
    return ph


def _device_tree(ctx, ph, limit=-1, device=1):
    ctx.set_option("photon_tree_device", device)
    ctx.set_option("photon_tree_depth_limit", limit)
    try:
        ctx.photon_map_build(2, ph, 1.0)
        return ctx.photon_map_tree(2, len(ph))
    finally:
        ctx.set_option("photon_tree_device", 1)
        ctx.set_option("photon_tree_depth_limit", -1)


@needs_ref
@pytest.mark.parametrize("kind", ["uniform", "clustered", "ties", "planes"])
@pytest.mark.parametrize("n", [9, 37, 1000, 65536, 300_001])
def test_device_tree_identical_to_reference(ctx, kind, n):
    ctx.upload(scenes.cornell_box(level=1))
    rng = np.random.default_rng(n * 7 + len(kind))
    ph = _photons(rng, n, kind)
    order, nodes = _device_tree(ctx, ph)
    ref_order, ref_nodes = oracle.RefPhotonMap(ph, 1.0).tree()
    assert np.array_equal(nodes, ref_nodes)
    assert np.array_equal(order, ref_order)


@needs_ref
def test_device_tree_of_traced_photons(ctx):
    ctx.upload(scenes.cornell_box(material="plastic"))
    ph, shot = ctx.photon_trace(abi.GATHER_SURFACE, 1_000_000, 8, 5)
    order, nodes = _device_tree(ctx, ph)
    ref_order, ref_nodes = oracle.RefPhotonMap(ph, 1.0 / shot).tree()
    assert np.array_equal(nodes, ref_nodes) and np.array_equal(order, ref_order)
    host_order, host_nodes = _device_tree(ctx, ph, device=0)
    assert np.array_equal(host_nodes, nodes) and np.array_equal(host_order, order)


@needs_ref
@pytest.mark.parametrize("limit", [0, 1, 3])
@pytest.mark.parametrize("kind", ["uniform", "ties"])
def test_heap_selection_path(ctx, limit, kind):
    ctx.upload(scenes.cornell_box(level=1))
    rng = np.random.default_rng(limit * 11 + len(kind))
    ph = _photons(rng, 20_000, kind)
    order, nodes = _device_tree(ctx, ph, limit=limit)
    ref_order, ref_nodes = oracle.photon_tree_limited(ph["position"], limit)
    assert np.array_equal(nodes, ref_nodes)
    assert np.array_equal(order, ref_order)
