"""The GPU SAH kd-tree build (lrt_kdtree_build_device, scene option kd_build_device).

Its trees must equal the host builder's -- which the host tests pin to the reference's
sah_kdtree::build -- node for node and leaf reference for leaf reference: single meshes from one
primitive to the level-6 sphere, flat and coincident boxes, signed zeros on a split plane, many meshes
built in one call, and a whole scene upload (the large 257-object scene) checked by its tree sizes and
by traced hits.
"""
import time

import numpy as np
import pytest

import lrt
import oracle
import scenes
from test_gpu_large import random_rays

pytestmark = pytest.mark.gpu
needs_ref = pytest.mark.skipif(not oracle.reference_available(), reason="reference build (oracle/_ref) missing")


def sphere_boxes(level, seed=20261203):
    pos, idx, _ = scenes.displaced_icosphere(level, scenes.SPHERE_CENTER, scenes.SPHERE_RADIUS, 0.05, seed)
    tri = pos[idx.reshape(-1, 3)]
    return tri.min(axis=1).astype(np.float32), tri.max(axis=1).astype(np.float32)


def soup(n, seed, size=0.05):
    rng = np.random.default_rng(seed)
    lo = rng.random((n, 3)).astype(np.float32)
    return lo, (lo + rng.random((n, 3)).astype(np.float32) * np.float32(size)).astype(np.float32)


def flat_and_coincident(n=3000, seed=7):
    lo, hi = soup(n, seed)
    hi[::5, 1] = lo[::5, 1]            # flat in y: planar events
    hi[::7] = lo[::7]                  # points
    lo[::11, 0] = np.float32(0.5)      # many events on one plane
    hi[::11, 0] = np.float32(0.5)
    lo[::13] = lo[0]                   # coincident boxes
    hi[::13] = hi[0]
    return lo, hi


def signed_zeros(n=2000, seed=11):
    """boxes starting or ending at x = -0.0 or +0.0, mixed: one sweep group holds both zeros"""
    lo, hi = soup(n, seed, 0.2)
    lo -= np.float32(0.5)
    hi -= np.float32(0.5)
    k = np.arange(n)
    zero = np.where(k % 2 == 0, np.float32(-0.0), np.float32(0.0)).astype(np.float32)
    a = k % 3 == 0
    lo[a, 0] = zero[a]
    hi[a, 0] = np.abs(hi[a, 0]) + np.float32(0.01)
    b = k % 3 == 1
    hi[b, 0] = zero[b]
    lo[b, 0] = -np.abs(lo[b, 0]) - np.float32(0.01)
    return lo, hi


def identical(n=500):
    return np.full((n, 3), 0.25, np.float32), np.full((n, 3), 0.75, np.float32)


def walls():
    """the axis-aligned quads of a box (two triangles per wall, all flat) plus a coarse sphere"""
    quads = []
    for axis in range(3):
        for v in (0.0, 1.0):
            lo = np.zeros(3, np.float32)
            hi = np.ones(3, np.float32)
            lo[axis] = hi[axis] = v
            quads += [(lo, hi), (lo, hi)]
    slo, shi = sphere_boxes(2)
    return (np.concatenate([np.array([q[0] for q in quads]), slo]).astype(np.float32),
            np.concatenate([np.array([q[1] for q in quads]), shi]).astype(np.float32))


CASES = {
    "one": soup(1, 1),
    "six": soup(6, 2),
    "seven": soup(7, 3),
    "forty": soup(40, 4, 0.3),
    "soup1000": soup(1000, 5),
    "soup30000": soup(30000, 6, 0.02),
    "flat_and_coincident": flat_and_coincident(),
    "signed_zeros": signed_zeros(),
    "identical": identical(),
    "walls": walls(),
    "sphere3": sphere_boxes(3),
    "sphere6": sphere_boxes(6),
}


def host_tree(bmin, bmax):
    nodes, refs, depth = lrt.kdtree_build(bmin, bmax)
    return nodes, refs, depth


def assert_same(gpu, host, name):
    (gn, gr, gd), (hn, hr, hd) = gpu, host
    assert gn.shape == hn.shape, "%s: %s nodes vs %s" % (name, gn.shape, hn.shape)
    assert np.array_equal(gn, hn), "%s: first differing node %d" % (name, int(np.argmax((gn != hn).any(axis=1))))
    assert np.array_equal(gr, hr), name
    assert gd == hd, name


@pytest.mark.parametrize("name", list(CASES))
def test_device_tree_equals_host_tree(ctx, name):
    bmin, bmax = CASES[name]
    assert_same(ctx.kdtree_build_device([(bmin, bmax)])[0], host_tree(bmin, bmax), name)


def test_many_meshes_in_one_build(ctx):
    names = list(CASES)
    trees = ctx.kdtree_build_device([CASES[n] for n in names])
    for name, tree in zip(names, trees):
        assert_same(tree, host_tree(*CASES[name]), name)


@needs_ref
def test_device_tree_equals_reference_tree(ctx):
    from test_host import _ref_tree
    bmin, bmax = CASES["sphere6"]
    nodes, refs, _ = ctx.kdtree_build_device([(bmin, bmax)])[0]
    rn, rr = _ref_tree(bmin, bmax)
    assert np.array_equal(nodes, rn) and np.array_equal(refs, rr)


def test_errors(ctx):
    lo, hi = soup(100, 9)
    lo[17, 2] = np.nan
    with pytest.raises(lrt.LrtError) as e:
        ctx.kdtree_build_device([(lo, hi)])
    assert e.value.status == -1
    with pytest.raises(lrt.LrtError) as e:
        ctx.kdtree_build_device([soup(10, 1), (np.zeros((0, 3), np.float32), np.zeros((0, 3), np.float32))])
    assert e.value.status == -1
    with pytest.raises(lrt.LrtError) as e:
        ctx.set_option("kd_build_device", 3)
    assert e.value.status == -5
    # the context stays usable
    assert_same(ctx.kdtree_build_device([CASES["forty"]])[0], host_tree(*CASES["forty"]), "forty")


def test_scene_upload_with_device_trees():
    """the large scene (256 level-5 spheres, ground quad, four lights): same trees, same hits, whichever
    builder the upload uses (0 host cores, 1 GPU; the default picks the GPU at this size)"""
    scene = scenes.large_scene()
    rng = np.random.default_rng(5)
    rays = random_rays(rng, 200_000, [-5.0, 0.0, -5.0], [5.0, 5.0, 5.0])
    out = {}
    for device in (0, 1):
        with lrt.Context(0) as c:
            c.set_option("kd_build_device", device)
            t0 = time.perf_counter()
            c.upload(scene)
            seconds = time.perf_counter() - t0
            info = [c.mesh_tree_info(i) for i in range(len(scene.objects))]
            out[device] = (info, c.trace(rays), seconds)
    print("scene upload: host trees %.2f s, device trees %.2f s" % (out[0][2], out[1][2]))
    assert out[0][0] == out[1][0]
    a, b = out[0][1], out[1][1]
    assert np.array_equal(a["object"], b["object"]) and np.array_equal(a["prim"], b["prim"])
    assert np.array_equal(a["t"].view(np.uint32), b["t"].view(np.uint32))
