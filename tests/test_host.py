"""CPU tests of liblrt's host side: the library loads and exports every C-ABI entry point, and the host
restatements (SAH kd-tree build, ggx.dat slicing, Fdr quadrature, Sobol table) match the reference.
No GPU work is launched here."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import ROOT

import lrt
import lrt_abi as abi
import oracle
import scenes


def header_symbols():
    text = open(os.path.join(ROOT, "include", "lrt.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|float|uint64_t|const char\*)\s+(lrt_\w+)\s*\(", text, re.M)))


def test_header_matches_binding_list():
    assert header_symbols() == sorted(lrt.EXPORTS)


def test_library_exports_every_declared_symbol():
    L = lrt.lib()
    for name in header_symbols():
        assert hasattr(L, name), name


def test_null_context_is_rejected_without_cuda():
    """entry points that take a context check it before any CUDA call (no GPU needed here)"""
    L = lrt.lib()
    tn, tr = C.c_uint64(7), C.c_uint64(7)
    assert L.lrt_kdtree_build_device(None, 0, None, None, None, None, 0, None, 0, None, None, None,
                                     C.byref(tn), C.byref(tr)) == -1
    cfg = abi.LaunchConfig()
    assert L.lrt_autotune(None, None, 0, 8, 3, None, None, C.byref(cfg)) == -1


def test_status_strings():
    L = lrt.lib()
    L.lrt_status_string.restype = C.c_char_p
    for code, name in abi.STATUS_NAMES.items():
        assert L.lrt_status_string(code).decode() == name


def test_create_without_gpu_reports_no_device():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    h = C.c_void_p()
    assert lrt.lib().lrt_create(0, None, C.byref(h)) == -9  # LRT_ERR_NO_DEVICE


def _tri_bounds(level):
    pos, idx, _ = scenes.displaced_icosphere(level, scenes.SPHERE_CENTER, scenes.SPHERE_RADIUS, 0.05, 20261203)
    tri = pos[idx.reshape(-1, 3)]
    return tri.min(axis=1).astype(np.float32), tri.max(axis=1).astype(np.float32)


def _ref_tree(bmin, bmax):
    lib = oracle.ref_lib()
    lib.ref_kdtree_packed.restype = C.c_int32
    cap = 8 * len(bmin) + 16
    rn = np.zeros((cap, 2), np.uint32)
    rr = np.zeros(cap, np.uint32)
    nn, nr = C.c_uint32(), C.c_uint32()
    assert lib.ref_kdtree_packed(abi.ptr(bmin, C.c_float), abi.ptr(bmax, C.c_float), len(bmin), abi.ptr(rn, C.c_uint32),
                                 cap, abi.ptr(rr, C.c_uint32), cap, C.byref(nn), C.byref(nr)) == 0
    return rn[: nn.value], rr[: nr.value]


needs_ref = pytest.mark.skipif(not oracle.reference_available(), reason="reference oracle not built")


@needs_ref
@pytest.mark.parametrize("level", [2, 4, 5, 6])
def test_kdtree_identical_to_reference(level):
    bmin, bmax = _tri_bounds(level)
    nodes, refs, depth = lrt.kdtree_build(bmin, bmax)
    rn, rr = _ref_tree(bmin, bmax)
    assert np.array_equal(nodes, rn)
    assert np.array_equal(refs, rr)
    assert depth <= 48


@needs_ref
def test_kdtree_degenerate_and_planar_boxes():
    rng = np.random.default_rng(7)
    n = 3000
    lo = rng.random((n, 3)).astype(np.float32)
    hi = lo + rng.random((n, 3)).astype(np.float32) * 0.05
    hi[::5, 1] = lo[::5, 1]            # planar in y
    hi[::7] = lo[::7]                  # points
    lo[::11, 0] = np.float32(0.5)      # many events on one plane
    hi[::11, 0] = np.float32(0.5)
    nodes, refs, _ = lrt.kdtree_build(lo, hi)
    rn, rr = _ref_tree(lo, hi)
    assert np.array_equal(nodes, rn) and np.array_equal(refs, rr)


def test_kdtree_small_inputs():
    nodes, refs, depth = lrt.kdtree_build(np.zeros((0, 3), np.float32), np.zeros((0, 3), np.float32))
    assert len(nodes) == 1 and len(refs) == 0
    nodes, refs, depth = lrt.kdtree_build(np.zeros((3, 3), np.float32), np.ones((3, 3), np.float32))
    assert len(nodes) == 1 and list(refs) == [0, 1, 2] and (nodes[0, 1] & 3) == 3


@needs_ref
@pytest.mark.parametrize("eta,alpha", [(1.49 / 1.000277, 0.15), (1.000277 / 1.49, 0.15), (1.7 / 1.000277, 0.2),
                                       (1.5, 0.05), (1.2, 0.9), (0.8, 2.0), (3.9, 0.001)])
def test_rough_transmittance_slice_bit_exact(eta, alpha):
    eta, alpha = np.float32(eta), np.float32(alpha)
    a, da = lrt.rough_transmittance_slice(oracle.GGX_PATH, eta, alpha)
    b, db = oracle.rough_transmittance(eta, alpha)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert np.float32(da).view(np.uint32) == np.float32(db).view(np.uint32)


@needs_ref
def test_rough_transmittance_errors():
    with pytest.raises(lrt.LrtError) as e:
        lrt.rough_transmittance_slice(oracle.GGX_PATH, 1.5, 5.0)
    assert e.value.status == -5
    with pytest.raises(lrt.LrtError) as e:
        lrt.rough_transmittance_slice("/nonexistent/ggx.dat", 1.5, 0.1)
    assert e.value.status == -4


@needs_ref
@pytest.mark.parametrize("eta", [1 / 1.49, 1.000277 / 1.49, 1.5, 1 / 1.7, 2.4, 1.01])
def test_fdr_matches_reference(eta):
    assert lrt.fresnel_diffuse_reflectance(eta) == oracle.fresnel_diffuse_reflectance(eta)


def test_scene_data_covers_workload_materials():
    for name in scenes.MATERIAL_NAMES:
        scenes.open_box(name, level=1)
        scenes.cornell_box(level=1, material=name)


@needs_ref
@pytest.mark.parametrize("alpha", [0.15, 0.2, 0.05, 0.3, 0.37, 0.6, 0.2 + 1e-3, 0.15 - 1e-3])
def test_scene_data_eta_slices_match_reference(alpha):
    """set_alpha on a stored eta slice = the reference's rough_transmittance at (eta, alpha), for the
    workload's alphas and the moved alphas of differentiation and optimisation"""
    data = scenes.load_scene_data()["eta_slices"]
    assert data
    for entry in data.values():
        eta = np.float32(entry["eta"])
        a, d = scenes.transmittance_table(eta, alpha)
        b, db = oracle.rough_transmittance(eta, np.float32(alpha))
        assert np.array_equal(a, b) and d == db


def test_rough_transmittance_at_alpha_errors():
    table, diffuse, rng = scenes.eta_slice(np.float32(1.49) / np.float32(1.000277))
    with pytest.raises(lrt.LrtError):
        lrt.rough_transmittance_at_alpha(table, diffuse, rng, float(rng[1]) + 1.0)
    with pytest.raises(lrt.LrtError):
        lrt.rough_transmittance_at_alpha(table[:1], diffuse[:1], rng, 0.2)


@needs_ref
def test_hosek_state_bit_exact():
    """lrt_hosek_state (the library's own cook over the model's RGB tables) against the reference's
    env_emitter state: fractional and integer turbidity (including the turbidity-10 edge, where the
    reference blends one turbidity only), ground albedo 0..1, the sun from below the horizon (the
    reference's cube root of a negative elevation is NaN, and so is the library's) to the zenith."""
    rng = np.random.default_rng(7)
    suns = [scenes.sun_direction(el, az) for el, az in [(30.0, 36.87), (0.5, 10.0), (89.0, 200.0), (60.0, 0.0)]]
    suns += [(0.6, 0.4, -0.7), (0.0, 1.0, 0.0), (1.0, 0.0, 0.0), (0.3, -0.2, 0.5)]
    suns += [tuple(rng.normal(size=3)) for _ in range(6)]
    cases = 0
    for sun in suns:
        for turbidity in (1.0, 1.5, 2.25, 3.0, 4.999, 7.3, 9.99, 10.0):
            for albedo in (0.0, 0.3, 0.77, 1.0):
                cfg, rad = lrt.hosek_state(sun, turbidity, albedo)
                rcfg, rrad = oracle.hosek_state(sun, turbidity, albedo)
                assert np.array_equal(cfg.view(np.uint64), rcfg.view(np.uint64)) or \
                    np.array_equal(cfg, rcfg, equal_nan=True), (sun, turbidity, albedo)
                assert np.array_equal(rad, rrad, equal_nan=True), (sun, turbidity, albedo)
                cases += 1
    assert cases == len(suns) * 32


def test_hosek_state_range_and_upload_cook():
    with pytest.raises(lrt.LrtError):
        lrt.hosek_state((0.0, 1.0, 0.0), 0.5, 0.3)
    with pytest.raises(lrt.LrtError):
        lrt.hosek_state((0.0, 1.0, 0.0), 10.5, 0.3)
    with pytest.raises(lrt.LrtError):
        lrt.hosek_state((0.0, 1.0, 0.0), 3.0, 1.5)
    with pytest.raises(lrt.LrtError):
        lrt.hosek_state((0.0, 0.0, 0.0), 3.0, 0.3)
    sky = scenes.sky_emitter()
    cfg, rad = scenes.hosek_state(sky["sun_direction"], sky["turbidity"], sky["albedo"])
    assert np.all(np.isfinite(cfg)) and np.all(rad > 0)


def test_diff_params_of_material_library():
    import diff
    scene, sphere, index = scenes.open_box_library(level=1)
    params = diff.scene_params(scene.materials)
    # the differentiation workload's 38 scalars: 5 roughnesses, 9 RGB albedos (three walls, the diffuse
    # sphere, plastic, rough plastic, the smooth coating's nested plastic, the two coat tints) and the
    # conductor's eta and k
    assert len(params) == 38
    assert sum(1 for p in params if p[1] == "alpha") == 5
    assert sum(1 for p in params if p[1] in ("diffuse_reflectance", "specular_reflectance")) == 27
    assert sum(1 for p in params if p[1] in ("eta", "k")) == 6
    assert diff.param_name(scene.materials, params[0]) == "m0.diffuse_reflectance[0]"
    rp = index["rough_plastic"]
    p = (rp, "alpha", None)
    assert p in params
    moved = diff.with_values(scene.materials, [p], [0.3])
    assert moved[rp]["alpha"] == 0.3 and scene.materials[rp]["alpha"] == 0.15
    assert not np.array_equal(moved[rp]["trans_table"], scene.materials[rp]["trans_table"])
    back = diff.with_values(moved, [p], [0.15])
    assert np.array_equal(back[rp]["trans_table"], scene.materials[rp]["trans_table"])


def test_diff_param_groups():
    import diff
    params = [(0, "diffuse_reflectance", 0), (0, "diffuse_reflectance", 1), (5, "alpha", None), (5, "eta", 2),
              (0, "diffuse_reflectance", 2), (5, "eta", 0), (7, "alpha", None)]
    group, chan, n = diff.param_groups(params)
    assert n == 4
    assert group == [0, 0, 1, 2, 0, 2, 3]
    assert chan == [0, 1, -1, 2, 2, 0, -1]


def test_autotune_keys_and_cache(tmp_path):
    import autotune
    scene, sphere, index = scenes.open_box_library(level=1)
    jobs, _ = scenes.batch_jobs(index, sphere, n_jobs=4)
    k1 = autotune.scene_key(scene, jobs)
    assert k1 == autotune.scene_key(scene, jobs) and k1.startswith("tris2^")
    tris = scene.triangle_count()
    paths = sum(j.width * j.height * j.spp for j in jobs)
    # the library's key: ceil(log2) of the triangle and path counts
    assert k1 == "tris2^%d_mats%d_emitters%d_paths2^%d" % ((tris - 1).bit_length(), len(scene.materials),
                                                          len(scene.emitters), (paths - 1).bit_length())
    path = str(tmp_path / "c.json")
    autotune.save_cache({k1: dict(autotune.DEFAULTS, seconds=0.5, trials=3)}, path)
    assert autotune.load_cache(path)[k1]["wave_capacity"] == autotune.DEFAULTS["wave_capacity"]
    assert autotune.load_cache(str(tmp_path / "missing.json")) == {}
    assert all(autotune.DEFAULTS[k] in autotune.CANDIDATES[k] for k in autotune.ORDER)


OBJ_TEXT = """# a quad, a pentagon fan, negative indices, normals, a degenerate triangle, CRLF lines
v 0 0 0\r
v 2 0 0\r
v 2 1.5 0\r
v 0 1.5 0\r
v 1 0.5 3.25\r
v 5 5 5
vn 0 0 2
vn 0.5 0.25 -1
vt 0.5 0.5

f 1 2 3 4
f 1//1 2//2 5//1
f -6/1/2 -5/1/1 -4 -3 -2
f 1 1 2
f 2 3 5
"""


def _write_obj(tmp_path, text=OBJ_TEXT, name="t.obj"):
    path = tmp_path / name
    path.write_bytes(text.encode())
    return str(path)


def test_load_obj_matches_reference_loader(tmp_path):
    path = _write_obj(tmp_path)
    pos, idx, nrm = lrt.load_obj(path)
    # 2 (quad) + 1 + 3 (pentagon fan) + 0 (degenerate) + 1 triangles
    assert idx.size == 3 * 7 and pos.shape == (6, 3) and nrm.shape == (21, 3)
    ext = pos[np.unique(idx)].max(0) - pos[np.unique(idx)].min(0)
    assert ext.max() == np.float32(1.0)
    if not oracle.reference_available():
        pytest.skip("reference oracle not built")
    rpos, ridx, rnrm = oracle.load_obj(path)
    assert np.array_equal(pos.view(np.uint32), rpos.view(np.uint32))
    assert np.array_equal(idx, ridx)
    assert np.array_equal(nrm.view(np.uint32), rnrm.view(np.uint32))


@pytest.mark.parametrize("text", ["v 0 0 0\nv 1 0 0\nf 1 2 3\n", "v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2\n",
                                  "v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1//4 2 3\n", "v 0 0 0\nv 1 0 0\nf 1 1 2\n"])
def test_load_obj_rejects_what_the_reference_rejects(tmp_path, text):
    path = _write_obj(tmp_path, text)
    with pytest.raises(lrt.LrtError):
        lrt.load_obj(path)
    if oracle.reference_available():
        assert oracle.load_obj(path) is None
    with pytest.raises(lrt.LrtError):
        lrt.load_obj(str(tmp_path / "missing.obj"))


@needs_ref
def test_load_obj_bunny_matches_reference():
    """the reference's own asset (src/main.cpp:69): 35,947 vertices, 69,451 faces"""
    if not os.path.exists(oracle.BUNNY_PATH):
        pytest.skip("bunny.obj not in the reference tree")
    pos, idx, nrm = lrt.load_obj(oracle.BUNNY_PATH)
    rpos, ridx, rnrm = oracle.load_obj(oracle.BUNNY_PATH)
    assert pos.shape == (35947, 3)
    assert np.array_equal(pos.view(np.uint32), rpos.view(np.uint32))
    assert np.array_equal(idx, ridx)
    assert np.array_equal(nrm.view(np.uint32), rnrm.view(np.uint32))
