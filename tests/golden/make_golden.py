"""Generates the golden fixtures in tests/golden/*.npz by running the reference itself (the unmodified
LinRT sources compiled by oracle/Makefile into oracle/_ref/liblrt_ref.so).

The reference ships no tests, golden vectors or known-answer data, so these files ARE the pinned
reference outputs: every input is stored beside the output it produced. Regenerate with
    make -C oracle ref && make -C ray-tracing_b200/csrc && python tests/golden/make_golden.py [fixture ...]
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "ray-tracing_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import lrt_abi as abi  # noqa: E402
import oracle  # noqa: E402
import scenes  # noqa: E402

SEED = 20261203


def save(name, **arrays):
    path = os.path.join(HERE, name)
    np.savez_compressed(path, **arrays)
    print("wrote", path, os.path.getsize(path), "bytes")


def unit(v):
    return v / np.linalg.norm(v, axis=-1, keepdims=True)


def random_dirs(rng, n):
    return unit(rng.normal(size=(n, 3))).astype(np.float32)


# ------------------------------------------------------------------------------------------------

def sampler_kat(rng):
    n = 256
    ps = np.zeros((n, 2), np.uint32)
    ps[:, 0] = rng.integers(0, 1 << 20, n)
    ps[:, 1] = rng.integers(0, 1 << 12, n)
    ps[:8] = [[0, 0], [0, 1], [1, 0], [12345, 63], [2**20 - 1, 4095], [7, 127], [262143, 255], [99, 1023]]
    values = oracle.sampler_values(ps, 40)
    save("sampler_kat.npz", pixel_sample=ps, values=values)


def trace_rays(rng, world, n_random=3072):
    """camera rays + interior rays in random / axis-aligned directions + bounded and outside rays"""
    w = h = 256
    n_cam = 1024
    ps = np.zeros((n_cam, 2), np.uint32)
    ps[:, 0] = rng.integers(0, w * h, n_cam)
    ps[:, 1] = rng.integers(0, 64, n_cam)
    cam = world.camera_rays(w, h, ps)
    rays = np.zeros(n_random, dtype=abi.RAY_DTYPE)
    o = np.stack([rng.uniform(-0.99, 0.99, n_random), rng.uniform(0.01, 1.99, n_random),
                  rng.uniform(-0.99, 1.49, n_random)], 1).astype(np.float32)
    d = random_dirs(rng, n_random)
    k = n_random // 8  # axis-aligned and zero-component directions (1/d = inf in traversal)
    axes = np.eye(3, dtype=np.float32)
    d[:k] = axes[rng.integers(0, 3, k)] * rng.choice([-1, 1], (k, 1)).astype(np.float32)
    d[k:2 * k, rng.integers(0, 3)] = 0.0
    d[k:2 * k] = unit(d[k:2 * k])
    # rays aimed at the sphere from the walls
    m = n_random // 4
    tgt = (np.array(scenes.SPHERE_CENTER) + rng.normal(scale=0.2, size=(m, 3))).astype(np.float32)
    d[2 * k:2 * k + m] = unit(tgt - o[2 * k:2 * k + m])
    rays["origin"], rays["direction"] = o, d
    rays["t_min"] = 0.001
    rays["t_max"] = np.float32(np.inf)
    rays["t_max"][-256:] = rng.uniform(0.05, 1.0, 256).astype(np.float32)  # bounded (shadow-like) rays
    # a few from outside the box
    rays["origin"][-512:-256] = (rng.normal(size=(256, 3)) * 3 + [0, 1, 0]).astype(np.float32)
    return np.concatenate([cam, rays])


def trace_kat(rng):
    out = {}
    for name, sc in [("cornell", scenes.cornell_box()), ("open", scenes.open_box("rough_coating"))]:
        world = oracle.RefWorld(sc)
        rays = trace_rays(rng, world)
        hits, tests = world.trace(rays)
        out[name + "_rays"] = rays
        out[name + "_hits"] = hits
        print(name, "hit rate", (hits["object"] >= 0).mean(), "triangle tests", tests)
    save("trace_kat.npz", **out)


def camera_kat(rng):
    world = oracle.RefWorld(scenes.cornell_box())
    ps = np.zeros((512, 2), np.uint32)
    ps[:, 0] = rng.integers(0, 256 * 256, 512)
    ps[:, 1] = rng.integers(0, 1 << 16, 512)
    save("camera_kat.npz", pixel_sample=ps, rays=world.camera_rays(256, 256, ps))


def material_zoo():
    """one scene carrying every BSDF configuration the BSDF KAT covers"""
    mats = [
        {"type": abi.MAT_DIFFUSE, "diffuse_reflectance": (0.8, 0.6, 0.4)},
        {"type": abi.MAT_ROUGH_CONDUCTOR, "eta": scenes.COPPER_ETA, "k": scenes.COPPER_K, "alpha": 0.1},
        {"type": abi.MAT_ROUGH_CONDUCTOR, "eta": scenes.COPPER_ETA, "k": scenes.COPPER_K, "alpha": 0.0},
        {"type": abi.MAT_DIELECTRIC, "int_ior": 1.5, "ext_ior": 1.0},
        {"type": abi.MAT_ROUGH_DIELECTRIC, "int_ior": 1.5, "ext_ior": 1.0, "alpha": 0.2},
        {"type": abi.MAT_PLASTIC, "int_ior": 1.49, "ext_ior": 1.000277, "diffuse_reflectance": (0.8, 0.8, 0.5)},
        {"type": abi.MAT_ROUGH_PLASTIC, "int_ior": 1.49, "ext_ior": 1.000277, "alpha": 0.15,
         "diffuse_reflectance": (0.8, 0.1, 0.05)},
        {"type": abi.MAT_COATING, "int_ior": 1.7, "ext_ior": 1.000277, "nested": 5, "specular_reflectance": (0.3, 0.6, 0.6)},
        {"type": abi.MAT_ROUGH_DIELECTRIC, "int_ior": 1.5, "ext_ior": 1.0, "alpha": 0.05},
        {"type": abi.MAT_ROUGH_COATING, "int_ior": 1.7, "ext_ior": 1.000277, "alpha": 0.2, "nested": 8},
        {"type": abi.MAT_COATING, "int_ior": 1.5, "ext_ior": 1.0, "nested": 0, "sigma_a": (0.5, 1.0, 2.0),
         "thickness": 0.5},
        {"type": abi.MAT_ROUGH_COATING, "int_ior": 1.7, "ext_ior": 1.000277, "alpha": 0.2, "nested": 1,
         "sigma_a": (0.2, 0.1, 0.3)},
        {"type": abi.MAT_PLASTIC, "int_ior": 1.49, "ext_ior": 1.000277, "diffuse_reflectance": (0.8, 0.3, 0.5),
         "nonlinear": 1},
    ]
    scenes.attach_tables(mats)
    quad = scenes.quad_mesh((-1, 0, -1), (-1, 0, 1), (1, 0, 1), (1, 0, -1), 0)
    emitters = [scenes.sky_emitter()]
    scenes.attach_hosek(emitters)
    return scenes.Scene([quad], mats, emitters, scenes.default_camera(), name="material_zoo")


def bsdf_queries(rng, n):
    q = np.zeros(n, dtype=abi.BSDF_QUERY_DTYPE)
    wi = random_dirs(rng, n)
    wi[: int(n * 0.85), 2] = np.abs(wi[: int(n * 0.85), 2])
    wo = random_dirs(rng, n)
    # a share of exact mirror / near-mirror directions so delta lobes evaluate non-zero
    m = n // 8
    wo[:m] = np.stack([-wi[:m, 0], -wi[:m, 1], wi[:m, 2]], 1)
    q["wi"], q["wo"] = wi, wo
    q["u"] = rng.random((n, 2), dtype=np.float32)
    q["lobe_sample"] = rng.random(n, dtype=np.float32)
    q["front_face"] = rng.random(n) < 0.8
    q["mode"] = (rng.random(n) < 0.3).astype(np.int32)
    masks = np.array([0xFFFFFFFF, abi.DIFFUSE | abi.GLOSSY, abi.SPECULAR | abi.REFLECTIVE | abi.DIELECTRIC,
                      abi.GLOSSY | abi.REFRACTIVE | abi.DIELECTRIC, abi.DIFFUSE], dtype=np.uint32)
    q["type_mask"] = masks[rng.choice(len(masks), n, p=[0.6, 0.2, 0.08, 0.06, 0.06])]
    q["component"] = rng.choice([-1, -1, -1, -1, 0, 1, 2], n)
    q["measure"] = np.where(rng.random(n) < 0.7, abi.MEASURE_SOLID_ANGLE, abi.MEASURE_DISCRETE)
    return q


def bsdf_kat(rng):
    sc = material_zoo()
    world = oracle.RefWorld(sc)
    out = {}
    for m in range(len(sc.materials)):
        q = bsdf_queries(rng, 768)
        out["q%d" % m] = q
        out["r%d" % m] = world.bsdf(m, q)
        out["flags%d" % m] = np.uint32(world.bsdf_flags(m))
    save("bsdf_kat.npz", **out)


def sky_kat(rng):
    world = oracle.RefWorld(scenes.open_box())
    d = random_dirs(rng, 1024)
    sun = np.array(scenes.sun_direction(), np.float64)
    d[:128] = unit(sun + rng.normal(scale=0.01, size=(128, 3))).astype(np.float32)  # around the sun
    d[128:256, 1] = rng.uniform(-1e-3, 2e-2, 128)                                     # near the horizon
    d[128:256] = unit(d[128:256])
    d[256:260] = [[0, 1, 0], [0, -1, 0], [1, 0, 0], [0, 0, 1]]
    save("sky_kat.npz", dirs=d, rgb=world.sky(d))


def emitter_kat(rng):
    out = {}
    for name, sc in [("cornell", scenes.cornell_box()), ("open", scenes.open_box())]:
        world = oracle.RefWorld(sc)
        n = 1024
        p = np.stack([rng.uniform(-0.99, 0.99, n), rng.uniform(0.0, 1.99, n), rng.uniform(-0.99, 1.49, n)],
                     1).astype(np.float32)
        u2 = rng.random((n, 2), dtype=np.float32)
        ds = world.emitter_sample(p, u2)
        dirs = random_dirs(rng, n)
        # half of the pdf queries along the sampled directions (inside the light / sun cone)
        ok = ds[:, 0] > 0
        dirs[ok[: n]] = np.where(rng.random((int(ok.sum()), 1)) < 0.5, ds[ok, 1:4], dirs[ok])
        out[name + "_points"], out[name + "_u2"], out[name + "_dirs"] = p, u2, dirs
        out[name + "_sample"] = ds
        out[name + "_pdf"] = world.emitter_pdf(p, dirs)
    save("emitter_kat.npz", **out)


def image_kat():
    """per-pixel mean and mean-of-squares of reference renders"""
    out = {}
    sc = scenes.cornell_box()
    world = oracle.RefWorld(sc)
    p = scenes.render_params(32, 32, 64, 6, 3)
    img, sq, secs = world.render(p, 0, True)
    out["cornell_64"], out["cornell_64_sq"] = img, sq
    print("cornell 64 spp", secs)
    p = scenes.render_params(32, 32, 4096, 6, 3, sample_offset=1 << 16)
    img, sq, secs = world.render(p, 0, True)
    out["cornell_4096"], out["cornell_4096_sq"] = img, sq
    print("cornell 4096 spp", secs)
    for name in scenes.MATERIAL_NAMES:
        world = oracle.RefWorld(scenes.open_box(name))
        p = scenes.render_params(24, 24, 256, 8, 3)
        img, sq, secs = world.render(p, 0, True)
        out["open_%s" % name], out["open_%s_sq" % name] = img, sq
        print("open", name, secs)
    save("image_kat.npz", **out)


def photon_kat(rng):
    out = {}
    for name in ["diffuse", "coating", "rough_dielectric"]:
        world = oracle.RefWorld(scenes.cornell_box(material=name))
        for kind in (abi.GATHER_SURFACE, abi.GATHER_CAUSTIC):
            ph, cnt = world.trace_particles(kind, 0, 2048, 8, 5, max_per=16)
            out["%s_%d_photons" % (name, kind)] = ph
            out["%s_%d_counts" % (name, kind)] = cnt
    save("photon_kat.npz", **out)


def knn_kat(rng):
    n = 6000
    photons = np.zeros(n, dtype=abi.PHOTON_DTYPE)
    centers = rng.random((12, 3)).astype(np.float32)
    photons["position"] = (centers[rng.integers(0, 12, n)] + rng.normal(scale=0.08, size=(n, 3))).astype(np.float32)
    photons["position"][:500] = rng.random((500, 3)).astype(np.float32)
    photons["direction"] = random_dirs(rng, n)
    photons["normal"] = random_dirs(rng, n)
    photons["power"] = rng.random((n, 3), dtype=np.float32)
    photons["depth"] = rng.integers(2, 9, n)
    q = (centers[rng.integers(0, 12, 400)] + rng.normal(scale=0.1, size=(400, 3))).astype(np.float32)
    normals = random_dirs(rng, 400)
    pm = oracle.RefPhotonMap(photons, scale=1.0 / 7777.0)
    out = {"photons": photons, "points": q, "normals": normals}
    for r2, k in [(0.0025, 16), (0.01, 64), (0.04, 100)]:
        idx, d2, cnt = pm.knn(q, r2, k)
        out["idx_%d" % k], out["d2_%d" % k], out["cnt_%d" % k] = idx, d2, cnt
    for radius, depth, k in [(0.05, 6, 64), (0.1, 4, 100)]:
        out["irr_%d" % k] = pm.irradiance(q, normals, radius, depth, k)
    save("knn_kat.npz", **out)


def light_kat():
    """area lights over a triangle mesh (scenes.mesh_light_box): emitter sampling and pdf at random
    points, and per-particle photons emitted from the mesh light"""
    rng = np.random.default_rng(SEED + 11)
    out = {}
    world = oracle.RefWorld(scenes.mesh_light_box(level=1))
    n = 2048
    p = np.stack([rng.uniform(-0.99, 0.99, n), rng.uniform(0.0, 1.99, n), rng.uniform(-0.99, 1.49, n)],
                 1).astype(np.float32)
    u2 = rng.random((n, 2), dtype=np.float32)
    ds = world.emitter_sample(p, u2)
    dirs = random_dirs(rng, n)
    ok = ds[:, 0] > 0
    dirs[ok] = np.where(rng.random((int(ok.sum()), 1)) < 0.7, ds[ok, 1:4], dirs[ok])
    out["mesh_points"], out["mesh_u2"], out["mesh_dirs"] = p, u2, dirs
    out["mesh_sample"] = ds
    out["mesh_pdf"] = world.emitter_pdf(p, dirs)
    world.close()
    world = oracle.RefWorld(scenes.mesh_light_box(level=3))
    ph, cnt = world.trace_particles(abi.GATHER_SURFACE, 0, 2048, 8, 5, max_per=16)
    out["mesh_photons"], out["mesh_photon_counts"] = ph, cnt
    world.close()
    save("light_kat.npz", **out)


def image_out_kat():
    """the image writer's float-to-byte conversion (io/image_write.cpp:10-20) and its vertical flip:
    special values, the values on either side of every byte boundary ((k/256)^2.2 and its float
    neighbours), and log-normal radiance, laid out as rows of 23 RGB pixels"""
    rng = np.random.default_rng(SEED + 13)
    special = np.array([0.0, -0.0, np.nan, np.inf, -np.inf, -1.0, -1e-30, 1e-45, 1e-38, 1e-30, 1e-10,
                        1.0, 0.5, 2.0, 1e30, 3.4e38], dtype=np.float32)
    edges = []
    for k in range(1, 257):
        e = np.float32((k / 256.0) ** 2.2)
        up, down = e, e
        edges.append(e)
        for _ in range(3):
            up = np.nextafter(up, np.float32(np.inf))
            down = np.nextafter(down, np.float32(-np.inf))
            edges += [up, down]
    edges = np.array(edges, dtype=np.float32)
    lognormal = np.exp(rng.normal(-1.5, 1.5, 6000)).astype(np.float32)
    values = np.concatenate([special, edges, lognormal])
    row = 23 * 3
    pad = (-len(values)) % row
    values = np.concatenate([values, rng.random(pad, dtype=np.float32)])
    rgb = values.reshape(-1, 23, 3)
    save("image_out_kat.npz", rgb=rgb, bytes=oracle.to_bytes(rgb), bytes_flipped=oracle.to_bytes(rgb, flip=True))


def main():
    if len(sys.argv) > 1:  # only the named fixtures, e.g. `make_golden.py light_kat`
        for name in sys.argv[1:]:
            globals()[name]()
        return
    rng = np.random.default_rng(SEED)
    sampler_kat(rng)
    camera_kat(rng)
    trace_kat(rng)
    bsdf_kat(rng)
    sky_kat(rng)
    emitter_kat(rng)
    knn_kat(rng)
    photon_kat(rng)
    image_kat()
    light_kat()
    image_out_kat()


if __name__ == "__main__":
    main()
