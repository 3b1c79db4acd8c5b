"""Seeded synthetic scenes of the LinRT rendering workloads.

Every scene is built from plain numpy arrays (float32 positions, uint32 indices, float32 corner
normals), so the GPU library and the reference harness receive identical inputs.

* ``cornell_box``: a closed box of 10 axis-aligned quads (20 triangles, each quad its own
  triangle_mesh), white walls 0.75, left wall (0.63, 0.06, 0.06), right wall (0.14, 0.45, 0.09), a
  ceiling quad area light of radiance (17, 12, 4), and an icosphere subdivided 6 times (81,920
  triangles) displaced radially by 5% with seeded 3-octave value noise, diffuse albedo 0.8.
  ``open_box`` removes the roof and the light and lights the box with a Hosek sky (turbidity 3, sun
  elevation 30 degrees, ground albedo 0.3); the sphere carries one of the seven materials.
* Materials follow the reference constructors and src/main.cpp:38-47 where the workload leaves a
  parameter open (plastic Kd, coating nests).

Rough-transmittance tables are caller-side inputs of the library (the reference slices them from its
ggx.dat at material construction): the eta slices the workload materials need are read from
``data/scene_data.json`` (``tests/golden/make_scene_data.py`` fills it) and cut to a 1-D table for any
alpha by the library. The Hosek sky state is cooked by the library (``lrt.hosek_state``).
"""
from __future__ import annotations

import base64
import functools
import json
import math
import os
from dataclasses import dataclass, field

import numpy as np

import lrt_abi as abi

DATA_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")
SCENE_DATA = os.path.join(DATA_DIR, "scene_data.json")

COPPER_ETA = (0.200438, 0.924033, 1.102212)   # fresnel.h:15-20
COPPER_K = (3.912948, 2.452847, 2.142188)

SKY_TURBIDITY = 3.0
SKY_ALBEDO = 0.3
SKY_SCALE = 0.05            # src/main.cpp:53
SUN_ELEVATION_DEG = 30.0
SUN_AZIMUTH_DEG = 36.87     # horizontal direction (0.6, 0, 0.8)

MATERIAL_NAMES = ["diffuse", "rough_dielectric", "rough_conductor", "plastic", "rough_plastic",
                  "coating", "rough_coating"]


@dataclass
class Scene:
    objects: list = field(default_factory=list)
    materials: list = field(default_factory=list)
    emitters: list = field(default_factory=list)
    camera: dict = field(default_factory=dict)
    name: str = ""

    def triangle_count(self) -> int:
        return sum(len(o["indices"]) // 3 for o in self.objects if o["kind"] == abi.OBJ_MESH)


# ---------------------------------------------------------------------------------------------
# caller-side tables (rough transmittance) and the cooked Hosek state

_scene_data_cache = None


def _f32_key(*values) -> str:
    return "_".join("%08x" % np.float32(v).view(np.uint32) for v in values)


def load_scene_data() -> dict:
    global _scene_data_cache
    if _scene_data_cache is None:
        if os.path.exists(SCENE_DATA):
            with open(SCENE_DATA) as f:
                _scene_data_cache = json.load(f)
        else:
            _scene_data_cache = {"eta_slices": {}}
    return _scene_data_cache


_eta_slice_cache = {}


def eta_slice(eta: float):
    """(sliced_table, sliced_diffuse, alpha_range) of the rough-transmittance data at eta (float32 key)."""
    key = _f32_key(eta)
    if key not in _eta_slice_cache:
        data = load_scene_data().get("eta_slices", {})
        if key not in data:
            raise KeyError("no rough-transmittance eta slice for eta=%r in %s; run tests/golden/make_scene_data.py"
                           % (float(eta), SCENE_DATA))
        e = data[key]
        n = e["n_alpha"]
        table = np.frombuffer(base64.b64decode(e["table_f32_b64"]), dtype="<f4").reshape(n, abi.TRANS_SAMPLES)
        diffuse = np.frombuffer(base64.b64decode(e["diffuse_f32_b64"]), dtype="<f4")
        _eta_slice_cache[key] = (table.astype(np.float32), diffuse.astype(np.float32),
                                 np.array(e["alpha_range"], dtype=np.float32))
    return _eta_slice_cache[key]


def transmittance_table(eta: float, alpha: float):
    """1-D rough-transmittance table and diffuse transmittance for (eta, alpha) as float32, by set_alpha
    (liblrt's host routine) on the stored eta slice."""
    import lrt
    table, diffuse, rng = eta_slice(eta)
    return lrt.rough_transmittance_at_alpha(table, diffuse, rng, float(np.float32(alpha)))


def hosek_state(sun_direction, turbidity: float, albedo: float):
    """(config (3, 9), radiance (3,)) of the sky, cooked by liblrt as env_emitter's constructor does."""
    import lrt
    return lrt.hosek_state(sun_direction, turbidity, albedo)


def required_tables(materials) -> list:
    """(eta, alpha) pairs whose tables the materials need."""
    out = []
    for m in materials:
        if m["type"] == abi.MAT_ROUGH_PLASTIC:
            eta = np.float32(m["int_ior"]) / np.float32(m["ext_ior"])
            out += [(eta, np.float32(m["alpha"])), (np.float32(1.0) / eta, np.float32(m["alpha"]))]
        elif m["type"] == abi.MAT_ROUGH_COATING:
            out.append((np.float32(m["int_ior"]) / np.float32(m["ext_ior"]), np.float32(m["alpha"])))
    return out


def attach_tables(materials) -> None:
    """Fill trans_table / trans_internal_diffuse of rough plastic and rough coating materials."""
    for m in materials:
        if m["type"] == abi.MAT_ROUGH_PLASTIC:
            eta = np.float32(m["int_ior"]) / np.float32(m["ext_ior"])
            m["trans_table"], _ = transmittance_table(eta, m["alpha"])
            _, m["trans_internal_diffuse"] = transmittance_table(np.float32(1.0) / eta, m["alpha"])
        elif m["type"] == abi.MAT_ROUGH_COATING:
            eta = np.float32(m["int_ior"]) / np.float32(m["ext_ior"])
            m["trans_table"], _ = transmittance_table(eta, m["alpha"])


def attach_hosek(emitters) -> None:
    for e in emitters:
        if e["kind"] == abi.EMITTER_ENV:
            e["hosek_config"], e["hosek_radiance"] = hosek_state(e["sun_direction"], e["turbidity"], e["albedo"])


def sun_direction(elevation_deg: float = SUN_ELEVATION_DEG, azimuth_deg: float = SUN_AZIMUTH_DEG):
    el, az = math.radians(elevation_deg), math.radians(azimuth_deg)
    return (math.cos(el) * math.sin(az), math.sin(el), math.cos(el) * math.cos(az))


# ---------------------------------------------------------------------------------------------
# geometry

def _hash3(ix, iy, iz, seed):
    """32-bit integer lattice hash -> [-1, 1)."""
    h = (ix.astype(np.uint32) * np.uint32(0x8DA6B343)) ^ (iy.astype(np.uint32) * np.uint32(0xD8163841)) \
        ^ (iz.astype(np.uint32) * np.uint32(0xCB1AB31F)) ^ np.uint32(seed)
    h ^= h >> np.uint32(16)
    h *= np.uint32(0x7FEB352D)
    h ^= h >> np.uint32(15)
    h *= np.uint32(0x846CA68B)
    h ^= h >> np.uint32(16)
    return h.astype(np.float64) * (2.0 / 4294967296.0) - 1.0


def value_noise(p: np.ndarray, seed: int) -> np.ndarray:
    """Trilinear lattice value noise with smoothstep weights, in [-1, 1]."""
    fl = np.floor(p)
    f = p - fl
    i = fl.astype(np.int64)
    w = f * f * (3.0 - 2.0 * f)
    out = np.zeros(p.shape[0])
    with np.errstate(over="ignore"):
        for dx in (0, 1):
            for dy in (0, 1):
                for dz in (0, 1):
                    v = _hash3(i[:, 0] + dx, i[:, 1] + dy, i[:, 2] + dz, seed)
                    wx = w[:, 0] if dx else 1.0 - w[:, 0]
                    wy = w[:, 1] if dy else 1.0 - w[:, 1]
                    wz = w[:, 2] if dz else 1.0 - w[:, 2]
                    out += v * wx * wy * wz
    return out


def fbm(p: np.ndarray, seed: int, octaves: int = 3) -> np.ndarray:
    """Octave sum with gains 1/2 and frequencies x2, normalised to [-1, 1]."""
    total = np.zeros(p.shape[0])
    norm = 0.0
    amp, freq = 1.0, 1.0
    for o in range(octaves):
        total += amp * value_noise(p * freq, seed + 1013 * o)
        norm += amp
        amp *= 0.5
        freq *= 2.0
    return total / norm


@functools.lru_cache(maxsize=8)
def icosphere(level: int):
    """Unit icosphere: 20 * 4**level triangles (float64 vertices, int64 faces)."""
    t = (1.0 + math.sqrt(5.0)) / 2.0
    v = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
                  [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], dtype=np.float64)
    f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4], [11, 10, 2],
                  [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5],
                  [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], dtype=np.int64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    for _ in range(level):
        a, b, c = f[:, 0], f[:, 1], f[:, 2]
        edges = np.stack([np.stack([a, b], 1), np.stack([b, c], 1), np.stack([c, a], 1)], 1).reshape(-1, 2)
        key = np.sort(edges, axis=1)
        uniq, inv = np.unique(key[:, 0] * (v.shape[0] + 1) + key[:, 1], return_inverse=True)
        e0 = uniq // (v.shape[0] + 1)
        e1 = uniq % (v.shape[0] + 1)
        mid = v[e0] + v[e1]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        mid_idx = (inv + v.shape[0]).reshape(-1, 3)
        v = np.concatenate([v, mid])
        ab, bc, ca = mid_idx[:, 0], mid_idx[:, 1], mid_idx[:, 2]
        f = np.concatenate([np.stack([a, ab, ca], 1), np.stack([b, bc, ab], 1), np.stack([c, ca, bc], 1),
                            np.stack([ab, bc, ca], 1)])
    return v, f


def displaced_icosphere(level: int, center, radius: float, amplitude: float, seed: int, frequency: float = 2.0):
    """Icosphere with radial displacement radius * (1 + amplitude * fbm(frequency * p)).

    Returns float32 positions, uint32 indices and float32 corner normals (area-weighted vertex normals)."""
    v, f = icosphere(level)
    r = radius * (1.0 + amplitude * fbm(v * frequency, seed))
    pos = v * r[:, None] + np.asarray(center, dtype=np.float64)[None, :]
    p0, p1, p2 = pos[f[:, 0]], pos[f[:, 1]], pos[f[:, 2]]
    fn = np.cross(p1 - p0, p2 - p0)
    vn = np.zeros_like(pos)
    for k in range(3):
        np.add.at(vn, f[:, k], fn)
    vn /= np.linalg.norm(vn, axis=1, keepdims=True)
    idx = f.reshape(-1).astype(np.uint32)
    corner_normals = vn[f.reshape(-1)].astype(np.float32)
    return pos.astype(np.float32), idx, corner_normals


def obj_mesh(path: str, material: int, scale: float = 1.0, offset=(0.0, 0.0, 0.0)) -> dict:
    """A mesh object from a Wavefront OBJ (liblrt's lrt_load_obj: the reference's load_obj, centred and
    scaled to a longest side of 1), then scaled and moved as given."""
    import lrt
    pos, idx, nrm = lrt.load_obj(path)
    if scale != 1.0 or any(offset):
        pos = (pos * np.float32(scale) + np.asarray(offset, dtype=np.float32)).astype(np.float32)
    return {"kind": abi.OBJ_MESH, "material": material, "positions": pos, "indices": idx, "corner_normals": nrm}


def quad_mesh(p0, p1, p2, p3, material: int):
    """Two-triangle mesh (p0,p1,p2), (p0,p2,p3) with flat corner normals."""
    pos = np.array([p0, p1, p2, p3], dtype=np.float32)
    idx = np.array([0, 1, 2, 0, 2, 3], dtype=np.uint32)
    n = np.cross(np.float64(pos[1]) - pos[0], np.float64(pos[2]) - pos[0])
    n /= np.linalg.norm(n)
    return {"kind": abi.OBJ_MESH, "material": material, "positions": pos, "indices": idx,
            "corner_normals": np.tile(n.astype(np.float32), (6, 1))}


# box extents: x in [-1, 1], y in [0, 2], z in [-1, 1.5]; light opening in the roof
BOX_X, BOX_Y, BOX_Z0, BOX_Z1 = 1.0, 2.0, -1.0, 1.5
HOLE = 0.3


def _box_quads(white: int, red: int, green: int, roof: bool):
    X, Y, Z0, Z1 = BOX_X, BOX_Y, BOX_Z0, BOX_Z1
    zm = 0.25
    quads = [
        quad_mesh((-X, 0, Z0), (-X, 0, zm), (X, 0, zm), (X, 0, Z0), white),     # floor, back half (normal +y)
        quad_mesh((-X, 0, zm), (-X, 0, Z1), (X, 0, Z1), (X, 0, zm), white),     # floor, front half
        quad_mesh((-X, 0, Z0), (X, 0, Z0), (X, Y, Z0), (-X, Y, Z0), white),     # back wall (normal +z)
        quad_mesh((-X, 0, Z1), (-X, Y, Z1), (X, Y, Z1), (X, 0, Z1), white),     # front wall (normal -z)
        quad_mesh((-X, 0, Z0), (-X, Y, Z0), (-X, Y, Z1), (-X, 0, Z1), red),     # left wall (normal +x)
        quad_mesh((X, 0, Z0), (X, 0, Z1), (X, Y, Z1), (X, Y, Z0), green),       # right wall (normal -x)
    ]
    if roof:
        h = HOLE
        quads += [  # roof strips around the light opening (normal -y)
            quad_mesh((-X, Y, Z0), (X, Y, Z0), (X, Y, -h), (-X, Y, -h), white),
            quad_mesh((-X, Y, h), (X, Y, h), (X, Y, Z1), (-X, Y, Z1), white),
            quad_mesh((-X, Y, -h), (-h, Y, -h), (-h, Y, h), (-X, Y, h), white),
            quad_mesh((h, Y, -h), (X, Y, -h), (X, Y, h), (h, Y, h), white),
        ]
    return quads


def material_library(name: str):
    """(materials list, index of the sphere material) for one of the seven materials; the three wall
    materials always come first (0 white, 1 red, 2 green)."""
    mats = [
        {"type": abi.MAT_DIFFUSE, "diffuse_reflectance": (0.75, 0.75, 0.75)},
        {"type": abi.MAT_DIFFUSE, "diffuse_reflectance": (0.63, 0.06, 0.06)},
        {"type": abi.MAT_DIFFUSE, "diffuse_reflectance": (0.14, 0.45, 0.09)},
    ]
    plastic = {"type": abi.MAT_PLASTIC, "int_ior": 1.49, "ext_ior": 1.000277, "specular_reflectance": (1, 1, 1),
               "diffuse_reflectance": (0.8, 0.8, 0.5)}
    if name == "diffuse":
        mats.append({"type": abi.MAT_DIFFUSE, "diffuse_reflectance": (0.8, 0.8, 0.8)})
    elif name == "rough_dielectric":
        mats.append({"type": abi.MAT_ROUGH_DIELECTRIC, "int_ior": 1.5, "ext_ior": 1.0, "alpha": 0.2})
    elif name == "rough_conductor":
        mats.append({"type": abi.MAT_ROUGH_CONDUCTOR, "eta": COPPER_ETA, "k": COPPER_K, "alpha": 0.1})
    elif name == "plastic":
        mats.append(plastic)
    elif name == "rough_plastic":
        mats.append({"type": abi.MAT_ROUGH_PLASTIC, "int_ior": 1.49, "ext_ior": 1.000277, "alpha": 0.15,
                     "specular_reflectance": (1, 1, 1), "diffuse_reflectance": (0.8, 0.1, 0.05)})
    elif name == "coating":
        mats.append(plastic)
        mats.append({"type": abi.MAT_COATING, "int_ior": 1.7, "ext_ior": 1.000277, "nested": len(mats) - 1,
                     "specular_reflectance": (0.3, 0.6, 0.6)})
    elif name == "rough_coating":
        mats.append({"type": abi.MAT_ROUGH_DIELECTRIC, "int_ior": 1.5, "ext_ior": 1.0, "alpha": 0.05})
        mats.append({"type": abi.MAT_ROUGH_COATING, "int_ior": 1.7, "ext_ior": 1.000277, "alpha": 0.2,
                     "nested": len(mats) - 1})
    elif name == "dielectric":
        mats.append({"type": abi.MAT_DIELECTRIC, "int_ior": 1.5, "ext_ior": 1.0})
    else:
        raise ValueError("unknown material %r" % name)
    return mats, len(mats) - 1


def default_camera(aspect: float = 1.0):
    return {"origin": (0.0, 1.0, 1.3), "look_at": (0.0, 0.55, 0.0), "up": (0.0, 1.0, 0.0), "fov": 60.0,
            "aspect": aspect}


SPHERE_CENTER = (0.0, 0.45, 0.0)
SPHERE_RADIUS = 0.42


def cornell_box(level: int = 6, seed: int = 20261203, material: str = "diffuse", aspect: float = 1.0,
                attach: bool = True) -> Scene:
    """Closed box + ceiling area light + displaced icosphere (diffuse 0.8 by default)."""
    mats, sphere_mat = material_library(material)
    objects = _box_quads(0, 1, 2, roof=True)
    pos, idx, nrm = displaced_icosphere(level, SPHERE_CENTER, SPHERE_RADIUS, 0.05, seed)
    objects.append({"kind": abi.OBJ_MESH, "material": sphere_mat, "positions": pos, "indices": idx,
                    "corner_normals": nrm})
    h = HOLE
    light = {"kind": abi.OBJ_RECTANGLE, "material": -1, "corner": (-h, BOX_Y - 1e-3, -h),
             "edge_u": (2 * h, 0.0, 0.0), "edge_v": (0.0, 0.0, 2 * h)}
    objects.append(light)
    emitters = [{"kind": abi.EMITTER_AREA, "object": len(objects) - 1, "radiance": (17.0, 12.0, 4.0)}]
    scene = Scene(objects, mats, emitters, default_camera(aspect), name="cornell_box_%s" % material)
    if attach:
        attach_tables(scene.materials)
    return scene


def mesh_box(path: str, material: str = "diffuse", scale: float = 0.9, aspect: float = 1.0, attach: bool = True) -> Scene:
    """The closed box and ceiling light of cornell_box with an OBJ mesh (e.g. the reference's bunny) in
    place of the sphere: loaded as the reference's load_obj loads it, scaled to `scale` and set on the
    floor."""
    mats, mesh_mat = material_library(material)
    objects = _box_quads(0, 1, 2, roof=True)
    mesh = obj_mesh(path, mesh_mat, scale)
    lo = mesh["positions"].min(axis=0)
    mesh["positions"] = (mesh["positions"] + np.array([0.0, 0.01 - lo[1], 0.0], dtype=np.float32)).astype(np.float32)
    objects.append(mesh)
    h = HOLE
    objects.append({"kind": abi.OBJ_RECTANGLE, "material": -1, "corner": (-h, BOX_Y - 1e-3, -h),
                    "edge_u": (2 * h, 0.0, 0.0), "edge_v": (0.0, 0.0, 2 * h)})
    emitters = [{"kind": abi.EMITTER_AREA, "object": len(objects) - 1, "radiance": (17.0, 12.0, 4.0)}]
    scene = Scene(objects, mats, emitters, default_camera(aspect), name="mesh_box_%s" % material)
    if attach:
        attach_tables(scene.materials)
    return scene


def demo_scene(bunny_path: str, aspect: float = 1.0, sphere_light: bool = False, attach: bool = True) -> Scene:
    """The reference's own demo scene (src/main.cpp:58-90): the bunny loaded by load_obj with the rough
    plastic of main.cpp:43 (alpha 0.1, Kd (0.8, 0.1, 0.05)), the ground as a sphere of radius 100 centred
    at (0, -100.5, 0) with diffuse (0.8, 0.8, 0), and the 1.2 x 1.2 rectangle light of radiance 12 at
    height 1.5; the camera at (0, 0.5, 3) looks at the origin (camera.h's default look_at) with a 60
    degree field of view. sphere_light adds the sphere light main.cpp:55-56 defines (radius 0.3 at
    (1.2, 0.4, 0), radiance 4) as an object and an emitter of the scene (main.cpp builds it but leaves it
    out)."""
    mats = [{"type": abi.MAT_ROUGH_PLASTIC, "int_ior": 1.49, "ext_ior": 1.000277, "alpha": 0.1,
             "specular_reflectance": (1, 1, 1), "diffuse_reflectance": (0.8, 0.1, 0.05)},
            {"type": abi.MAT_DIFFUSE, "diffuse_reflectance": (0.8, 0.8, 0.0)}]
    objects = [obj_mesh(bunny_path, 0),
               {"kind": abi.OBJ_SPHERE, "material": 1, "center": (0.0, -100.5, 0.0), "radius": 100.0},
               {"kind": abi.OBJ_RECTANGLE, "material": -1, "corner": (-0.6, 1.5, -0.6), "edge_u": (1.2, 0.0, 0.0),
                "edge_v": (0.0, 0.0, 1.2)}]
    emitters = [{"kind": abi.EMITTER_AREA, "object": 2, "radiance": (12.0, 12.0, 12.0)}]
    if sphere_light:
        objects.append({"kind": abi.OBJ_SPHERE, "material": -1, "center": (1.2, 0.4, 0.0), "radius": 0.3})
        emitters.append({"kind": abi.EMITTER_AREA, "object": 3, "radiance": (4.0, 4.0, 4.0)})
    camera = {"origin": (0.0, 0.5, 3.0), "look_at": (0.0, 0.0, 0.0), "up": (0.0, 1.0, 0.0), "fov": 60.0,
              "aspect": aspect}
    scene = Scene(objects, mats, emitters, camera, name="demo_scene" + ("_sphere_light" if sphere_light else ""))
    if attach:
        attach_tables(scene.materials)
    return scene


def mesh_light_box(level: int = 6, light_level: int = 2, seed: int = 20261203, material: str = "diffuse",
                   aspect: float = 1.0, attach: bool = True) -> Scene:
    """The closed box and displaced sphere of cornell_box lit by an emitting triangle mesh instead of the
    ceiling rectangle: a displaced icosphere (level 2, 320 triangles, radius 0.16) near the ceiling with
    radiance (9, 6, 3) and a white diffuse surface, an area light over a mesh as area_emitter takes any
    hittable (area_emitter.h:17-49, triangle_mesh.h:109-138). A second emitter, a small rectangle on the
    back wall of radiance (2, 3, 6), makes the light pick of scene::sample_emitter_direction matter."""
    mats, sphere_mat = material_library(material)
    objects = _box_quads(0, 1, 2, roof=True)
    pos, idx, nrm = displaced_icosphere(level, SPHERE_CENTER, SPHERE_RADIUS, 0.05, seed)
    objects.append({"kind": abi.OBJ_MESH, "material": sphere_mat, "positions": pos, "indices": idx,
                    "corner_normals": nrm})
    lpos, lidx, lnrm = displaced_icosphere(light_level, (0.35, 1.55, 0.2), 0.16, 0.1, seed + 7)
    objects.append({"kind": abi.OBJ_MESH, "material": 0, "positions": lpos, "indices": lidx, "corner_normals": lnrm})
    emitters = [{"kind": abi.EMITTER_AREA, "object": len(objects) - 1, "radiance": (9.0, 6.0, 3.0)}]
    objects.append({"kind": abi.OBJ_RECTANGLE, "material": -1, "corner": (-0.7, 0.6, BOX_Z0 + 1e-3),
                    "edge_u": (0.3, 0.0, 0.0), "edge_v": (0.0, 0.3, 0.0)})  # normal +z, into the box
    emitters.append({"kind": abi.EMITTER_AREA, "object": len(objects) - 1, "radiance": (2.0, 3.0, 6.0)})
    scene = Scene(objects, mats, emitters, default_camera(aspect), name="mesh_light_box_%s" % material)
    if attach:
        attach_tables(scene.materials)
    return scene


def sky_emitter():
    return {"kind": abi.EMITTER_ENV, "sun_direction": sun_direction(), "turbidity": SKY_TURBIDITY,
            "albedo": SKY_ALBEDO, "scale": SKY_SCALE}


def open_box(material: str = "diffuse", level: int = 6, seed: int = 20261203, aspect: float = 1.0,
             attach: bool = True) -> Scene:
    """The box without roof and light, open to the Hosek sky; the sphere carries `material`."""
    mats, sphere_mat = material_library(material)
    objects = _box_quads(0, 1, 2, roof=False)
    pos, idx, nrm = displaced_icosphere(level, SPHERE_CENTER, SPHERE_RADIUS, 0.05, seed)
    objects.append({"kind": abi.OBJ_MESH, "material": sphere_mat, "positions": pos, "indices": idx,
                    "corner_normals": nrm})
    emitters = [sky_emitter()]
    scene = Scene(objects, mats, emitters, default_camera(aspect), name="open_box_%s" % material)
    if attach:
        attach_tables(scene.materials)
        attach_hosek(scene.emitters)
    return scene


def open_box_library(level: int = 6, seed: int = 20261203, aspect: float = 1.0, attach: bool = True):
    """The open box with every material of MATERIAL_NAMES in one material list, for batched jobs that
    each put one of them on the sphere. Returns (scene, sphere object index, {name: material index});
    the sphere carries the diffuse material by default."""
    mats = []
    index = {}
    for name in MATERIAL_NAMES:
        lib_mats, sphere = material_library(name)
        if not mats:
            mats.extend(dict(m) for m in lib_mats[:3])
        offset = len(mats) - 3
        for m in lib_mats[3:]:
            m = dict(m)
            if "nested" in m:
                m["nested"] += offset
            mats.append(m)
        index[name] = sphere + offset
    scene = open_box("diffuse", level, seed, aspect, attach=False)
    sphere_obj = next(i for i, o in enumerate(scene.objects) if o["kind"] == abi.OBJ_MESH and len(o["indices"]) > 6 * 3)
    scene.objects[sphere_obj]["material"] = index["diffuse"]
    scene.materials = mats
    scene.name = "open_box_library"
    if attach:
        attach_tables(scene.materials)
        attach_hosek(scene.emitters)
    return scene, sphere_obj, index


def job_desc(camera: dict, width: int, height: int, spp: int, sample_offset: int = 0, override_object: int = -1,
             override_material: int = -1, output_offset: int = 0):
    return abi.JobDesc(abi.camera_desc(camera), width, height, spp, sample_offset, override_object,
                       override_material, output_offset)


def large_scene(level: int = 5, grid=(8, 8, 4), seed: int = 20261206, spacing: float = 1.15, aspect: float = 1.0,
                attach: bool = True) -> Scene:
    """The large photon-mapping scene: an 8 x 8 x 4 grid of seeded displaced icospheres (level 5,
    20,480 triangles each, radii uniform in [0.2, 0.5], each carrying one of the seven materials at
    random) above a ground quad, lit by the Hosek sky and four quad lights facing down. Each sphere is
    its own mesh object, as a reference scene built from triangle_mesh objects would hold them
    (256 x 20,480 = 5,242,880 sphere triangles)."""
    rng = np.random.default_rng(seed)
    mats = [{"type": abi.MAT_DIFFUSE, "diffuse_reflectance": (0.5, 0.5, 0.5)}]  # ground
    index = {}
    for name in MATERIAL_NAMES:
        lib_mats, sphere = material_library(name)
        offset = len(mats) - 3
        for m in lib_mats[3:]:
            m = dict(m)
            if "nested" in m:
                m["nested"] += offset
            mats.append(m)
        index[name] = sphere + offset
    nx, nz, ny = grid
    S = 0.5 * spacing * max(nx, nz) + 2.0
    objects = [quad_mesh((-S, 0.0, S), (S, 0.0, S), (S, 0.0, -S), (-S, 0.0, -S), 0)]
    for iy in range(ny):
        for iz in range(nz):
            for ix in range(nx):
                center = ((ix - 0.5 * (nx - 1)) * spacing, 0.55 + iy * spacing, (iz - 0.5 * (nz - 1)) * spacing)
                radius = float(rng.uniform(0.2, 0.5))
                material = MATERIAL_NAMES[int(rng.integers(len(MATERIAL_NAMES)))]
                sphere_seed = int(rng.integers(1 << 30))
                pos, idx, nrm = displaced_icosphere(level, center, radius, 0.05, sphere_seed)
                objects.append({"kind": abi.OBJ_MESH, "material": index[material], "positions": pos,
                                "indices": idx, "corner_normals": nrm})
    emitters = []
    top = 0.55 + ny * spacing + 1.5
    h = 0.75
    for cx, cz in ((-2.5, -2.5), (2.5, -2.5), (-2.5, 2.5), (2.5, 2.5)):
        objects.append({"kind": abi.OBJ_RECTANGLE, "material": -1, "corner": (cx - h, top, cz - h),
                        "edge_u": (2 * h, 0.0, 0.0), "edge_v": (0.0, 0.0, 2 * h)})
        emitters.append({"kind": abi.EMITTER_AREA, "object": len(objects) - 1, "radiance": (12.0, 11.0, 9.0)})
    emitters.append(sky_emitter())
    camera = {"origin": (10.0, 4.0, 12.0), "look_at": (0.0, 2.2, 0.0), "up": (0.0, 1.0, 0.0), "fov": 45.0,
              "aspect": aspect}
    scene = Scene(objects, mats, emitters, camera, name="large_grid_%dx%dx%d_level%d" % (nx, nz, ny, level))
    if attach:
        attach_tables(scene.materials)
        attach_hosek(scene.emitters)
    return scene


# workloads -----------------------------------------------------------------------------------

CONFIG0 = {"width": 256, "height": 256, "spp": 16, "max_depth": 6, "rr_depth": 3}
CONFIG3 = {"width": 1024, "height": 1024, "spp": 32, "photons": 16_000_000, "photon_depth": 8, "k": 100,
           "radius_cap": 0.05}
CONFIG1 = {"width": 512, "height": 512, "spp": 64, "max_depth": 8, "rr_depth": 3,
           "photons": 1_000_000, "k": 64}


BATCH_RESOLUTIONS = [(128, 128), (256, 256), (512, 512), (1024, 768)]
BATCH_SEED = 20261204


def batch_jobs(scene_index: dict, sphere: int, n_jobs: int = 64, seed: int = BATCH_SEED, spp_range=(4, 256)):
    """The batched workload: n_jobs jobs drawn from `seed`, each with a resolution from BATCH_RESOLUTIONS,
    spp uniform in spp_range (inclusive), a camera on a sphere of radius 3-5 around the origin looking at
    it (upper hemisphere, 10-70 degrees elevation, so that it sees into the open box), and one of the
    seven materials on the sphere. Jobs are packed back to back in the output buffer. Returns
    (jobs, specs) with specs the per-job dicts."""
    rng = np.random.default_rng(seed)
    jobs, specs, offset = [], [], 0
    for _ in range(n_jobs):
        w, h = BATCH_RESOLUTIONS[int(rng.integers(len(BATCH_RESOLUTIONS)))]
        spp = int(rng.integers(spp_range[0], spp_range[1] + 1))
        radius = float(rng.uniform(3.0, 5.0))
        elev = np.radians(float(rng.uniform(10.0, 70.0)))
        azim = np.radians(float(rng.uniform(0.0, 360.0)))
        origin = (radius * np.cos(elev) * np.sin(azim), radius * np.sin(elev), radius * np.cos(elev) * np.cos(azim))
        material = MATERIAL_NAMES[int(rng.integers(len(MATERIAL_NAMES)))]
        cam = {"origin": tuple(float(x) for x in origin), "look_at": (0.0, 0.3, 0.0), "up": (0.0, 1.0, 0.0),
               "fov": 30.0, "aspect": w / h}
        spec = {"camera": cam, "width": w, "height": h, "spp": spp, "material": material, "output_offset": offset}
        jobs.append(job_desc(cam, w, h, spp, 0, sphere, scene_index[material], offset))
        specs.append(spec)
        offset += 3 * w * h
    return jobs, specs


def render_params(width, height, spp, max_depth, rr_depth, sample_offset=0, row_begin=0, row_end=0):
    return abi.RenderParams(width, height, spp, max_depth, rr_depth, sample_offset, row_begin, row_end)
