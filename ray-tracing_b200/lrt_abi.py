"""ctypes mirrors of the C ABI in include/lrt.h, and helpers that turn a Python scene into an
``lrt_scene_desc`` whose arrays stay alive as long as the returned holder.

The same structures are passed to liblrt (the product) and, in tests, to the reference harness, so both
sides are built from identical arrays.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

LRT_OK = 0
STATUS_NAMES = {
    0: "LRT_OK", -1: "LRT_ERR_INVALID_ARGUMENT", -2: "LRT_ERR_CUDA", -3: "LRT_ERR_OUT_OF_MEMORY",
    -4: "LRT_ERR_IO", -5: "LRT_ERR_RANGE", -6: "LRT_ERR_NO_SCENE", -9: "LRT_ERR_NO_DEVICE",
}
for _code, _name in STATUS_NAMES.items():
    globals()[_name] = _code

# BSDF flags (src/material/bsdf.h:18-28)
DIFFUSE, SPECULAR, REFLECTIVE, TRANSPARENT = 1, 2, 4, 8
GLOSSY, METALLIC, DIELECTRIC, REFRACTIVE = 16, 32, 64, 128
MEASURE_SOLID_ANGLE, MEASURE_DISCRETE = 1, 5
MODE_RADIANCE, MODE_IMPORTANCE = 0, 1

MAT_DIFFUSE, MAT_ROUGH_CONDUCTOR, MAT_DIELECTRIC, MAT_ROUGH_DIELECTRIC = 0, 1, 2, 3
MAT_PLASTIC, MAT_ROUGH_PLASTIC, MAT_COATING, MAT_ROUGH_COATING = 4, 5, 6, 7
OBJ_MESH, OBJ_RECTANGLE, OBJ_SPHERE = 0, 1, 2
EMITTER_AREA, EMITTER_ENV = 0, 1
GATHER_SURFACE, GATHER_CAUSTIC = 0, 1
TRANS_SAMPLES = 100

STAGE_NAMES = ["raygen", "extend", "sort", "shade", "shadow", "accumulate"]


class MaterialDesc(C.Structure):
    _fields_ = [
        ("type", C.c_int32), ("nested", C.c_int32), ("nonlinear", C.c_int32),
        ("int_ior", C.c_float), ("ext_ior", C.c_float), ("alpha", C.c_float), ("thickness", C.c_float),
        ("diffuse_reflectance", C.c_float * 3), ("specular_reflectance", C.c_float * 3),
        ("specular_transmittance", C.c_float * 3), ("eta", C.c_float * 3), ("k", C.c_float * 3),
        ("sigma_a", C.c_float * 3), ("trans_table", C.c_float * TRANS_SAMPLES),
        ("trans_internal_diffuse", C.c_float), ("eta_pair", C.c_float * 2),
    ]


class ObjectDesc(C.Structure):
    _fields_ = [
        ("kind", C.c_int32), ("material", C.c_int32), ("n_vertices", C.c_uint32), ("n_indices", C.c_uint32),
        ("positions", C.POINTER(C.c_float)), ("indices", C.POINTER(C.c_uint32)),
        ("corner_normals", C.POINTER(C.c_float)),
        ("corner", C.c_float * 3), ("edge_u", C.c_float * 3), ("edge_v", C.c_float * 3),
        ("center", C.c_float * 3), ("radius", C.c_float),
    ]


class EmitterDesc(C.Structure):
    _fields_ = [
        ("kind", C.c_int32), ("object", C.c_int32), ("radiance", C.c_float * 3),
        ("sun_direction", C.c_float * 3), ("turbidity", C.c_float), ("albedo", C.c_float), ("scale", C.c_float),
        ("hosek_config", (C.c_double * 9) * 3), ("hosek_radiance", C.c_double * 3),
    ]


class CameraDesc(C.Structure):
    _fields_ = [
        ("origin", C.c_float * 3), ("look_at", C.c_float * 3), ("up", C.c_float * 3),
        ("fov_degrees", C.c_float), ("aspect_ratio", C.c_float),
    ]


class SceneDesc(C.Structure):
    _fields_ = [
        ("n_objects", C.c_uint32), ("objects", C.POINTER(ObjectDesc)),
        ("n_materials", C.c_uint32), ("materials", C.POINTER(MaterialDesc)),
        ("n_emitters", C.c_uint32), ("emitters", C.POINTER(EmitterDesc)),
        ("camera", CameraDesc),
    ]


class Ray(C.Structure):
    _fields_ = [("origin", C.c_float * 3), ("direction", C.c_float * 3), ("t_min", C.c_float), ("t_max", C.c_float)]


class Hit(C.Structure):
    _fields_ = [("t", C.c_float), ("object", C.c_int32), ("prim", C.c_int32), ("front_face", C.c_int32),
                ("p", C.c_float * 3), ("normal", C.c_float * 3)]


class BsdfQuery(C.Structure):
    _fields_ = [("wi", C.c_float * 3), ("wo", C.c_float * 3), ("u", C.c_float * 2), ("lobe_sample", C.c_float),
                ("front_face", C.c_int32), ("mode", C.c_int32), ("type_mask", C.c_uint32),
                ("component", C.c_int32), ("measure", C.c_int32)]


class BsdfResult(C.Structure):
    _fields_ = [("sample_weight", C.c_float * 3), ("sample_wo", C.c_float * 3), ("sample_pdf", C.c_float),
                ("sample_eta", C.c_float), ("sampled_type", C.c_uint32), ("sampled_component", C.c_int32),
                ("eval", C.c_float * 3), ("pdf", C.c_float)]


class Photon(C.Structure):
    _fields_ = [("position", C.c_float * 3), ("direction", C.c_float * 3), ("normal", C.c_float * 3),
                ("power", C.c_float * 3), ("depth", C.c_uint32)]


class RenderParams(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("spp", C.c_uint32), ("max_depth", C.c_int32),
                ("rr_depth", C.c_int32), ("sample_offset", C.c_uint32), ("row_begin", C.c_uint32),
                ("row_end", C.c_uint32)]


def camera_desc(camera: dict) -> CameraDesc:
    cam = CameraDesc()
    cam.origin = _f3(camera["origin"])
    cam.look_at = _f3(camera["look_at"])
    cam.up = _f3(camera["up"])
    cam.fov_degrees = camera["fov"]
    cam.aspect_ratio = camera["aspect"]
    return cam


class DiffParam(C.Structure):
    _fields_ = [("group", C.c_uint32), ("channel", C.c_int32)]


class JobDesc(C.Structure):
    _fields_ = [("camera", CameraDesc), ("width", C.c_uint32), ("height", C.c_uint32), ("spp", C.c_uint32),
                ("sample_offset", C.c_uint32), ("override_object", C.c_int32), ("override_material", C.c_int32),
                ("output_offset", C.c_uint64)]


class LaunchConfig(C.Structure):
    _fields_ = [("wave_capacity", C.c_uint32), ("pixel_tile", C.c_uint32), ("blocks_per_sm", C.c_uint32),
                ("from_cache", C.c_uint32), ("seconds", C.c_float), ("trials", C.c_uint32)]


class PhotonRenderParams(C.Structure):
    _fields_ = [("global_map", C.c_int32), ("caustic_map", C.c_int32), ("global_radius", C.c_float),
                ("caustic_radius", C.c_float), ("max_depth", C.c_int32), ("max_specular_depth", C.c_int32),
                ("direct_samples", C.c_int32), ("glossy_samples", C.c_int32), ("lookup_size", C.c_uint32)]

    @classmethod
    def reference_defaults(cls, lookup_size=120):
        """photon_integrator.h:57-65"""
        return cls(-1, -1, 0.0, 0.0, 128, 4, 16, 32, lookup_size)


class RenderStats(C.Structure):
    _fields_ = [("paths", C.c_uint64), ("extension_rays", C.c_uint64), ("shadow_rays", C.c_uint64),
                ("nodes_visited", C.c_uint64), ("triangles_tested", C.c_uint64),
                ("shadow_nodes_visited", C.c_uint64), ("shadow_triangles_tested", C.c_uint64),
                ("shading_events", C.c_uint64),
                ("kernel_launches", C.c_uint64), ("stage_ms", C.c_float * 6), ("stage_launches", C.c_uint32 * 6),
                ("rays_at_depth", C.c_uint64 * 16), ("knn_queries", C.c_uint64), ("knn_nodes_visited", C.c_uint64),
                ("knn_photons_tested", C.c_uint64), ("knn_photons_found", C.c_uint64)]


# numpy views of the record arrays
RAY_DTYPE = np.dtype([("origin", "<f4", 3), ("direction", "<f4", 3), ("t_min", "<f4"), ("t_max", "<f4")])
HIT_DTYPE = np.dtype([("t", "<f4"), ("object", "<i4"), ("prim", "<i4"), ("front_face", "<i4"),
                      ("p", "<f4", 3), ("normal", "<f4", 3)])
BSDF_QUERY_DTYPE = np.dtype([("wi", "<f4", 3), ("wo", "<f4", 3), ("u", "<f4", 2), ("lobe_sample", "<f4"),
                             ("front_face", "<i4"), ("mode", "<i4"), ("type_mask", "<u4"), ("component", "<i4"),
                             ("measure", "<i4")])
BSDF_RESULT_DTYPE = np.dtype([("sample_weight", "<f4", 3), ("sample_wo", "<f4", 3), ("sample_pdf", "<f4"),
                              ("sample_eta", "<f4"), ("sampled_type", "<u4"), ("sampled_component", "<i4"),
                              ("eval", "<f4", 3), ("pdf", "<f4")])
PHOTON_DTYPE = np.dtype([("position", "<f4", 3), ("direction", "<f4", 3), ("normal", "<f4", 3),
                         ("power", "<f4", 3), ("depth", "<u4")])
assert RAY_DTYPE.itemsize == C.sizeof(Ray)
assert HIT_DTYPE.itemsize == C.sizeof(Hit)
assert BSDF_QUERY_DTYPE.itemsize == C.sizeof(BsdfQuery)
assert BSDF_RESULT_DTYPE.itemsize == C.sizeof(BsdfResult)
assert PHOTON_DTYPE.itemsize == C.sizeof(Photon)


def ptr(array: np.ndarray, ctype=None):
    """Pointer to a C-contiguous numpy array (the array must outlive the call)."""
    assert array.flags["C_CONTIGUOUS"], "array must be C-contiguous"
    return array.ctypes.data_as(C.POINTER(ctype) if ctype is not None else C.c_void_p)


def _f3(values) -> "C.Array":
    v = np.asarray(values, dtype=np.float32).reshape(3)
    return (C.c_float * 3)(*[float(x) for x in v])


def material_descs(materials, out=None, start=0):
    """lrt_material_desc records of a material list (into `out` from index `start` when given)."""
    if out is None:
        out = (MaterialDesc * max(1, len(materials)))()
    for i, m in enumerate(materials):
        d = out[start + i]
        d.type = m["type"]
        d.nested = m.get("nested", -1)
        d.nonlinear = int(m.get("nonlinear", 0))
        d.int_ior = m.get("int_ior", 1.5)
        d.ext_ior = m.get("ext_ior", 1.0)
        d.alpha = m.get("alpha", 0.0)
        d.thickness = m.get("thickness", 1.0)
        d.diffuse_reflectance = _f3(m.get("diffuse_reflectance", (0.5, 0.5, 0.5)))
        d.specular_reflectance = _f3(m.get("specular_reflectance", (1, 1, 1)))
        d.specular_transmittance = _f3(m.get("specular_transmittance", (1, 1, 1)))
        d.eta = _f3(m.get("eta", (0, 0, 0)))
        d.k = _f3(m.get("k", (0, 0, 0)))
        d.sigma_a = _f3(m.get("sigma_a", (0, 0, 0)))
        table = m.get("trans_table")
        if table is not None:
            t = np.asarray(table, dtype=np.float32)
            assert t.size == TRANS_SAMPLES
            d.trans_table = (C.c_float * TRANS_SAMPLES)(*[float(x) for x in t])
        d.trans_internal_diffuse = float(m.get("trans_internal_diffuse", 0.0))
        pair = m.get("eta_pair")
        if pair is not None:
            d.eta_pair = (C.c_float * 2)(float(pair[0]), float(pair[1]))
    return out


class SceneHolder:
    """Owns the ctypes descriptors and numpy buffers of one lrt_scene_desc."""

    def __init__(self, scene):
        self.scene = scene
        self.keep = []
        objs = (ObjectDesc * max(1, len(scene.objects)))()
        for i, o in enumerate(scene.objects):
            d = objs[i]
            d.kind = o["kind"]
            d.material = o.get("material", -1)
            if o["kind"] == OBJ_MESH:
                pos = np.ascontiguousarray(o["positions"], dtype=np.float32).reshape(-1)
                idx = np.ascontiguousarray(o["indices"], dtype=np.uint32).reshape(-1)
                nrm = np.ascontiguousarray(o["corner_normals"], dtype=np.float32).reshape(-1)
                assert nrm.size == idx.size * 3
                self.keep += [pos, idx, nrm]
                d.n_vertices = pos.size // 3
                d.n_indices = idx.size
                d.positions = ptr(pos, C.c_float)
                d.indices = ptr(idx, C.c_uint32)
                d.corner_normals = ptr(nrm, C.c_float)
            elif o["kind"] == OBJ_RECTANGLE:
                d.corner, d.edge_u, d.edge_v = _f3(o["corner"]), _f3(o["edge_u"]), _f3(o["edge_v"])
            else:
                d.center = _f3(o["center"])
                d.radius = float(np.float32(o["radius"]))
        mats = material_descs(scene.materials)
        ems = (EmitterDesc * max(1, len(scene.emitters)))()
        for i, e in enumerate(scene.emitters):
            d = ems[i]
            d.kind = e["kind"]
            d.object = e.get("object", -1)
            d.radiance = _f3(e.get("radiance", (0, 0, 0)))
            if e["kind"] == EMITTER_ENV:
                d.sun_direction = _f3(e["sun_direction"])
                d.turbidity = e["turbidity"]
                d.albedo = e["albedo"]
                d.scale = e["scale"]
                cfg = e.get("hosek_config")
                if cfg is not None:
                    cfg = np.asarray(cfg, dtype=np.float64).reshape(3, 9)
                    for c in range(3):
                        for j in range(9):
                            d.hosek_config[c][j] = float(cfg[c, j])
                    for c in range(3):
                        d.hosek_radiance[c] = float(e["hosek_radiance"][c])
        cam = camera_desc(scene.camera)
        self.objects, self.materials, self.emitters = objs, mats, ems
        self.desc = SceneDesc(len(scene.objects), objs, len(scene.materials), mats, len(scene.emitters), ems, cam)

    @property
    def ref(self):
        return C.byref(self.desc)
