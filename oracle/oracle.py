"""TEST INFRASTRUCTURE: ctypes loader of the reference oracle (oracle/_ref/liblrt_ref.so, the
unmodified reference compiled by oracle/Makefile) and of the C restatement (oracle/build/liblrt_oracle.so).

Only tests/, the smoke check and the CPU-baseline leg of bench.py use this module.
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "ray-tracing_b200"))
import lrt_abi as abi  # noqa: E402

ORACLE_DIR = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(ORACLE_DIR, "_ref")
REF_LIB = os.path.join(REF_DIR, "liblrt_ref.so")
GGX_PATH = os.path.join(REF_DIR, "third_party", "data", "ggx.dat")
RESTATEMENT_LIB = os.path.join(ORACLE_DIR, "build", "liblrt_oracle.so")

_ref = {}
TIMING_LIBS = {v: os.path.join(REF_DIR, "liblrt_ref_timing_%s.so" % v) for v in ("v3", "v4")}


def reference_available() -> bool:
    return os.path.exists(REF_LIB) and os.path.exists(GGX_PATH)


def _load(path):
    if True:
        lib = C.CDLL(path)
        vp, u32, i32, f32 = C.c_void_p, C.c_uint32, C.c_int32, C.c_float
        P = C.POINTER
        lib.ref_last_error.restype = C.c_char_p
        lib.ref_world_create.restype = vp
        lib.ref_world_create.argtypes = [P(abi.SceneDesc), C.c_char_p]
        lib.ref_world_destroy.argtypes = [vp]
        lib.ref_trace.restype = C.c_int64
        lib.ref_trace.argtypes = [vp, P(abi.Ray), u32, P(abi.Hit), P(C.c_uint64)]
        lib.ref_bsdf_query.argtypes = [vp, i32, P(abi.BsdfQuery), u32, P(abi.BsdfResult)]
        lib.ref_bsdf_flags.restype = u32
        lib.ref_bsdf_flags.argtypes = [vp, i32]
        lib.ref_sky_eval.argtypes = [vp, P(f32), u32, P(f32)]
        lib.ref_emitter_sample.argtypes = [vp, P(f32), P(f32), u32, P(f32)]
        lib.ref_emitter_pdf.argtypes = [vp, P(f32), P(f32), u32, P(f32)]
        lib.ref_sampler_values.argtypes = [P(u32), u32, u32, P(f32)]
        lib.ref_camera_rays.argtypes = [vp, u32, u32, P(u32), u32, P(abi.Ray)]
        lib.ref_render.restype = C.c_double
        lib.ref_render.argtypes = [vp, P(abi.RenderParams), u32, P(f32), P(f32)]
        lib.ref_render_window.restype = C.c_double
        lib.ref_render_window.argtypes = [vp, P(abi.RenderParams), u32, u32, u32, P(f32), P(f32)]
        lib.ref_photon_render.restype = C.c_double
        lib.ref_photon_render.argtypes = [vp, P(abi.RenderParams), u32, P(abi.Photon), u32, f32, P(abi.Photon), u32, f32,
                                          P(abi.PhotonRenderParams), P(f32), P(f32)]
        lib.ref_trace_particles.argtypes = [vp, i32, u32, u32, i32, i32, u32, P(abi.Photon), P(u32)]
        lib.ref_photon_gather.restype = u32
        lib.ref_photon_gather.argtypes = [vp, i32, u32, i32, i32, P(abi.Photon), P(C.c_uint64), P(C.c_double)]
        lib.ref_photon_map_create.restype = vp
        lib.ref_photon_map_create.argtypes = [P(abi.Photon), u32, f32]
        lib.ref_photon_map_destroy.argtypes = [vp]
        lib.ref_photon_map_tree.restype = i32
        lib.ref_photon_map_tree.argtypes = [vp, P(u32), P(i32), C.c_uint64, P(u32)]
        lib.ref_photon_tree_limited.restype = i32
        lib.ref_photon_tree_limited.argtypes = [P(f32), u32, C.c_int, P(u32), P(i32), C.c_uint64, P(u32)]
        lib.ref_photon_map_knn.argtypes = [vp, P(f32), u32, f32, u32, P(u32), P(f32), P(u32)]
        lib.ref_photon_map_irradiance.argtypes = [vp, P(f32), P(f32), u32, f32, i32, u32, P(f32)]
        lib.ref_rough_transmittance.restype = i32
        lib.ref_rough_transmittance.argtypes = [C.c_char_p, f32, f32, P(f32), P(f32)]
        lib.ref_rough_transmittance_eval.restype = f32
        lib.ref_rough_transmittance_eval.argtypes = [C.c_char_p, f32, f32, f32]
        lib.ref_fresnel_diffuse_reflectance.restype = f32
        lib.ref_fresnel_diffuse_reflectance.argtypes = [f32]
        lib.ref_hosek_state.argtypes = [P(f32), f32, f32, P(C.c_double), P(C.c_double)]
        lib.ref_hardware_concurrency.restype = u32
        lib.ref_to_bytes.argtypes = [P(f32), C.c_int, C.c_int, C.c_int, P(C.c_uint8)]
        return lib


def ref_lib(timing: bool = False):
    """The parity build (timing=False: -O2/-O3 -ffp-contract=off, the reference's own arithmetic), or
    the timing build for this host (timing=True: -O3 for the widest x86-64 level its CPU supports,
    with GCC's default contraction), falling back to the parity build when none was made."""
    global _ref
    if not reference_available():
        raise FileNotFoundError("reference oracle not built: run `make -C oracle ref` (needs the reference sources)")
    key = timing_variant() if timing else "parity"
    if key not in _ref:
        _ref[key] = _load(TIMING_LIBS.get(key, REF_LIB))
    return _ref[key]


def cpu_flags() -> set:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    return set(line.split(":", 1)[1].split())
    except OSError:
        pass
    return set()


def timing_variant() -> str:
    """'v4' (AVX-512), 'v3' (AVX2 + FMA) or 'parity': the widest timing build this host can run"""
    flags = cpu_flags()
    v3 = {"avx", "avx2", "bmi1", "bmi2", "f16c", "fma", "abm", "movbe", "xsave"}
    v4 = v3 | {"avx512f", "avx512bw", "avx512cd", "avx512dq", "avx512vl"}
    for name, need in (("v4", v4), ("v3", v3)):
        if need <= flags and os.path.exists(TIMING_LIBS[name]):
            return name
    return "parity"


def timing_build_flags() -> str:
    v = timing_variant()
    return "-O3 -ffp-contract=off (parity build)" if v == "parity" else "-O3 -march=x86-64-%s" % v


def _p(a, t=C.c_float):
    return abi.ptr(a, t)


class RefWorld:
    """Reference objects built from the same scene description as the GPU library."""

    def __init__(self, scene, timing: bool = False):
        """timing=True: the timing build (the CPU baseline); otherwise the parity build."""
        self.holder = abi.SceneHolder(scene)
        self.lib = ref_lib(timing)
        self.handle = self.lib.ref_world_create(C.byref(self.holder.desc), REF_DIR.encode())
        if not self.handle:
            raise RuntimeError("reference scene construction failed: %s" % self.lib.ref_last_error().decode())

    def close(self):
        if self.handle:
            self.lib.ref_world_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def trace(self, rays: np.ndarray):
        rays = np.ascontiguousarray(rays, dtype=abi.RAY_DTYPE)
        hits = np.zeros(len(rays), dtype=abi.HIT_DTYPE)
        tests = C.c_uint64(0)
        mism = self.lib.ref_trace(self.handle, _p(rays, abi.Ray), len(rays), _p(hits, abi.Hit), C.byref(tests))
        assert mism == 0, "harness object loop disagrees with scene::hit on %d rays" % mism
        return hits, tests.value

    def bsdf(self, material: int, queries: np.ndarray):
        queries = np.ascontiguousarray(queries, dtype=abi.BSDF_QUERY_DTYPE)
        out = np.zeros(len(queries), dtype=abi.BSDF_RESULT_DTYPE)
        self.lib.ref_bsdf_query(self.handle, material, _p(queries, abi.BsdfQuery), len(queries),
                                 _p(out, abi.BsdfResult))
        return out

    def bsdf_flags(self, material: int) -> int:
        return self.lib.ref_bsdf_flags(self.handle, material)

    def sky(self, dirs: np.ndarray):
        dirs = np.ascontiguousarray(dirs, dtype=np.float32)
        out = np.zeros((len(dirs), 3), dtype=np.float32)
        self.lib.ref_sky_eval(self.handle, _p(dirs), len(dirs), _p(out))
        return out

    def emitter_sample(self, points, u2):
        points = np.ascontiguousarray(points, dtype=np.float32)
        u2 = np.ascontiguousarray(u2, dtype=np.float32)
        out = np.zeros((len(points), 16), dtype=np.float32)
        self.lib.ref_emitter_sample(self.handle, _p(points), _p(u2), len(points), _p(out))
        return out

    def emitter_pdf(self, points, dirs):
        points = np.ascontiguousarray(points, dtype=np.float32)
        dirs = np.ascontiguousarray(dirs, dtype=np.float32)
        out = np.zeros(len(points), dtype=np.float32)
        self.lib.ref_emitter_pdf(self.handle, _p(points), _p(dirs), len(points), _p(out))
        return out

    def camera_rays(self, width, height, pixel_sample):
        ps = np.ascontiguousarray(pixel_sample, dtype=np.uint32)
        rays = np.zeros(len(ps), dtype=abi.RAY_DTYPE)
        self.lib.ref_camera_rays(self.handle, width, height, _p(ps, C.c_uint32), len(ps), _p(rays, abi.Ray))
        return rays

    def render(self, params: abi.RenderParams, threads: int = 0, want_sq: bool = False):
        img = np.zeros((params.height, params.width, 3), dtype=np.float32)
        sq = np.zeros_like(img) if want_sq else None
        secs = self.lib.ref_render(self.handle, C.byref(params), threads, _p(img),
                                    _p(sq) if sq is not None else None)
        return img, sq, secs

    def render_window(self, params: abi.RenderParams, col_begin: int, col_end: int, threads: int = 0):
        """Mean and mean of squares over rows [row_begin, row_end) x columns [col_begin, col_end) of the
        full frame (the crop of a render, pixel for pixel); the image arrays are full-frame sized."""
        img = np.zeros((params.height, params.width, 3), dtype=np.float32)
        sq = np.zeros_like(img)
        secs = self.lib.ref_render_window(self.handle, C.byref(params), col_begin, col_end, threads, _p(img), _p(sq))
        return img, sq, secs

    def render_photon(self, params, pp, global_photons, global_scale, caustic_photons, caustic_scale, threads=0,
                      want_sq=True):
        """photon_integrator::radiance over the image with maps built from the given photon arrays"""
        g = np.ascontiguousarray(global_photons, dtype=abi.PHOTON_DTYPE)
        c = np.ascontiguousarray(caustic_photons, dtype=abi.PHOTON_DTYPE)
        img = np.zeros((params.height, params.width, 3), dtype=np.float32)
        sq = np.zeros_like(img) if want_sq else None
        secs = self.lib.ref_photon_render(self.handle, C.byref(params), threads, _p(g, abi.Photon) if len(g) else None,
                                           len(g), global_scale, _p(c, abi.Photon) if len(c) else None, len(c),
                                           caustic_scale, C.byref(pp), _p(img), _p(sq) if sq is not None else None)
        return img, sq, secs

    def trace_particles(self, kind, first, count, max_depth, rr_depth, max_per=64):
        photons = np.zeros(count * max_per, dtype=abi.PHOTON_DTYPE)
        counts = np.zeros(count, dtype=np.uint32)
        self.lib.ref_trace_particles(self.handle, kind, first, count, max_depth, rr_depth, max_per,
                                      _p(photons, abi.Photon), _p(counts, C.c_uint32))
        return photons.reshape(count, max_per), counts

    def photon_gather(self, kind, requested, max_depth, rr_depth):
        photons = np.zeros(requested, dtype=abi.PHOTON_DTYPE)
        shot = C.c_uint64(0)
        secs = C.c_double(0)
        n = self.lib.ref_photon_gather(self.handle, kind, requested, max_depth, rr_depth,
                                        _p(photons, abi.Photon), C.byref(shot), C.byref(secs))
        return photons[:n], shot.value, secs.value


class RefPhotonMap:
    def __init__(self, photons: np.ndarray, scale: float = 1.0):
        self.photons = np.ascontiguousarray(photons, dtype=abi.PHOTON_DTYPE)
        self.handle = ref_lib().ref_photon_map_create(_p(self.photons, abi.Photon), len(self.photons), scale)

    def tree(self):
        """(order, nodes) of the reference's build in lrt_photon_map_tree's layout"""
        n = len(self.photons)
        order = np.zeros(max(1, n), dtype=np.uint32)
        cap = max(1, n // 2 + 16)
        nodes = np.zeros((cap, 4), dtype=np.int32)
        nn = C.c_uint32(0)
        assert ref_lib().ref_photon_map_tree(self.handle, _p(order, C.c_uint32), _p(nodes, C.c_int32), cap,
                                             C.byref(nn)) == 0
        return order[:n], nodes[: nn.value]

    def knn(self, points, r2, k):
        points = np.ascontiguousarray(points, dtype=np.float32)
        n = len(points)
        idx = np.full((n, k), 0xFFFFFFFF, dtype=np.uint32)
        d2 = np.zeros((n, k), dtype=np.float32)
        cnt = np.zeros(n, dtype=np.uint32)
        ref_lib().ref_photon_map_knn(self.handle, _p(points), n, r2, k, _p(idx, C.c_uint32), _p(d2),
                                     _p(cnt, C.c_uint32))
        return idx, d2, cnt

    def irradiance(self, points, normals, radius, max_depth, k):
        points = np.ascontiguousarray(points, dtype=np.float32)
        normals = np.ascontiguousarray(normals, dtype=np.float32)
        out = np.zeros((len(points), 3), dtype=np.float32)
        ref_lib().ref_photon_map_irradiance(self.handle, _p(points), _p(normals), len(points), radius, max_depth,
                                            k, _p(out))
        return out

    def __del__(self):
        try:
            if self.handle:
                ref_lib().ref_photon_map_destroy(self.handle)
                self.handle = None
        except Exception:
            pass


def load_obj(path: str):
    """the reference's load_obj: (positions [n, 3], indices [m], corner_normals [m, 3]), or None when it
    returns no mesh. It runs in its own process (oracle/_ref/ref_obj_dump): the reference reads numbers
    with the iostream extractors, which crash in a Python process whose numpy brought in another C++
    runtime."""
    import subprocess
    import tempfile
    with tempfile.TemporaryDirectory() as tmp:
        out = os.path.join(tmp, "mesh.bin")
        rc = subprocess.run([OBJ_DUMP, path, out], capture_output=True).returncode
        if rc == 1:
            return None
        if rc != 0:
            raise RuntimeError("ref_obj_dump failed (%d)" % rc)
        raw = open(out, "rb").read()
    nv, ni = np.frombuffer(raw[:8], dtype="<u4")
    o = 8
    pos = np.frombuffer(raw[o:o + 12 * nv], dtype="<f4").reshape(nv, 3).copy()
    o += 12 * nv
    idx = np.frombuffer(raw[o:o + 4 * ni], dtype="<u4").copy()
    o += 4 * ni
    nrm = np.frombuffer(raw[o:o + 12 * ni], dtype="<f4").reshape(ni, 3).copy()
    return pos, idx, nrm


OBJ_DUMP = os.path.join(REF_DIR, "ref_obj_dump")
BUNNY_PATH = os.path.join(REF_DIR, "assets", "bunny.obj")


def sampler_values(pixel_sample, n_dims):
    ps = np.ascontiguousarray(pixel_sample, dtype=np.uint32)
    out = np.zeros((len(ps), n_dims), dtype=np.float32)
    ref_lib().ref_sampler_values(_p(ps, C.c_uint32), len(ps), n_dims, _p(out))
    return out


def rough_transmittance(eta, alpha, ggx_path=GGX_PATH):
    table = np.zeros(abi.TRANS_SAMPLES, dtype=np.float32)
    diffuse = C.c_float(0)
    n = ref_lib().ref_rough_transmittance(ggx_path.encode(), eta, alpha, _p(table), C.byref(diffuse))
    if n < 0:
        raise RuntimeError(ref_lib().ref_last_error().decode())
    assert n == abi.TRANS_SAMPLES
    return table, np.float32(diffuse.value)


def fresnel_diffuse_reflectance(eta):
    return np.float32(ref_lib().ref_fresnel_diffuse_reflectance(eta))


def hosek_state(sun_direction, turbidity, albedo):
    sd = np.asarray(sun_direction, dtype=np.float32)
    cfg = np.zeros(27, dtype=np.float64)
    rad = np.zeros(3, dtype=np.float64)
    ref_lib().ref_hosek_state(_p(sd), turbidity, albedo, _p(cfg, C.c_double), _p(rad, C.c_double))
    return cfg.reshape(3, 9), rad


def photon_tree_limited(positions, limit):
    """photon_map::build_range over positions with libstdc++'s introselect given `limit` partitions per
    node (-1: std::nth_element's own budget); (order, nodes) in lrt_photon_map_tree's layout"""
    pos = np.ascontiguousarray(positions, dtype=np.float32).reshape(-1, 3)
    n = len(pos)
    order = np.zeros(max(1, n), dtype=np.uint32)
    cap = max(1, n // 2 + 16)
    nodes = np.zeros((cap, 4), dtype=np.int32)
    nn = C.c_uint32(0)
    assert ref_lib().ref_photon_tree_limited(_p(pos), n, limit, _p(order, C.c_uint32), _p(nodes, C.c_int32), cap,
                                             C.byref(nn)) == 0
    return order[:n], nodes[: nn.value]


def to_bytes(rgb, flip=False):
    """The reference image writer's 8-bit RGB of a (height, width, 3) float image (image_write.cpp)."""
    rgb = np.ascontiguousarray(rgb, dtype=np.float32)
    h, w = rgb.shape[0], rgb.shape[1]
    out = np.empty((h, w, 3), dtype=np.uint8)
    ref_lib().ref_to_bytes(_p(rgb), w, h, int(bool(flip)), _p(out, C.c_uint8))
    return out


def hardware_concurrency() -> int:
    return int(ref_lib().ref_hardware_concurrency())
