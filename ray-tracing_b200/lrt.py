"""Python host binding of liblrt (ctypes over the C ABI in include/lrt.h).

This is the host-side mirror of the reference's integrator/scene interfaces for tests and benchmarks:
``Context.upload(scene)`` replaces building LinRT::scene, ``Context.render(...)`` replaces the tile loop
of src/main.cpp around path_integrator::radiance, and the query methods expose the per-function parity
entry points (traversal, BSDFs, sky, sampler, emitters, photons).

The library is loaded from this directory (``liblrt.so``, built by ``make -C csrc``). There is no CPU
fallback: a missing library or a missing GPU raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

import lrt_abi as abi
from lrt_abi import ptr

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblrt.so")

# every entry point include/lrt.h declares (checked by the CPU test suite)
EXPORTS = [
    "lrt_create", "lrt_destroy", "lrt_last_error", "lrt_status_string", "lrt_rough_transmittance_slice",
    "lrt_fresnel_diffuse_reflectance", "lrt_hosek_state", "lrt_kdtree_build", "lrt_kdtree_build_device", "lrt_scene_upload", "lrt_scene_device_bytes",
    "lrt_scene_set_camera_frame", "lrt_tonemap", "lrt_tonemap_dev", "lrt_tonemap_table", "lrt_device_allocations",
    "lrt_mesh_tree_info", "lrt_trace", "lrt_trace_dev", "lrt_occluded", "lrt_bsdf_evaluate", "lrt_sky_eval",
    "lrt_sampler_values", "lrt_camera_rays", "lrt_emitter_query", "lrt_render", "lrt_render_dev",
    "lrt_render_dev_noalloc", "lrt_render_batch", "lrt_render_batch_dev",
    "lrt_render_plain", "lrt_render_plain_dev", "lrt_autotune", "lrt_load_obj", "lrt_rough_transmittance_eta_slice",
    "lrt_rough_transmittance_at_alpha", "lrt_scene_update_materials", "lrt_diff_setup", "lrt_render_adjoint",
    "lrt_render_adjoint_dev",
    "lrt_render_stats_get", "lrt_render_stats_reset", "lrt_set_option", "lrt_photon_trace",
    "lrt_photon_trace_particles", "lrt_photon_map_build", "lrt_photon_map_tree", "lrt_photon_knn", "lrt_photon_irradiance",
    "lrt_photon_irradiance_dev",
    "lrt_photon_preprocess", "lrt_render_photon", "lrt_render_photon_dev",
]


def tonemap_table() -> np.ndarray:
    """The 256 byte thresholds of the image writer's float-to-byte conversion (host only)."""
    out = np.zeros(256, dtype=np.float32)
    st = lib().lrt_tonemap_table(ptr(out, C.c_float))
    if st != 0:
        raise LrtError(st, "lrt_tonemap_table")
    return out


class LrtError(RuntimeError):
    def __init__(self, status, message):
        super().__init__("%s: %s" % (abi.STATUS_NAMES.get(status, status), message))
        self.status = status


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError("liblrt.so is not built (run `make -C %s`)" % os.path.join(HERE, "csrc"))
        L = C.CDLL(LIB_PATH)
        vp, u32, i32, f32, u64 = C.c_void_p, C.c_uint32, C.c_int32, C.c_float, C.c_uint64
        P = C.POINTER
        L.lrt_create.argtypes = [C.c_int, vp, P(vp)]
        L.lrt_destroy.argtypes = [vp]
        L.lrt_last_error.restype = C.c_char_p
        L.lrt_last_error.argtypes = [vp]
        L.lrt_status_string.restype = C.c_char_p
        L.lrt_status_string.argtypes = [C.c_int]
        L.lrt_rough_transmittance_slice.argtypes = [C.c_char_p, f32, f32, P(f32), P(f32)]
        L.lrt_fresnel_diffuse_reflectance.restype = f32
        L.lrt_fresnel_diffuse_reflectance.argtypes = [f32]
        L.lrt_hosek_state.argtypes = [P(f32), f32, f32, P(C.c_double), P(C.c_double)]
        L.lrt_kdtree_build.argtypes = [P(f32), P(f32), u32, P(u32), u32, P(u32), u32, P(u32), P(u32), P(u32)]
        L.lrt_kdtree_build_device.argtypes = [vp, u32, P(u32), P(f32), P(f32), P(u32), u64, P(u32), u64, P(u32),
                                              P(u32), P(u32), P(u64), P(u64)]
        L.lrt_scene_upload.argtypes = [vp, P(abi.SceneDesc)]
        L.lrt_scene_device_bytes.restype = u64
        L.lrt_scene_device_bytes.argtypes = [vp]
        L.lrt_scene_set_camera_frame.argtypes = [vp, P(f32), P(f32), P(f32), P(f32)]
        L.lrt_device_allocations.restype = u64
        L.lrt_device_allocations.argtypes = []
        L.lrt_tonemap.argtypes = [vp, P(f32), u32, u32, C.c_int, P(C.c_uint8)]
        L.lrt_tonemap_dev.argtypes = [vp, vp, u32, u32, C.c_int, vp]
        L.lrt_tonemap_table.argtypes = [P(f32)]
        L.lrt_mesh_tree_info.argtypes = [vp, u32, P(u32), P(u32), P(u32)]
        L.lrt_trace.argtypes = [vp, P(abi.Ray), u32, P(abi.Hit)]
        L.lrt_trace_dev.argtypes = [vp, vp, u32, vp]
        L.lrt_occluded.argtypes = [vp, P(abi.Ray), u32, i32, P(C.c_uint8)]
        L.lrt_bsdf_evaluate.argtypes = [vp, i32, P(abi.BsdfQuery), u32, P(abi.BsdfResult)]
        L.lrt_sky_eval.argtypes = [vp, P(f32), u32, P(f32)]
        L.lrt_sampler_values.argtypes = [vp, P(u32), u32, u32, P(f32)]
        L.lrt_camera_rays.argtypes = [vp, u32, u32, P(u32), u32, P(abi.Ray)]
        L.lrt_emitter_query.argtypes = [vp, P(f32), P(f32), P(f32), u32, P(f32), P(f32)]
        L.lrt_render.argtypes = [vp, P(abi.RenderParams), P(f32)]
        L.lrt_render_dev.argtypes = [vp, P(abi.RenderParams), vp]
        L.lrt_render_dev_noalloc.argtypes = [vp, P(abi.RenderParams), vp]
        L.lrt_render_batch.argtypes = [vp, P(abi.JobDesc), u32, i32, i32, P(f32)]
        L.lrt_render_batch_dev.argtypes = [vp, P(abi.JobDesc), u32, i32, i32, vp]
        L.lrt_render_plain.argtypes = [vp, P(abi.JobDesc), u32, i32, i32, P(f32)]
        L.lrt_render_plain_dev.argtypes = [vp, P(abi.JobDesc), u32, i32, i32, vp]
        L.lrt_autotune.argtypes = [vp, P(abi.JobDesc), u32, i32, i32, vp, C.c_char_p, P(abi.LaunchConfig)]
        L.lrt_load_obj.argtypes = [C.c_char_p, P(u32), P(u32), P(f32), u32, P(u32), P(f32), u32]
        L.lrt_rough_transmittance_eta_slice.argtypes = [C.c_char_p, f32, P(f32), P(f32), u32, P(u32), P(f32)]
        L.lrt_rough_transmittance_at_alpha.argtypes = [P(f32), P(f32), u32, P(f32), f32, P(f32), P(f32)]
        L.lrt_scene_update_materials.argtypes = [vp, P(abi.MaterialDesc), u32]
        L.lrt_diff_setup.argtypes = [vp, u32, P(f32), P(abi.MaterialDesc), P(abi.MaterialDesc), u32,
                                     P(abi.DiffParam)]
        L.lrt_render_adjoint.argtypes = [vp, P(abi.JobDesc), u32, i32, i32, P(f32), P(C.c_double)]
        L.lrt_render_adjoint_dev.argtypes = [vp, P(abi.JobDesc), u32, i32, i32, vp, vp]
        L.lrt_render_stats_get.argtypes = [vp, P(abi.RenderStats)]
        L.lrt_render_stats_reset.argtypes = [vp]
        L.lrt_set_option.argtypes = [vp, C.c_char_p, C.c_int64]
        L.lrt_photon_trace.argtypes = [vp, i32, u32, i32, i32, P(abi.Photon), P(u32), P(u64)]
        L.lrt_photon_trace_particles.argtypes = [vp, i32, u32, u32, i32, i32, u32, P(abi.Photon), P(u32)]
        L.lrt_photon_map_build.argtypes = [vp, i32, P(abi.Photon), u32, f32]
        L.lrt_photon_map_tree.argtypes = [vp, i32, P(u32), P(i32), u64, P(u32)]
        L.lrt_photon_knn.argtypes = [vp, i32, P(f32), u32, f32, u32, P(u32), P(f32), P(u32)]
        L.lrt_photon_irradiance.argtypes = [vp, i32, P(f32), P(f32), u32, f32, i32, u32, P(f32)]
        L.lrt_photon_irradiance_dev.argtypes = [vp, i32, vp, vp, u32, f32, i32, u32, vp]
        L.lrt_photon_preprocess.argtypes = [vp, u32, u32, i32, i32, f32, P(abi.PhotonRenderParams), P(u64)]
        L.lrt_render_photon.argtypes = [vp, P(abi.RenderParams), P(abi.PhotonRenderParams), P(f32)]
        L.lrt_render_photon_dev.argtypes = [vp, P(abi.RenderParams), P(abi.PhotonRenderParams), vp]
        _lib = L
    return _lib


def hosek_state(sun_direction, turbidity: float, albedo: float):
    """The Hosek-Wilkie RGB sky state env_emitter's constructor cooks: (config (3, 9), radiance (3,)) as
    float64, bit-identical to the reference."""
    sun = np.ascontiguousarray(sun_direction, dtype=np.float32).reshape(3)
    cfg = np.zeros((3, 9), dtype=np.float64)
    rad = np.zeros(3, dtype=np.float64)
    st = lib().lrt_hosek_state(ptr(sun, C.c_float), float(np.float32(turbidity)), float(np.float32(albedo)),
                               ptr(cfg, C.c_double), ptr(rad, C.c_double))
    if st != 0:
        raise LrtError(st, "Hosek state: turbidity must lie in [1, 10], albedo in [0, 1]")
    return cfg, rad


def rough_transmittance_slice(ggx_path: str, eta: float, alpha: float):
    table = np.zeros(abi.TRANS_SAMPLES, dtype=np.float32)
    diffuse = C.c_float(0.0)
    st = lib().lrt_rough_transmittance_slice(ggx_path.encode(), eta, alpha, ptr(table, C.c_float), C.byref(diffuse))
    if st != 0:
        raise LrtError(st, "rough transmittance slice failed")
    return table, np.float32(diffuse.value)


def load_obj(path: str):
    """(positions [n, 3], indices [m], corner_normals [m, 3]) of a Wavefront OBJ, read as the reference's
    load_obj reads it (centred, longest side 1)"""
    nv, ni = C.c_uint32(0), C.c_uint32(0)
    st = lib().lrt_load_obj(path.encode(), C.byref(nv), C.byref(ni), None, 0, None, None, 0)
    if st != 0:
        raise LrtError(st, "cannot load %s" % path)
    pos = np.zeros((nv.value, 3), dtype=np.float32)
    idx = np.zeros(ni.value, dtype=np.uint32)
    nrm = np.zeros((ni.value, 3), dtype=np.float32)
    st = lib().lrt_load_obj(path.encode(), C.byref(nv), C.byref(ni), ptr(pos, C.c_float), nv.value, ptr(idx, C.c_uint32),
                            ptr(nrm, C.c_float), ni.value)
    if st != 0:
        raise LrtError(st, "cannot load %s" % path)
    return pos, idx, nrm


def rough_transmittance_eta_slice(ggx_path: str, eta: float):
    """(sliced_table [n_alpha, TRANS_SAMPLES], sliced_diffuse [n_alpha], alpha_range [2]) of ggx.dat at eta"""
    cap = 4096
    table = np.zeros(cap * abi.TRANS_SAMPLES, dtype=np.float32)
    diffuse = np.zeros(cap, dtype=np.float32)
    n = C.c_uint32(0)
    rng = np.zeros(2, dtype=np.float32)
    st = lib().lrt_rough_transmittance_eta_slice(ggx_path.encode(), eta, ptr(table, C.c_float), ptr(diffuse, C.c_float),
                                                 cap, C.byref(n), ptr(rng, C.c_float))
    if st != 0:
        raise LrtError(st, "rough transmittance eta slice failed")
    k = n.value
    return table[:k * abi.TRANS_SAMPLES].reshape(k, abi.TRANS_SAMPLES).copy(), diffuse[:k].copy(), rng


def rough_transmittance_at_alpha(sliced_table, sliced_diffuse, alpha_range, alpha: float):
    t = np.ascontiguousarray(sliced_table, dtype=np.float32)
    d = np.ascontiguousarray(sliced_diffuse, dtype=np.float32)
    r = np.ascontiguousarray(alpha_range, dtype=np.float32)
    table = np.zeros(abi.TRANS_SAMPLES, dtype=np.float32)
    diffuse = C.c_float(0.0)
    st = lib().lrt_rough_transmittance_at_alpha(ptr(t, C.c_float), ptr(d, C.c_float), len(d), ptr(r, C.c_float), alpha,
                                                ptr(table, C.c_float), C.byref(diffuse))
    if st != 0:
        raise LrtError(st, "rough transmittance at alpha %r failed" % alpha)
    return table, np.float32(diffuse.value)


def fresnel_diffuse_reflectance(eta: float) -> np.float32:
    return np.float32(lib().lrt_fresnel_diffuse_reflectance(eta))


def kdtree_build(bmin: np.ndarray, bmax: np.ndarray):
    """Host SAH kd-tree: (nodes (n,2) uint32, refs uint32, depth)."""
    bmin = np.ascontiguousarray(bmin, dtype=np.float32)
    bmax = np.ascontiguousarray(bmax, dtype=np.float32)
    n = len(bmin)
    nn, nr, depth = C.c_uint32(0), C.c_uint32(0), C.c_uint32(0)
    cap_nodes, cap_refs = max(16, 8 * n), max(16, 8 * n)
    for _ in range(4):
        nodes = np.zeros((cap_nodes, 2), dtype=np.uint32)
        refs = np.zeros(cap_refs, dtype=np.uint32)
        st = lib().lrt_kdtree_build(ptr(bmin, C.c_float), ptr(bmax, C.c_float), n, ptr(nodes, C.c_uint32), cap_nodes,
                                    ptr(refs, C.c_uint32), cap_refs, C.byref(nn), C.byref(nr), C.byref(depth))
        if st == 0:
            return nodes[: nn.value], refs[: nr.value], depth.value
        if st != -5:
            raise LrtError(st, "kd-tree build failed")
        cap_nodes, cap_refs = nn.value, nr.value
    raise LrtError(-5, "kd-tree build: output sizing failed")


class Context:
    """One liblrt context (one GPU, one CUDA stream)."""

    def __init__(self, device: int = 0, stream: int | None = None):
        self.handle = C.c_void_p()
        st = lib().lrt_create(device, C.c_void_p(stream) if stream else None, C.byref(self.handle))
        if st != 0:
            raise LrtError(st, "lrt_create(device=%d) failed" % device)
        self.scene = None
        self.holder = None

    def _check(self, st):
        if st != 0:
            raise LrtError(st, lib().lrt_last_error(self.handle).decode())

    def close(self):
        if self.handle:
            lib().lrt_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- scene ----
    def upload(self, scene):
        holder = abi.SceneHolder(scene)
        self._check(lib().lrt_scene_upload(self.handle, C.byref(holder.desc)))
        self.scene, self.holder = scene, holder
        return self

    def scene_bytes(self) -> int:
        return int(lib().lrt_scene_device_bytes(self.handle))

    def tonemap(self, rgb, flip=False):
        """8-bit RGB of a (height, width, 3) float image as the reference's image writer converts it."""
        rgb = np.ascontiguousarray(rgb, dtype=np.float32)
        h, w = rgb.shape[0], rgb.shape[1]
        out = np.empty((h, w, 3), dtype=np.uint8)
        self._check(lib().lrt_tonemap(self.handle, ptr(rgb, C.c_float), w, h, int(bool(flip)), ptr(out, C.c_uint8)))
        return out

    def set_camera_frame(self, origin, lower_left_corner, horizontal, vertical):
        """Render with a constructed camera's own frame vectors instead of the uploaded camera's."""
        v = [np.ascontiguousarray(x, dtype=np.float32).reshape(3) for x in
             (origin, lower_left_corner, horizontal, vertical)]
        self._check(lib().lrt_scene_set_camera_frame(self.handle, *[ptr(x, C.c_float) for x in v]))
        return self

    def kdtree_build_device(self, meshes):
        """GPU SAH kd-trees of several meshes at once; meshes = [(bmin, bmax), ...] with (n, 3) float32
        boxes. Returns [(nodes (n,2) uint32, refs uint32, depth)] as kdtree_build does per mesh."""
        counts = np.array([len(b) for b, _ in meshes], dtype=np.uint32)
        bmin = np.ascontiguousarray(np.concatenate([np.asarray(b, np.float32).reshape(-1, 3) for b, _ in meshes]))
        bmax = np.ascontiguousarray(np.concatenate([np.asarray(b, np.float32).reshape(-1, 3) for _, b in meshes]))
        m = len(meshes)
        nc, rc, dp = np.zeros(m, np.uint32), np.zeros(m, np.uint32), np.zeros(m, np.uint32)
        tn, tr = C.c_uint64(0), C.c_uint64(0)
        cap_n, cap_r = max(16, 8 * len(bmin)), max(16, 8 * len(bmin))
        for _ in range(2):
            nodes = np.empty((cap_n, 2), dtype=np.uint32)
            refs = np.empty(cap_r, dtype=np.uint32)
            st = lib().lrt_kdtree_build_device(self.handle, m, ptr(counts, C.c_uint32), ptr(bmin, C.c_float),
                                               ptr(bmax, C.c_float), ptr(nodes, C.c_uint32), cap_n,
                                               ptr(refs, C.c_uint32), cap_r, ptr(nc, C.c_uint32), ptr(rc, C.c_uint32),
                                               ptr(dp, C.c_uint32), C.byref(tn), C.byref(tr))
            if st == 0:
                out, on, orf = [], 0, 0
                for k in range(m):
                    out.append((nodes[on: on + nc[k]], refs[orf: orf + rc[k]], int(dp[k])))
                    on += int(nc[k])
                    orf += int(rc[k])
                return out
            if st != -5:
                self._check(st)
            cap_n, cap_r = tn.value, tr.value
        raise LrtError(-5, "kd-tree build: output sizing failed")

    def mesh_tree_info(self, obj: int):
        n, r, d = C.c_uint32(), C.c_uint32(), C.c_uint32()
        self._check(lib().lrt_mesh_tree_info(self.handle, obj, C.byref(n), C.byref(r), C.byref(d)))
        return n.value, r.value, d.value

    # ---- parity queries ----
    def trace(self, rays: np.ndarray) -> np.ndarray:
        rays = np.ascontiguousarray(rays, dtype=abi.RAY_DTYPE)
        hits = np.zeros(len(rays), dtype=abi.HIT_DTYPE)
        self._check(lib().lrt_trace(self.handle, ptr(rays, abi.Ray), len(rays), ptr(hits, abi.Hit)))
        return hits

    def occluded(self, rays: np.ndarray, light: int) -> np.ndarray:
        rays = np.ascontiguousarray(rays, dtype=abi.RAY_DTYPE)
        out = np.zeros(len(rays), dtype=np.uint8)
        self._check(lib().lrt_occluded(self.handle, ptr(rays, abi.Ray), len(rays), light, ptr(out, C.c_uint8)))
        return out

    def trace_dev(self, rays_ptr: int, n: int, hits_ptr: int):
        self._check(lib().lrt_trace_dev(self.handle, C.c_void_p(rays_ptr), n, C.c_void_p(hits_ptr)))

    def bsdf(self, material: int, queries: np.ndarray) -> np.ndarray:
        queries = np.ascontiguousarray(queries, dtype=abi.BSDF_QUERY_DTYPE)
        out = np.zeros(len(queries), dtype=abi.BSDF_RESULT_DTYPE)
        self._check(lib().lrt_bsdf_evaluate(self.handle, material, ptr(queries, abi.BsdfQuery), len(queries),
                                            ptr(out, abi.BsdfResult)))
        return out

    def sky(self, dirs: np.ndarray) -> np.ndarray:
        dirs = np.ascontiguousarray(dirs, dtype=np.float32)
        out = np.zeros((len(dirs), 3), dtype=np.float32)
        self._check(lib().lrt_sky_eval(self.handle, ptr(dirs, C.c_float), len(dirs), ptr(out, C.c_float)))
        return out

    def sampler_values(self, pixel_sample: np.ndarray, n_dims: int) -> np.ndarray:
        ps = np.ascontiguousarray(pixel_sample, dtype=np.uint32)
        out = np.zeros((len(ps), n_dims), dtype=np.float32)
        self._check(lib().lrt_sampler_values(self.handle, ptr(ps, C.c_uint32), len(ps), n_dims, ptr(out, C.c_float)))
        return out

    def camera_rays(self, width: int, height: int, pixel_sample: np.ndarray) -> np.ndarray:
        ps = np.ascontiguousarray(pixel_sample, dtype=np.uint32)
        rays = np.zeros(len(ps), dtype=abi.RAY_DTYPE)
        self._check(lib().lrt_camera_rays(self.handle, width, height, ptr(ps, C.c_uint32), len(ps), ptr(rays, abi.Ray)))
        return rays

    def emitter_query(self, points, u2, dirs):
        points = np.ascontiguousarray(points, dtype=np.float32)
        u2 = np.ascontiguousarray(u2, dtype=np.float32)
        dirs = np.ascontiguousarray(dirs, dtype=np.float32)
        out = np.zeros((len(points), 16), dtype=np.float32)
        pdf = np.zeros(len(points), dtype=np.float32)
        self._check(lib().lrt_emitter_query(self.handle, ptr(points, C.c_float), ptr(u2, C.c_float), ptr(dirs, C.c_float),
                                            len(points), ptr(out, C.c_float), ptr(pdf, C.c_float)))
        return out, pdf

    # ---- rendering ----
    def render(self, params: abi.RenderParams, out: np.ndarray | None = None) -> np.ndarray:
        if out is None:
            out = np.zeros((params.height, params.width, 3), dtype=np.float32)
        assert out.dtype == np.float32 and out.flags["C_CONTIGUOUS"] and out.size == params.width * params.height * 3
        self._check(lib().lrt_render(self.handle, C.byref(params), ptr(out, C.c_float)))
        return out

    def render_dev(self, params: abi.RenderParams, rgb_ptr: int):
        self._check(lib().lrt_render_dev(self.handle, C.byref(params), C.c_void_p(rgb_ptr)))

    def render_batch(self, jobs, max_depth: int, rr_depth: int, out: np.ndarray | None = None) -> np.ndarray:
        """Renders every job (abi.JobDesc) in shared waves; returns the flat output buffer."""
        arr = (abi.JobDesc * len(jobs))(*jobs)
        floats = max((j.output_offset + 3 * j.width * j.height for j in jobs), default=0)
        if out is None:
            out = np.zeros(max(1, floats), dtype=np.float32)
        assert out.dtype == np.float32 and out.flags["C_CONTIGUOUS"] and out.size >= floats
        self._check(lib().lrt_render_batch(self.handle, arr, len(jobs), max_depth, rr_depth, ptr(out, C.c_float)))
        return out

    def render_batch_dev(self, jobs, max_depth: int, rr_depth: int, rgb_ptr: int):
        arr = (abi.JobDesc * len(jobs))(*jobs)
        self._check(lib().lrt_render_batch_dev(self.handle, arr, len(jobs), max_depth, rr_depth, C.c_void_p(rgb_ptr)))

    def autotune(self, jobs, max_depth: int, rr_depth: int, rgb_ptr: int, cache_path: str | None = None) -> dict:
        """lrt_autotune: times the batch's launch shapes, leaves the fastest on the context and returns it."""
        arr = (abi.JobDesc * len(jobs))(*jobs)
        cfg = abi.LaunchConfig()
        self._check(lib().lrt_autotune(self.handle, arr, len(jobs), max_depth, rr_depth, C.c_void_p(rgb_ptr),
                                       cache_path.encode() if cache_path else None, C.byref(cfg)))
        return {"wave_capacity": cfg.wave_capacity, "pixel_tile": cfg.pixel_tile, "blocks_per_sm": cfg.blocks_per_sm,
                "from_cache": bool(cfg.from_cache), "seconds": cfg.seconds, "trials": cfg.trials}

    def render_plain(self, jobs, max_depth: int, rr_depth: int, out: np.ndarray | None = None) -> np.ndarray:
        """The plain one-launch-per-job path tracer over the same jobs and output layout."""
        arr = (abi.JobDesc * len(jobs))(*jobs)
        floats = max((j.output_offset + 3 * j.width * j.height for j in jobs), default=0)
        if out is None:
            out = np.zeros(max(1, floats), dtype=np.float32)
        assert out.dtype == np.float32 and out.flags["C_CONTIGUOUS"] and out.size >= floats
        self._check(lib().lrt_render_plain(self.handle, arr, len(jobs), max_depth, rr_depth, ptr(out, C.c_float)))
        return out

    def render_plain_dev(self, jobs, max_depth: int, rr_depth: int, rgb_ptr: int):
        arr = (abi.JobDesc * len(jobs))(*jobs)
        self._check(lib().lrt_render_plain_dev(self.handle, arr, len(jobs), max_depth, rr_depth, C.c_void_p(rgb_ptr)))

    def set_option(self, name: str, value: int):
        self._check(lib().lrt_set_option(self.handle, name.encode(), int(value)))

    def stats(self) -> dict:
        s = abi.RenderStats()
        self._check(lib().lrt_render_stats_get(self.handle, C.byref(s)))
        return {
            "paths": s.paths, "extension_rays": s.extension_rays, "shadow_rays": s.shadow_rays,
            "nodes_visited": s.nodes_visited, "triangles_tested": s.triangles_tested,
            "shadow_nodes_visited": s.shadow_nodes_visited, "shadow_triangles_tested": s.shadow_triangles_tested,
            "shading_events": s.shading_events, "kernel_launches": s.kernel_launches,
            "stage_ms": {abi.STAGE_NAMES[i]: s.stage_ms[i] for i in range(6)},
            "stage_launches": {abi.STAGE_NAMES[i]: s.stage_launches[i] for i in range(6)},
            "rays_at_depth": [int(s.rays_at_depth[i]) for i in range(16)],
            "knn_queries": s.knn_queries, "knn_nodes_visited": s.knn_nodes_visited,
            "knn_photons_tested": s.knn_photons_tested, "knn_photons_found": s.knn_photons_found,
        }

    def reset_stats(self):
        self._check(lib().lrt_render_stats_reset(self.handle))

    # ---- photons ----
    def photon_trace(self, kind: int, requested: int, max_depth: int, rr_depth: int):
        photons = np.zeros(max(1, requested), dtype=abi.PHOTON_DTYPE)
        n = C.c_uint32(0)
        shot = C.c_uint64(0)
        self._check(lib().lrt_photon_trace(self.handle, kind, requested, max_depth, rr_depth, ptr(photons, abi.Photon),
                                           C.byref(n), C.byref(shot)))
        return photons[: n.value], shot.value

    def photon_trace_particles(self, kind, first, count, max_depth, rr_depth, max_per=64):
        photons = np.zeros(count * max_per, dtype=abi.PHOTON_DTYPE)
        counts = np.zeros(count, dtype=np.uint32)
        self._check(lib().lrt_photon_trace_particles(self.handle, kind, first, count, max_depth, rr_depth, max_per,
                                                     ptr(photons, abi.Photon), ptr(counts, C.c_uint32)))
        return photons.reshape(count, max_per), counts

    def photon_map_build(self, map_id: int, photons: np.ndarray, scale: float):
        photons = np.ascontiguousarray(photons, dtype=abi.PHOTON_DTYPE)
        self._check(lib().lrt_photon_map_build(self.handle, map_id, ptr(photons, abi.Photon), len(photons), scale))

    def photon_map_tree(self, map_id: int, n_photons: int):
        """(order, nodes): the built map's photon order (indices into the build's array) and its nodes,
        (n_nodes, 4) int32 in depth-first order (interior: left, right, axis, split bits; leaf: first, count, 3, 0)"""
        order = np.zeros(max(1, n_photons), dtype=np.uint32)
        cap = max(1, n_photons // 2 + 16)
        nodes = np.zeros((cap, 4), dtype=np.int32)
        nn = C.c_uint32(0)
        self._check(lib().lrt_photon_map_tree(self.handle, map_id, ptr(order, C.c_uint32), ptr(nodes, C.c_int32), cap,
                                              C.byref(nn)))
        return order[:n_photons], nodes[: nn.value]

    def photon_knn(self, map_id: int, points, r2: float, k: int):
        points = np.ascontiguousarray(points, dtype=np.float32)
        n = len(points)
        idx = np.full((n, k), 0xFFFFFFFF, dtype=np.uint32)
        d2 = np.zeros((n, k), dtype=np.float32)
        cnt = np.zeros(n, dtype=np.uint32)
        self._check(lib().lrt_photon_knn(self.handle, map_id, ptr(points, C.c_float), n, r2, k, ptr(idx, C.c_uint32),
                                         ptr(d2, C.c_float), ptr(cnt, C.c_uint32)))
        return idx, d2, cnt

    def photon_preprocess(self, global_photons: int, caustic_photons: int, max_depth: int = 128, rr_depth: int = 5,
                          radius_cap: float = float("inf"), lookup_size: int = 120):
        pp = abi.PhotonRenderParams.reference_defaults(lookup_size)
        pp.max_depth = max_depth
        shots = (C.c_uint64 * 2)()
        self._check(lib().lrt_photon_preprocess(self.handle, global_photons, caustic_photons, max_depth, rr_depth,
                                                radius_cap, C.byref(pp), shots))
        return pp, (shots[0], shots[1])

    def render_photon(self, params: abi.RenderParams, pp: abi.PhotonRenderParams, out: np.ndarray | None = None):
        if out is None:
            out = np.zeros((params.height, params.width, 3), dtype=np.float32)
        self._check(lib().lrt_render_photon(self.handle, C.byref(params), C.byref(pp), ptr(out, C.c_float)))
        return out

    def render_photon_dev(self, params: abi.RenderParams, pp: abi.PhotonRenderParams, rgb_ptr: int):
        self._check(lib().lrt_render_photon_dev(self.handle, C.byref(params), C.byref(pp), C.c_void_p(rgb_ptr)))

    def photon_irradiance_dev(self, map_id: int, points_ptr: int, normals_ptr: int, n: int, radius: float,
                              max_depth: int, k: int, rgb_ptr: int):
        self._check(lib().lrt_photon_irradiance_dev(self.handle, map_id, C.c_void_p(points_ptr),
                                                    C.c_void_p(normals_ptr), n, radius, max_depth, k,
                                                    C.c_void_p(rgb_ptr)))

    def photon_irradiance(self, map_id: int, points, normals, radius: float, max_depth: int, k: int):
        points = np.ascontiguousarray(points, dtype=np.float32)
        normals = np.ascontiguousarray(normals, dtype=np.float32)
        out = np.zeros((len(points), 3), dtype=np.float32)
        self._check(lib().lrt_photon_irradiance(self.handle, map_id, ptr(points, C.c_float), ptr(normals, C.c_float),
                                                len(points), radius, max_depth, k, ptr(out, C.c_float)))
        return out
