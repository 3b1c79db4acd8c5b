"""Material parameters of a scene as a flat vector, and the caller side of liblrt's path-replay adjoint.

A parameter is one scalar of one material: an albedo channel (diffuse_reflectance of diffuse, plastic
and rough plastic; the coat tint specular_reflectance of the smooth and rough coatings), a roughness
(alpha of the rough materials) or a conductor eta / k channel. On the seven-material differentiation
workload (the three wall albedos, the seven sphere materials and the coatings' nested plastic and rough
glass) that is 38 scalars: 5 roughnesses, 9 RGB albedos and the conductor's eta and k. The
channels of one field form a group, moved together, since channel c of a BSDF value moves only with
channel c of the field; a roughness is a group of its own. For each group the library receives the
scene's material list moved by +step and by -step (with the rough-transmittance tables re-sliced
where alpha moves) and differentiates the BSDF values on every path by those records
(lrt_diff_setup, lrt_render_adjoint).
"""
from __future__ import annotations

import copy
import ctypes as C

import numpy as np

import lrt
import lrt_abi as abi
import scenes

ALBEDO_TYPES = (abi.MAT_DIFFUSE, abi.MAT_PLASTIC, abi.MAT_ROUGH_PLASTIC)
ROUGH_TYPES = (abi.MAT_ROUGH_DIELECTRIC, abi.MAT_ROUGH_CONDUCTOR, abi.MAT_ROUGH_PLASTIC, abi.MAT_ROUGH_COATING)
COATING_TYPES = (abi.MAT_COATING, abi.MAT_ROUGH_COATING)


def scene_params(materials, only=None):
    """[(material, field, channel)] of every differentiable scalar, in material order: alpha first, then
    diffuse_reflectance (coatings: specular_reflectance), eta, k channels. `only`: restrict to these
    material indices."""
    out = []
    for i, m in enumerate(materials):
        if only is not None and i not in only:
            continue
        t = m["type"]
        if t in ROUGH_TYPES:
            out.append((i, "alpha", None))
        if t in ALBEDO_TYPES:
            out += [(i, "diffuse_reflectance", c) for c in range(3)]
        if t in COATING_TYPES:
            out += [(i, "specular_reflectance", c) for c in range(3)]
        if t == abi.MAT_ROUGH_CONDUCTOR:
            out += [(i, "eta", c) for c in range(3)] + [(i, "k", c) for c in range(3)]
    return out


def param_name(materials, p) -> str:
    i, field, c = p
    return "m%d.%s%s" % (i, field, "" if c is None else "[%d]" % c)


# the values lrt_abi.material_descs gives a field a material dict leaves out
FIELD_DEFAULTS = {"specular_reflectance": (1.0, 1.0, 1.0), "diffuse_reflectance": (0.5, 0.5, 0.5),
                  "eta": (0.0, 0.0, 0.0), "k": (0.0, 0.0, 0.0), "alpha": 0.0}


def get_value(materials, p) -> float:
    i, field, c = p
    v = materials[i].get(field, FIELD_DEFAULTS[field])
    return float(v if c is None else v[c])


def set_value(materials, p, value) -> None:
    i, field, c = p
    if c is None:
        materials[i][field] = float(value)
    else:
        v = [float(x) for x in materials[i].get(field, FIELD_DEFAULTS[field])]
        v[c] = float(value)
        materials[i][field] = tuple(v)


def param_groups(params):
    """(group of each parameter, channel of each parameter (-1: scalar), number of groups)"""
    keys, group, chan = {}, [], []
    for (m, field, c) in params:
        key = (m, field) if c is not None else (m, field, "scalar")
        if key not in keys:
            keys[key] = len(keys)
        group.append(keys[key])
        chan.append(-1 if c is None else int(c))
    return group, chan, len(keys)


def with_values(materials, params, values):
    """a copy of the material list with the parameters set (tables re-sliced)"""
    mats = copy.deepcopy(materials)
    for p, v in zip(params, values):
        set_value(mats, p, v)
    scenes.attach_tables(mats)
    return mats


class Differentiable:
    """The material parameters of the scene uploaded to `ctx`, with their adjoint.

    set_values() moves the scene's materials (lrt_scene_update_materials) and rebuilds the +/- step
    records (lrt_diff_setup); adjoint() returns d(sum_pixels <adjoint, image>)/d(params)."""

    def __init__(self, ctx: lrt.Context, scene, params=None, step: float = 1e-3):
        self.ctx = ctx
        self.scene = scene
        self.params = list(params) if params is not None else scene_params(scene.materials)
        if not self.params or len(self.params) > 64:
            raise ValueError("between 1 and 64 parameters are supported, got %d" % len(self.params))
        self.steps = np.full(len(self.params), step, dtype=np.float32)
        self.materials = copy.deepcopy(scene.materials)
        self._setup()

    def names(self):
        return [param_name(self.materials, p) for p in self.params]

    def values(self) -> np.ndarray:
        return np.array([get_value(self.materials, p) for p in self.params], dtype=np.float64)

    def set_values(self, values, setup: bool = True) -> None:
        """move the scene's materials to `values`; setup=False skips the +/- records (renders only)"""
        self.materials = with_values(self.materials, self.params, values)
        descs = abi.material_descs(self.materials)
        self.ctx._check(lrt.lib().lrt_scene_update_materials(self.ctx.handle, descs, len(self.materials)))
        if setup:
            self._setup()

    def _setup(self) -> None:
        nm = len(self.materials)
        group, chan, n_groups = param_groups(self.params)
        plus = (abi.MaterialDesc * (n_groups * nm))()
        minus = (abi.MaterialDesc * (n_groups * nm))()
        base = self.values()
        steps = np.zeros(n_groups, dtype=np.float32)
        for g in range(n_groups):
            members = [j for j in range(len(self.params)) if group[j] == g]
            steps[g] = self.steps[members[0]]
            for arr, sign in ((plus, 1.0), (minus, -1.0)):
                moved = copy.deepcopy(self.materials)
                for j in members:
                    set_value(moved, self.params[j], base[j] + sign * float(steps[g]))
                scenes.attach_tables(moved)
                abi.material_descs(moved, arr, g * nm)
        desc = (abi.DiffParam * len(self.params))(*[abi.DiffParam(g, c) for g, c in zip(group, chan)])
        self.ctx._check(lrt.lib().lrt_diff_setup(self.ctx.handle, n_groups, lrt.ptr(steps, C.c_float), plus, minus,
                                                 len(self.params), desc))

    def adjoint(self, jobs, max_depth: int, rr_depth: int, adjoint_image: np.ndarray) -> np.ndarray:
        arr = (abi.JobDesc * len(jobs))(*jobs)
        adj = np.ascontiguousarray(adjoint_image, dtype=np.float32).reshape(-1)
        floats = max(j.output_offset + 3 * j.width * j.height for j in jobs)
        assert adj.size >= floats
        grad = np.zeros(len(self.params), dtype=np.float64)
        self.ctx._check(lrt.lib().lrt_render_adjoint(self.ctx.handle, arr, len(jobs), max_depth, rr_depth,
                                                     lrt.ptr(adj, C.c_float), lrt.ptr(grad, C.c_double)))
        return grad

    def adjoint_dev(self, jobs, max_depth: int, rr_depth: int, adjoint_ptr: int, grad_ptr: int) -> None:
        arr = (abi.JobDesc * len(jobs))(*jobs)
        self.ctx._check(lrt.lib().lrt_render_adjoint_dev(self.ctx.handle, arr, len(jobs), max_depth, rr_depth,
                                                         C.c_void_p(adjoint_ptr), C.c_void_p(grad_ptr)))
