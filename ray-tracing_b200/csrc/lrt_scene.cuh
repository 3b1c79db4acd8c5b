// lrt_scene.cuh — device-side scene queries: kd-tree traversal with Moller-Trumbore triangle tests,
// analytic shapes, the linear object list, emitters (area lights and the Hosek sky) and the camera.
//
// Traversal restates sah_kdtree::intersect (src/accelerator/sah_kdtree.h:62-121) over 8-byte nodes:
// same front-to-back order, same [mint, maxt] intervals, same early exit, so the same leaves and
// triangles are tested in the same order and the closest hit (ties: the later triangle wins,
// triangle_mesh.h:77) is bit-identical.
#pragma once

#include "lrt_bsdf.cuh"
#include "lrt_math.cuh"
#include "lrt_types.h"

namespace lrt {

constexpr float kInf = __builtin_huge_valf();
constexpr int kStackSize = 48;  // sah_kdtree.h:80 (depth limit <= 48 keeps the stack within bounds)

// One deferred far child of the kd traversal. The reference's stack item also holds the child's
// entry distance (sah_kdtree.h:82-84), but that value always equals the current exit distance at
// the moment the item is popped: a push sets the near child's maxt to the split distance, which is
// the far child's mint, and every later push is popped before this one while nothing else changes
// maxt. So a pop sets mint = maxt, then restores maxt from the item, and an item fits in 8 bytes.
struct __align__(8) TravItem {
    uint32_t node;
    float maxt;
};

struct Ray {
    f3 o;
    f3 d;
};

// per-ray traversal counters (algorithmic-bytes accounting); compiled out unless requested
struct TraceCount {
    uint32_t nodes;
    uint32_t tris;
};

struct HitInfo {
    float t;
    int32_t object;     // -1 miss
    int32_t prim;       // triangle within the mesh, -1 analytic
    bool front_face;
    f3 p;
    f3 normal;          // hit_record::normal (faces the ray)
};

#ifdef __CUDACC__
__device__ __forceinline__ uint2 ld_node(const uint2* p) { return __ldg(p); }
__device__ __forceinline__ float4 ld_tri(const float4* p) { return __ldg(p); }
#endif

// Moller-Trumbore as triangle_mesh::hit_triangle (triangle_mesh.h:43-99), on a leaf record
// (p0 | degenerate, edge1, edge2). Returns true and updates closest/u/v when accepted.
__device__ __forceinline__ bool hit_tri_record(const float4* rec, const Ray& r, float t0, float t1, float& closest,
                                               float& out_u, float& out_v) {
    const float4 a = ld_tri(rec);
    const float4 b = ld_tri(rec + 1);
    const float4 c = ld_tri(rec + 2);
    if(a.w != 0.0f) return false;  // cross(edge1, edge2).length_squared() <= 0
    const f3 p0{a.x, a.y, a.z};
    const f3 edge1{b.x, b.y, b.z};
    const f3 edge2{c.x, c.y, c.z};
    const f3 pvec = cross(r.d, edge2);
    const float det = dot(edge1, pvec);
    if(fabsf(det) < 1e-8f) return false;
    const float inv_det = 1.0f / det;
    const f3 tvec = r.o - p0;
    const float u = dot(tvec, pvec) * inv_det;
    if(u < 0.0f || u > 1.0f) return false;
    const f3 qvec = cross(tvec, edge1);
    const float v = dot(r.d, qvec) * inv_det;
    if(v < 0.0f || u + v > 1.0f) return false;
    const float t = dot(edge2, qvec) * inv_det;
    if(t < t0 || t > t1) return false;
    closest = t;
    out_u = u;
    out_v = v;
    return true;
}

struct MeshHit {
    float t;
    float u, v;
    uint32_t ref;  // leaf reference of the last accepted triangle
};

// Conservative box cull: false only when the ray's [t_min, t_max] interval cannot reach the box
// [lo, hi] grown by 1e-3 (+ 1e-4 relative), so nothing inside it can be accepted. Directions with a zero
// component are handled per slab. t_entry: where the interval enters the grown box.
__device__ __forceinline__ bool box_reach(const float* lo_v, const float* hi_v, const Ray& r, float t_min, float t_max,
                                          float& t_entry) {
    float tn = t_min, tf = t_max;
#pragma unroll
    for(int a = 0; a < 3; ++a) {
        const float lo = lo_v[a], hi = hi_v[a];
        const float pad = 1e-3f + 1e-4f * (fabsf(lo) + fabsf(hi));
        const float oa = comp(r.o, a), da = comp(r.d, a);
        if(da == 0.0f) {
            if(oa < lo - pad || oa > hi + pad) return false;
            continue;
        }
        const float inv = 1.0f / da;
        float t0 = (lo - pad - oa) * inv;
        float t1 = (hi + pad - oa) * inv;
        if(t0 > t1) {
            const float t = t0;
            t0 = t1;
            t1 = t;
        }
        tn = fmaxf(tn, t0 - 1e-4f * fabsf(t0));
        tf = fminf(tf, t1 + 1e-4f * fabsf(t1));
    }
    t_entry = tn;
    return !(tn > tf);
}

// the object cull: a mesh none of whose triangles the ray's interval can reach is skipped
__device__ __forceinline__ bool ray_may_hit_box(const ObjRec& o, const Ray& r, float t_min, float t_max) {
    float t_entry;
    return box_reach(o.bmin, o.bmax, r, t_min, t_max, t_entry);
}

// Object-list walk: f(object) for every object the ray may reach, in list order, or -- when the scene
// has an object hierarchy -- in front-to-back node order, pruned by limit() (the current closest hit,
// read at every node). f returns true to stop (any-hit queries). The closest-hit callers resolve equal
// t by object index, the list's "later object wins", so both orders give the same hit.
template <typename Limit, typename F>
__device__ __forceinline__ void for_each_object(const DeviceScene& s, const Ray& r, float t_min, Limit limit, F f) {
    if(s.n_tlas == 0) {
        for(int32_t i = 0; i < s.n_objects; ++i) {
            if(f(i)) return;
        }
        return;
    }
    int32_t stack[kTlasStack];
    int top = 0;
    stack[top++] = 0;
    while(top > 0) {
        const int32_t node = stack[--top];
        const float4 a = __ldg(s.tlas + 2 * node), b = __ldg(s.tlas + 2 * node + 1);
        const float lo[3] = {a.x, a.y, a.z}, hi[3] = {b.x, b.y, b.z};
        float t_entry;
        if(!box_reach(lo, hi, r, t_min, limit(), t_entry)) continue;
        const int32_t right = __float_as_int(b.w);
        if(right < 0) {
            const int32_t first = __float_as_int(a.w);
            for(int32_t k = first; k < first - right; ++k) {
                if(f(__ldg(s.tlas_objs + k))) return;
            }
            continue;
        }
        const int32_t left = __float_as_int(a.w);
        // nearer child on top
        const float4 la = __ldg(s.tlas + 2 * left), ra = __ldg(s.tlas + 2 * right);
        const float4 lb = __ldg(s.tlas + 2 * left + 1), rb = __ldg(s.tlas + 2 * right + 1);
        const float llo[3] = {la.x, la.y, la.z}, lhi[3] = {lb.x, lb.y, lb.z};
        const float rlo[3] = {ra.x, ra.y, ra.z}, rhi[3] = {rb.x, rb.y, rb.z};
        float tl = kInf, tr = kInf;
        const bool hl = box_reach(llo, lhi, r, t_min, limit(), tl);
        const bool hr = box_reach(rlo, rhi, r, t_min, limit(), tr);
        if(top + 2 > kTlasStack) continue;  // unreachable: the build caps the depth below the stack size
        if(hl && hr) {
            stack[top++] = tl <= tr ? right : left;
            stack[top++] = tl <= tr ? left : right;
        } else if(hl) {
            stack[top++] = left;
        } else if(hr) {
            stack[top++] = right;
        }
    }
}

// Queue segment of a ray: 1 when it may reach the box of one of the scene's heavy meshes (the ones whose
// traversal dominates), 0 otherwise. Only a scheduling hint: every ray is traced the same way.
__device__ __forceinline__ int heavy_key(const DeviceScene& s, const Ray& r, float t_min, float t_max) {
    for(int32_t h = 0; h < s.n_heavy; ++h) {
        if(ray_may_hit_box(s.objects[s.heavy[h]], r, t_min, t_max)) return 1;
    }
    return 0;
}

// sah_kdtree::intersect over one mesh's tree with the triangle_mesh::hit leaf callback, written as
// a descend loop and a leaf loop (same node and triangle order as the reference's single loop, fewer
// divergent branches per warp). kAny: stop at the first accepted triangle (occlusion queries).
template <bool kCount, bool kAny>
__device__ __forceinline__ bool trace_mesh(const DeviceScene& s, const ObjRec& o, const Ray& r, float t_min, float t_max,
                                           MeshHit& h, TraceCount& cnt) {
    const uint2* nodes = s.nodes + o.node_base;
    const float4* tris = s.tris + 3ull * o.ref_base;
    float closest = t_max;
    bool hit_any = false;
    const float inv_x = 1.0f / r.d.x, inv_y = 1.0f / r.d.y, inv_z = 1.0f / r.d.z;
    TravItem stack[kStackSize];
    int top = 0;
    float mint = t_min;
    float maxt = closest;
    uint32_t node = 0;
    while(true) {
        uint2 n;
        // descend through interior nodes until a leaf (sah_kdtree.h:105-120)
        while(true) {
            if(closest < mint) return hit_any;
            n = ld_node(nodes + node);
            if(kCount) ++cnt.nodes;
            if((n.y & 3u) == kLeafTag) break;
            const uint32_t axis = n.y & 3u;
            const float split = __uint_as_float(n.x);
            const float o_a = comp(r.o, axis);
            const float d_a = comp(r.d, axis);
            const float t_plane = (split - o_a) * (axis == 0 ? inv_x : (axis == 1 ? inv_y : inv_z));
            const bool left_of_split = o_a < split || (o_a == split && d_a <= 0.0f);
            const uint32_t right = n.y >> 2;
            const uint32_t first_child = left_of_split ? node + 1 : right;
            const uint32_t second_child = left_of_split ? right : node + 1;
            if(t_plane > maxt || t_plane <= 0.0f) {
                node = first_child;
            } else if(t_plane < mint) {
                node = second_child;
            } else {
                if(top < kStackSize) stack[top++] = TravItem{second_child, maxt};
                node = first_child;
                maxt = t_plane;
            }
        }
        // leaf: the callback for each triangle with (mint, min(maxt, closest)) (sah_kdtree.h:86-93)
        const uint32_t count = n.y >> 2;
        const uint32_t first = n.x;
        float limit = smin(maxt, closest);
        for(uint32_t i = 0; i < count; ++i) {
            if(kCount) ++cnt.tris;
            float u, v;
            if(hit_tri_record(tris + 3ull * (first + i), r, mint, limit, closest, u, v)) {
                hit_any = true;
                h.t = closest;
                h.u = u;
                h.v = v;
                h.ref = first + i;
                if(kAny) return true;
            }
            limit = smin(maxt, closest);
        }
        if(top == 0) break;
        --top;
        node = stack[top].node;
        mint = maxt;
        maxt = stack[top].maxt;
    }
    return hit_any;
}

// rectangle::hit (src/geometry/rectangle.h:18-55)
__device__ __forceinline__ bool hit_rectangle(const ObjRec& o, const Ray& r, float t_min, float t_max, float& t_out,
                                              f3& p_out) {
    const f3 normal = load3(o.normal);
    const float denom = dot(normal, r.d);
    if(fabsf(denom) < 1e-8f) return false;
    const f3 corner = load3(o.corner);
    const float t = dot(corner - r.o, normal) / denom;
    if(t < t_min || t > t_max) return false;
    const f3 p = r.o + t * r.d;
    const f3 d = p - corner;
    const f3 eu = load3(o.edge_u);
    const f3 ev = load3(o.edge_v);
    const float uu = dot(eu, eu);
    const float vv = dot(ev, ev);
    const float uv = dot(eu, ev);
    const float du = dot(d, eu);
    const float dv = dot(d, ev);
    const float det = uu * vv - uv * uv;
    if(fabsf(det) < 1e-12f) return false;
    const float u = (vv * du - uv * dv) / det;
    const float v = (uu * dv - uv * du) / det;
    if(u < 0.0f || u > 1.0f || v < 0.0f || v > 1.0f) return false;
    t_out = t;
    p_out = p;
    return true;
}

// sphere::hit (src/geometry/sphere.h:21-49)
__device__ __forceinline__ bool hit_sphere(const ObjRec& o, const Ray& r, float t_min, float t_max, float& t_out) {
    const f3 center = load3(o.center);
    const f3 oc = r.o - center;
    const float a = length_squared(r.d);
    const float half_b = dot(oc, r.d);
    const float c = length_squared(oc) - o.radius * o.radius;
    const float discriminant = half_b * half_b - a * c;
    if(discriminant < 0.0f) return false;
    const float sqrtd = sqrtf(discriminant);
    float root = (-half_b - sqrtd) / a;
    if(root < t_min || root > t_max) {
        root = (-half_b + sqrtd) / a;
        if(root < t_min || root > t_max) return false;
    }
    t_out = root;
    return true;
}

// The full hit record of the object list's closest hit (hittable_list::hit, hittable_list.h:19-34,
// then the record each shape writes).
template <bool kCount>
__device__ __forceinline__ bool scene_hit(const DeviceScene& s, const Ray& r, float t_min, float t_max, HitInfo& out,
                                          TraceCount& cnt) {
    float closest_so_far = t_max;
    int32_t best = -1;
    MeshHit best_mesh{};
    // hittable_list::hit: an object replaces the best on a nearer hit, or an equal one later in the list
    for_each_object(s, r, t_min, [&]() { return closest_so_far; }, [&](int32_t i) {
        const ObjRec& o = s.objects[i];
        if(o.kind == LRT_OBJECT_MESH) {
            MeshHit mh;
            if(ray_may_hit_box(o, r, t_min, closest_so_far) &&
               trace_mesh<kCount, false>(s, o, r, t_min, closest_so_far, mh, cnt) &&
               (mh.t < closest_so_far || i > best)) {
                closest_so_far = mh.t;
                best = i;
                best_mesh = mh;
            }
        } else if(o.kind == LRT_OBJECT_RECTANGLE) {
            float t;
            f3 p;
            if(hit_rectangle(o, r, t_min, closest_so_far, t, p) && (t < closest_so_far || i > best)) {
                closest_so_far = t;
                best = i;
            }
        } else {
            float t;
            if(hit_sphere(o, r, t_min, closest_so_far, t) && (t < closest_so_far || i > best)) {
                closest_so_far = t;
                best = i;
            }
        }
        return false;
    });
    out.object = best;
    out.prim = -1;
    if(best < 0) return false;
    const ObjRec& o = s.objects[best];
    const float t = closest_so_far;
    out.t = t;
    out.p = r.o + t * r.d;
    if(o.kind == LRT_OBJECT_MESH) {
        // triangle_mesh.h:80-96: face normal from the geometric cross product, then the interpolated
        // shading normal flipped toward the ray.
        const uint32_t ref = o.ref_base + best_mesh.ref;
        const uint32_t tri = __ldg(s.ref_prim + ref);
        out.prim = static_cast<int32_t>(tri);
        const float4 b = ld_tri(s.tris + 3ull * ref + 1);
        const float4 c = ld_tri(s.tris + 3ull * ref + 2);
        const f3 geometric = cross(f3{b.x, b.y, b.z}, f3{c.x, c.y, c.z});
        const f3 outward = geometric / length(geometric);
        out.front_face = dot(r.d, outward) < 0.0f;
        out.normal = out.front_face ? outward : -outward;
        const float u = best_mesh.u;
        const float v = best_mesh.v;
        const float b0 = 1.0f - u - v;
        const float4* cn = s.normals + 3ull * (o.tri_base + tri);
        const float4 n0 = __ldg(cn), n1 = __ldg(cn + 1), n2 = __ldg(cn + 2);
        f3 shading = b0 * f3{n0.x, n0.y, n0.z} + u * f3{n1.x, n1.y, n1.z} + v * f3{n2.x, n2.y, n2.z};
        if(length_squared(shading) > 0.0f) {
            shading = shading / length(shading);
            if(dot(r.d, shading) > 0.0f) shading = -shading;
            out.normal = shading;
        }
    } else if(o.kind == LRT_OBJECT_RECTANGLE) {
        const f3 normal = load3(o.normal);
        out.front_face = dot(r.d, normal) < 0.0f;
        out.normal = out.front_face ? normal : -normal;
    } else {
        const f3 outward = (out.p - load3(o.center)) / o.radius;
        out.front_face = dot(r.d, outward) < 0.0f;
        out.normal = out.front_face ? outward : -outward;
    }
    return true;
}

// Shadow-ray query with the closest-hit semantics the path integrator needs
// (path_integrator.h:113-115): returns the emitter index of the closest object within [t_min, t_max],
// -1 for a non-emitting object, -2 for no hit.
template <bool kCount>
__device__ __forceinline__ int32_t scene_hit_emitter(const DeviceScene& s, const Ray& r, float t_min, float t_max,
                                                     TraceCount& cnt) {
    float closest_so_far = t_max;
    int32_t best = -1;
    for_each_object(s, r, t_min, [&]() { return closest_so_far; }, [&](int32_t i) {
        const ObjRec& o = s.objects[i];
        if(o.kind == LRT_OBJECT_MESH) {
            MeshHit mh;
            if(ray_may_hit_box(o, r, t_min, closest_so_far) &&
               trace_mesh<kCount, false>(s, o, r, t_min, closest_so_far, mh, cnt) &&
               (mh.t < closest_so_far || i > best)) {
                closest_so_far = mh.t;
                best = i;
            }
        } else if(o.kind == LRT_OBJECT_RECTANGLE) {
            float t;
            f3 p;
            if(hit_rectangle(o, r, t_min, closest_so_far, t, p) && (t < closest_so_far || i > best)) {
                closest_so_far = t;
                best = i;
            }
        } else {
            float t;
            if(hit_sphere(o, r, t_min, closest_so_far, t) && (t < closest_so_far || i > best)) {
                closest_so_far = t;
                best = i;
            }
        }
        return false;
    });
    if(best < 0) return -2;
    return s.objects[best].emitter;
}

// Whether an occlusion ray towards an area light can reach the light's own shape within [t_min, t_max]
// (the rule of scene_occluded); for a mesh light: whether any of its triangles is accepted.
static __device__ __noinline__ bool mesh_light_reachable(const DeviceScene& s, const ObjRec& o, const Ray& r, float t_min,
                                                  float t_max) {
    MeshHit mh;
    TraceCount cnt{0, 0};
    return ray_may_hit_box(o, r, t_min, t_max) && trace_mesh<false, true>(s, o, r, t_min, t_max, mh, cnt);
}

__device__ __forceinline__ bool light_shape_reachable(const DeviceScene& s, const ObjRec& o, const Ray& r, float t_min,
                                                      float t_max) {
    float t;
    f3 p;
    if(o.kind == LRT_OBJECT_RECTANGLE) return hit_rectangle(o, r, t_min, t_max, t, p);
    if(o.kind == LRT_OBJECT_SPHERE) return hit_sphere(o, r, t_min, t_max, t);
    return mesh_light_reachable(s, o, r, t_min, t_max);
}

// Shadow test of path_integrator.h:113-115: blocked = (closest hit exists) && (its emitter != light).
// When the light's own shape cannot be hit within [t_min, t_max] (always the case for the sky), the
// closest hit is never the light, so blocked == "any object has an accepted hit": objects are tested
// in list order and each traversal stops at its first accepted triangle. Otherwise the closest-hit
// query decides.
template <bool kCount>
__device__ __forceinline__ bool scene_occluded(const DeviceScene& s, const Ray& r, float t_min, float t_max,
                                               int32_t light, TraceCount& cnt) {
    const EmitRec& e = s.emitters[light];
    if(e.kind == LRT_EMITTER_AREA) {
        if(light_shape_reachable(s, s.objects[e.object], r, t_min, t_max)) {
            const int32_t hit = scene_hit_emitter<kCount>(s, r, t_min, t_max, cnt);
            return hit != -2 && hit != light;
        }
    }
    bool blocked = false;
    for_each_object(s, r, t_min, [&]() { return t_max; }, [&](int32_t i) {
        const ObjRec& o = s.objects[i];
        if(o.kind == LRT_OBJECT_MESH) {
            MeshHit mh;
            blocked = ray_may_hit_box(o, r, t_min, t_max) && trace_mesh<kCount, true>(s, o, r, t_min, t_max, mh, cnt);
        } else if(o.kind == LRT_OBJECT_RECTANGLE) {
            float t;
            f3 p;
            blocked = hit_rectangle(o, r, t_min, t_max, t, p);
        } else {
            float t;
            blocked = hit_sphere(o, r, t_min, t_max, t);
        }
        return blocked;
    });
    return blocked;
}

// ---- resumable traversal (persistent kernels) ----
//
// The object-list walk of scene_hit (and of the occlusion test) as a state machine that advances one
// unit of work per call: either scans objects up to the next mesh whose box the ray may reach (testing
// analytic shapes on the way), or runs one descend-to-leaf + leaf of the current mesh's traversal. The
// nodes, triangles and their order per ray are exactly those of trace_mesh / scene_hit; persistent
// kernels interleave rays so that a lane whose ray finishes takes a new one at once.
struct TravState {
    Ray r;
    float t_min;
    float t_max;          // occlusion: the shadow ray's tmax; closest hit: +inf
    int32_t obj;          // the mesh being traversed
    int32_t cursor;       // list walk: next object; hierarchy walk: next entry of the current leaf
    int32_t leaf_end;
    int32_t tl_top;       // hierarchy stack depth, -1 before the root is pushed
    bool in_mesh;
    bool any_mode;        // occlusion without a reachable light: stop at the first accepted hit
    uint32_t node;
    float mint, maxt;
    int32_t top;
    float closest;        // closest inside the current mesh
    float closest_so_far; // across the list
    int32_t best;
    MeshHit best_mesh;
    MeshHit cur;
    bool cur_hit;
    float inv_x, inv_y, inv_z;
};

__device__ __forceinline__ void trav_begin(TravState& st, const Ray& r, float t_min, float t_max, bool any_mode) {
    st.r = r;
    st.t_min = t_min;
    st.t_max = t_max;
    st.obj = -1;
    st.cursor = 0;
    st.leaf_end = 0;
    st.tl_top = -1;
    st.in_mesh = false;
    st.any_mode = any_mode;
    st.closest_so_far = t_max;
    st.best = -1;
    st.cur_hit = false;
    st.inv_x = 1.0f / r.d.x;
    st.inv_y = 1.0f / r.d.y;
    st.inv_z = 1.0f / r.d.z;
}

// The next object of the walk that the ray may reach (-1: none left): the list in order, or the
// hierarchy's leaves front to back, pruned by the closest hit so far.
__device__ __forceinline__ int32_t trav_next_object(const DeviceScene& s, TravState& st, int32_t* tl_stack) {
    if(s.n_tlas == 0) return st.cursor < s.n_objects ? st.cursor++ : -1;
    while(true) {
        if(st.cursor < st.leaf_end) return __ldg(s.tlas_objs + st.cursor++);
        if(st.tl_top < 0) {
            tl_stack[0] = 0;
            st.tl_top = 1;
        }
        if(st.tl_top == 0) return -1;
        const int32_t node = tl_stack[--st.tl_top];
        const float4 a = __ldg(s.tlas + 2 * node), b = __ldg(s.tlas + 2 * node + 1);
        const float lo[3] = {a.x, a.y, a.z}, hi[3] = {b.x, b.y, b.z};
        float t_entry;
        if(!box_reach(lo, hi, st.r, st.t_min, st.closest_so_far, t_entry)) continue;
        const int32_t right = __float_as_int(b.w);
        if(right < 0) {
            st.cursor = __float_as_int(a.w);
            st.leaf_end = st.cursor - right;
            continue;
        }
        const int32_t left = __float_as_int(a.w);
        const float4 la = __ldg(s.tlas + 2 * left), ra = __ldg(s.tlas + 2 * right);
        const float4 lb = __ldg(s.tlas + 2 * left + 1), rb = __ldg(s.tlas + 2 * right + 1);
        const float llo[3] = {la.x, la.y, la.z}, lhi[3] = {lb.x, lb.y, lb.z};
        const float rlo[3] = {ra.x, ra.y, ra.z}, rhi[3] = {rb.x, rb.y, rb.z};
        float tl = kInf, tr = kInf;
        const bool hl = box_reach(llo, lhi, st.r, st.t_min, st.closest_so_far, tl);
        const bool hr = box_reach(rlo, rhi, st.r, st.t_min, st.closest_so_far, tr);
        if(st.tl_top + 2 > kTlasStack) continue;  // unreachable: the build caps the depth below the stack size
        if(hl && hr) {
            tl_stack[st.tl_top++] = tl <= tr ? right : left;
            tl_stack[st.tl_top++] = tl <= tr ? left : right;
        } else if(hl) {
            tl_stack[st.tl_top++] = left;
        } else if(hr) {
            tl_stack[st.tl_top++] = right;
        }
    }
}

// One unit of work; returns true when the ray is finished (result in best / best_mesh / closest_so_far;
// in any_mode best >= 0 means "hit"). Equal t is resolved by object index, as the list's order does.
// kLeafInline: one-leaf meshes are tested during the object scan (faster for occlusion rays; for
// closest-hit rays the longer scan loop costs more than the saved steps).
template <bool kCount, bool kLeafInline = false>
__device__ __forceinline__ bool trav_step(const DeviceScene& s, TravState& st, TravItem* stack, int32_t* tl_stack,
                                          TraceCount& cnt) {
    if(!st.in_mesh) {
        while(true) {
            const int32_t i = trav_next_object(s, st, tl_stack);
            if(i < 0) return true;
            const ObjRec& o = s.objects[i];
            if(o.kind == LRT_OBJECT_MESH) {
                if(kLeafInline && o.n_nodes == 1 && ray_may_hit_box(o, st.r, st.t_min, st.closest_so_far)) {
                    // a tree that is one leaf (a quad, a few triangles): its traversal is that leaf's
                    // triangles in order over [t_min, closest] -- done here, without entering the mesh
                    const uint2 n = ld_node(s.nodes + o.node_base);
                    if(kCount) ++cnt.nodes;
                    const float4* tris = s.tris + 3ull * o.ref_base;
                    const uint32_t count = n.y >> 2;
                    float closest = st.closest_so_far;
                    bool hit = false;
                    MeshHit mh{};
                    for(uint32_t k = 0; k < count; ++k) {
                        if(kCount) ++cnt.tris;
                        float u, v;
                        if(hit_tri_record(tris + 3ull * (n.x + k), st.r, st.t_min, closest, closest, u, v)) {
                            hit = true;
                            mh = MeshHit{closest, u, v, n.x + k};
                            if(st.any_mode) {
                                st.best = i;
                                return true;
                            }
                        }
                    }
                    if(hit && (mh.t < st.closest_so_far || i > st.best)) {
                        st.closest_so_far = mh.t;
                        st.best = i;
                        st.best_mesh = mh;
                    }
                    continue;
                }
                if(ray_may_hit_box(o, st.r, st.t_min, st.closest_so_far)) {
                    st.obj = i;
                    st.in_mesh = true;
                    st.node = 0;
                    st.mint = st.t_min;
                    st.maxt = st.closest_so_far;
                    st.closest = st.closest_so_far;
                    st.top = 0;
                    st.cur_hit = false;
                    return false;
                }
            } else if(o.kind == LRT_OBJECT_RECTANGLE) {
                float t;
                f3 p;
                if(hit_rectangle(o, st.r, st.t_min, st.closest_so_far, t, p) && (t < st.closest_so_far || i > st.best)) {
                    st.closest_so_far = t;
                    st.best = i;
                    if(st.any_mode) return true;
                }
            } else {
                float t;
                if(hit_sphere(o, st.r, st.t_min, st.closest_so_far, t) && (t < st.closest_so_far || i > st.best)) {
                    st.closest_so_far = t;
                    st.best = i;
                    if(st.any_mode) return true;
                }
            }
        }
    }
    const ObjRec& o = s.objects[st.obj];
    const uint2* nodes = s.nodes + o.node_base;
    bool mesh_done = false;
    uint2 n;
    while(true) {  // descend (sah_kdtree.h:105-120)
        if(st.closest < st.mint) {
            mesh_done = true;
            break;
        }
        n = ld_node(nodes + st.node);
        if(kCount) ++cnt.nodes;
        if((n.y & 3u) == kLeafTag) break;
        const uint32_t axis = n.y & 3u;
        const float split = __uint_as_float(n.x);
        const float o_a = comp(st.r.o, axis);
        const float d_a = comp(st.r.d, axis);
        const float t_plane = (split - o_a) * (axis == 0 ? st.inv_x : (axis == 1 ? st.inv_y : st.inv_z));
        const bool left_of_split = o_a < split || (o_a == split && d_a <= 0.0f);
        const uint32_t right = n.y >> 2;
        const uint32_t first_child = left_of_split ? st.node + 1 : right;
        const uint32_t second_child = left_of_split ? right : st.node + 1;
        if(t_plane > st.maxt || t_plane <= 0.0f) {
            st.node = first_child;
        } else if(t_plane < st.mint) {
            st.node = second_child;
        } else {
            if(st.top < kStackSize) stack[st.top++] = TravItem{second_child, st.maxt};
            st.node = first_child;
            st.maxt = t_plane;
        }
    }
    if(!mesh_done) {  // leaf (sah_kdtree.h:86-93)
        const float4* tris = s.tris + 3ull * o.ref_base;
        const uint32_t count = n.y >> 2;
        const uint32_t first = n.x;
        float limit = smin(st.maxt, st.closest);
        for(uint32_t i = 0; i < count; ++i) {
            if(kCount) ++cnt.tris;
            float u, v;
            if(hit_tri_record(tris + 3ull * (first + i), st.r, st.mint, limit, st.closest, u, v)) {
                st.cur_hit = true;
                st.cur.t = st.closest;
                st.cur.u = u;
                st.cur.v = v;
                st.cur.ref = first + i;
                if(st.any_mode) {
                    st.best = st.obj;
                    return true;
                }
            }
            limit = smin(st.maxt, st.closest);
        }
        if(st.top == 0) {
            mesh_done = true;
        } else {
            --st.top;
            st.node = stack[st.top].node;
            st.mint = st.maxt;
            st.maxt = stack[st.top].maxt;
        }
    }
    if(mesh_done) {
        if(st.cur_hit && (st.cur.t < st.closest_so_far || st.obj > st.best)) {
            st.closest_so_far = st.cur.t;
            st.best = st.obj;
            st.best_mesh = st.cur;
        }
        st.in_mesh = false;
    }
    return false;
}

// The hit record of a finished closest-hit traversal (the second half of scene_hit).
__device__ __forceinline__ void hit_record_of(const DeviceScene& s, const Ray& r, int32_t best, float t,
                                              const MeshHit& best_mesh, HitInfo& out) {
    out.object = best;
    out.prim = -1;
    const ObjRec& o = s.objects[best];
    out.t = t;
    out.p = r.o + t * r.d;
    if(o.kind == LRT_OBJECT_MESH) {
        const uint32_t ref = o.ref_base + best_mesh.ref;
        const uint32_t tri = __ldg(s.ref_prim + ref);
        out.prim = static_cast<int32_t>(tri);
        const float4 b = ld_tri(s.tris + 3ull * ref + 1);
        const float4 c = ld_tri(s.tris + 3ull * ref + 2);
        const f3 geometric = cross(f3{b.x, b.y, b.z}, f3{c.x, c.y, c.z});
        const f3 outward = geometric / length(geometric);
        out.front_face = dot(r.d, outward) < 0.0f;
        out.normal = out.front_face ? outward : -outward;
        const float u = best_mesh.u;
        const float v = best_mesh.v;
        const float b0 = 1.0f - u - v;
        const float4* cn = s.normals + 3ull * (o.tri_base + tri);
        const float4 n0 = __ldg(cn), n1 = __ldg(cn + 1), n2 = __ldg(cn + 2);
        f3 shading = b0 * f3{n0.x, n0.y, n0.z} + u * f3{n1.x, n1.y, n1.z} + v * f3{n2.x, n2.y, n2.z};
        if(length_squared(shading) > 0.0f) {
            shading = shading / length(shading);
            if(dot(r.d, shading) > 0.0f) shading = -shading;
            out.normal = shading;
        }
    } else if(o.kind == LRT_OBJECT_RECTANGLE) {
        const f3 normal = load3(o.normal);
        out.front_face = dot(r.d, normal) < 0.0f;
        out.normal = out.front_face ? normal : -normal;
    } else {
        const f3 outward = (out.p - load3(o.center)) / o.radius;
        out.front_face = dot(r.d, outward) < 0.0f;
        out.normal = out.front_face ? outward : -outward;
    }
}

// ---- sky: env_emitter::eval (env_emitter.h:71-88) + ArHosekSkyModel_GetRadianceInternal (double) ----
// The terms of ArHosekSkyModel_GetRadianceInternal that do not depend on the channel, computed once per
// direction (the same double values the per-channel evaluation computes).
struct HosekAngles {
    double gamma, cos_gamma, cos_theta, zenith;
};

__device__ __forceinline__ HosekAngles hosek_angles(double theta, double gamma) {
    HosekAngles h;
    h.gamma = gamma;
    h.cos_gamma = cos(gamma);
    h.cos_theta = cos(theta);
    h.zenith = sqrt(h.cos_theta);
    return h;
}

__device__ __forceinline__ double hosek_radiance(const double* cfg, const HosekAngles& h) {
    const double expM = exp(cfg[4] * h.gamma);
    const double rayM = h.cos_gamma * h.cos_gamma;
    const double mieM = (1.0 + h.cos_gamma * h.cos_gamma) / pow((1.0 + cfg[8] * cfg[8] - 2.0 * cfg[8] * h.cos_gamma), 1.5);
    return (1.0 + cfg[0] * exp(cfg[1] / (h.cos_theta + 0.01))) *
           (cfg[2] + cfg[3] * expM + cfg[5] * rayM + cfg[6] * mieM + cfg[7] * h.zenith);
}

__device__ __forceinline__ f3 env_eval(const EmitRec& e, f3 direction) {
    const f3 dir = normalize(direction);
    if(dir.y <= 0.0f) return mk(1.0f);
    const float theta = acos_rn(sclamp(dir.y, 0.0f, 1.0f));
    const float gamma = acos_rn(sclamp(dot(dir, load3(e.sun)), -1.0f, 1.0f));
    const HosekAngles h = hosek_angles(theta, gamma);
    const f3 c{static_cast<float>(hosek_radiance(e.cfg[0], h) * e.rad[0]),
               static_cast<float>(hosek_radiance(e.cfg[1], h) * e.rad[1]),
               static_cast<float>(hosek_radiance(e.cfg[2], h) * e.rad[2])};
    return c * e.scale;
}

// scene::eval_environment (scene.h:62-70)
__device__ __forceinline__ f3 eval_environment(const DeviceScene& s, f3 direction) {
    f3 emitted = mk(0.0f);
    for(int32_t i = 0; i < s.n_emitters; ++i) {
        if(s.emitters[i].kind == LRT_EMITTER_ENV) emitted += env_eval(s.emitters[i], direction);
    }
    return emitted;
}

struct DirectSample {
    f3 direction;
    f3 point;
    f3 radiance;
    float pdf;
    float distance;
    int32_t emitter;
};

// triangle_mesh::sample_position (triangle_mesh.h:109-138): sample.x picks a triangle by area through
// the mesh's float area CDF (std::upper_bound), its remainder and sample.y place a point by the
// square-root barycentric warp; the normal is the unit geometric normal.
static __device__ __noinline__ void mesh_light_sample_position(const DeviceScene& s, const EmitRec& e, float sx, float sy,
                                                        f3& p, f3& n, float& pdf) {
    pdf = 0.0f;
    if(e.area <= 0.0f || e.n_tris == 0) return;
    const float* cdf = s.light_cdf + e.tri_first;
    const float target = smin(sx, 0.999999f) * e.area;
    uint32_t first = 0, count = e.n_tris;  // std::upper_bound: the first entry greater than target
    while(count > 0) {
        const uint32_t step = count / 2;
        if(!(target < cdf[first + step])) {
            first += step + 1;
            count -= step + 1;
        } else {
            count = step;
        }
    }
    const uint32_t tri = first < e.n_tris ? first : e.n_tris - 1;
    const float prev = tri == 0 ? 0.0f : cdf[tri - 1];
    const float span = cdf[tri] - prev;
    const float u0 = span > 0.0f ? (target - prev) / span : 0.0f;
    const float su = sqrtf(u0);
    const float b0 = 1.0f - su;
    const float b1 = sy * su;
    const float b2 = 1.0f - b0 - b1;
    const float4* c = s.light_tri + 3ull * (e.tri_first + tri);
    const f3 p0{c[0].x, c[0].y, c[0].z}, p1{c[1].x, c[1].y, c[1].z}, p2{c[2].x, c[2].y, c[2].z};
    p = b0 * p0 + b1 * p1 + b2 * p2;
    const f3 geometric = cross(p1 - p0, p2 - p0);
    n = geometric / length(geometric);
    pdf = 1.0f / e.area;
}

// hittable::sample_position of the emitter's shape (rectangle.h:65-69, sphere.h:60-67,
// triangle_mesh.h:109-138). kMeshLights = false compiles the mesh branch out, for kernels that only
// run on scenes whose lights are rectangles and spheres (the out-of-line mesh call costs registers
// in every caller that keeps it).
template <bool kMeshLights = true>
__device__ __forceinline__ void emitter_sample_position(const DeviceScene& s, const EmitRec& e, float sx, float sy,
                                                        f3& p, f3& n, float& pdf) {
    const ObjRec& o = s.objects[e.object];
    if(kMeshLights && o.kind == LRT_OBJECT_MESH) {
        mesh_light_sample_position(s, e, sx, sy, p, n, pdf);
    } else if(o.kind == LRT_OBJECT_RECTANGLE) {
        p = load3(o.corner) + sx * load3(o.edge_u) + sy * load3(o.edge_v);
        n = load3(o.normal);
        pdf = 1.0f / o.area;
    } else {
        const float z = 1.0f - 2.0f * sy;
        const float ring = sqrtf(smax(0.0f, 1.0f - z * z));
        const float phi = 2.0f * kPi * sx;
        float sin_phi, cos_phi;
        sincos_rn(phi, sin_phi, cos_phi);
        n = f3{ring * cos_phi, ring * sin_phi, z};
        p = load3(o.center) + o.radius * n;
        pdf = 1.0f / o.area;
    }
}

// area_emitter::sample (area_emitter.h:17-49)
template <bool kMeshLights = true>
__device__ __forceinline__ bool area_sample(const DeviceScene& s, const EmitRec& e, f3 shading_point, float sx,
                                            float sy, DirectSample& out) {
    if(e.area <= 0.0f) return false;
    f3 p, n;
    float pdf_area = 0.0f;
    emitter_sample_position<kMeshLights>(s, e, sx, sy, p, n, pdf_area);
    const f3 to_light = p - shading_point;
    const float dist2 = length_squared(to_light);
    if(dist2 < 1e-8f) return false;
    const float dist = sqrtf(dist2);
    const f3 direction = to_light / dist;
    const float cos_light = dot(n, -direction);
    if(cos_light <= 0.0f) return false;
    out.point = p;
    out.direction = direction;
    out.distance = dist;
    out.pdf = pdf_area * dist2 / cos_light;
    out.radiance = load3(e.radiance);
    return true;
}

// env_emitter::sample (env_emitter.h:33-53); kRadiance = false leaves out.radiance to the caller (the
// path tracer evaluates the sky only for shadow rays that turn out unoccluded)
template <bool kRadiance = true>
__device__ __forceinline__ bool env_sample(const EmitRec& e, float sx, float sy, DirectSample& out) {
    if(!e.sun_active) return false;
    const float cos_theta = (1.0f - sx) + sx * e.cos_cutoff;
    const float sin_theta = sqrtf(smax(0.0f, 1.0f - cos_theta * cos_theta));
    const float phi = 2.0f * kPi * sy;
    float sin_phi, cos_phi;
    sincos_rn(phi, sin_phi, cos_phi);
    const f3 local{cos_phi * sin_theta, sin_phi * sin_theta, cos_theta};
    const f3 a0 = load3(e.frame[0]), a1 = load3(e.frame[1]), a2 = load3(e.frame[2]);
    out.direction = a0 * local.x + a1 * local.y + a2 * local.z;
    out.pdf = e.cone_pdf;
    out.radiance = kRadiance ? env_eval(e, out.direction) : mk(0.0f);
    out.distance = kInf;
    return true;
}

// scene::sample_emitter_direction (scene.h:73-93): uniform 1/n light pick on sample.x
template <bool kMeshLights = true, bool kEnvRadiance = true>
__device__ __forceinline__ bool sample_emitter_direction(const DeviceScene& s, f3 shading_point, float sx, float sy,
                                                         DirectSample& out) {
    const int32_t count = s.n_emitters;
    if(count <= 0) return false;
    const float scaled = sx * static_cast<float>(count);
    int32_t index = static_cast<int32_t>(scaled);
    if(index >= count) index = count - 1;
    const float rx = scaled - static_cast<float>(index);
    const EmitRec& e = s.emitters[index];
    out.distance = kInf;
    out.pdf = 0.0f;
    const bool ok = e.kind == LRT_EMITTER_ENV ? env_sample<kEnvRadiance>(e, rx, sy, out)
                                              : area_sample<kMeshLights>(s, e, shading_point, rx, sy, out);
    if(!ok) return false;
    out.emitter = index;
    out.pdf *= 1.0f / static_cast<float>(count);
    return out.pdf > 0.0f;
}

// triangle_mesh::hit of a mesh light over [0.001, inf) (area_emitter.h:60): the closest triangle's
// t, front_face and hit-record normal (the shading normal turned toward the ray)
static __device__ __noinline__ bool mesh_light_hit(const DeviceScene& s, int32_t object, const Ray& r, float& t, f3& normal) {
    const ObjRec& o = s.objects[object];
    MeshHit mh;
    TraceCount cnt{0, 0};
    if(!ray_may_hit_box(o, r, 0.001f, kInf) || !trace_mesh<false, false>(s, o, r, 0.001f, kInf, mh, cnt)) return false;
    HitInfo h;
    hit_record_of(s, r, object, mh.t, mh, h);
    if(!h.front_face) return false;
    t = mh.t;
    normal = h.normal;
    return true;
}

// area_emitter::pdf (area_emitter.h:51-72): re-intersects the light shape
template <bool kMeshLights = true>
__device__ __forceinline__ float area_pdf(const DeviceScene& s, const EmitRec& e, f3 shading_point, f3 direction) {
    if(e.area <= 0.0f) return 0.0f;
    const f3 dir = normalize(direction);
    const Ray r{shading_point, dir};
    const ObjRec& o = s.objects[e.object];
    float t;
    f3 normal;
    if(o.kind == LRT_OBJECT_MESH) {
        if(!kMeshLights || !mesh_light_hit(s, e.object, r, t, normal)) return 0.0f;
    } else if(o.kind == LRT_OBJECT_RECTANGLE) {
        f3 p;
        if(!hit_rectangle(o, r, 0.001f, kInf, t, p)) return 0.0f;
        normal = load3(o.normal);
        if(!(dot(r.d, normal) < 0.0f)) return 0.0f;  // !rec.front_face
    } else {
        if(!hit_sphere(o, r, 0.001f, kInf, t)) return 0.0f;
        const f3 p = r.o + t * r.d;
        normal = (p - load3(o.center)) / o.radius;
        if(!(dot(r.d, normal) < 0.0f)) return 0.0f;
    }
    const float cos_light = dot(normal, -dir);
    if(cos_light <= 0.0f) return 0.0f;
    return t * t / (e.area * cos_light);
}

// env_emitter::pdf (env_emitter.h:55-69)
__device__ __forceinline__ float env_pdf(const EmitRec& e, f3 direction) {
    if(!e.sun_active) return 0.0f;
    const f3 dir = normalize(direction);
    if(dot(dir, load3(e.sun)) + 1e-5f < e.cos_cutoff) return 0.0f;
    return e.cone_pdf;
}

// scene::pdf_emitter_direction (scene.h:96-108)
template <bool kMeshLights = true>
__device__ __forceinline__ float pdf_emitter_direction(const DeviceScene& s, f3 shading_point, f3 direction) {
    const int32_t count = s.n_emitters;
    if(count <= 0) return 0.0f;
    const float selection = 1.0f / static_cast<float>(count);
    float sum = 0.0f;
    for(int32_t i = 0; i < count; ++i) {
        const EmitRec& e = s.emitters[i];
        const float p = e.kind == LRT_EMITTER_ENV ? env_pdf(e, direction) : area_pdf<kMeshLights>(s, e, shading_point, direction);
        sum += selection * p;
    }
    return sum;
}

// area_emitter::emitted (area_emitter.h:79-85)
__device__ __forceinline__ f3 area_emitted(const EmitRec& e, f3 normal, f3 outgoing) {
    if(dot(normal, outgoing) <= 0.0f) return mk(0.0f);
    return load3(e.radiance);
}

// camera::get_ray for a pinhole (camera.h:53-60)
__device__ __forceinline__ Ray camera_ray(const CamRec& c, float s, float t) {
    const f3 origin = load3(c.origin);
    const f3 target = load3(c.llc) + s * load3(c.horizontal) + t * load3(c.vertical) - origin;
    return Ray{origin, normalize(target)};
}

LRT_HD float power_heuristic(float pdf_strategy, float pdf_other) {
    const float a = pdf_strategy * pdf_strategy;
    const float b = pdf_other * pdf_other;
    const float sum = a + b;
    return sum > 0.0f ? a / sum : 0.0f;
}

}  // namespace lrt
