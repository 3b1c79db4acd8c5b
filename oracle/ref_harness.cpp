/*
 * ref_harness.cpp — TEST INFRASTRUCTURE, not product code.
 *
 * A thin extern "C" harness around the UNMODIFIED LinRT reference sources, compiled from where they
 * lie (see oracle/Makefile) into oracle/_ref/liblrt_ref.so. Only tests/, the smoke check and the CPU
 * baseline leg of bench.py load it: it is the checker and the CPU baseline, never the thing measured.
 *
 * What it exposes, each a direct call into reference code:
 *   ref_world_create      builds reference objects (bsdfs, triangle_mesh/rectangle/sphere, area_emitter,
 *                         env_emitter, camera, scene) from the same lrt_scene_desc the GPU library takes
 *   ref_trace             scene::hit, with the hit object/triangle recovered through the kd-tree leaf callback
 *                         exactly as triangle_mesh::hit (src/geometry/triangle_mesh.h:30-41) forms it
 *   ref_bsdf_query        bsdf::sample / eval / pdf (src/material/bsdf.h:78-88)
 *   ref_sky_eval          scene::eval_environment (src/core/scene.h:62-70)
 *   ref_render            the tile loop of src/main.cpp:103-147 around path_integrator::radiance, with
 *                         max_depth / rr_depth made run-time settings (generated header copy, oracle/Makefile)
 *   ref_trace_particles   photon_tracer::trace_particle per particle index (photon_gather.h:45-49)
 *   ref_photon_gather     photon_gather::run (thread-completion order, as the reference)
 *   ref_photon_map_*      photon_map::build / nearest / estimate_irradiance
 *   ref_rough_transmittance, ref_fresnel_diffuse_reflectance, ref_hosek_state: host-side tables
 *
 * `private` is defined to `public` while the reference headers are read, so that the harness can reach
 * the kd-tree of a mesh, the photon map's internals and the sky state; no reference code is changed.
 */
#include <algorithm>
#include <array>
#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <functional>
#include <limits>
#include <memory>
#include <queue>
#include <stdexcept>
#include <string>
#include <thread>
#include <unordered_map>
#include <utility>
#include <vector>
#include <unistd.h>

int lrt_ref_max_depth = 50;  // path_integrator.h:173, made settable in the generated copy
int lrt_ref_rr_depth = 5;    // path_integrator.h:19
// photon_integrator.h:57-64, made settable in the generated copy
int lrt_ref_pm_max_depth = 128;
int lrt_ref_pm_max_specular_depth = 4;
int lrt_ref_pm_rr_depth = 5;
int lrt_ref_pm_direct_samples = 16;
int lrt_ref_pm_glossy_samples = 32;
std::size_t lrt_ref_pm_global_photons = 250000;
std::size_t lrt_ref_pm_caustic_photons = 250000;
std::size_t lrt_ref_pm_lookup_size = 120;

#define private public
#include "core/scene.h"
#include "core/camera.h"
#include "core/sampler.h"
#include "core/hittable_list.h"
#include "geometry/triangle_mesh.h"
#include "geometry/rectangle.h"
#include "geometry/sphere.h"
#include "material/diffuse_bsdf.h"
#include "material/rough_conductor_bsdf.h"
#include "material/dielectric_bsdf.h"
#include "material/rough_dielectric_bsdf.h"
#include "material/plastic_bsdf.h"
#include "material/rough_plastic_bsdf.h"
#include "material/coating_bsdf.h"
#include "material/rough_coating_bsdf.h"
#include "emitter/area_emitter.h"
#include "emitter/env_emitter.h"
#include "accelerator/thread_pool.h"
#include "integrator/path/path_integrator.h"
#include "integrator/photonmapper/photon_map.h"
#include "integrator/photonmapper/photon_tracer.h"
#include "integrator/photonmapper/photon_gather.h"
#include "integrator/photonmapper/photon_integrator.h"
#undef private

#include "lrt.h"

using namespace LinRT;

namespace {

thread_local std::string g_error;

vec3 v3(const float* p) { return vec3(p[0], p[1], p[2]); }
void put3(float* dst, const vec3& v) { dst[0] = v.x; dst[1] = v.y; dst[2] = v.z; }

struct ref_world {
    std::vector<std::shared_ptr<bsdf>> materials;
    std::vector<std::shared_ptr<hittable>> objects;
    std::vector<int> kinds;
    std::vector<std::shared_ptr<emitter>> emitters;
    std::unique_ptr<scene> world;
    camera cam;
};

struct cwd_guard {
    char saved[4096];
    bool ok = false;
    explicit cwd_guard(const char* dir) {
        if(dir && *dir && getcwd(saved, sizeof(saved)) != nullptr) {
            ok = chdir(dir) == 0;
        }
    }
    ~cwd_guard() {
        if(ok) {
            if(chdir(saved) != 0) { /* nothing sensible to do */ }
        }
    }
};

std::shared_ptr<bsdf> make_material(const lrt_material_desc& m, const std::vector<std::shared_ptr<bsdf>>& made) {
    switch(m.type) {
    case LRT_DIFFUSE:
        return std::make_shared<diffuse_bsdf>(v3(m.diffuse_reflectance));
    case LRT_ROUGH_CONDUCTOR:
        return std::make_shared<rough_conductor_bsdf>(conductor_ior{v3(m.eta), v3(m.k)}, m.alpha,
                                                      v3(m.specular_reflectance));
    case LRT_DIELECTRIC:
        return std::make_shared<dielectric_bsdf>(m.int_ior, m.ext_ior, v3(m.specular_reflectance),
                                                 v3(m.specular_transmittance));
    case LRT_ROUGH_DIELECTRIC:
        return std::make_shared<rough_dielectric_bsdf>(m.int_ior, m.ext_ior, m.alpha, v3(m.specular_reflectance),
                                                       v3(m.specular_transmittance));
    case LRT_PLASTIC:
        return std::make_shared<plastic_bsdf>(m.int_ior, m.ext_ior, v3(m.specular_reflectance),
                                              v3(m.diffuse_reflectance), m.nonlinear != 0);
    case LRT_ROUGH_PLASTIC:
        return std::make_shared<rough_plastic_bsdf>(m.int_ior, m.ext_ior, m.alpha, v3(m.specular_reflectance),
                                                    v3(m.diffuse_reflectance), m.nonlinear != 0);
    case LRT_COATING:
        if(m.nested < 0 || static_cast<size_t>(m.nested) >= made.size()) {
            throw std::runtime_error("coating: nested material must come first");
        }
        return std::make_shared<coating_bsdf>(m.int_ior, m.ext_ior, made[static_cast<size_t>(m.nested)],
                                              v3(m.specular_reflectance), v3(m.sigma_a), m.thickness);
    case LRT_ROUGH_COATING:
        if(m.nested < 0 || static_cast<size_t>(m.nested) >= made.size()) {
            throw std::runtime_error("rough coating: nested material must come first");
        }
        return std::make_shared<rough_coating_bsdf>(m.int_ior, m.ext_ior, m.alpha, made[static_cast<size_t>(m.nested)],
                                                    v3(m.specular_reflectance), v3(m.sigma_a), m.thickness);
    default:
        throw std::runtime_error("unknown material type");
    }
}

// Closest hit over the object list in list order, with the hit object and triangle index recovered.
// The loop is hittable_list::hit (src/core/hittable_list.h:19-34); for meshes the per-triangle leaf
// callback is the lambda of triangle_mesh::hit (src/geometry/triangle_mesh.h:34-38) plus a record of the
// triangle index.
bool world_hit(const ref_world& w, const ray& r, float t_min, float t_max, hit_record& rec, int& object,
               int& prim, uint64_t* tests) {
    hit_record temp;
    bool hit_anything = false;
    float closest_so_far = t_max;
    object = -1;
    prim = -1;
    for(size_t i = 0; i < w.objects.size(); ++i) {
        int tri = -1;
        bool h = false;
        if(w.kinds[i] == LRT_OBJECT_MESH) {
            const auto* mesh = static_cast<const triangle_mesh*>(w.objects[i].get());
            auto closest = closest_so_far;
            mesh->kdtree.intersect(r, t_min, closest, [&](std::uint32_t triangle, float mint, float maxt) {
                if(tests) { ++*tests; }
                if(mesh->hit_triangle(triangle, r, mint, maxt, closest, temp)) {
                    h = true;
                    tri = static_cast<int>(triangle);
                }
            });
        } else {
            h = w.objects[i]->hit(r, t_min, closest_so_far, temp);
        }
        if(h) {
            hit_anything = true;
            closest_so_far = temp.t;
            rec = temp;
            object = static_cast<int>(i);
            prim = tri;
        }
    }
    return hit_anything;
}

bool same_bits(float a, float b) { return std::memcmp(&a, &b, sizeof(float)) == 0; }

void fill_photon(lrt_photon& out, const photon& p) {
    put3(out.position, p.position);
    put3(out.direction, p.direction);
    put3(out.normal, p.normal);
    put3(out.power, p.power);
    out.depth = p.depth;
}

photon to_photon(const lrt_photon& p) {
    photon out;
    out.position = v3(p.position);
    out.direction = v3(p.direction);
    out.normal = v3(p.normal);
    out.power = v3(p.power);
    out.depth = static_cast<std::uint16_t>(p.depth);
    return out;
}

struct ref_photon_map {
    photon_map map;
    std::vector<uint32_t> original;  // post-build position -> index in the caller's array
};

// The tile loop of src/main.cpp:103-147 (32x32 tiles on a thread_pool of `threads` workers) around
// `radiance(ray, sampler)`. rgb = per-pixel mean; rgb_sq (optional) = per-pixel mean of squares. Returns
// the wall-clock seconds of the tile loop (steady_clock, as main.cpp:103,148).
// Columns [col_begin, col_end) only when col_end > col_begin (a crop window of the full frame: the camera
// and pixel indices are those of the whole image).
template <typename Radiance>
double render_tiles(const ref_world& w, const lrt_render_params* p, uint32_t threads, float* rgb, float* rgb_sq,
                    Radiance&& radiance, uint32_t col_begin = 0, uint32_t col_end = 0) {
    const int width = static_cast<int>(p->width);
    const int height = static_cast<int>(p->height);
    const int x_begin = col_end > col_begin ? static_cast<int>(col_begin) : 0;
    const int x_end = col_end > col_begin ? static_cast<int>(std::min<uint32_t>(col_end, p->width)) : width;
    const int row_begin = p->row_end > p->row_begin ? static_cast<int>(p->row_begin) : 0;
    const int row_end = p->row_end > p->row_begin ? static_cast<int>(p->row_end) : height;
    const int spp = static_cast<int>(p->spp);
    constexpr int tile = 32;
    const auto start = std::chrono::steady_clock::now();
    {
        thread_pool pool(threads == 0 ? std::thread::hardware_concurrency() : threads);
        for(int y0 = row_begin; y0 < row_end; y0 += tile) {
            for(int x0 = x_begin; x0 < x_end; x0 += tile) {
                const int x1 = std::min(x0 + tile, x_end);
                const int y1 = std::min(y0 + tile, row_end);
                pool.submit([&, x0, y0, x1, y1] {
                    for(int y = y0; y < y1; ++y) {
                        for(int x = x0; x < x1; ++x) {
                            color sum(0.0f);
                            color sum_sq(0.0f);
                            for(int s = 0; s < spp; ++s) {
                                const auto pixel_index = static_cast<uint32_t>(y * width + x);
                                sampler smp;
                                smp.start(pixel_index, static_cast<uint32_t>(s) + p->sample_offset);
                                const auto offset = smp.next_2d();
                                const auto u = (static_cast<float>(x) + offset.x) / static_cast<float>(width - 1);
                                const auto v = (static_cast<float>(y) + offset.y) / static_cast<float>(height - 1);
                                auto r = w.world->sensor().get_ray(u, v);
                                const auto L = radiance(r, smp);
                                sum += L;
                                sum_sq += L * L;
                            }
                            const size_t o = 3 * (static_cast<size_t>(y) * width + x);
                            put3(rgb + o, sum / static_cast<float>(spp));
                            if(rgb_sq) { put3(rgb_sq + o, sum_sq / static_cast<float>(spp)); }
                        }
                    }
                });
            }
        }
        pool.wait();
    }
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count();
}

}  // namespace

// the image writer's float-to-byte conversion (io/image_write.cpp:10-20); it has external linkage in
// the reference but no declaration in image_write.h
namespace LinRT {
unsigned char to_byte(global_precision value);
}

extern "C" {

const char* ref_last_error() { return g_error.c_str(); }


void* ref_world_create(const lrt_scene_desc* desc, const char* data_root) {
    try {
        auto w = std::make_unique<ref_world>();
        {
            // rough_transmittance opens "third_party/data/ggx.dat" relative to the working directory
            // (src/material/func/rough_transmittance.h:18).
            cwd_guard guard(data_root);
            for(uint32_t i = 0; i < desc->n_materials; ++i) {
                w->materials.push_back(make_material(desc->materials[i], w->materials));
            }
        }
        hittable_list shapes;
        for(uint32_t i = 0; i < desc->n_objects; ++i) {
            const auto& o = desc->objects[i];
            std::shared_ptr<hittable> obj;
            if(o.kind == LRT_OBJECT_MESH) {
                std::vector<vec3> positions(o.n_vertices);
                for(uint32_t v = 0; v < o.n_vertices; ++v) { positions[v] = v3(o.positions + 3 * v); }
                std::vector<std::uint32_t> indices(o.indices, o.indices + o.n_indices);
                std::vector<vec3> normals(o.n_indices);
                for(uint32_t c = 0; c < o.n_indices; ++c) { normals[c] = v3(o.corner_normals + 3 * c); }
                obj = std::make_shared<triangle_mesh>(std::move(positions), std::move(indices), std::move(normals));
            } else if(o.kind == LRT_OBJECT_RECTANGLE) {
                obj = std::make_shared<rectangle>(v3(o.corner), v3(o.edge_u), v3(o.edge_v));
            } else if(o.kind == LRT_OBJECT_SPHERE) {
                obj = std::make_shared<sphere>(v3(o.center), o.radius);
            } else {
                throw std::runtime_error("unknown object kind");
            }
            if(o.material >= 0) {
                obj->set_material(w->materials.at(static_cast<size_t>(o.material)));
            }
            w->objects.push_back(obj);
            w->kinds.push_back(o.kind);
            shapes.add(obj);
        }
        for(uint32_t i = 0; i < desc->n_emitters; ++i) {
            const auto& e = desc->emitters[i];
            if(e.kind == LRT_EMITTER_AREA) {
                w->emitters.push_back(std::make_shared<area_emitter>(w->objects.at(static_cast<size_t>(e.object)),
                                                                     v3(e.radiance)));
            } else if(e.kind == LRT_EMITTER_ENV) {
                w->emitters.push_back(std::make_shared<env_emitter>(v3(e.sun_direction), e.turbidity, e.albedo,
                                                                    e.scale));
            } else {
                throw std::runtime_error("unknown emitter kind");
            }
        }
        w->cam.origin = v3(desc->camera.origin);
        w->cam.look_at = v3(desc->camera.look_at);
        w->cam.update(v3(desc->camera.up), desc->camera.fov_degrees, desc->camera.aspect_ratio);
        auto emitters_copy = w->emitters;
        w->world = std::make_unique<scene>(std::move(shapes), std::move(emitters_copy), w->cam);
        return w.release();
    } catch(const std::exception& ex) {
        g_error = ex.what();
        return nullptr;
    }
}

void ref_world_destroy(void* handle) { delete static_cast<ref_world*>(handle); }

// Closest hits. Returns the number of rays whose record differs from scene::hit's own (must be 0).
int64_t ref_trace(void* handle, const lrt_ray* rays, uint32_t n, lrt_hit* hits, uint64_t* triangle_tests) {
    const auto& w = *static_cast<ref_world*>(handle);
    int64_t mismatches = 0;
    for(uint32_t i = 0; i < n; ++i) {
        const ray r(v3(rays[i].origin), v3(rays[i].direction));
        hit_record rec;
        int object = -1;
        int prim = -1;
        const bool h = world_hit(w, r, rays[i].t_min, rays[i].t_max, rec, object, prim, triangle_tests);
        hit_record check;
        const bool h2 = w.world->hit(r, rays[i].t_min, rays[i].t_max, check);
        if(h != h2 || (h && (!same_bits(rec.t, check.t) || !same_bits(rec.normal.x, check.normal.x)
                             || !same_bits(rec.normal.y, check.normal.y) || !same_bits(rec.normal.z, check.normal.z)))) {
            ++mismatches;
        }
        auto& out = hits[i];
        std::memset(&out, 0, sizeof(out));
        out.object = -1;
        out.prim = -1;
        if(h) {
            out.t = rec.t;
            out.object = object;
            out.prim = prim;
            out.front_face = rec.front_face ? 1 : 0;
            put3(out.p, rec.p);
            put3(out.normal, rec.normal);
        }
    }
    return mismatches;
}

void ref_bsdf_query(void* handle, int32_t material, const lrt_bsdf_query* q, uint32_t n, lrt_bsdf_result* out) {
    const auto& w = *static_cast<ref_world*>(handle);
    const auto& m = w.materials.at(static_cast<size_t>(material));
    for(uint32_t i = 0; i < n; ++i) {
        bsdf_context ctx;
        ctx.mode = q[i].mode == LRT_MODE_IMPORTANCE ? bsdf_context::transport_mode::IMPORTANCE
                                                    : bsdf_context::transport_mode::RADIANCE;
        ctx.type_mask = q[i].type_mask;
        ctx.component = q[i].component;
        ctx.lobe_sample = q[i].lobe_sample;

        bsdf_sample_record s;
        s.wi = v3(q[i].wi);
        s.front_face = q[i].front_face != 0;
        const auto weight = m->sample(ctx, s, vec2(q[i].u[0], q[i].u[1]));
        auto& r = out[i];
        put3(r.sample_weight, weight);
        put3(r.sample_wo, s.wo);
        r.sample_pdf = s.pdf;
        r.sample_eta = s.eta;
        r.sampled_type = s.sampled_type;
        r.sampled_component = s.sampled_component;

        bsdf_sample_record e;
        e.wi = v3(q[i].wi);
        e.wo = v3(q[i].wo);
        e.front_face = q[i].front_face != 0;
        const auto meas = q[i].measure == LRT_MEASURE_DISCRETE ? measure::discrete : measure::solid_angle;
        put3(r.eval, m->eval(ctx, e, meas));
        r.pdf = m->pdf(ctx, e, meas);
    }
}

uint32_t ref_bsdf_flags(void* handle, int32_t material) {
    const auto& w = *static_cast<ref_world*>(handle);
    return w.materials.at(static_cast<size_t>(material))->flags();
}

void ref_sky_eval(void* handle, const float* directions, uint32_t n, float* rgb) {
    const auto& w = *static_cast<ref_world*>(handle);
    for(uint32_t i = 0; i < n; ++i) {
        put3(rgb + 3 * i, w.world->eval_environment(v3(directions + 3 * i)));
    }
}

// scene::sample_emitter_direction + pdf_emitter_direction (src/core/scene.h:73-108).
// out per query: ok, dir[3], point[3], normal[3], pdf, distance, radiance[3], emitter index, pdf of dir.
void ref_emitter_sample(void* handle, const float* points, const float* u2, uint32_t n, float* out) {
    const auto& w = *static_cast<ref_world*>(handle);
    for(uint32_t i = 0; i < n; ++i) {
        direct_sample ds;
        const bool ok = w.world->sample_emitter_direction(v3(points + 3 * i), vec2(u2[2 * i], u2[2 * i + 1]), ds);
        float* o = out + 16 * i;
        o[0] = ok ? 1.0f : 0.0f;
        put3(o + 1, ds.direction);
        put3(o + 4, ds.point);
        put3(o + 7, ds.normal);
        o[10] = ds.pdf;
        o[11] = ds.distance;
        put3(o + 12, ds.radiance);
        int idx = -1;
        for(size_t e = 0; e < w.emitters.size(); ++e) {
            if(w.emitters[e].get() == ds.emitter_ptr) { idx = static_cast<int>(e); }
        }
        o[15] = static_cast<float>(idx);
    }
}

void ref_emitter_pdf(void* handle, const float* points, const float* dirs, uint32_t n, float* pdf) {
    const auto& w = *static_cast<ref_world*>(handle);
    for(uint32_t i = 0; i < n; ++i) {
        pdf[i] = w.world->pdf_emitter_direction(v3(points + 3 * i), v3(dirs + 3 * i));
    }
}

void ref_sampler_values(const uint32_t* pixel_sample, uint32_t n, uint32_t n_dims, float* values) {
    for(uint32_t i = 0; i < n; ++i) {
        sampler s;
        s.start(pixel_sample[2 * i], pixel_sample[2 * i + 1]);
        for(uint32_t d = 0; d < n_dims; ++d) {
            values[static_cast<size_t>(i) * n_dims + d] = s.next_1d();
        }
    }
}

// Camera rays exactly as src/main.cpp:121-132 forms them.
void ref_camera_rays(void* handle, uint32_t width, uint32_t height, const uint32_t* pixel_sample, uint32_t n,
                     lrt_ray* rays) {
    const auto& w = *static_cast<ref_world*>(handle);
    for(uint32_t i = 0; i < n; ++i) {
        const uint32_t pixel = pixel_sample[2 * i];
        const uint32_t x = pixel % width;
        const uint32_t y = pixel / width;
        sampler s;
        s.start(pixel, pixel_sample[2 * i + 1]);
        const auto offset = s.next_2d();
        const auto u = (static_cast<float>(x) + offset.x) / static_cast<float>(width - 1);
        const auto v = (static_cast<float>(y) + offset.y) / static_cast<float>(height - 1);
        const auto r = w.world->sensor().get_ray(u, v);
        put3(rays[i].origin, r.origin);
        put3(rays[i].direction, r.direction);
        rays[i].t_min = 0.001f;
        rays[i].t_max = INFINITY;
    }
}

// Path-traced image (path_integrator::radiance with run-time max_depth / rr_depth).
double ref_render(void* handle, const lrt_render_params* p, uint32_t threads, float* rgb, float* rgb_sq) {
    const auto& w = *static_cast<ref_world*>(handle);
    lrt_ref_max_depth = p->max_depth;
    lrt_ref_rr_depth = p->rr_depth;
    const path_integrator integrator;
    return render_tiles(w, p, threads, rgb, rgb_sq,
                        [&](ray& r, sampler& smp) { return integrator.radiance(r, *w.world, smp); });
}

// The same over a window of columns (rows from p): the crop of a large frame, pixel for pixel.
double ref_render_window(void* handle, const lrt_render_params* p, uint32_t col_begin, uint32_t col_end,
                         uint32_t threads, float* rgb, float* rgb_sq) {
    const auto& w = *static_cast<ref_world*>(handle);
    lrt_ref_max_depth = p->max_depth;
    lrt_ref_rr_depth = p->rr_depth;
    const path_integrator integrator;
    return render_tiles(
        w, p, threads, rgb, rgb_sq, [&](ray& r, sampler& smp) { return integrator.radiance(r, *w.world, smp); },
        col_begin, col_end);
}

// Photon-mapper image: photon_integrator::radiance with the given photon maps (built by
// photon_map::build from the arrays) and radii in place of preprocess(), and run-time constants.
double ref_photon_render(void* handle, const lrt_render_params* p, uint32_t threads, const lrt_photon* global,
                         uint32_t n_global, float global_scale, const lrt_photon* caustic, uint32_t n_caustic,
                         float caustic_scale, const lrt_photon_render_params* pp, float* rgb, float* rgb_sq) {
    const auto& w = *static_cast<ref_world*>(handle);
    lrt_ref_pm_max_depth = pp->max_depth;
    lrt_ref_pm_max_specular_depth = pp->max_specular_depth;
    lrt_ref_pm_direct_samples = pp->direct_samples;
    lrt_ref_pm_glossy_samples = pp->glossy_samples;
    lrt_ref_pm_lookup_size = pp->lookup_size;
    photon_integrator integrator;
    std::vector<photon> g(n_global), c(n_caustic);
    for(uint32_t i = 0; i < n_global; ++i) { g[i] = to_photon(global[i]); }
    for(uint32_t i = 0; i < n_caustic; ++i) { c[i] = to_photon(caustic[i]); }
    if(n_global) { integrator.global_map.build(g, global_scale); }
    if(n_caustic) { integrator.caustic_map.build(c, caustic_scale); }
    integrator.global_radius = pp->global_radius;
    integrator.caustic_radius = pp->caustic_radius;
    return render_tiles(w, p, threads, rgb, rgb_sq,
                        [&](ray& r, sampler& smp) { return integrator.radiance(r, *w.world, smp); });
}

// photon_tracer::trace_particle for particles [first, first+count), sampler.start(0, index) as
// photon_gather.h:45-48. counts[i] = photons of particle first+i; at most max_per are copied per particle.
void ref_trace_particles(void* handle, int32_t kind, uint32_t first, uint32_t count, int32_t max_depth,
                         int32_t rr_depth, uint32_t max_per, lrt_photon* photons, uint32_t* counts) {
    const auto& w = *static_cast<ref_world*>(handle);
    const auto g = kind == LRT_GATHER_CAUSTIC ? photon_tracer::gather::caustic : photon_tracer::gather::surface;
    std::vector<photon> out;
    for(uint32_t i = 0; i < count; ++i) {
        out.clear();
        sampler s;
        s.start(0, first + i);
        photon_tracer::trace_particle(*w.world, g, s, max_depth, rr_depth, out);
        counts[i] = static_cast<uint32_t>(out.size());
        for(size_t j = 0; j < out.size() && j < max_per; ++j) {
            fill_photon(photons[static_cast<size_t>(i) * max_per + j], out[j]);
        }
    }
}

// photon_gather::run (src/integrator/photonmapper/photon_gather.h:15-61): hardware_concurrency workers,
// batches appended in completion order. Returns the photon count; *shot = particles counted.
uint32_t ref_photon_gather(void* handle, int32_t kind, uint32_t requested, int32_t max_depth, int32_t rr_depth,
                           lrt_photon* photons, uint64_t* shot, double* seconds) {
    const auto& w = *static_cast<ref_world*>(handle);
    const auto g = kind == LRT_GATHER_CAUSTIC ? photon_tracer::gather::caustic : photon_tracer::gather::surface;
    photon_gather gather;
    const auto start = std::chrono::steady_clock::now();
    const auto result = gather.run(*w.world, g, requested, max_depth, rr_depth);
    if(seconds) { *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count(); }
    for(size_t i = 0; i < result.photons.size(); ++i) { fill_photon(photons[i], result.photons[i]); }
    *shot = result.shot;
    return static_cast<uint32_t>(result.photons.size());
}

void* ref_photon_map_create(const lrt_photon* photons, uint32_t n, float scale) {
    auto pm = std::make_unique<ref_photon_map>();
    std::vector<photon> v(n);
    for(uint32_t i = 0; i < n; ++i) { v[i] = to_photon(photons[i]); }
    pm->map.build(v, scale);
    // recover the permutation nth_element applied: match each stored record to the caller's array
    std::unordered_map<std::string, uint32_t> key_to_index;
    key_to_index.reserve(n * 2);
    auto key_of = [](const photon& p) {
        std::string k(sizeof(float) * 12 + 2, '\0');
        std::memcpy(&k[0], &p.position, sizeof(float) * 3);
        std::memcpy(&k[12], &p.direction, sizeof(float) * 3);
        std::memcpy(&k[24], &p.normal, sizeof(float) * 3);
        std::memcpy(&k[36], &p.power, sizeof(float) * 3);
        std::memcpy(&k[48], &p.depth, 2);
        return k;
    };
    for(uint32_t i = 0; i < n; ++i) { key_to_index.emplace(key_of(v[i]), i); }
    pm->original.resize(n);
    for(uint32_t i = 0; i < n; ++i) {
        const auto it = key_to_index.find(key_of(pm->map.photons[i]));
        pm->original[i] = it == key_to_index.end() ? 0xffffffffu : it->second;
    }
    return pm.release();
}

void ref_photon_map_destroy(void* handle) { delete static_cast<ref_photon_map*>(handle); }

// the built tree (photon_map.h:74-81, 83-114): order[i] = caller index of the photon at position i;
// nodes as 4 words, interior {left, right, axis, split bits}, leaf {start, count, 3, 0}
int ref_photon_map_tree(void* handle, uint32_t* order, int32_t* nodes, uint64_t max_nodes, uint32_t* n_nodes) {
    const auto* pm = static_cast<ref_photon_map*>(handle);
    *n_nodes = static_cast<uint32_t>(pm->map.nodes.size());
    if(pm->map.nodes.size() > max_nodes) return -1;
    std::copy(pm->original.begin(), pm->original.end(), order);
    for(size_t i = 0; i < pm->map.nodes.size(); ++i) {
        const auto& nd = pm->map.nodes[i];
        int32_t* o = nodes + 4 * i;
        if(nd.leaf) {
            o[0] = nd.start;
            o[1] = nd.count;
            o[2] = 3;
            o[3] = 0;
        } else {
            o[0] = nd.left;
            o[1] = nd.right;
            o[2] = nd.axis;
            std::memcpy(&o[3], &nd.split, 4);
        }
    }
    return 0;
}

// photon_map::build_range's recursion (photon_map.h:83-114) over bare positions with libstdc++'s
// introselect given an explicit partition budget per node (std::nth_element's is 2*floor(log2(n))), so
// that a small budget drives its heap-selection path. Test infrastructure for the device build.
namespace {
struct limited_item {
    float p[3];
    uint32_t index;
};
int limited_build(std::vector<limited_item>& v, int start, int count, int limit, std::vector<std::array<int32_t, 4>>& out) {
    const int index = static_cast<int>(out.size());
    out.push_back({start, count, 3, 0});
    if(count <= 8) return index;
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for(int i = 0; i < count; ++i) {
        for(int a = 0; a < 3; ++a) {
            lo[a] = std::min(lo[a], v[start + i].p[a]);
            hi[a] = std::max(hi[a], v[start + i].p[a]);
        }
    }
    const float ext[3] = {hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]};
    int axis = 0;
    if(ext[1] > ext[axis]) axis = 1;
    if(ext[2] > ext[axis]) axis = 2;
    const int mid = start + count / 2;
    auto cmp = [axis](const limited_item& a, const limited_item& b) { return a.p[axis] < b.p[axis]; };
    const int budget = limit >= 0 ? limit : 2 * std::__lg(count);
    std::__introselect(v.begin() + start, v.begin() + mid, v.begin() + start + count, budget,
                       __gnu_cxx::__ops::__iter_comp_iter(cmp));
    const int left = limited_build(v, start, mid - start, limit, out);
    const int right = limited_build(v, mid, start + count - mid, limit, out);
    int32_t split_bits;
    std::memcpy(&split_bits, &v[mid].p[axis], 4);
    out[index] = {left, right, axis, split_bits};
    return index;
}
}  // namespace

int ref_photon_tree_limited(const float* positions, uint32_t n, int limit, uint32_t* order, int32_t* nodes,
                            uint64_t max_nodes, uint32_t* n_nodes) {
    std::vector<limited_item> v(n);
    for(uint32_t i = 0; i < n; ++i) v[i] = limited_item{{positions[3 * i], positions[3 * i + 1], positions[3 * i + 2]}, i};
    std::vector<std::array<int32_t, 4>> out;
    if(n > 0) limited_build(v, 0, static_cast<int>(n), limit, out);
    *n_nodes = static_cast<uint32_t>(out.size());
    if(out.size() > max_nodes) return -1;
    for(uint32_t i = 0; i < n; ++i) order[i] = v[i].index;
    for(size_t i = 0; i < out.size(); ++i) std::memcpy(nodes + 4 * i, out[i].data(), 16);
    return 0;
}

// photon_map::nearest (photon_map.h:117-130): results in max-heap pop order (descending (d2, index)).
void ref_photon_map_knn(void* handle, const float* points, uint32_t n, float r2, uint32_t k, uint32_t* idx,
                        float* d2, uint32_t* count) {
    const auto& pm = *static_cast<ref_photon_map*>(handle);
    for(uint32_t i = 0; i < n; ++i) {
        count[i] = 0;
        if(pm.map.photons.empty()) { continue; }
        const auto result = pm.map.nearest(v3(points + 3 * i), r2, k);
        count[i] = static_cast<uint32_t>(result.size());
        for(size_t j = 0; j < result.size(); ++j) {
            idx[static_cast<size_t>(i) * k + j] = pm.original[result[j].second];
            d2[static_cast<size_t>(i) * k + j] = result[j].first;
        }
    }
}

void ref_photon_map_irradiance(void* handle, const float* points, const float* normals, uint32_t n, float radius,
                               int32_t max_depth, uint32_t k, float* rgb) {
    const auto& pm = *static_cast<ref_photon_map*>(handle);
    for(uint32_t i = 0; i < n; ++i) {
        put3(rgb + 3 * i, pm.map.estimate_irradiance(v3(points + 3 * i), v3(normals + 3 * i), radius, max_depth, k));
    }
}

// rough_transmittance(eta, alpha) after set_eta/set_alpha: the 1-D table in cos^(1/4) theta and
// eval_diffuse(). Returns the table length, or -1 (message in ref_last_error) on the reference's throw.
int32_t ref_rough_transmittance(const char* ggx_path, float eta, float alpha, float* table, float* diffuse) {
    try {
        rough_transmittance rt(eta, alpha, ggx_path);
        for(size_t i = 0; i < rt.trans.size(); ++i) { table[i] = rt.trans[i]; }
        *diffuse = rt.eval_diffuse();
        return static_cast<int32_t>(rt.trans.size());
    } catch(const std::exception& ex) {
        g_error = ex.what();
        return -1;
    }
}

float ref_rough_transmittance_eval(const char* ggx_path, float eta, float alpha, float cos_theta) {
    rough_transmittance rt(eta, alpha, ggx_path);
    return rt.eval(cos_theta);
}

float ref_fresnel_diffuse_reflectance(float eta) { return fresnel_diffuse_reflectance(eta); }

// The cooked RGB Hosek state of an env_emitter built as env_emitter.h:13-30 does.
void ref_hosek_state(const float* sun_direction, float turbidity, float albedo, double* config27, double* radiance3) {
    env_emitter e(v3(sun_direction), turbidity, albedo, 1.0f);
    for(int c = 0; c < 3; ++c) {
        for(int i = 0; i < 9; ++i) { config27[c * 9 + i] = e.state->configs[c][i]; }
        radiance3[c] = e.state->radiances[c];
    }
}

uint32_t ref_hardware_concurrency() { return std::max(1u, std::thread::hardware_concurrency()); }

// The reference sah_kdtree built over the given primitive bounds, with its reachable nodes written out
// depth-first (left child next, right child after the left subtree) in the packed two-word form of
// lrt_kdtree_build, so that trees can be compared word for word. Returns 0, or -1 if arrays are small.
int32_t ref_kdtree_packed(const float* bmin, const float* bmax, uint32_t n, uint32_t* nodes_out, uint32_t max_nodes,
                          uint32_t* refs_out, uint32_t max_refs, uint32_t* n_nodes, uint32_t* n_refs) {
    std::vector<aabb> boxes(n);
    for(uint32_t i = 0; i < n; ++i) {
        boxes[i].minimum = v3(bmin + 3 * i);
        boxes[i].maximum = v3(bmax + 3 * i);
    }
    sah_kdtree tree;
    tree.build(boxes);
    std::vector<std::uint32_t> nodes;
    std::vector<std::uint32_t> refs;
    std::function<uint32_t(int)> pack = [&](int raw) -> uint32_t {
        const uint32_t index = static_cast<uint32_t>(nodes.size() / 2);
        nodes.push_back(0);
        nodes.push_back(0);
        const auto& nd = tree.nodes[static_cast<size_t>(raw)];
        if(nd.leaf) {
            nodes[2 * index] = static_cast<uint32_t>(refs.size());
            nodes[2 * index + 1] = (static_cast<uint32_t>(nd.count) << 2) | 3u;
            for(int i = 0; i < nd.count; ++i) refs.push_back(tree.ordered[static_cast<size_t>(nd.first + i)]);
            return index;
        }
        pack(nd.left);
        const uint32_t right = pack(nd.right);
        std::uint32_t bits;
        std::memcpy(&bits, &nd.split, 4);
        nodes[2 * index] = bits;
        nodes[2 * index + 1] = (right << 2) | static_cast<uint32_t>(nd.axis);
        return index;
    };
    if(!tree.nodes.empty()) pack(0);
    *n_nodes = static_cast<uint32_t>(nodes.size() / 2);
    *n_refs = static_cast<uint32_t>(refs.size());
    if(*n_nodes > max_nodes || *n_refs > max_refs) return -1;
    std::copy(nodes.begin(), nodes.end(), nodes_out);
    std::copy(refs.begin(), refs.end(), refs_out);
    return 0;
}

// ImageWriter::save's byte conversion and vertical flip (image_write.cpp:53-69) of width*height RGB
// pixels into out (3 bytes per pixel)
void ref_to_bytes(const float* rgb, int width, int height, int flip, unsigned char* out) {
    const size_t n = static_cast<size_t>(width) * static_cast<size_t>(height);
    for(size_t i = 0; i < 3 * n; ++i) out[i] = LinRT::to_byte(rgb[i]);
    if(flip) {
        for(int y = 0; y < height / 2; ++y) {
            unsigned char* a = out + 3ull * static_cast<size_t>(y) * width;
            unsigned char* b = out + 3ull * static_cast<size_t>(height - 1 - y) * width;
            std::swap_ranges(a, a + 3ull * width, b);
        }
    }
}

}  // extern "C"
