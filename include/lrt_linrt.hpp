// lrt_linrt.hpp — the reference-side drop-in of liblrt for LinRT (Lincacc/Ray-Tracing): integrators with
// the reference's preprocess/render shape that run its rendering hot path on a B200 through the C ABI of
// lrt.h, and the translation of a LinRT scene into an lrt_scene_desc.
//
// What it replaces (paths inside the reference project):
//   gpu_path_integrator     path_integrator (src/integrator/path/path_integrator.h:18-182) together with
//                           the tile loop of src/main.cpp:103-147 that calls it: render() fills the image
//   gpu_photon_integrator   photon_integrator (src/integrator/photonmapper/photon_integrator.h:15-296):
//                           preprocess() traces the global and caustic photons and builds the maps with
//                           the reference's counts, depth and radii; render() runs the eye pass
//   translate()             walks the scene's hittable_list (hittable_list::for_each, hittable_list.h:36-41)
//                           and emitter list into an lrt_scene_desc: triangle meshes, rectangles and spheres
//                           in list order, the eight BSDFs, area and sky emitters, the camera's frame
//
// Include it after the LinRT headers it reads (core/scene.h, geometry/{triangle_mesh,rectangle,sphere}.h,
// the material headers, emitter/{area_emitter,env_emitter}.h). Reading a constructed scene needs members
// that LinRT keeps private; each class involved grants them to `LinRT::lrt_linrt_access` with the line
//     friend struct lrt_linrt_access;
// in scene, hittable, triangle_mesh, rectangle, area_emitter, env_emitter, rough_transmittance,
// ggx_distribution and the eight BSDF classes (diffuse_bsdf, rough_conductor_bsdf, dielectric_bsdf,
// rough_dielectric_bsdf, plastic_bsdf, rough_plastic_bsdf, coating_bsdf, rough_coating_bsdf). A BSDF is translated from what its object holds, so a translated
// scene renders exactly as the reference's own objects do: the rough-transmittance tables are copied from
// the objects, a coating's eta and 1/eta are passed as held (lrt_material_desc::eta_pair), the camera as
// its frame (lrt_scene_set_camera_frame), the sky as its cooked Hosek state.
//
// Errors are thrown as lrt_linrt::error (status and liblrt's message); LinRT itself reports errors by
// return values and nullptr, so the calls that replace its integrators are the only places that throw.
#pragma once

#include <cstdint>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include "lrt.h"

namespace LinRT {

// Read access to the members the translation needs (granted by `friend struct lrt_linrt_access;`).
struct lrt_linrt_access {
    static const hittable_list& shapes(const scene& s) { return s.shapes; }
    static const std::vector<std::shared_ptr<emitter>>& emitters(const scene& s) { return s.emitters; }

    static const std::vector<vec3>& positions(const triangle_mesh& m) { return m.positions; }
    static const std::vector<std::uint32_t>& indices(const triangle_mesh& m) { return m.indices; }
    static const std::vector<vec3>& corner_normals(const triangle_mesh& m) { return m.corner_normals; }
    static vec3 corner(const rectangle& r) { return r.corner; }
    static vec3 edge_u(const rectangle& r) { return r.edge_u; }
    static vec3 edge_v(const rectangle& r) { return r.edge_v; }

    static const hittable* shape_of(const area_emitter& e) { return e.shape_ptr.get(); }
    static color radiance_of(const area_emitter& e) { return e.radiance; }
    static vec3 sun_direction(const env_emitter& e) { return e.sun_direction; }
    static global_precision scale(const env_emitter& e) { return e.scale; }
    static const ArHosekSkyModelState* sky_state(const env_emitter& e) { return e.state.get(); }

    // every BSDF's members, by type
    static void read(const diffuse_bsdf& b, lrt_material_desc& d) { put(d.diffuse_reflectance, b.albedo); }
    static void read(const rough_conductor_bsdf& b, lrt_material_desc& d) {
        d.alpha = b.alpha;
        put(d.eta, b.eta);
        put(d.k, b.k);
        put(d.specular_reflectance, b.specular_reflectance);
    }
    static void read(const dielectric_bsdf& b, lrt_material_desc& d) {
        d.int_ior = b.int_ior;
        d.ext_ior = b.ext_ior;
        put(d.specular_reflectance, b.specular_reflectance);
        put(d.specular_transmittance, b.specular_transmittance);
    }
    static void read(const rough_dielectric_bsdf& b, lrt_material_desc& d) {
        d.int_ior = b.int_ior;
        d.ext_ior = b.ext_ior;
        d.alpha = b.alpha;
        put(d.specular_reflectance, b.specular_reflectance);
        put(d.specular_transmittance, b.specular_transmittance);
    }
    // the plastics hold eta = int_ior / ext_ior: (eta, 1) reproduces it, and everything derived from it
    static void read(const plastic_bsdf& b, lrt_material_desc& d) {
        d.int_ior = b.eta;
        d.ext_ior = 1.0f;
        d.nonlinear = b.nonlinear ? 1 : 0;
        put(d.specular_reflectance, b.specular_reflectance);
        put(d.diffuse_reflectance, b.diffuse_reflectance);
    }
    static void read(const rough_plastic_bsdf& b, lrt_material_desc& d) {
        d.int_ior = b.eta;
        d.ext_ior = 1.0f;
        d.alpha = b.alpha;
        d.nonlinear = b.nonlinear ? 1 : 0;
        put(d.specular_reflectance, b.specular_reflectance);
        put(d.diffuse_reflectance, b.diffuse_reflectance);
        copy_table(b.external, d);
        d.trans_internal_diffuse = b.internal.diff_trans[0];
    }
    static void read(const coating_bsdf& b, lrt_material_desc& d) {
        d.eta_pair[0] = b.eta;
        d.eta_pair[1] = b.inv_eta;
        d.thickness = b.thickness;
        put(d.sigma_a, b.sigma_a);
        put(d.specular_reflectance, b.specular_reflectance);
    }
    static void read(const rough_coating_bsdf& b, lrt_material_desc& d) {
        d.eta_pair[0] = b.eta;
        d.eta_pair[1] = b.inv_eta;
        d.thickness = b.thickness;
        d.alpha = b.distribution.alpha;
        put(d.sigma_a, b.sigma_a);
        put(d.specular_reflectance, b.specular_reflectance);
        copy_table(b.transmittance, d);
    }
    static const bsdf* nested(const coating_bsdf& b) { return b.nested.get(); }
    static const bsdf* nested(const rough_coating_bsdf& b) { return b.nested.get(); }

    static void put(float* out, const vec3& v) {
        out[0] = v.x;
        out[1] = v.y;
        out[2] = v.z;
    }
    static void copy_table(const rough_transmittance& t, lrt_material_desc& d) {
        const std::size_t n = t.trans.size() < LRT_TRANS_SAMPLES ? t.trans.size() : LRT_TRANS_SAMPLES;
        for(std::size_t i = 0; i < n; ++i) d.trans_table[i] = t.trans[i];
    }
};

}  // namespace LinRT

namespace lrt_linrt {

class error : public std::runtime_error {
public:
    error(int status, const std::string& what) : std::runtime_error(what), status(status) {}
    int status;
};

// The arrays an lrt_scene_desc points into, kept alive with it.
struct scene_arrays {
    std::vector<lrt_object_desc> objects;
    std::vector<lrt_material_desc> materials;
    std::vector<lrt_emitter_desc> emitters;
    std::vector<std::vector<float>> positions, corner_normals;
    std::vector<std::vector<std::uint32_t>> indices;
    float camera_frame[4][3] = {};  // origin, lower_left_corner, horizontal, vertical

    lrt_scene_desc desc() const {
        lrt_scene_desc d{};
        d.n_objects = static_cast<uint32_t>(objects.size());
        d.objects = objects.data();
        d.n_materials = static_cast<uint32_t>(materials.size());
        d.materials = materials.data();
        d.n_emitters = static_cast<uint32_t>(emitters.size());
        d.emitters = emitters.data();
        return d;
    }
};

namespace detail {

using A = LinRT::lrt_linrt_access;

inline void put3(float* out, const LinRT::vec3& v) { A::put(out, v); }

// the material list in an order where a coating's nested BSDF precedes it; index of every BSDF
inline int material_index(const LinRT::bsdf* b, scene_arrays& out, std::unordered_map<const LinRT::bsdf*, int>& seen) {
    using namespace LinRT;
    if(!b) return -1;
    const auto it = seen.find(b);
    if(it != seen.end()) return it->second;
    lrt_material_desc d{};
    d.nested = -1;
    d.int_ior = 1.5f;
    d.ext_ior = 1.0f;
    d.thickness = 1.0f;
    for(int c = 0; c < 3; ++c) d.specular_reflectance[c] = d.specular_transmittance[c] = 1.0f;
    if(const auto* x = dynamic_cast<const diffuse_bsdf*>(b)) {
        d.type = LRT_DIFFUSE;
        A::read(*x, d);
    } else if(const auto* x = dynamic_cast<const rough_conductor_bsdf*>(b)) {
        d.type = LRT_ROUGH_CONDUCTOR;
        A::read(*x, d);
    } else if(const auto* x = dynamic_cast<const dielectric_bsdf*>(b)) {
        d.type = LRT_DIELECTRIC;
        A::read(*x, d);
    } else if(const auto* x = dynamic_cast<const rough_dielectric_bsdf*>(b)) {
        d.type = LRT_ROUGH_DIELECTRIC;
        A::read(*x, d);
    } else if(const auto* x = dynamic_cast<const plastic_bsdf*>(b)) {
        d.type = LRT_PLASTIC;
        A::read(*x, d);
    } else if(const auto* x = dynamic_cast<const rough_plastic_bsdf*>(b)) {
        d.type = LRT_ROUGH_PLASTIC;
        A::read(*x, d);
    } else if(const auto* x = dynamic_cast<const coating_bsdf*>(b)) {
        d.type = LRT_COATING;
        d.nested = material_index(A::nested(*x), out, seen);
        A::read(*x, d);
    } else if(const auto* x = dynamic_cast<const rough_coating_bsdf*>(b)) {
        d.type = LRT_ROUGH_COATING;
        d.nested = material_index(A::nested(*x), out, seen);
        A::read(*x, d);
    } else {
        throw error(LRT_ERR_INVALID_ARGUMENT, "lrt_linrt: a BSDF type liblrt does not know");
    }
    const int index = static_cast<int>(out.materials.size());
    out.materials.push_back(d);
    seen[b] = index;
    return index;
}

}  // namespace detail

// The scene as liblrt takes it: objects in the hittable_list's order (its ties: the later object wins),
// each mesh's positions, indices and corner normals as the triangle_mesh holds them, materials as their
// objects hold them, emitters in the scene's order (area lights point at their shape's object, the sky
// carries its cooked state), the camera's frame.
inline scene_arrays translate(const LinRT::scene& sc) {
    using namespace LinRT;
    using A = lrt_linrt_access;
    scene_arrays out;
    std::unordered_map<const bsdf*, int> seen;
    std::unordered_map<const hittable*, int> object_of;
    A::shapes(sc).for_each([&](const hittable& h) {
        lrt_object_desc o{};
        o.material = detail::material_index(h.get_material().get(), out, seen);
        if(const auto* m = dynamic_cast<const triangle_mesh*>(&h)) {
            o.kind = LRT_OBJECT_MESH;
            std::vector<float> pos, nrm;
            for(const vec3& p : A::positions(*m)) pos.insert(pos.end(), {p.x, p.y, p.z});
            for(const vec3& n : A::corner_normals(*m)) nrm.insert(nrm.end(), {n.x, n.y, n.z});
            out.positions.push_back(std::move(pos));
            out.corner_normals.push_back(std::move(nrm));
            out.indices.push_back(A::indices(*m));
        } else if(const auto* r = dynamic_cast<const rectangle*>(&h)) {
            o.kind = LRT_OBJECT_RECTANGLE;
            o.material = -1;  // rectangle::hit leaves the record without a BSDF (rectangle.h:50)
            detail::put3(o.corner, A::corner(*r));
            detail::put3(o.edge_u, A::edge_u(*r));
            detail::put3(o.edge_v, A::edge_v(*r));
        } else if(const auto* q = dynamic_cast<const sphere*>(&h)) {
            o.kind = LRT_OBJECT_SPHERE;
            detail::put3(o.center, q->center);
            o.radius = q->radius;
        } else {
            throw error(LRT_ERR_INVALID_ARGUMENT, "lrt_linrt: a shape type liblrt does not know");
        }
        object_of[&h] = static_cast<int>(out.objects.size());
        out.objects.push_back(o);
    });
    // mesh arrays are bound once every vector is in place (their buffers do not move after this)
    for(std::size_t i = 0, m = 0; i < out.objects.size(); ++i) {
        lrt_object_desc& o = out.objects[i];
        if(o.kind != LRT_OBJECT_MESH) continue;
        o.n_vertices = static_cast<uint32_t>(out.positions[m].size() / 3);
        o.n_indices = static_cast<uint32_t>(out.indices[m].size());
        o.positions = out.positions[m].data();
        o.indices = out.indices[m].data();
        o.corner_normals = out.corner_normals[m].data();
        ++m;
    }
    for(const auto& e : A::emitters(sc)) {
        lrt_emitter_desc d{};
        d.object = -1;
        if(const auto* a = dynamic_cast<const area_emitter*>(e.get())) {
            d.kind = LRT_EMITTER_AREA;
            const auto it = object_of.find(A::shape_of(*a));
            if(it == object_of.end()) {
                throw error(LRT_ERR_INVALID_ARGUMENT, "lrt_linrt: an area light whose shape is not in the scene");
            }
            d.object = it->second;
            detail::put3(d.radiance, A::radiance_of(*a));
        } else if(const auto* s = dynamic_cast<const env_emitter*>(e.get())) {
            d.kind = LRT_EMITTER_ENV;
            detail::put3(d.sun_direction, A::sun_direction(*s));
            d.scale = A::scale(*s);
            const ArHosekSkyModelState* st = A::sky_state(*s);
            d.turbidity = static_cast<float>(st->turbidity);
            d.albedo = static_cast<float>(st->albedo);
            for(int c = 0; c < 3; ++c) {
                for(int k = 0; k < 9; ++k) d.hosek_config[c][k] = st->configs[c][k];
                d.hosek_radiance[c] = st->radiances[c];
            }
        } else {
            throw error(LRT_ERR_INVALID_ARGUMENT, "lrt_linrt: an emitter type liblrt does not know");
        }
        out.emitters.push_back(d);
    }
    const camera& cam = sc.sensor();
    if(cam.lens_radius > 0.0f) throw error(LRT_ERR_INVALID_ARGUMENT, "lrt_linrt: only pinhole cameras (aperture 0)");
    detail::put3(out.camera_frame[0], cam.origin);
    detail::put3(out.camera_frame[1], cam.lower_left_corner);
    detail::put3(out.camera_frame[2], cam.horizontal);
    detail::put3(out.camera_frame[3], cam.vertical);
    return out;
}

// One liblrt context (device, its own CUDA stream, the uploaded scene).
class context {
public:
    explicit context(int device = 0) { check(lrt_create(device, nullptr, &ctx_)); }
    ~context() {
        if(ctx_) lrt_destroy(ctx_);
    }
    context(const context&) = delete;
    context& operator=(const context&) = delete;

    lrt_context* get() const { return ctx_; }

    void check(int status) const {
        if(status != LRT_OK) {
            throw error(status, std::string(lrt_status_string(status)) + ": " + (ctx_ ? lrt_last_error(ctx_) : ""));
        }
    }

    // the scene's objects, materials, emitters and camera, translated and uploaded (kd-trees built)
    void upload(const LinRT::scene& sc) {
        const scene_arrays a = translate(sc);
        const lrt_scene_desc d = a.desc();
        check(lrt_scene_upload(ctx_, &d));
        check(lrt_scene_set_camera_frame(ctx_, a.camera_frame[0], a.camera_frame[1], a.camera_frame[2],
                                         a.camera_frame[3]));
    }

    // pixels[y * width + x] = the mean of samples sample_offset .. sample_offset + spp - 1 of pixel (x, y)
    void copy_out(const std::vector<float>& rgb, std::vector<LinRT::color>& pixels) const {
        pixels.resize(rgb.size() / 3);
        for(std::size_t i = 0; i < pixels.size(); ++i) pixels[i] = LinRT::color(rgb[3 * i], rgb[3 * i + 1], rgb[3 * i + 2]);
    }

private:
    lrt_context* ctx_ = nullptr;
};

// path_integrator (path_integrator.h:18-182) on the GPU. preprocess() uploads the scene; render() is the
// tile loop of main.cpp:103-147 with path_integrator::radiance for every (pixel, sample): sample s of
// pixel (x, y) starts sampler.start(y * width + x, s), offsets the camera ray by next_2d() and divides
// the sum by spp -- the image main.cpp writes. max_depth and rr_depth default to the reference's
// constants (path_integrator.h:173, :19).
class gpu_path_integrator {
public:
    explicit gpu_path_integrator(int device = 0, int max_depth = 50, int rr_depth = 5)
        : ctx_(device), max_depth_(max_depth), rr_depth_(rr_depth) {}

    void preprocess(const LinRT::scene& sc) { ctx_.upload(sc); }

    void render(int width, int height, int spp, std::vector<LinRT::color>& pixels, uint32_t sample_offset = 0) {
        if(width < 2 || height < 2 || spp < 1) throw error(LRT_ERR_INVALID_ARGUMENT, "lrt_linrt: image size or spp");
        lrt_render_params p{};
        p.width = static_cast<uint32_t>(width);
        p.height = static_cast<uint32_t>(height);
        p.spp = static_cast<uint32_t>(spp);
        p.max_depth = max_depth_;
        p.rr_depth = rr_depth_;
        p.sample_offset = sample_offset;
        std::vector<float> rgb(3ull * width * height);
        ctx_.check(lrt_render(ctx_.get(), &p, rgb.data()));
        ctx_.copy_out(rgb, pixels);
    }

    context& lrt() { return ctx_; }

private:
    context ctx_;
    int max_depth_, rr_depth_;
};

// photon_integrator (photon_integrator.h:15-296) on the GPU with the reference's constants
// (photon_integrator.h:57-65): preprocess() traces the global and caustic photons (250,000 each; the
// caustic gather only when the scene has a specular BSDF), builds the maps and sets the radii from the
// scene's bounding sphere (photon_integrator.h:15-37); render() is main.cpp's tile loop around
// photon_integrator::radiance.
class gpu_photon_integrator {
public:
    explicit gpu_photon_integrator(int device = 0) : ctx_(device) {
        params_.global_map = params_.caustic_map = -1;
        params_.max_depth = 128;
        params_.max_specular_depth = 4;
        params_.direct_samples = 16;
        params_.glossy_samples = 32;
        params_.lookup_size = 120;
    }

    std::size_t global_photons = 250000;
    std::size_t caustic_photons = 250000;
    int rr_depth = 5;

    void preprocess(const LinRT::scene& sc) {
        ctx_.upload(sc);
        uint64_t shots[2] = {0, 0};
        ctx_.check(lrt_photon_preprocess(ctx_.get(), static_cast<uint32_t>(global_photons),
                                         static_cast<uint32_t>(caustic_photons), params_.max_depth, rr_depth,
                                         __builtin_huge_valf(), &params_, shots));
    }

    void render(int width, int height, int spp, std::vector<LinRT::color>& pixels, uint32_t sample_offset = 0) {
        if(width < 2 || height < 2 || spp < 1) throw error(LRT_ERR_INVALID_ARGUMENT, "lrt_linrt: image size or spp");
        lrt_render_params p{};
        p.width = static_cast<uint32_t>(width);
        p.height = static_cast<uint32_t>(height);
        p.spp = static_cast<uint32_t>(spp);
        p.max_depth = params_.max_depth;
        p.rr_depth = rr_depth;
        p.sample_offset = sample_offset;
        std::vector<float> rgb(3ull * width * height);
        ctx_.check(lrt_render_photon(ctx_.get(), &p, &params_, rgb.data()));
        ctx_.copy_out(rgb, pixels);
    }

    const lrt_photon_render_params& params() const { return params_; }
    context& lrt() { return ctx_; }

private:
    context ctx_;
    lrt_photon_render_params params_{};
};

}  // namespace lrt_linrt
