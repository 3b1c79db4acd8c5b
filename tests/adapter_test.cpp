// Test of the reference-side adapter (include/lrt_linrt.hpp): the reference's own demo scene
// (src/main.cpp:38-90), built from the reference's classes, rendered through gpu_path_integrator /
// gpu_photon_integrator and by the reference's integrators on the CPU, compared per pixel.
//
//     adapter_test <bunny.obj> path|photon <width> <height> <spp>
//
// Prints one JSON line: pixels, the fraction beyond 3 Monte Carlo standard errors of the reference's
// per-pixel spread, the image means. path: path_integrator with its own constants (max_depth 50,
// rr_depth 5) against gpu_path_integrator on the same samples. photon: the GPU traces the photons
// (gpu_photon_integrator::preprocess, the reference's counts and radii); the reference's
// photon_integrator renders with maps built by photon_map::build from the same photon arrays.
//
// Test infrastructure: the adapter reads members LinRT keeps private, which a maintainer grants with
// `friend struct lrt_linrt_access;` in each class; this test, which must not change the reference,
// compiles the reference headers with private and protected read as public instead.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <thread>
#include <vector>

#define private public
#define protected public
#include "core/camera.h"
#include "core/hittable_list.h"
#include "core/sampler.h"
#include "core/scene.h"
#include "emitter/area_emitter.h"
#include "emitter/env_emitter.h"
#include "geometry/rectangle.h"
#include "geometry/sphere.h"
#include "geometry/triangle_mesh.h"
#include "integrator/path/path_integrator.h"
#include "integrator/photonmapper/photon_integrator.h"
#include "io/obj_loader.h"
#include "material/coating_bsdf.h"
#include "material/dielectric_bsdf.h"
#include "material/diffuse_bsdf.h"
#include "material/plastic_bsdf.h"
#include "material/rough_coating_bsdf.h"
#include "material/rough_conductor_bsdf.h"
#include "material/rough_dielectric_bsdf.h"
#include "material/rough_plastic_bsdf.h"
#undef private
#undef protected

#include "lrt_linrt.hpp"

using namespace LinRT;

namespace {

// main.cpp:38-90 with the sphere light of main.cpp:55-56 added to the scene (it defines it but leaves it
// out), so that the sphere's emitter sampling and hit are exercised too
std::unique_ptr<scene> demo_scene(const char* bunny, int width, int height) {
    const auto rough_plastic = std::make_shared<rough_plastic_bsdf>(1.49f, 1.000277f, 0.1f, color(1.0f),
                                                                    color(0.8f, 0.1f, 0.05f));
    camera cam;
    cam.origin = vec3(0.0f, 0.5f, 3.0f);
    cam.update(vec3(0.0f, 1.0f, 0.0f), 60.0f,
               static_cast<global_precision>(width) / static_cast<global_precision>(height));
    hittable_list world;
    auto mesh = load_obj(bunny);
    if(!mesh) return nullptr;
    mesh->translate(vec3(0.0f, 0.0f, 0.0f));
    mesh->set_material(rough_plastic);
    world.add(mesh);
    auto plane = std::make_shared<sphere>(vec3(0.0f, -100.5f, 0.0f), 100.0f);
    plane->set_material(std::make_shared<diffuse_bsdf>(color(.8f, .8f, .0f)));
    world.add(plane);
    auto rect = std::make_shared<rectangle>(vec3(-0.6f, 1.5f, -0.6f), vec3(1.2f, 0.0f, 0.0f), vec3(0.0f, 0.0f, 1.2f));
    auto rect_emitter = std::make_shared<area_emitter>(rect, color(12.0f));
    world.add(rect);
    auto ball = std::make_shared<sphere>(vec3(1.2f, 0.4f, 0.0f), 0.3f);
    auto ball_emitter = std::make_shared<area_emitter>(ball, color(4.0f));
    world.add(ball);
    std::vector<std::shared_ptr<emitter>> emitters{rect_emitter, ball_emitter};
    return std::make_unique<scene>(std::move(world), std::move(emitters), cam);
}

// the tile loop of main.cpp:110-147 on all host threads: per-pixel mean and mean of squares
template <typename Radiance>
void cpu_render(const scene& sc, int width, int height, int spp, std::vector<double>& mean, std::vector<double>& sq,
                Radiance radiance) {
    mean.assign(3ull * width * height, 0.0);
    sq.assign(3ull * width * height, 0.0);
    const unsigned n_threads = std::max(1u, std::thread::hardware_concurrency());
    std::vector<std::thread> pool;
    for(unsigned t = 0; t < n_threads; ++t) {
        pool.emplace_back([&, t] {
            for(int y = static_cast<int>(t); y < height; y += static_cast<int>(n_threads)) {
                for(int x = 0; x < width; ++x) {
                    double s[3] = {0, 0, 0}, s2[3] = {0, 0, 0};
                    for(int k = 0; k < spp; ++k) {
                        sampler smp;
                        smp.start(static_cast<uint32_t>(y * width + x), static_cast<uint32_t>(k));
                        const auto offset = smp.next_2d();
                        const auto u = (static_cast<global_precision>(x) + offset.x) / static_cast<global_precision>(width - 1);
                        const auto v = (static_cast<global_precision>(y) + offset.y) / static_cast<global_precision>(height - 1);
                        auto r = sc.sensor().get_ray(u, v);
                        const color c = radiance(r, smp);
                        const double ch[3] = {c.x, c.y, c.z};
                        for(int i = 0; i < 3; ++i) {
                            s[i] += ch[i];
                            s2[i] += ch[i] * ch[i];
                        }
                    }
                    const size_t o = 3ull * (static_cast<size_t>(y) * width + x);
                    for(int i = 0; i < 3; ++i) {
                        mean[o + i] = s[i] / spp;
                        sq[o + i] = s2[i] / spp;
                    }
                }
            }
        });
    }
    for(auto& th : pool) th.join();
}

}  // namespace

int main(int argc, char** argv) {
    if(argc != 6) {
        std::fprintf(stderr, "usage: adapter_test <bunny.obj> path|photon <width> <height> <spp>\n");
        return 2;
    }
    const std::string mode = argv[2];
    const int width = std::atoi(argv[3]), height = std::atoi(argv[4]), spp = std::atoi(argv[5]);
    const auto sc = demo_scene(argv[1], width, height);
    if(!sc) {
        std::fprintf(stderr, "cannot load %s\n", argv[1]);
        return 2;
    }
    std::vector<color> gpu;
    std::vector<double> mean, sq;
    try {
        if(mode == "path") {
            lrt_linrt::gpu_path_integrator integrator;
            integrator.preprocess(*sc);
            integrator.render(width, height, spp, gpu);
            const path_integrator reference;
            cpu_render(*sc, width, height, spp, mean, sq,
                       [&](ray& r, sampler& smp) { return reference.radiance(r, *sc, smp); });
        } else if(mode == "photon") {
            lrt_linrt::gpu_photon_integrator integrator;
            integrator.preprocess(*sc);
            integrator.render(width, height, spp, gpu);
            // the same photon arrays (the gathers are deterministic), into the reference's maps
            const lrt_photon_render_params& pp = integrator.params();
            photon_integrator reference;
            lrt_context* ctx = integrator.lrt().get();
            const int kinds[2] = {LRT_GATHER_SURFACE, LRT_GATHER_CAUSTIC};
            const int maps[2] = {pp.global_map, pp.caustic_map};
            const std::size_t requested[2] = {integrator.global_photons, integrator.caustic_photons};
            for(int m = 0; m < 2; ++m) {
                if(maps[m] < 0) continue;
                std::vector<lrt_photon> ph(requested[m]);
                uint32_t n = 0;
                uint64_t shot = 0;
                integrator.lrt().check(lrt_photon_trace(ctx, kinds[m], static_cast<uint32_t>(requested[m]),
                                                        pp.max_depth - 1, integrator.rr_depth, ph.data(), &n, &shot));
                std::vector<photon> list(n);
                for(uint32_t i = 0; i < n; ++i) {
                    list[i].position = vec3(ph[i].position[0], ph[i].position[1], ph[i].position[2]);
                    list[i].direction = vec3(ph[i].direction[0], ph[i].direction[1], ph[i].direction[2]);
                    list[i].normal = vec3(ph[i].normal[0], ph[i].normal[1], ph[i].normal[2]);
                    list[i].power = color(ph[i].power[0], ph[i].power[1], ph[i].power[2]);
                    list[i].depth = static_cast<std::uint16_t>(ph[i].depth);
                }
                (m == 0 ? reference.global_map : reference.caustic_map)
                    .build(list, 1.0f / static_cast<global_precision>(shot));
            }
            reference.global_radius = pp.global_radius;
            reference.caustic_radius = pp.caustic_radius;
            cpu_render(*sc, width, height, spp, mean, sq,
                       [&](ray& r, sampler& smp) { return reference.radiance(r, *sc, smp); });
        } else {
            std::fprintf(stderr, "mode must be path or photon\n");
            return 2;
        }
    } catch(const lrt_linrt::error& e) {
        std::printf("{\"error\": \"%s\", \"status\": %d}\n", e.what(), e.status);
        return 1;
    }
    std::size_t beyond = 0, nonfinite = 0;
    double gsum = 0.0, rsum = 0.0;
    for(std::size_t i = 0; i < gpu.size(); ++i) {
        const double g[3] = {gpu[i].x, gpu[i].y, gpu[i].z};
        for(int c = 0; c < 3; ++c) {
            const double m = mean[3 * i + c];
            if(!std::isfinite(g[c]) || !std::isfinite(m)) {
                ++nonfinite;
                continue;
            }
            const double se = std::sqrt(std::max(sq[3 * i + c] - m * m, 0.0) / spp);
            if(std::fabs(g[c] - m) > 3.0 * se + 1e-6 * std::max(std::fabs(m), 1e-3)) ++beyond;
            gsum += g[c];
            rsum += m;
        }
    }
    const double values = 3.0 * gpu.size();
    std::printf("{\"mode\": \"%s\", \"pixels\": %zu, \"beyond_3se\": %.6f, \"nonfinite\": %zu, \"gpu_mean\": %.8g, "
                "\"reference_mean\": %.8g}\n",
                mode.c_str(), gpu.size(), beyond / values, nonfinite, gsum / values, rsum / values);
    return 0;
}
