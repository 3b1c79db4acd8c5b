// lrt_host.h — host-side scene assembly (no CUDA calls): SAH kd-tree build, device record packing,
// rough-transmittance slicing, Fdr quadrature, camera and emitter precomputation.
#pragma once

#include <stdint.h>

#include <functional>
#include <memory>
#include <utility>
#include <string>
#include <vector>

#include "lrt.h"
#include "lrt_types.h"

namespace lrt {

struct MeshTreeInfo {
    uint32_t nodes;  // reachable nodes after packing
    uint32_t refs;   // leaf references after packing
    uint32_t depth;  // deepest leaf (root = 1)
};

// An allocator whose resize leaves new elements uninitialised, for the large arrays that the scene
// assembly fills on all host cores: their pages are first touched by the threads that write them.
template <typename T>
struct UninitAlloc : std::allocator<T> {
    template <typename U>
    struct rebind {
        using other = UninitAlloc<U>;
    };
    UninitAlloc() = default;
    template <typename U>
    UninitAlloc(const UninitAlloc<U>&) {}
    template <typename U>
    void construct(U* p) noexcept {
        ::new(static_cast<void*>(p)) U;
    }
    template <typename U, typename... Args>
    void construct(U* p, Args&&... args) {
        ::new(static_cast<void*>(p)) U(std::forward<Args>(args)...);
    }
};
template <typename T>
using BigVec = std::vector<T, UninitAlloc<T>>;

struct HostScene {
    BigVec<uint2> nodes;
    BigVec<float4> tris;
    BigVec<uint32_t> ref_prim;
    BigVec<float4> normals;
    std::vector<ObjRec> objects;
    std::vector<MatRec> materials;
    std::vector<float> tables;
    std::vector<EmitRec> emitters;
    std::vector<MeshTreeInfo> mesh_info;  // per object (zeros for analytic shapes)
    CamRec cam{};
    int32_t n_infinite = 0;
    // scene::sample_emitter_ray's luminance CDF over emitters with positive power (scene.h:21-34)
    std::vector<float> emission_cdf;
    std::vector<int32_t> emission_index;
    float emission_power = 0.0f;
    // area lights over meshes: per triangle the running area sum and the corner positions
    std::vector<float> light_cdf;
    std::vector<float4> light_tri;
    float bounding_radius = 0.0f;  // scene::bounding_sphere_radius (scene.h:41-45)
    bool has_delta_bsdf = false;   // scene::has_delta_bsdf (scene.h:48-57)
    // meshes of more than 64 triangles, largest first; queue segmentation is off when there are > 4
    int32_t n_heavy = 0;
    int32_t heavy[4] = {-1, -1, -1, -1};
    // object hierarchy (empty when the list is short): nodes as the device reads them, leaf objects
    std::vector<float4> tlas;
    std::vector<int32_t> tlas_objs;
};


// SAH kd-tree over triangle AABBs, the tree sah_kdtree::build produces (src/accelerator/sah_kdtree.h:35-57,
// 175-347), packed depth-first into 8-byte nodes with leaf references in leaf order.
struct PackedTree {
    std::vector<uint2> nodes;
    std::vector<uint32_t> refs;  // triangle index per leaf reference
    uint32_t depth = 0;
};

// Builds the kd-trees of several meshes at once: primitive boxes concatenated mesh after mesh (3 floats
// each), `counts` primitives per mesh (each at least 1); one tree per mesh in `out`.
using KdBatchBuilder = std::function<int(const std::vector<uint32_t>& counts, const BigVec<float>& bmin,
                                         const BigVec<float>& bmax, std::vector<PackedTree>& out,
                                         std::string& error)>;

// Validates and packs a scene description. Returns LRT_OK or an LRT_ERR_* with a message. The meshes'
// kd-trees are built on the host cores, or by `kd` when it is given.
int build_host_scene(const lrt_scene_desc* desc, HostScene& out, std::string& error,
                     const KdBatchBuilder* kd = nullptr);

void build_kdtree(const float* bmin, const float* bmax, uint32_t count, PackedTree& out);

// What a kd-tree build of `count` boxes starts from (sah_kdtree.h:35-57): the root voxel, extended box
// by box in order; the depth limit min(48, int(8 + 1.3 log2 count)), at least 1; the number of sweep
// events (two per axis, one where the box is flat on that axis).
struct KdRootInfo {
    float lo[3], hi[3];
    int32_t depth_limit;
    uint64_t n_events;
};
KdRootInfo kd_root_info(const float* bmin, const float* bmax, uint32_t count);

// load_obj (src/io/obj_loader.h:44-141): positions (3 floats each, centred and unitised), triangle
// indices and per-corner normals (3 floats per index)
int load_obj(const char* path, std::vector<float>& positions, std::vector<uint32_t>& indices,
             std::vector<float>& corner_normals, std::string& error);

// camera::update for a pinhole with focus distance 1 (src/core/camera.h:20-44)
CamRec camera_from_desc(const lrt_camera_desc& c);

// Packs a material list into device records; rough plastic / rough coating tables are appended to `tables`.
int pack_materials(const lrt_material_desc* mats, uint32_t n, std::vector<MatRec>& out, std::vector<float>& tables,
                   std::string& error);

// rough_transmittance (src/material/func/rough_transmittance.h:67-185) in two steps: set_eta on the
// file's data gives an eta slice (n_alpha x LRT_TRANS_SAMPLES values, n_alpha diffuse values), set_alpha
// on that slice gives the 1-D table; rough_transmittance_slice runs both.
int rough_transmittance_eta(const char* path, float eta, std::vector<float>& sliced_t, std::vector<float>& sliced_d,
                            float& alpha_min, float& alpha_max, std::string& error);
int rough_transmittance_alpha(const float* sliced_t, const float* sliced_d, uint32_t n_alpha, float alpha_min,
                              float alpha_max, float alpha, float* table, float* diffuse, std::string& error);
int rough_transmittance_slice(const char* path, float eta, float alpha, float* table, float* diffuse, std::string& error);
float fresnel_diffuse_reflectance(float eta);
// The Hosek-Wilkie RGB sky state env_emitter's constructor cooks (src/emitter/env_emitter.h:13-30 ->
// arhosek_rgb_skymodelstate_alloc_init, third_party/hosek/ArHosekSkyModel.cc:602-635): per channel the
// nine radiance-distribution coefficients and the radiance scale, bit-identical to the reference.
int hosek_state(const float sun_direction[3], float turbidity, float albedo, double config[3][9], double radiance[3],
                std::string& error);
void sobol_direction_table(uint32_t table[16][32]);

}  // namespace lrt
