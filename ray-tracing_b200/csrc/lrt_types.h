// lrt_types.h — device-resident scene records shared by the host builder and the kernels.
//
// HBM layout (all arrays device-resident for the life of a scene):
//   nodes      uint2  [total kd nodes]   8-byte SAH kd-tree nodes, every mesh's tree concatenated
//   tris       float4 [3 * total refs]   per leaf reference: (p0, degenerate flag), edge1, edge2, stored in
//                                        leaf order so one leaf is one contiguous run of 48-byte records
//   ref_prim   uint32 [total refs]       leaf reference -> triangle index inside its mesh
//   normals    float4 [3 * total tris]   per triangle: the three corner normals (read once per closest hit)
//   objects    ObjRec [n_objects]        the linear object list in reference order
//   materials  MatRec [n_materials]
//   tables     float  [100 * n_tables]   rough-transmittance 1-D tables
//   emitters   EmitRec[n_emitters]
//   tlas       float4 [2 * nodes]       bounding-volume hierarchy over the objects (scenes of > 16 objects)
//   tlas_objs  int32  [n_objects]       object indices in leaf order
//   light_cdf  float  [mesh-light tris]  area CDF of every mesh that is an area light, mesh after mesh
//   light_tri  float4 [3 * same]         corner positions of those triangles (area-light sampling)
#pragma once

#include <stdint.h>
#include <vector_types.h>

namespace lrt {

// kd node word1 low 2 bits: split axis 0..2, or 3 for a leaf.
//   interior: word0 = split (float bits), word1 = (right_child << 2) | axis; left child = this + 1
//   leaf:     word0 = first reference,    word1 = (count << 2) | 3
constexpr uint32_t kLeafTag = 3u;

// object-list hierarchies are built above this many objects; their depth stays below the stack size
constexpr uint32_t kTlasMinObjects = 16;
constexpr int kTlasStack = 32;

struct ObjRec {
    int32_t kind;        // LRT_OBJECT_*
    int32_t material;    // -1 none (rectangles always none)
    int32_t emitter;     // emitter index, -1 none
    uint32_t node_base;  // mesh: first node of its tree
    uint32_t ref_base;   // mesh: first leaf reference
    uint32_t tri_base;   // mesh: first triangle (normals)
    uint32_t n_tris;
    uint32_t n_nodes;
    float bmin[3];       // mesh bounds (for the conservative object skip)
    float bmax[3];
    float corner[3];     // rectangle
    float edge_u[3];
    float edge_v[3];
    float normal[3];
    float area;          // rectangle / sphere / mesh surface area
    float center[3];     // sphere
    float radius;
};

struct MatRec {
    int32_t type;
    int32_t nested;              // coatings: nested material index
    uint32_t flags;              // bsdf::flags()
    int32_t component_count;     // bsdf::component_count()
    float int_ior, ext_ior;
    float alpha;                 // raw alpha (rough conductor: <= 0 means smooth)
    float dist_alpha;            // ggx_distribution alpha = max(alpha, 1e-4)
    float eta;                   // plastic/coatings: int_ior / ext_ior
    float inv_eta;               // coatings: ext_ior / int_ior; plastic: 1 / (eta*eta) (inv_eta2)
    float fdr;                   // plastic: fdr_int; rough plastic: internal diffuse transmittance
    float specular_sampling_weight;
    float thickness;
    int32_t nonlinear;
    int32_t table;               // index of the 1-D rough-transmittance table, -1 none
    int32_t specular_component;  // coatings
    float diffuse[3];
    float spec_refl[3];
    float spec_trans[3];
    float cond_eta[3];
    float cond_k[3];
    float sigma_a[3];
    int32_t sigma_zero;          // sigma_a.is_zero()
};

struct EmitRec {
    int32_t kind;        // LRT_EMITTER_*
    int32_t object;      // area: object index
    int32_t shape;       // area: LRT_OBJECT_* of that object
    int32_t sun_active;  // env
    float radiance[3];   // area
    float area;          // area: shape area
    uint32_t tri_first;  // area over a mesh: its first entry in light_cdf / light_tri
    uint32_t n_tris;     // area over a mesh: its triangle count
    // env
    float sun[3];
    float frame[3][3];   // onb built from sun (axis 0, 1, 2)
    float cos_cutoff;
    float cone_pdf;
    float scale;
    double cfg[3][9];
    double rad[3];
};

struct CamRec {
    float origin[3];
    float llc[3];
    float horizontal[3];
    float vertical[3];
};

// one job of a batched render: its paths occupy [path_begin, path_begin + width*height*spp) of the
// batch's path index space, ordered by (pixel, sample)
struct JobRec {
    CamRec cam;
    uint32_t width, height, spp, sample_offset;
    int32_t override_obj, override_mat;
    unsigned long long path_begin;
    unsigned long long out_offset;  // float offset of the job's image in the output
};

struct DeviceScene {
    const uint2* nodes;
    const float4* tris;
    const uint32_t* ref_prim;
    const float4* normals;
    const ObjRec* objects;
    const MatRec* materials;
    const float* tables;
    const EmitRec* emitters;
    const uint32_t* sobol;          // 16 x 32 Sobol direction numbers
    const float* emission_cdf;      // scene::sample_emitter_ray luminance CDF (scene.h:21-34)
    const int32_t* emission_index;  // emitter index of each CDF bin
    const float* light_cdf;         // mesh lights: running triangle area per triangle (triangle_mesh.h:17-24)
    const float4* light_tri;        // mesh lights: the triangle's three corner positions
    int32_t n_objects;
    int32_t n_materials;
    int32_t n_emitters;
    int32_t n_infinite;      // emitters with is_infinite()
    int32_t n_emission;      // CDF bins
    float emission_power;    // total luminance of emitted power
    int32_t n_heavy;         // meshes large enough that rays reaching their box are queued apart
    int32_t heavy[4];
    CamRec cam;
    // bounding-volume hierarchy over the object list (scenes with many objects); n_tlas = 0: the
    // object list is walked in order
    const float4* tlas;      // 2 per node: (bmin, first object | left child), (bmax, -count | right child)
    const int32_t* tlas_objs;
    int32_t n_tlas;
};

}  // namespace lrt
