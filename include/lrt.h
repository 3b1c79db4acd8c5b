/*
 * lrt.h — C ABI of liblrt, the B200 (sm_100a) rendering hot path of the LinRT CPU ray tracer.
 *
 * Every entry point returns an int status (LRT_OK = 0, negative LRT_ERR_* on failure); no C++
 * exception crosses this boundary. lrt_last_error() gives the message of the last failure on a
 * context. All device work of a context is ordered on the CUDA stream given to lrt_create(). A
 * context is not thread-safe: use one per host thread, or serialise calls.
 *
 * Entry points that take host pointers copy them (host <-> device copies happen inside the call);
 * the *_dev variants take device pointers that the caller owns.
 *
 * Reference interfaces replaced (paths inside the reference project):
 *   scene build + upload        src/core/scene.h:21-34, src/core/hittable_list.h:10-34,
 *                               src/geometry/triangle_mesh.h:14-28,148-157, src/accelerator/sah_kdtree.h:35-57
 *   lrt_trace                   scene::hit src/core/scene.h:36-38 -> hittable_list::hit src/core/hittable_list.h:19-34
 *                               -> triangle_mesh::hit src/geometry/triangle_mesh.h:30-99 -> sah_kdtree::intersect
 *                               src/accelerator/sah_kdtree.h:62-121; rectangle::hit src/geometry/rectangle.h:18-55;
 *                               sphere::hit src/geometry/sphere.h:21-49
 *   lrt_bsdf_evaluate           bsdf::sample/eval/pdf src/material/bsdf.h:55-89 and the eight BSDFs in src/material/
 *   lrt_sky_eval                scene::eval_environment src/core/scene.h:61-70 -> env_emitter::eval
 *                               src/emitter/env_emitter.h:71-88
 *   lrt_render                  the tile loop of src/main.cpp:103-147 around path_integrator::radiance
 *                               src/integrator/path/path_integrator.h:18-170
 *   lrt_photon_trace            photon_gather::run src/integrator/photonmapper/photon_gather.h:15-61 with
 *                               photon_tracer::trace_particle src/integrator/photonmapper/photon_tracer.h:23-96
 *   lrt_photon_map_build        photon_map::build src/integrator/photonmapper/photon_map.h:26-33
 *   lrt_photon_knn              photon_map::nearest/search src/integrator/photonmapper/photon_map.h:117-165
 *   lrt_photon_irradiance       photon_map::estimate_irradiance src/integrator/photonmapper/photon_map.h:38-70
 *   lrt_rough_transmittance_slice  rough_transmittance ctor src/material/func/rough_transmittance.h:15-24,67-185
 *   lrt_fresnel_diffuse_reflectance fresnel_diffuse_reflectance src/material/func/fresnel.h:128-133
 *   lrt_tonemap                 to_byte + the flip of ImageWriter::save src/io/image_write.cpp:10-20,60-69
 *   lrt_hosek_state             env_emitter ctor src/emitter/env_emitter.h:13-30 -> arhosek_rgb_skymodelstate_alloc_init
 *                               third_party/hosek/ArHosekSkyModel.cc:602-635
 */
#ifndef LRT_H
#define LRT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define LRT_OK                    0
#define LRT_ERR_INVALID_ARGUMENT (-1)
#define LRT_ERR_CUDA             (-2)
#define LRT_ERR_OUT_OF_MEMORY    (-3)
#define LRT_ERR_IO               (-4)
#define LRT_ERR_RANGE            (-5)
#define LRT_ERR_NO_SCENE         (-6)
/* -7, -8 and -10 are not used: no kernel of the library waits on a queue or a flag */
#define LRT_ERR_NO_DEVICE        (-9)

/* ---- BSDF flags (src/material/bsdf.h:18-28) ---- */
#define LRT_BSDF_NONE        0u
#define LRT_BSDF_DIFFUSE     (1u << 0)
#define LRT_BSDF_SPECULAR    (1u << 1)
#define LRT_BSDF_REFLECTIVE  (1u << 2)
#define LRT_BSDF_TRANSPARENT (1u << 3)
#define LRT_BSDF_GLOSSY      (1u << 4)
#define LRT_BSDF_METALLIC    (1u << 5)
#define LRT_BSDF_DIELECTRIC  (1u << 6)
#define LRT_BSDF_REFRACTIVE  (1u << 7)

/* measure (src/material/bsdf.h:9-16) */
#define LRT_MEASURE_SOLID_ANGLE 1
#define LRT_MEASURE_DISCRETE    5

/* transport mode (src/material/bsdf.h:31-34) */
#define LRT_MODE_RADIANCE   0
#define LRT_MODE_IMPORTANCE 1

/* material types: one per BSDF class in src/material/ */
#define LRT_DIFFUSE          0  /* diffuse_bsdf.h */
#define LRT_ROUGH_CONDUCTOR  1  /* rough_conductor_bsdf.h (alpha <= 0: smooth mirror) */
#define LRT_DIELECTRIC       2  /* dielectric_bsdf.h */
#define LRT_ROUGH_DIELECTRIC 3  /* rough_dielectric_bsdf.h */
#define LRT_PLASTIC          4  /* plastic_bsdf.h */
#define LRT_ROUGH_PLASTIC    5  /* rough_plastic_bsdf.h */
#define LRT_COATING          6  /* coating_bsdf.h */
#define LRT_ROUGH_COATING    7  /* rough_coating_bsdf.h */

/* rough-transmittance table length in cos^(1/4) theta (ggx.dat theta samples) */
#define LRT_TRANS_SAMPLES 100

/*
 * Material description. Field meaning follows the reference constructors:
 *   diffuse:          diffuse_reflectance = albedo
 *   rough_conductor:  eta, k, alpha, specular_reflectance
 *   dielectric:       int_ior, ext_ior, specular_reflectance, specular_transmittance
 *   rough_dielectric: int_ior, ext_ior, alpha, specular_reflectance, specular_transmittance
 *   plastic:          int_ior, ext_ior, specular_reflectance, diffuse_reflectance, nonlinear
 *   rough_plastic:    int_ior, ext_ior, alpha, specular_reflectance, diffuse_reflectance, nonlinear,
 *                     trans_table = rough_transmittance(int/ext, alpha) sliced 1-D table,
 *                     trans_internal_diffuse = rough_transmittance(ext/int, alpha).eval_diffuse()
 *   coating:          int_ior, ext_ior, nested, specular_reflectance, sigma_a, thickness
 *   rough_coating:    int_ior, ext_ior, alpha, nested, specular_reflectance, sigma_a, thickness,
 *                     trans_table = rough_transmittance(int/ext, alpha) sliced 1-D table
 * The tables come from lrt_rough_transmittance_slice() (or any caller holding the same data).
 * A coating's nested material must have a smaller index than the coating and must not itself be
 * a coating (the reference allows deeper nesting; the device path supports one level).
 */
typedef struct lrt_material_desc {
    int32_t type;
    int32_t nested;
    int32_t nonlinear;
    float int_ior;
    float ext_ior;
    float alpha;
    float thickness;
    float diffuse_reflectance[3];
    float specular_reflectance[3];
    float specular_transmittance[3];
    float eta[3];
    float k[3];
    float sigma_a[3];
    float trans_table[LRT_TRANS_SAMPLES];
    float trans_internal_diffuse;
    /* coatings: {eta, 1/eta} exactly as a constructed coating_bsdf holds them (coating.h keeps the
     * ratio and its reciprocal, not the two indices); eta_pair[0] > 0 overrides int_ior/ext_ior */
    float eta_pair[2];
} lrt_material_desc;

/* objects of the linear object list (src/core/hittable_list.h); order is significant */
#define LRT_OBJECT_MESH      0  /* triangle_mesh: one SAH kd-tree per mesh */
#define LRT_OBJECT_RECTANGLE 1  /* rectangle: never carries a BSDF (rectangle.h:50) */
#define LRT_OBJECT_SPHERE    2  /* sphere */

typedef struct lrt_object_desc {
    int32_t kind;
    int32_t material;          /* index into materials, -1 = none */
    uint32_t n_vertices;
    uint32_t n_indices;        /* 3 per triangle */
    const float* positions;    /* n_vertices * 3 */
    const uint32_t* indices;   /* n_indices */
    const float* corner_normals; /* n_indices * 3: one normal per triangle corner */
    float corner[3];           /* rectangle */
    float edge_u[3];
    float edge_v[3];
    float center[3];           /* sphere */
    float radius;
} lrt_object_desc;

#define LRT_EMITTER_AREA 0  /* area_emitter over an object (area_emitter.h) */
#define LRT_EMITTER_ENV  1  /* Hosek sky (env_emitter.h) */

/*
 * Emitter description. For LRT_EMITTER_ENV, hosek_config/hosek_radiance are the RGB model state
 * (ArHosekSkyModelState configs[0..2] and radiances[0..2]) cooked by
 * arhosek_rgb_skymodelstate_alloc_init(turbidity, albedo, asin(normalize(sun_direction).y)); left all
 * zero, the upload cooks it from sun_direction, turbidity and albedo (lrt_hosek_state).
 */
typedef struct lrt_emitter_desc {
    int32_t kind;
    int32_t object;            /* area: index of the emitting object */
    float radiance[3];         /* area */
    float sun_direction[3];    /* env: normalised inside, as env_emitter.h:17 */
    float turbidity;
    float albedo;
    float scale;
    double hosek_config[3][9];
    double hosek_radiance[3];
} lrt_emitter_desc;

/* pinhole camera (src/core/camera.h:20-44); aperture must be 0 */
typedef struct lrt_camera_desc {
    float origin[3];
    float look_at[3];
    float up[3];
    float fov_degrees;
    float aspect_ratio;
} lrt_camera_desc;

typedef struct lrt_scene_desc {
    uint32_t n_objects;
    const lrt_object_desc* objects;
    uint32_t n_materials;
    const lrt_material_desc* materials;
    uint32_t n_emitters;
    const lrt_emitter_desc* emitters;
    lrt_camera_desc camera;
} lrt_scene_desc;

/* ---- queries ---- */

/* one ray: origin, direction, t_min, t_max */
typedef struct lrt_ray {
    float origin[3];
    float direction[3];
    float t_min;
    float t_max;
} lrt_ray;

typedef struct lrt_hit {
    float t;
    int32_t object;      /* -1 on miss */
    int32_t prim;        /* triangle index inside the mesh; -1 for analytic shapes */
    int32_t front_face;
    float p[3];
    float normal[3];     /* shading normal, facing the incoming ray (hit_record::normal) */
} lrt_hit;

typedef struct lrt_bsdf_query {
    float wi[3];
    float wo[3];
    float u[2];
    float lobe_sample;
    int32_t front_face;
    int32_t mode;          /* LRT_MODE_* */
    uint32_t type_mask;
    int32_t component;
    int32_t measure;       /* for eval/pdf: LRT_MEASURE_* */
} lrt_bsdf_query;

typedef struct lrt_bsdf_result {
    float sample_weight[3];
    float sample_wo[3];
    float sample_pdf;
    float sample_eta;
    uint32_t sampled_type;
    int32_t sampled_component;
    float eval[3];
    float pdf;
} lrt_bsdf_result;

/* photon record (photon_map.h:16-22) */
typedef struct lrt_photon {
    float position[3];
    float direction[3];
    float normal[3];
    float power[3];
    uint32_t depth;
} lrt_photon;

#define LRT_GATHER_SURFACE 0
#define LRT_GATHER_CAUSTIC 1

typedef struct lrt_render_params {
    uint32_t width;
    uint32_t height;
    uint32_t spp;
    int32_t max_depth;       /* path_integrator.h:173 */
    int32_t rr_depth;        /* path_integrator.h:19 */
    uint32_t sample_offset;  /* first sample index (replicas render disjoint sample ranges) */
    uint32_t row_begin;      /* render rows [row_begin, row_end); 0,0 = all rows */
    uint32_t row_end;
} lrt_render_params;

/* per-stage device time of the wavefront renderer, accumulated while stage timing is on */
#define LRT_STAGE_RAYGEN  0
#define LRT_STAGE_EXTEND  1
#define LRT_STAGE_SORT    2
#define LRT_STAGE_SHADE   3
#define LRT_STAGE_SHADOW  4
#define LRT_STAGE_ACCUM   5
#define LRT_STAGE_COUNT   6
#define LRT_MAX_STAT_DEPTH 16

typedef struct lrt_render_stats {
    uint64_t paths;              /* camera paths traced */
    uint64_t extension_rays;     /* closest-hit rays traced */
    uint64_t shadow_rays;        /* NEE shadow rays traced */
    uint64_t nodes_visited;      /* kd nodes visited by extension rays (option count_work) */
    uint64_t triangles_tested;   /* triangle tests of extension rays (option count_work) */
    uint64_t shadow_nodes_visited;     /* the same for shadow rays */
    uint64_t shadow_triangles_tested;
    uint64_t shading_events;
    uint64_t kernel_launches;
    float stage_ms[LRT_STAGE_COUNT];
    uint32_t stage_launches[LRT_STAGE_COUNT];
    uint64_t rays_at_depth[LRT_MAX_STAT_DEPTH];  /* extension rays per bounce (option count_work) */
    /* k-nearest-photon queries of lrt_photon_irradiance(_dev) with option count_work */
    uint64_t knn_queries;
    uint64_t knn_nodes_visited;   /* photon-map nodes read */
    uint64_t knn_photons_tested;  /* photon positions whose distance was computed */
    uint64_t knn_photons_found;   /* photons returned (<= k per query) and read by the estimate */
} lrt_render_stats;

/* ---- context ---- */
typedef struct lrt_context lrt_context;

int lrt_create(int device, void* cuda_stream, lrt_context** out);
int lrt_destroy(lrt_context* ctx);
const char* lrt_last_error(const lrt_context* ctx);
const char* lrt_status_string(int status);

/* the float-to-byte conversion of the image writer (src/io/image_write.cpp:10-20: NaN -> 0,
 * value^(1/2.2), clamp to [0, 0.999], truncate value*256) applied to width*height RGB pixels, with the
 * writer's optional vertical flip (image_write.cpp:60-69) when flip != 0; bytes holds 3 per pixel.
 * The bytes are those of the reference's to_byte with the host's powf (see lrt_tonemap_table). */
int lrt_tonemap(lrt_context* ctx, const float* rgb, uint32_t width, uint32_t height, int flip, uint8_t* bytes);
int lrt_tonemap_dev(lrt_context* ctx, const float* rgb_dev, uint32_t width, uint32_t height, int flip,
                    uint8_t* bytes_dev);
/* the 256 byte thresholds these use (host only, no device work): thresholds[k] for k = 1..255 is the
 * smallest float whose byte is >= k under the reference's to_byte evaluated with this process's C
 * library powf, thresholds[0] = 0; a finite value v >= 0 converts to the number of k >= 1 with
 * thresholds[k] <= v. LRT_ERR_RANGE if the host powf made the steps non-monotonic. */
int lrt_tonemap_table(float* thresholds /* 256 */);

/* host-side utilities (no device work) */
int lrt_rough_transmittance_slice(const char* ggx_path, float eta, float alpha,
                                  float* table_out /* LRT_TRANS_SAMPLES */, float* diffuse_out);
float lrt_fresnel_diffuse_reflectance(float eta);
/* The Hosek-Wilkie RGB sky state of env_emitter's constructor (src/emitter/env_emitter.h:13-30:
 * elevation = asin(normalize(sun_direction).y) in float, then arhosek_rgb_skymodelstate_alloc_init,
 * third_party/hosek/ArHosekSkyModel.cc:602-635, in double): config = configs[0..2][0..8] (27 doubles),
 * radiance = radiances[0..2]; bit-identical to the reference. The model's tables cover turbidity
 * 1..10 and ground albedo 0..1: other values give LRT_ERR_RANGE (the reference reads outside its
 * tables there). lrt_scene_upload cooks the state itself when an env emitter's hosek_config is all
 * zero. */
int lrt_hosek_state(const float* sun_direction /* 3 */, float turbidity, float albedo, double* config /* 27 */,
                    double* radiance /* 3 */);
/* The same table in two steps, so that a caller without ggx.dat can re-slice for any alpha: the eta
 * slice (set_eta, rough_transmittance.h:129-167) = n_alpha x LRT_TRANS_SAMPLES transmittance values
 * (alpha-major) and n_alpha diffuse values, with the file's alpha range; then set_alpha on it
 * (rough_transmittance.h:169-185). `capacity` is the n_alpha the two buffers hold. */
int lrt_rough_transmittance_eta_slice(const char* ggx_path, float eta, float* sliced_table, float* sliced_diffuse,
                                      uint32_t capacity, uint32_t* n_alpha_out, float* alpha_range_out /* 2 */);
int lrt_rough_transmittance_at_alpha(const float* sliced_table, const float* sliced_diffuse, uint32_t n_alpha,
                                     const float* alpha_range /* 2 */, float alpha,
                                     float* table_out /* LRT_TRANS_SAMPLES */, float* diffuse_out);

/* Wavefront OBJ as the reference's load_obj (src/io/obj_loader.h:44-141): 'v', 'vn' and 'f' lines
 * (faces fanned from their first corner; 1-based or negative indices; corners "p", "p/t", "p//n",
 * "p/t/n"), triangles with a zero-length cross product dropped, corners without a normal given the
 * triangle's unit geometric normal, positions centred on the box of the referenced positions and
 * scaled to a longest side of 1. The arrays are those an lrt_object_desc mesh takes. Call with null
 * arrays to get the counts, then with arrays of at least those sizes (capacities in vertices and
 * indices). Errors: LRT_ERR_IO (file), LRT_ERR_INVALID_ARGUMENT (bad index or face, no triangle),
 * LRT_ERR_RANGE (capacity too small). */
int lrt_load_obj(const char* path, uint32_t* n_vertices, uint32_t* n_indices, float* positions,
                 uint32_t vertex_capacity, uint32_t* indices, float* corner_normals, uint32_t index_capacity);

/* Host-only SAH kd-tree build over n primitive bounds (3 floats each in bmin/bmax): the tree
 * sah_kdtree::build makes (src/accelerator/sah_kdtree.h:35-57,175-347), packed depth-first into
 * 8-byte nodes (2 uint32 words each: interior = split bits, right<<2|axis; leaf = first, count<<2|3)
 * with leaf references in leaf order. Returns LRT_ERR_RANGE (and the needed sizes) when the output
 * arrays are too small. */
int lrt_kdtree_build(const float* bmin, const float* bmax, uint32_t n, uint32_t* nodes_out,
                     uint32_t max_nodes, uint32_t* refs_out, uint32_t max_refs, uint32_t* n_nodes,
                     uint32_t* n_refs, uint32_t* depth);

/* The trees lrt_kdtree_build makes, for n_meshes meshes at once, built on the context's GPU: all nodes
 * of a tree level are swept together (event lists sorted once and partitioned stably into the
 * children, SAH costs from prefix counts, the reference's tie, leaf and retract rules). Boxes are
 * concatenated mesh after mesh, counts[m] boxes each (at least 1). Each mesh's packed nodes (2 words
 * each, right-child indices within the mesh) and leaf references follow the previous mesh's in
 * nodes_out / refs_out; node_counts, ref_counts and depths (may be null) get the per-mesh sizes and
 * *total_nodes, *total_refs the totals. LRT_ERR_RANGE when the outputs are too small (the totals are
 * set), LRT_ERR_INVALID_ARGUMENT for a NaN bound or an empty mesh. */
int lrt_kdtree_build_device(lrt_context* ctx, uint32_t n_meshes, const uint32_t* counts, const float* bmin,
                            const float* bmax, uint32_t* nodes_out, uint64_t max_nodes, uint32_t* refs_out,
                            uint64_t max_refs, uint32_t* node_counts, uint32_t* ref_counts, uint32_t* depths,
                            uint64_t* total_nodes, uint64_t* total_refs);

/* scene: builds the per-mesh SAH kd-trees (on the GPU or the host cores, option "kd_build_device") and
 * uploads everything to the device */
int lrt_scene_upload(lrt_context* ctx, const lrt_scene_desc* desc);
/* bytes the last upload copied host->device */
uint64_t lrt_scene_device_bytes(const lrt_context* ctx);
/* replaces the uploaded scene's camera by a constructed camera's own frame (camera.h:20-44 keeps
 * origin, lower_left_corner, horizontal and vertical; the render reads only these), so a caller
 * holding a built camera renders with its exact vectors; LRT_ERR_NO_SCENE before an upload */
int lrt_scene_set_camera_frame(lrt_context* ctx, const float* origin, const float* lower_left_corner,
                               const float* horizontal, const float* vertical);
/* kd-tree of one mesh object: node count, leaf-list length, maximum depth */
int lrt_mesh_tree_info(const lrt_context* ctx, uint32_t object, uint32_t* nodes, uint32_t* refs,
                       uint32_t* depth);

/* closest-hit queries (parity) */
int lrt_trace(lrt_context* ctx, const lrt_ray* rays, uint32_t n, lrt_hit* hits);
int lrt_trace_dev(lrt_context* ctx, const lrt_ray* rays_dev, uint32_t n, lrt_hit* hits_dev);

/* shadow-ray test of path_integrator.h:113-115 towards emitter `light`: blocked[i] = 1 when the
 * closest hit in [t_min, t_max] exists and is not that emitter's shape */
int lrt_occluded(lrt_context* ctx, const lrt_ray* rays, uint32_t n, int32_t light, uint8_t* blocked);

/* BSDF sample + eval + pdf of material `material` for each query (parity) */
int lrt_bsdf_evaluate(lrt_context* ctx, int32_t material, const lrt_bsdf_query* q, uint32_t n,
                      lrt_bsdf_result* out);
/* environment radiance for directions (n * 3 floats in, n * 3 out) */
int lrt_sky_eval(lrt_context* ctx, const float* directions, uint32_t n, float* rgb);
/* sampler values for (pixel, sample) pairs: n_dims floats per pair (parity; src/core/sampler.h:12-27) */
int lrt_sampler_values(lrt_context* ctx, const uint32_t* pixel_sample, uint32_t n, uint32_t n_dims,
                       float* values);
/* camera rays of (pixel, sample) pairs exactly as src/main.cpp:121-132 forms them (parity) */
int lrt_camera_rays(lrt_context* ctx, uint32_t width, uint32_t height, const uint32_t* pixel_sample,
                    uint32_t n, lrt_ray* rays);
/* scene::sample_emitter_direction at (point, u2) and scene::pdf_emitter_direction at (point, dir)
 * (src/core/scene.h:73-108). sample_out: 16 floats per query = ok, direction[3], point[3], 0,0,0,
 * pdf, distance, radiance[3], emitter index. */
int lrt_emitter_query(lrt_context* ctx, const float* points, const float* u2, const float* dirs,
                      uint32_t n, float* sample_out, float* pdf_out);

/* path-traced image: rgb is width*height*3 floats, row-major from row 0 (as src/main.cpp) */
int lrt_render(lrt_context* ctx, const lrt_render_params* params, float* rgb);
int lrt_render_dev(lrt_context* ctx, const lrt_render_params* params, float* rgb_dev);
/* Allocation-free lrt_render_dev (no counterpart in the reference). For callers that must not have a
 * library call cudaMalloc: a cudaMalloc can synchronise the whole device, which a frame loop sharing the
 * GPU with other streams cannot afford, and it fails where the device memory is already committed to a
 * caching allocator or a fixed budget. This entry point allocates nothing: its path state lives in one
 * 32 MiB file-scope device array that every GPU loading the library holds until exit; the caller
 * passes the output buffer and has uploaded the scene. Limits: max_depth <= 64 (LRT_ERR_RANGE beyond).
 * Its first call on a device looks the array up (cudaGetSymbolAddress) and should come before any
 * stream capture; later calls outside a capture look it up again (a device reset between calls gets the
 * new address). Calls share the array: calls that overlap on the GPU race. The render statistics count
 * its paths and launches, but the options count_work and stage_timing are not honoured here (their
 * counters and events would need buffers of their own). */
int lrt_render_dev_noalloc(lrt_context* ctx, const lrt_render_params* params, float* rgb_dev);
/* Device allocations (cudaMalloc, pool allocations) the library has made in this process so far, for
 * callers that check a call allocated nothing (no counterpart in the reference). */
uint64_t lrt_device_allocations(void);

/* One render job of a batch: its own pinhole camera, resolution, samples and (optionally) the material
 * of one object replaced, rendered over the uploaded scene exactly as lrt_render would render it with
 * that camera and material. Its image (width*height*3 floats, layout of lrt_render) starts at float
 * `output_offset` of the batch's output buffer. */
typedef struct lrt_job_desc {
    lrt_camera_desc camera;
    uint32_t width;
    uint32_t height;
    uint32_t spp;
    uint32_t sample_offset;
    int32_t override_object;    /* -1: none */
    int32_t override_material;
    uint64_t output_offset;
} lrt_job_desc;

/* Many jobs in shared waves: the paths of all jobs fill the same wavefront queues, and the launch
 * sequence of one wave is captured once as a CUDA graph and replayed for every wave (the wave cursor
 * lives in device memory). No counterpart in the reference, whose main renders one image; a
 * reference-side caller would otherwise loop lrt_render over its jobs. */
int lrt_render_batch(lrt_context* ctx, const lrt_job_desc* jobs, uint32_t n_jobs, int32_t max_depth,
                     int32_t rr_depth, float* rgb);
int lrt_render_batch_dev(lrt_context* ctx, const lrt_job_desc* jobs, uint32_t n_jobs, int32_t max_depth,
                         int32_t rr_depth, float* rgb_dev);

/* Launch-shape autotuner of lrt_render_batch: times the jobs (spp scaled to about 150M paths per trial)
 * over paths per wave {2^19 .. 2^24}, pixel_tile {1, 4, 8, 16} and blocks_per_sm {0, 2, 3}, one knob at a
 * time from the defaults, and leaves the fastest on the context (the same as lrt_set_option of the
 * three). With a cache_path (a text file, one line per size class: triangles and paths rounded up to
 * powers of two, material and emitter counts), a cached class is applied without timing and a timed one
 * is appended. The knobs change speed only, never images. No reference counterpart. */
typedef struct lrt_launch_config {
    uint32_t wave_capacity;
    uint32_t pixel_tile;
    uint32_t blocks_per_sm;
    uint32_t from_cache;  /* 1: read from cache_path; 0: timed by this call */
    float seconds;        /* the best trial's time */
    uint32_t trials;      /* configurations timed by this call */
} lrt_launch_config;
int lrt_autotune(lrt_context* ctx, const lrt_job_desc* jobs, uint32_t n_jobs, int32_t max_depth, int32_t rr_depth,
                 float* rgb_dev, const char* cache_path, lrt_launch_config* out);

/* The plain GPU path tracer, for comparison: one kernel launch per job, one thread per pixel running
 * the reference's render loop (main.cpp:121-136 over path_integrator::li, path_integrator.h:23-166)
 * with the whole path in registers. Same jobs, output layout and images as lrt_render_batch. */
int lrt_render_plain(lrt_context* ctx, const lrt_job_desc* jobs, uint32_t n_jobs, int32_t max_depth,
                     int32_t rr_depth, float* rgb);
int lrt_render_plain_dev(lrt_context* ctx, const lrt_job_desc* jobs, uint32_t n_jobs, int32_t max_depth,
                         int32_t rr_depth, float* rgb_dev);

/* ---- differentiation: path-replay adjoint of the path tracer ----
 *
 * Parameters are scalars of the material list (an albedo channel, a roughness, a conductor eta/k
 * channel ...). They are moved in groups: group g is described by two full material lists, the
 * scene's list with every parameter of g moved by +steps[g] and by -steps[g] (rough-transmittance
 * tables re-sliced where alpha moved), which the library packs like lrt_scene_upload. A parameter
 * names its group and a colour channel: channel c (0..2) when it moves only channel c of every BSDF
 * value (the three channels of an albedo, of a conductor's eta or k, which therefore share one
 * group), -1 when it moves all channels (then it is its group's only parameter). The adjoint replays
 * every path of the jobs from its sampler state and adds sum over paths of
 * <adjoint[pixel] / spp, dL_path / dparam> into grad, with dL_path/dparam from the derivative of each
 * BSDF value on the path (central difference of the packed +/- records) under detached sampling:
 * sampled directions, lobe choices, Russian roulette and MIS weights do not move with the
 * parameters. No counterpart in the reference. */
#define LRT_MAX_DIFF_PARAMS 64
#define LRT_MAX_ADJOINT_DEPTH 16
#define LRT_MAX_GROUPS_PER_MATERIAL 8
typedef struct lrt_diff_param {
    uint32_t group;
    int32_t channel;
} lrt_diff_param;
/* replace the material values of the uploaded scene (same count, types, nesting and BSDF flags);
 * clears the differentiation setup */
int lrt_scene_update_materials(lrt_context* ctx, const lrt_material_desc* materials, uint32_t n_materials);
/* plus / minus: n_groups consecutive material lists of the scene's material count each */
int lrt_diff_setup(lrt_context* ctx, uint32_t n_groups, const float* steps, const lrt_material_desc* plus,
                   const lrt_material_desc* minus, uint32_t n_params, const lrt_diff_param* params);
/* adjoint: dLoss/dimage in the batch output layout of `jobs`; grad: n_params doubles, added to */
int lrt_render_adjoint(lrt_context* ctx, const lrt_job_desc* jobs, uint32_t n_jobs, int32_t max_depth,
                       int32_t rr_depth, const float* adjoint, double* grad);
int lrt_render_adjoint_dev(lrt_context* ctx, const lrt_job_desc* jobs, uint32_t n_jobs, int32_t max_depth,
                           int32_t rr_depth, const float* adjoint_dev, double* grad_dev);

/* statistics of the renders since the last reset; counting adds per-ray node/triangle counters */
int lrt_render_stats_get(lrt_context* ctx, lrt_render_stats* out);
int lrt_render_stats_reset(lrt_context* ctx);
/* options: "stage_timing", "count_work" (0/1), "wave_capacity" (paths per wave, 1024..2^26;
 * 0, the default: 2^24 for forward renders, 2^21 for adjoint renders; a wave never holds more paths than
 * its call renders),
 * "photon_eye_slot_mb" (8192: device memory for the wavefront eye pass's sample slots, up to 2^20 slots),
 * "photon_eye_sort" (1, the default: the wavefront eye pass shades its slots grouped by the material type of
 * the surface each walk resumes on; 0: in slot order -- same images),
 * "photon_eye_tail" (65536: once every sample of a wavefront eye pass has started and at most this many
 * queries are queued, the remaining walks finish in place, one thread each; 0: never -- same images),
 * "knn_shared_heap" (1, the default: irradiance lookups with k <= 64 keep their k-nearest heaps in shared memory;
 * 0: in local memory -- same results),
 * "batch_queue" (0, the default: batches as shared path waves; 1: one persistent megakernel that pulls
 * (job, 32-pixel tile) items from a device queue, costliest jobs first -- identical images),
 * "photon_tree_device" (1, the default: photon maps' kd-trees built on the GPU; 0: on the host cores with
 * std::nth_element; the trees are identical), "photon_tree_depth_limit" (-1, the default: the partition
 * budget std::nth_element gives a node, 2*floor(log2(n)); k >= 0: k partitions, then the heap selection
 * -- a test setting for that path), "batch_graph" (1: one CUDA graph per wave sequence, 0: direct launches),
 * "adjoint_megakernel" (1: the one-thread-per-path adjoint instead of the wavefront one),
 * "blocks_per_sm" (cap on resident blocks per SM of every grid, 0: occupancy's maximum),
 * "pixel_tile" (batch path order: bands of this many rows walked column by column; 1: row-major),
 * "kd_build_device" (where lrt_scene_upload builds the meshes' kd-trees, the same trees either way: 0 the
 * host cores, 1 the GPU, 2 (default) the GPU for scenes of at least 2^15 triangles), "object_bvh" (1: scenes of more than 16 objects are walked through a hierarchy over the objects'
 * boxes; 0: the object list in order, as hittable_list::hit does), "photon_eye_kernel" (the
 * photon-mapper eye pass: 2 wavefront -- samples in device-memory slots, their rays traced in queues
 * by the persistent traversal; 1: persistent lanes tracing a warp's rays together; 0: one camera
 * sample per thread tracing each ray where it is issued). The last six change speed only, never an
 * image or a hit. */
int lrt_set_option(lrt_context* ctx, const char* name, int64_t value);

/* photons: particles [0, ...) traced in index order until `requested` photons are stored */
int lrt_photon_trace(lrt_context* ctx, int32_t kind, uint32_t requested, int32_t max_depth,
                     int32_t rr_depth, lrt_photon* photons_out, uint32_t* n_out, uint64_t* shot_out);
/* photons of particles [first, first+count), with per-particle photon counts (parity) */
int lrt_photon_trace_particles(lrt_context* ctx, int32_t kind, uint32_t first, uint32_t count,
                               int32_t max_depth, int32_t rr_depth, uint32_t max_per_particle,
                               lrt_photon* photons_out, uint32_t* counts_out);
int lrt_photon_map_build(lrt_context* ctx, int32_t map, const lrt_photon* photons, uint32_t n,
                         float scale);
/* The built map's tree (photon_map.h:74-81): order[i] = the index (in the array given to the build) of
 * the photon at tree position i; nodes: 4 words per node in depth-first order -- interior {left,
 * right, axis, split as float bits}, leaf {first photon, count, 3, 0}. n_nodes gets the node count
 * (max_nodes too small: LRT_ERR_RANGE). */
int lrt_photon_map_tree(lrt_context* ctx, int32_t map, uint32_t* order, int32_t* nodes, uint64_t max_nodes,
                        uint32_t* n_nodes);
/* k nearest photons within squared radius r2 (photon_map.h:117-165). Indices refer to the array
 * given to lrt_photon_map_build; each query's results are sorted by (d2, index) descending as the
 * reference pops its max-heap. */
int lrt_photon_knn(lrt_context* ctx, int32_t map, const float* points, uint32_t n, float r2,
                   uint32_t k, uint32_t* idx_out, float* d2_out, uint32_t* count_out);
/* The same with caller-owned device buffers (points, normals: 3 floats each; rgb_dev: 3 floats per
 * query), ordered on the context's stream, no synchronisation. */
int lrt_photon_irradiance_dev(lrt_context* ctx, int32_t map, const float* points_dev, const float* normals_dev,
                              uint32_t n, float radius, int32_t max_depth, uint32_t k, float* rgb_dev);
int lrt_photon_irradiance(lrt_context* ctx, int32_t map, const float* points, const float* normals,
                          uint32_t n, float radius, int32_t max_depth, uint32_t k, float* rgb_out);

/* photon-mapper eye pass settings (photon_integrator.h:15-17,57-65) */
typedef struct lrt_photon_render_params {
    int32_t global_map;          /* photon map id, -1 = empty */
    int32_t caustic_map;
    float global_radius;
    float caustic_radius;
    int32_t max_depth;           /* 128 in the reference */
    int32_t max_specular_depth;  /* 4 */
    int32_t direct_samples;      /* 16 */
    int32_t glossy_samples;      /* 32 */
    uint32_t lookup_size;        /* k, 120 in the reference; at most 128 */
} lrt_photon_render_params;

/* photon_integrator::preprocess (photon_integrator.h:15-37): radii 0.05 R and 0.0125 R of the scene's
 * bounding sphere (each capped at radius_cap; pass INFINITY for none), a global gather and -- when the
 * scene has a specular BSDF -- a caustic gather with photon depth max_depth - 1, and maps 0 / 1 for the
 * gathers that stored their request. Fills the map ids and radii of *out; shots[2] gets the particle
 * counts (may be null). */
int lrt_photon_preprocess(lrt_context* ctx, uint32_t global_photons, uint32_t caustic_photons,
                          int32_t max_depth, int32_t rr_depth, float radius_cap,
                          lrt_photon_render_params* out, uint64_t* shots);
/* photon-mapper image: photon_integrator::radiance for every (pixel, sample) of the tile loop of
 * src/main.cpp:103-147 */
int lrt_render_photon(lrt_context* ctx, const lrt_render_params* params, const lrt_photon_render_params* pp,
                      float* rgb);
int lrt_render_photon_dev(lrt_context* ctx, const lrt_render_params* params,
                          const lrt_photon_render_params* pp, float* rgb_dev);

#ifdef __cplusplus
}
#endif

#endif /* LRT_H */
