// lrt_context.cuh — the context object behind the C ABI and small device/launch helpers shared by
// the library's translation units.
#pragma once

#include <cuda_runtime.h>

#include <atomic>

#include <cstdarg>
#include <cstdio>
#include <string>
#include <vector>

#include "lrt.h"
#include "lrt_host.h"
#include "lrt_math.cuh"
#include "lrt_types.h"

namespace lrt {

// device allocations the library has made in this process (lrt_device_allocations)
inline std::atomic<uint64_t> g_device_allocations{0};

struct DevBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    void release() {
        if(ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
    }
    cudaError_t ensure(size_t n) {
        if(n <= bytes) return cudaSuccess;
        release();
        cudaError_t e = cudaMalloc(&ptr, n);
        if(e == cudaSuccess) {
            bytes = n;
            ++g_device_allocations;
        }
        return e;
    }
    template <typename T>
    T* as() const { return static_cast<T*>(ptr); }
};

constexpr int kKeys = 10;  // shading keys: 0 miss, 1 hit without BSDF, 2 + material type
constexpr int kBlock = 128;
constexpr int kMaxPhotonMaps = 4;
constexpr uint32_t kMaxKnn = 128;

// per-bounce device counters of one wave. The active and shadow queues have two segments of
// `capacity` entries: rays that may reach the box of a heavy mesh (segment 1) and the others, so that a
// warp's rays share the cost of the large traversals.
struct BounceCounters {
    uint32_t active[2];  // paths entering this bounce, per segment
    uint32_t shadow[2];  // shadow rays emitted by this bounce, per segment
    uint32_t key_count[kKeys];
    uint32_t pad[2];
};
static_assert(sizeof(BounceCounters) == 64, "counter layout");

struct WaveState {
    uint32_t capacity = 0;
    DevBuf o, d, tp, L, misc, id, hit_p, hit_n, q0, q1, keyed, sh_o, sh_d, sh_c, sh_s, sum;
};

// photon map in tree order: positions carry the caller's index in w (bits)
struct PhotonNode {
    int32_t a;      // interior: left child; leaf: first photon
    int32_t b;      // interior: right child; leaf: photon count
    int32_t axis;   // 0..2, or 3 for a leaf
    float split;
};

struct PhotonMap {
    uint32_t n = 0;
    float scale = 1.0f;
    DevBuf pos;     // float4 x, y, z, caller index
    DevBuf dir;     // float4 direction, depth (as float)
    DevBuf nrm;     // float4 normal
    DevBuf pow;     // float4 power
    DevBuf nodes;   // PhotonNode
    uint32_t n_nodes = 0;
    uint32_t depth = 0;
};

}  // namespace lrt

struct lrt_context {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int sm_count = 0;
    std::string error;
    // scene
    bool has_scene = false;
    lrt::HostScene host;
    lrt::DeviceScene ds{};
    lrt::DevBuf nodes, tris, ref_prim, normals, objects, materials, tables, emitters, emission, sobol, tlas, tlas_objs;
    lrt::DevBuf light_cdf, light_tri;
    bool object_bvh = true;  // false: walk the object list in order even where a hierarchy was built
    uint64_t scene_bytes = 0;
    // render
    lrt::WaveState wave;
    lrt::DevBuf out_rgb, scratch_a, scratch_b, counters;
    lrt::DevBuf batch_jobs, batch_path_job, batch_sums, batch_cursor, batch_out;
    bool batch_graph = true;
    // differentiation: per parameter the material list moved by +step and by -step
    uint32_t diff_params = 0;  // 0: no lrt_diff_setup for the current materials
    uint32_t diff_groups = 0;
    uint32_t diff_kmax = 0;             // most groups that move one material
    bool adjoint_megakernel = false;    // true: the one-thread-per-path adjoint kernel
    lrt::DevBuf adj_vmask, adj_vmid, adj_lsnap, adj_dlog, adj_sh_mid, adj_sh_vis, adj_sh_prod;
    lrt::DevBuf diff_mats, diff_tables, diff_inv2step, diff_aff_begin, diff_aff_list, diff_group_begin,
        diff_group_params, diff_adjoint, diff_grad;
    lrt_render_stats stats{};
    bool stage_timing = false;
    bool count_work = false;
    uint32_t wave_capacity = 0;      // paths per wave; 0: kForwardWaveCapacity / kAdjointWaveCapacity
    uint32_t blocks_per_sm_cap = 0;  // 0: as many resident blocks per SM as occupancy allows
    uint32_t pixel_tile = 1;         // batch path order: bands of this many rows, column by column
    std::vector<cudaEvent_t> events;
    std::vector<int> event_stage;
    // photons
    uint64_t photon_eye_slot_mb = 8192;  // device memory for the wavefront eye pass's slots (frames, queries)
    bool photon_eye_sort = true;  // the wavefront eye pass shades slots grouped by the surface's material type
    uint32_t photon_eye_tail = 65536;  // queued queries below which the eye pass finishes its walks in place
    bool knn_shared_heap = true;  // photon lookups keep their k-NN heaps in shared memory (false: local memory)
    bool batch_queue = false;  // true: a batch as one persistent megakernel over (job, tile) items
    bool photon_tree_device = true;  // the reference's photon tree built on the GPU (false: on the host cores)
    int photon_tree_depth_limit = -1;  // introselect's partition budget per node (-1: 2*floor(log2(n)), as std::nth_element)
    bool shade_per_key = true;  // one shading kernel per material type present (false: one for all)
    uint32_t shade_keys = 3u;    // bit k: shading key k can occur in the uploaded scene
    bool has_mesh_lights = false;
    bool has_sky = false;  // an env emitter: the path tracer's sky NEE radiance is evaluated after visibility  // a mesh is an area light: the one all-keys shading kernel runs
    int kd_build_device = 2;  // lrt_scene_upload's kd-trees: 0 host cores, 1 GPU, 2 GPU from 2^15 triangles
    int photon_eye_kernel = 2;  // 0: one sample per thread; 1: persistent lanes; 2: wavefront slots
    lrt::DevBuf eye_slots, eye_frames, eye_queue, eye_L, eye_queries;
    lrt::DevBuf knn_work;  // k-NN counters (option count_work): queries, nodes, photons tested, found
    lrt::PhotonMap maps[lrt::kMaxPhotonMaps];
    lrt::DevBuf ph_counts, ph_offsets, ph_out, ph_tmp, ph_keys, ph_vals, ph_cub, ph_seg, ph_eye, ph_stage;
};

namespace lrt {

inline int fail(lrt_context* ctx, int code, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if(ctx) ctx->error = buf;
    return code;
}

// A failed runtime call also sets the thread's last-error state; it is cleared here so that the next
// launch check (cudaGetLastError) of a later call does not report this failure again.
#define LRT_CUDA(ctx, call)                                                                                   \
    do {                                                                                                      \
        cudaError_t e_ = (call);                                                                              \
        if(e_ != cudaSuccess) {                                                                               \
            (void)cudaGetLastError();                                                                         \
            return ::lrt::fail(ctx, e_ == cudaErrorMemoryAllocation ? LRT_ERR_OUT_OF_MEMORY : LRT_ERR_CUDA,   \
                               "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__);          \
        }                                                                                                     \
    } while(0)

// A batch's jobs as one persistent megakernel launch pulling (job, tile) items from a device queue
// (lrt_plain.cu, option batch_queue); images identical to the per-job plain launches.
int render_batch_queue(lrt_context* ctx, const std::vector<JobRec>& recs, unsigned long long total, int32_t max_depth,
                       int32_t rr_depth, float* rgb_dev);

// The photon map's kd-tree of photons_dev built on the GPU, identical to photon_map::build's
// (lrt_photon_tree.cu); fills pm's search arrays and nodes.
int photon_tree_build_device(lrt_context* ctx, PhotonMap& pm, const lrt_photon* photons_dev, uint32_t n,
                             int depth_limit);

// Validates a batch's jobs and lays out their path ranges (pixel-major, samples inner) and outputs;
// total = the batch's paths, out_floats = the output floats the jobs reach.
int job_records(lrt_context* ctx, const lrt_job_desc* jobs, uint32_t n_jobs, std::vector<JobRec>& recs,
                unsigned long long& total, unsigned long long& out_floats);

// The kd-trees of several meshes built together on the context's GPU (lrt_kdbuild.cu); the trees are
// those build_kdtree makes. Signature of a KdBatchBuilder.
int build_kdtrees_device(lrt_context* ctx, const std::vector<uint32_t>& counts, const BigVec<float>& bmin,
                         const BigVec<float>& bmax, std::vector<PackedTree>& out, std::string& err);

inline uint32_t blocks_for(uint32_t n) { return (n + kBlock - 1) / kBlock; }

inline int grid_for(lrt_context* ctx, const void* kernel, int block) {
    int per_sm = 0;
    if(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, 0) != cudaSuccess || per_sm < 1) per_sm = 1;
    if(ctx->blocks_per_sm_cap > 0 && per_sm > static_cast<int>(ctx->blocks_per_sm_cap)) {
        per_sm = static_cast<int>(ctx->blocks_per_sm_cap);
    }
    return ctx->sm_count * per_sm;
}

#ifdef __CUDACC__
__device__ __forceinline__ const uint32_t (*sobol_table(const DeviceScene& s))[32] {
    return reinterpret_cast<const uint32_t(*)[32]>(s.sobol);
}

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

// warp-aggregated append: one atomic per warp (ballot + popc), slot per lane
__device__ __forceinline__ uint32_t warp_append(uint32_t* counter) {
    const uint32_t mask = __activemask();
    const int leader = __ffs(mask) - 1;
    uint32_t base = 0;
    if(static_cast<int>(lane_id()) == leader) base = atomicAdd(counter, static_cast<uint32_t>(__popc(mask)));
    base = __shfl_sync(mask, base, leader);
    return base + __popc(mask & ((1u << lane_id()) - 1u));
}

// warp-aggregated append into one of several queues: lanes with equal keys share one atomic
__device__ __forceinline__ uint32_t warp_append_keyed(uint32_t* counters, int key) {
    const uint32_t active = __activemask();
    const uint32_t peers = __match_any_sync(active, key);
    const int leader = __ffs(peers) - 1;
    uint32_t base = 0;
    if(static_cast<int>(lane_id()) == leader) base = atomicAdd(counters + key, static_cast<uint32_t>(__popc(peers)));
    base = __shfl_sync(peers, base, leader);
    return base + __popc(peers & ((1u << lane_id()) - 1u));
}

__device__ __forceinline__ uint32_t lanemask_lt() { return (1u << lane_id()) - 1u; }

// fetch queue indices for the idle lanes of a warp (all 32 lanes call it): this lane's index, or >= n
__device__ __forceinline__ uint32_t warp_fetch(uint32_t* counter, bool idle, uint32_t n, bool& exhausted) {
    const unsigned full = 0xffffffffu;
    const unsigned want = __ballot_sync(full, idle);
    uint32_t base = 0;
    const int leader = __ffs(want) - 1;
    if(static_cast<int>(lane_id()) == leader) base = atomicAdd(counter, static_cast<uint32_t>(__popc(want)));
    base = __shfl_sync(full, base, leader);
    if(base + static_cast<uint32_t>(__popc(want)) >= n) exhausted = true;
    return base + __popc(want & lanemask_lt());
}

// warp reduce then one atomic per warp
__device__ __forceinline__ void add_count(unsigned long long* dst, uint32_t v) {
    const uint32_t mask = __activemask();
    unsigned long long x = v;
    for(int off = 16; off > 0; off >>= 1) x += __shfl_down_sync(mask, x, off);
    if(lane_id() == static_cast<uint32_t>(__ffs(mask) - 1) && x) atomicAdd(dst, x);
}
#endif

}  // namespace lrt
