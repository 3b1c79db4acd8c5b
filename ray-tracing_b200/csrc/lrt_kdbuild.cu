// lrt_kdbuild.cu — SAH kd-tree build on the GPU: the tree sah_kdtree::build makes
// (src/accelerator/sah_kdtree.h:35-57, 141-347), for many meshes at once.
//
// The reference builds depth first and sorts every node's events anew. This build runs level by level
// over all nodes of all meshes together:
//   1. every primitive's sweep events (start and end per axis, one planar event on an axis where the
//      box is flat) are sorted once by (mesh, axis, position, type), primitive order kept among equal
//      keys, with an LSD radix sort. A child's events are its primitives' events unchanged (boxes are
//      not clipped), a subsequence of its parent's sorted list, so a stable partition hands every
//      node the list it would have sorted itself;
//   2. per level, exclusive scans of per-event counts give, at each group of events with equal axis
//      and position, the primitives left and right of that plane exactly as the reference's sweep
//      counts them (sah_kdtree.h:233-283). Each group's SAH cost enters a per-node minimum keyed by
//      (cost, event index): the first minimum in sweep order wins, as the sweep's strict `<` does;
//   3. each node takes the reference's decision (leaf rules, bad refines, sah_kdtree.h:183-190,
//      285-288) and its primitive list and events are partitioned stably into its two children
//      (the side rules of sah_kdtree.h:290-306);
//   4. once no node splits, costs run bottom up and a node whose split costs no less than a leaf is
//      retracted to one (sah_kdtree.h:330-345); the reachable nodes are laid out depth first into the
//      packed 8-byte format with leaf references in leaf order.
// Every float expression is the host builder's, in its order (the library is built with -fmad=false),
// so costs, and with them the chosen planes, are bit-identical.
#include "lrt_context.cuh"

#include <algorithm>
#include <memory>

namespace lrt {

namespace {

constexpr float kTraversalCost = 15.0f;
constexpr float kQueryCost = 20.0f;
constexpr float kEmptySpaceBonus = 0.9f;
constexpr uint32_t kStopPrims = 6;
constexpr uint32_t kMaxBadRefines = 3;
constexpr int kMaxLevels = 64;  // the depth limit is at most 48

constexpr int kThreads = 256;

// grid of a grid-stride loop over n items
inline int grid_of(size_t n) {
    return static_cast<int>(std::max<size_t>(1, std::min<size_t>((n + kThreads - 1) / kThreads, 148 * 32)));
}
// grid of one thread per item (per-node kernels)
inline int grid_each(size_t n) { return static_cast<int>(std::max<size_t>(1, (n + kThreads - 1) / kThreads)); }

// ------------------------------------------------------------------------------------------------
// device memory: the build's buffers grow level by level; they come from a stream-ordered pool of this
// build (released at its end), so growing one neither synchronises nor returns memory to the driver

struct BuildPool {
    cudaMemPool_t pool = nullptr;
    cudaStream_t stream = nullptr;
    cudaError_t create(int device, cudaStream_t s) {
        stream = s;
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        cudaError_t e = cudaMemPoolCreate(&pool, &props);
        if(e != cudaSuccess) return e;
        uint64_t keep = ~0ull;  // keep freed blocks for reuse until the pool is destroyed
        return cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    ~BuildPool() {
        if(pool) cudaMemPoolDestroy(pool);  // memory still in flight is released when its frees complete
    }
};
thread_local BuildPool* t_pool = nullptr;

struct PBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
    PBuf() = default;
    PBuf(const PBuf&) = delete;
    PBuf& operator=(const PBuf&) = delete;
    ~PBuf() { release(); }
    void release() {
        if(ptr) cudaFreeAsync(ptr, t_pool->stream);
        ptr = nullptr;
        bytes = 0;
    }
    // at least n bytes, growing by a quarter more than asked; the contents are not kept
    cudaError_t ensure(size_t n) {
        if(n <= bytes) return cudaSuccess;
        release();
        n += n / 4;
        const cudaError_t e = cudaMallocFromPoolAsync(&ptr, n, t_pool->pool, t_pool->stream);
        if(e == cudaSuccess) ++g_device_allocations;
        if(e == cudaSuccess) bytes = n;
        return e;
    }
    template <typename T>
    T* as() const {
        return static_cast<T*>(ptr);
    }
};

// ------------------------------------------------------------------------------------------------
// exclusive scans (out has n + 1 entries; out[n] is the total)

struct U2 {
    uint32_t a, b;
};
struct U4 {
    uint32_t a, b, c, d;
};
__host__ __device__ inline U2 operator+(U2 x, U2 y) { return U2{x.a + y.a, x.b + y.b}; }
__host__ __device__ inline U4 operator+(U4 x, U4 y) { return U4{x.a + y.a, x.b + y.b, x.c + y.c, x.d + y.d}; }
__host__ __device__ inline uint32_t zero_of(uint32_t) { return 0u; }
__host__ __device__ inline U2 zero_of(U2) { return U2{0u, 0u}; }
__host__ __device__ inline U4 zero_of(U4) { return U4{0u, 0u, 0u, 0u}; }

constexpr int kScanPer = 4;
constexpr int kScanTile = kThreads * kScanPer;

// exclusive scan of one value per thread over the block; `total` gets the block's sum
template <typename T>
__device__ T block_exclusive(T v, T* sh, T& total) {
    const int tid = threadIdx.x;
    sh[tid] = v;
    __syncthreads();
    for(int off = 1; off < kThreads; off <<= 1) {
        const T t = tid >= off ? sh[tid - off] : zero_of(v);
        __syncthreads();
        sh[tid] = sh[tid] + t;
        __syncthreads();
    }
    const T excl = tid ? sh[tid - 1] : zero_of(v);
    total = sh[kThreads - 1];
    __syncthreads();
    return excl;
}

// a scan's input: in(i) for i in [0, n), read from an array or computed from the build's arrays
template <typename T>
struct ArrayIn {
    const T* p;
    __device__ T operator()(uint32_t i) const { return p[i]; }
};

template <typename T, typename In>
__global__ void __launch_bounds__(kThreads) k_scan_reduce(In in, uint32_t n, T* sums) {
    __shared__ T sh[kThreads];
    const size_t base = static_cast<size_t>(blockIdx.x) * kScanTile + threadIdx.x * kScanPer;
    T acc = zero_of(T{});
    for(int j = 0; j < kScanPer; ++j) {
        if(base + j < n) acc = acc + in(static_cast<uint32_t>(base + j));
    }
    T total;
    block_exclusive(acc, sh, total);
    if(threadIdx.x == 0) sums[blockIdx.x] = total;
}

template <typename T, typename In>
__global__ void __launch_bounds__(kThreads) k_scan_apply(In in, T* out, uint32_t n, const T* offsets) {
    __shared__ T sh[kThreads];
    const size_t base = static_cast<size_t>(blockIdx.x) * kScanTile + threadIdx.x * kScanPer;
    T v[kScanPer];
    T acc = zero_of(T{});
    for(int j = 0; j < kScanPer; ++j) {
        v[j] = base + j < n ? in(static_cast<uint32_t>(base + j)) : zero_of(T{});
        acc = acc + v[j];
    }
    T total;
    T run = block_exclusive(acc, sh, total);
    const T off = offsets ? offsets[blockIdx.x] : zero_of(T{});
    run = off + run;
    for(int j = 0; j < kScanPer; ++j) {
        if(base + j < n) out[base + j] = run;
        run = run + v[j];
    }
    if(blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) out[n] = off + total;
}

struct ScanTemp {
    PBuf level[8];
};

template <typename T, typename In>
cudaError_t scan_exclusive(In in, T* out, uint32_t n, ScanTemp& tmp, cudaStream_t s, int depth = 0) {
    if(n == 0) return cudaMemsetAsync(out, 0, sizeof(T), s);
    const uint32_t nb = (n + kScanTile - 1) / kScanTile;
    if(nb == 1) {
        k_scan_apply<T, In><<<1, kThreads, 0, s>>>(in, out, n, nullptr);
        return cudaGetLastError();
    }
    if(depth >= 7) return cudaErrorInvalidValue;
    cudaError_t e = tmp.level[depth].ensure(sizeof(T) * (2ull * nb + 1));
    if(e != cudaSuccess) return e;
    T* sums = tmp.level[depth].as<T>();
    T* scanned = sums + nb;
    k_scan_reduce<T, In><<<nb, kThreads, 0, s>>>(in, n, sums);
    e = scan_exclusive(ArrayIn<T>{sums}, scanned, nb, tmp, s, depth + 1);
    if(e != cudaSuccess) return e;
    k_scan_apply<T, In><<<nb, kThreads, 0, s>>>(in, out, n, scanned);
    return cudaGetLastError();
}

// ------------------------------------------------------------------------------------------------
// LSD radix sort of (64-bit key, 32-bit value) pairs, 8 bits per pass, stable

constexpr int kSortRounds = 8;
constexpr int kSortTile = kThreads * kSortRounds;

__global__ void __launch_bounds__(kThreads) k_radix_hist(const uint64_t* keys, uint32_t n, int shift, uint32_t* hist,
                                                         uint32_t n_tiles) {
    __shared__ uint32_t cnt[256];
    cnt[threadIdx.x] = 0;
    __syncthreads();
    const size_t base = static_cast<size_t>(blockIdx.x) * kSortTile;
    for(int r = 0; r < kSortRounds; ++r) {
        const size_t i = base + r * kThreads + threadIdx.x;
        if(i < n) atomicAdd(&cnt[(keys[i] >> shift) & 255u], 1u);
    }
    __syncthreads();
    hist[static_cast<size_t>(threadIdx.x) * n_tiles + blockIdx.x] = cnt[threadIdx.x];
}

// Items of a tile go in rounds of 256 consecutive items; within a round a lane's rank among the
// warp's lanes with its digit, then the warps' counts in warp order, keep the order of equal digits.
__global__ void __launch_bounds__(kThreads) k_radix_scatter(const uint64_t* kin, const uint32_t* vin, uint64_t* kout,
                                                            uint32_t* vout, uint32_t n, int shift,
                                                            const uint32_t* offsets, uint32_t n_tiles) {
    __shared__ uint32_t running[256];
    __shared__ uint32_t wc[kThreads / 32][256];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    running[tid] = offsets[static_cast<size_t>(tid) * n_tiles + blockIdx.x];
    const size_t base = static_cast<size_t>(blockIdx.x) * kSortTile;
    for(int r = 0; r < kSortRounds; ++r) {
        for(int w = 0; w < kThreads / 32; ++w) wc[w][tid] = 0;
        __syncthreads();
        const size_t i = base + r * kThreads + tid;
        const bool valid = i < n;
        uint64_t k = 0;
        uint32_t v = 0, d = 256;
        if(valid) {
            k = kin[i];
            v = vin[i];
            d = static_cast<uint32_t>(k >> shift) & 255u;
        }
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        const uint32_t rank = __popc(peers & ((1u << lane) - 1u));
        if(valid && rank == 0) wc[warp][d] = __popc(peers);
        __syncthreads();
        {
            uint32_t acc = running[tid];
            for(int w = 0; w < kThreads / 32; ++w) {
                const uint32_t c = wc[w][tid];
                wc[w][tid] = acc;
                acc += c;
            }
            running[tid] = acc;
        }
        __syncthreads();
        if(valid) {
            const uint32_t dst = wc[warp][d] + rank;
            kout[dst] = k;
            vout[dst] = v;
        }
        __syncthreads();
    }
}

struct SortBufs {
    PBuf keys2, vals2, hist;
};

// sorts keys[0, n) by bits [0, bits) carrying vals; the result ends in (keys, vals)
cudaError_t radix_sort(uint64_t* keys, uint32_t* vals, uint32_t n, int bits, SortBufs& b, ScanTemp& st, cudaStream_t s) {
    if(n <= 1) return cudaSuccess;
    const uint32_t n_tiles = (n + kSortTile - 1) / kSortTile;
    cudaError_t e;
    if((e = b.keys2.ensure(8ull * n)) != cudaSuccess) return e;
    if((e = b.vals2.ensure(4ull * n)) != cudaSuccess) return e;
    if((e = b.hist.ensure(4ull * (256ull * n_tiles + 1) * 2)) != cudaSuccess) return e;
    uint32_t* hist = b.hist.as<uint32_t>();
    uint32_t* offsets = hist + 256ull * n_tiles + 1;
    uint64_t* ka = keys;
    uint32_t* va = vals;
    uint64_t* kb = b.keys2.as<uint64_t>();
    uint32_t* vb = b.vals2.as<uint32_t>();
    int passes = 0;
    for(int shift = 0; shift < bits; shift += 8, ++passes) {
        k_radix_hist<<<n_tiles, kThreads, 0, s>>>(ka, n, shift, hist, n_tiles);
        if((e = scan_exclusive(ArrayIn<uint32_t>{hist}, offsets, 256u * n_tiles, st, s)) != cudaSuccess) return e;
        k_radix_scatter<<<n_tiles, kThreads, 0, s>>>(ka, va, kb, vb, n, shift, offsets, n_tiles);
        std::swap(ka, kb);
        std::swap(va, vb);
    }
    if(passes & 1) {
        if((e = cudaMemcpyAsync(keys, ka, 8ull * n, cudaMemcpyDeviceToDevice, s)) != cudaSuccess) return e;
        if((e = cudaMemcpyAsync(vals, va, 4ull * n, cudaMemcpyDeviceToDevice, s)) != cudaSuccess) return e;
    }
    return cudaGetLastError();
}

// ------------------------------------------------------------------------------------------------
// the build

struct KdNode {  // a node of the level being split
    float lo[3], hi[3];
    uint32_t ev_begin, ev_count;    // its events in the level's event arrays
    uint32_t pe_begin, prim_count;  // its primitives in the level's primitive list (ascending)
    uint32_t mesh, depth, bad, active;
    // the decision
    uint32_t split, axis, planar_left, bad_next;
    float pos;
};

struct KdRaw {  // a node of the finished tree, one array per level
    float lo[3], hi[3];
    float split;
    uint32_t left, right;           // children in the next level's array
    uint32_t pe_begin, prim_count;  // its primitives in this level's primitive list
    uint32_t mesh, axis, leaf, reach;
    float cost;
    uint32_t sub_nodes, sub_refs;   // reachable nodes and leaf references of its subtree
    uint32_t out_index, out_ref;    // depth-first index and first leaf reference within its mesh
};

struct EventArrays {
    uint32_t* node;
    uint32_t* prim;
    float* pos;
    uint8_t* at;  // axis << 2 | type (0 end, 1 planar, 2 start)
};

struct EventBufs {
    PBuf node, prim, pos, at;
    cudaError_t ensure(size_t n) {
        cudaError_t e;
        if((e = node.ensure(4 * n + 4)) != cudaSuccess) return e;
        if((e = prim.ensure(4 * n + 4)) != cudaSuccess) return e;
        if((e = pos.ensure(4 * n + 4)) != cudaSuccess) return e;
        return at.ensure(n + 4);
    }
    EventArrays view() const { return EventArrays{node.as<uint32_t>(), prim.as<uint32_t>(), pos.as<float>(), at.as<uint8_t>()}; }
};

// aabb::surface_area (aabb.h:24-27)
__device__ inline float surface_area(const float lo[3], const float hi[3]) {
    const float ex = hi[0] - lo[0], ey = hi[1] - lo[1], ez = hi[2] - lo[2];
    return 2.0f * (ex * ey + ex * ez + ey * ez);
}

// sah_kdtree::split_probability (sah_kdtree.h:141-173)
__device__ inline void split_probability(const float lo[3], const float hi[3], uint32_t axis, float left_width,
                                         float right_width, float& p_left, float& p_right) {
    const float ex = hi[0] - lo[0], ey = hi[1] - lo[1], ez = hi[2] - lo[2];
    const float denom = ex * ey + ey * ez + ex * ez;
    const float temp = 1.0f / denom;
    float face, perimeter;
    if(axis == 0) {
        face = ey * ez;
        perimeter = ey + ez;
    } else if(axis == 1) {
        face = ex * ez;
        perimeter = ex + ez;
    } else {
        face = ex * ey;
        perimeter = ex + ey;
    }
    p_left = (face + perimeter * left_width) * temp;
    p_right = (face + perimeter * right_width) * temp;
}

// the leaf rules checked before a node's sweep (sah_kdtree.h:183-190)
__device__ inline uint32_t splittable(const KdNode& n, const int32_t* limits) {
    return !(n.prim_count <= kStopPrims || static_cast<int32_t>(n.depth) >= limits[n.mesh] ||
             surface_area(n.lo, n.hi) <= 0.0f);
}

// which child a primitive goes to: 1 left only, 2 right only, 0 both (sah_kdtree.h:290-306; its end
// event at or below the plane puts it left, its start event at or above puts it right, a planar
// event compares with the plane and the planar_left choice)
__device__ inline uint32_t side_of(float lo, float hi, float plane, uint32_t planar_left) {
    if(lo == hi) return (lo < plane || (lo == plane && planar_left)) ? 1u : 2u;
    if(hi <= plane) return 1u;
    if(lo >= plane) return 2u;
    return 0u;
}

// orderable bits of a position with -0 taken as +0 (the sweep compares positions with ==)
__device__ inline uint32_t order_bits(float p) {
    const uint32_t u = __float_as_uint(p == 0.0f ? 0.0f : p);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

// six event slots per primitive: (axis, start-or-planar) and (axis, end); the end slot of a flat
// axis is empty and sorts last
__global__ void k_event_keys(uint32_t n_prims, const float* bmin, const float* bmax, const uint32_t* prim_mesh,
                             uint64_t* keys, uint32_t* vals, uint32_t* error) {
    const size_t n = 6ull * n_prims;
    for(size_t s = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; s < n;
        s += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const uint32_t prim = static_cast<uint32_t>(s / 6);
        const uint32_t axis = static_cast<uint32_t>(s % 6) / 2;
        const uint32_t end = static_cast<uint32_t>(s & 1);
        const float lo = bmin[3ull * prim + axis], hi = bmax[3ull * prim + axis];
        if(lo != lo || hi != hi) atomicOr(error, 1u);
        uint64_t key = ~0ull;
        if(!(end && lo == hi)) {
            const uint32_t type = end ? 0u : (lo == hi ? 1u : 2u);
            key = (static_cast<uint64_t>(prim_mesh[prim]) << 36) | (static_cast<uint64_t>(axis) << 34) |
                  (static_cast<uint64_t>(order_bits(end ? hi : lo)) << 2) | type;
        }
        keys[s] = key;
        vals[s] = static_cast<uint32_t>(s);
    }
}

__global__ void k_event_decode(uint32_t n, const uint64_t* keys, const uint32_t* vals, const float* bmin,
                               const float* bmax, EventArrays ev) {
    for(uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t v = vals[i];
        const uint32_t prim = v / 6;
        const uint32_t axis = (v % 6) / 2;
        const uint32_t end = v & 1u;
        const float lo = bmin[3ull * prim + axis], hi = bmax[3ull * prim + axis];
        const uint32_t type = end ? 0u : (lo == hi ? 1u : 2u);
        ev.node[i] = static_cast<uint32_t>(keys[i] >> 36);
        ev.prim[i] = prim;
        ev.pos[i] = end ? hi : lo;
        ev.at[i] = static_cast<uint8_t>(axis << 2 | type);
    }
}

__global__ void k_level0_prims(uint32_t n, const uint32_t* prim_mesh, uint32_t* pe_prim, uint32_t* pe_node) {
    for(uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        pe_prim[i] = i;
        pe_node[i] = prim_mesh[i];
    }
}

__global__ void k_level0_active(uint32_t k, KdNode* nodes, const int32_t* limits) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i < k) nodes[i].active = splittable(nodes[i], limits);
}

__device__ inline bool group_starts(const EventArrays& ev, uint32_t e, uint32_t begin) {
    return e == begin || (ev.at[e - 1] >> 2) != (ev.at[e] >> 2) || ev.pos[e - 1] != ev.pos[e];
}

// per event: start-or-planar, planar-or-end, planar, first of its (axis, position) group
struct EventCounts {
    EventArrays ev;
    const KdNode* nodes;
    __device__ U4 operator()(uint32_t e) const {
        const uint32_t type = ev.at[e] & 3u;
        const bool head = group_starts(ev, e, nodes[ev.node[e]].ev_begin);
        return U4{type != 0u ? 1u : 0u, type != 2u ? 1u : 0u, type == 1u ? 1u : 0u, head ? 1u : 0u};
    }
};

// the last event of each group, and the first event of each (node, axis) segment
__global__ void k_group_tails(uint32_t n, EventArrays ev, const KdNode* nodes, const U4* scan, uint32_t* tail_of,
                              uint32_t* axis_begin) {
    for(uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const uint32_t node = ev.node[e];
        const KdNode& nd = nodes[node];
        const uint32_t axis = ev.at[e] >> 2;
        if(e == nd.ev_begin || (ev.at[e - 1] >> 2) != axis) axis_begin[3ull * node + axis] = e;
        const bool last = e + 1 == nd.ev_begin + nd.ev_count || group_starts(ev, e + 1, nd.ev_begin);
        if(last) tail_of[scan[e + 1].d - 1] = e;
    }
}

// the sweep's cost at each group (sah_kdtree.h:233-283) into the node's minimum of (cost, event)
__global__ void __launch_bounds__(kThreads) k_group_costs(uint32_t n, EventArrays ev, const KdNode* nodes,
                                                          const U4* scan, const uint32_t* tail_of,
                                                          const uint32_t* axis_begin, unsigned long long* best,
                                                          uint8_t* planar_left_of, uint32_t* error) {
    const uint32_t stride = gridDim.x * blockDim.x;
    for(uint32_t base = blockIdx.x * blockDim.x; base < n; base += stride) {
        const uint32_t e = base + threadIdx.x;
        uint32_t node = 0xffffffffu;
        unsigned long long key = ~0ull;
        if(e < n && scan[e + 1].d != scan[e].d) {
            const uint32_t nd_i = ev.node[e];
            const KdNode& nd = nodes[nd_i];
            const uint32_t axis = ev.at[e] >> 2;
            const float position = ev.pos[e];
            if(nd.active && position > nd.lo[axis] && position < nd.hi[axis]) {
                const uint32_t t = tail_of[scan[e].d];
                const uint32_t ab = axis_begin[3ull * nd_i + axis];
                const int n_l = static_cast<int>(scan[e].a - scan[ab].a);
                const int n_r = static_cast<int>(nd.prim_count) - static_cast<int>(scan[t + 1].b - scan[ab].b);
                const int num_planar = static_cast<int>(scan[t + 1].c - scan[e].c);
                float p_left, p_right;
                split_probability(nd.lo, nd.hi, axis, position - nd.lo[axis], nd.hi[axis] - position, p_left, p_right);
                float cost;
                uint32_t planar_left = 0;
                if(num_planar == 0) {
                    cost = kTraversalCost + kQueryCost * (p_left * static_cast<float>(n_l) + p_right * static_cast<float>(n_r));
                    if(n_l == 0 || n_r == 0) cost *= kEmptySpaceBonus;
                } else {
                    float cost_left = kTraversalCost + kQueryCost * (p_left * static_cast<float>(n_l + num_planar) +
                                                                     p_right * static_cast<float>(n_r));
                    float cost_right = kTraversalCost + kQueryCost * (p_left * static_cast<float>(n_l) +
                                                                      p_right * static_cast<float>(n_r + num_planar));
                    if(n_l + num_planar == 0 || n_r == 0) cost_left *= kEmptySpaceBonus;
                    if(n_l == 0 || n_r + num_planar == 0) cost_right *= kEmptySpaceBonus;
                    if(cost_left != cost_left || cost_right != cost_right) atomicOr(error, 2u);
                    planar_left = cost_left < cost_right ? 1u : 0u;
                    cost = planar_left ? cost_left : cost_right;
                }
                planar_left_of[e] = static_cast<uint8_t>(planar_left);
                if(cost != cost) {
                    atomicOr(error, 2u);
                } else if(cost < __int_as_float(0x7f800000)) {  // an infinite cost never beats the start
                    node = nd_i;
                    key = (static_cast<unsigned long long>(__float_as_uint(cost)) << 32) | e;
                }
            }
        }
        // one atomic per warp where all lanes share the node (costs are positive: their bits order)
        const uint32_t peers = __match_any_sync(0xffffffffu, node);
        if(peers == 0xffffffffu) {
            for(int off = 16; off > 0; off >>= 1) {
                const unsigned long long o = __shfl_xor_sync(0xffffffffu, key, off);
                key = o < key ? o : key;
            }
            if((threadIdx.x & 31) == 0 && node != 0xffffffffu) atomicMin(&best[node], key);
        } else if(node != 0xffffffffu) {
            atomicMin(&best[node], key);
        }
    }
}

// leaf or split (sah_kdtree.h:183-190, 285-288); writes the node's tree record
__global__ void k_node_decide(uint32_t k, KdNode* nodes, const unsigned long long* best, EventArrays ev,
                              const uint8_t* planar_left_of, KdRaw* raw, uint32_t level) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= k) return;
    KdNode& nd = nodes[i];
    KdRaw r{};
    for(int a = 0; a < 3; ++a) {
        r.lo[a] = nd.lo[a];
        r.hi[a] = nd.hi[a];
    }
    r.pe_begin = nd.pe_begin;
    r.prim_count = nd.prim_count;
    r.mesh = nd.mesh;
    r.leaf = 1;
    r.reach = level == 0 ? 1u : 0u;
    uint32_t split = 0;
    if(nd.active) {
        const unsigned long long key = best[i];
        const float best_cost = key == ~0ull ? __int_as_float(0x7f800000) : __uint_as_float(static_cast<uint32_t>(key >> 32));
        const float leaf_cost = static_cast<float>(nd.prim_count) * kQueryCost;
        uint32_t bad = nd.bad;
        split = 1;
        if(best_cost >= leaf_cost) {
            if((best_cost > 4.0f * leaf_cost && nd.prim_count < 16) || bad >= kMaxBadRefines ||
               best_cost == __int_as_float(0x7f800000)) {
                split = 0;
            } else {
                ++bad;
            }
        }
        if(split) {
            const uint32_t h = static_cast<uint32_t>(key);
            nd.axis = ev.at[h] >> 2;
            nd.pos = ev.pos[h];
            nd.planar_left = planar_left_of[h];
            nd.bad_next = bad;
            r.leaf = 0;
            r.axis = nd.axis;
            r.split = nd.pos;
        }
    }
    nd.split = split;
    raw[i] = r;
}

struct SplitFlags {
    const KdNode* nodes;
    __device__ uint32_t operator()(uint32_t i) const { return nodes[i].split; }
};

// (to the left child, to the right child) of an event or a primitive entry
__device__ inline U2 child_flags(const KdNode& nd, uint32_t prim, const float* bmin, const float* bmax) {
    if(!nd.split) return U2{0u, 0u};
    const uint32_t side = side_of(bmin[3ull * prim + nd.axis], bmax[3ull * prim + nd.axis], nd.pos, nd.planar_left);
    return U2{side != 2u ? 1u : 0u, side != 1u ? 1u : 0u};
}

struct EventSides {
    EventArrays ev;
    const KdNode* nodes;
    const float* bmin;
    const float* bmax;
    __device__ U2 operator()(uint32_t e) const { return child_flags(nodes[ev.node[e]], ev.prim[e], bmin, bmax); }
};

struct PrimSides {
    const uint32_t* pe_prim;
    const uint32_t* pe_node;
    const KdNode* nodes;
    const float* bmin;
    const float* bmax;
    __device__ U2 operator()(uint32_t i) const { return child_flags(nodes[pe_node[i]], pe_prim[i], bmin, bmax); }
};

// the two children of every split node, at 2 x (split nodes before it) in the next level
__global__ void k_children(uint32_t k, const KdNode* nodes, const uint32_t* split_scan, const U2* ev_scan,
                           const U2* pe_scan, KdRaw* raw, KdNode* next, const int32_t* limits) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= k) return;
    const KdNode& nd = nodes[i];
    if(!nd.split) return;
    const uint32_t c = 2 * split_scan[i];
    raw[i].left = c;
    raw[i].right = c + 1;
    const uint32_t b = nd.ev_begin, en = nd.ev_begin + nd.ev_count;
    const uint32_t pb = nd.pe_begin, pn = nd.pe_begin + nd.prim_count;
    KdNode L{}, R{};
    for(int a = 0; a < 3; ++a) {
        L.lo[a] = R.lo[a] = nd.lo[a];
        L.hi[a] = R.hi[a] = nd.hi[a];
    }
    L.hi[nd.axis] = nd.pos;
    R.lo[nd.axis] = nd.pos;
    L.ev_begin = ev_scan[b].a + ev_scan[b].b;
    L.ev_count = ev_scan[en].a - ev_scan[b].a;
    R.ev_begin = ev_scan[en].a + ev_scan[b].b;
    R.ev_count = ev_scan[en].b - ev_scan[b].b;
    L.pe_begin = pe_scan[pb].a + pe_scan[pb].b;
    L.prim_count = pe_scan[pn].a - pe_scan[pb].a;
    R.pe_begin = pe_scan[pn].a + pe_scan[pb].b;
    R.prim_count = pe_scan[pn].b - pe_scan[pb].b;
    L.mesh = R.mesh = nd.mesh;
    L.depth = R.depth = nd.depth + 1;
    L.bad = R.bad = nd.bad_next;
    L.active = splittable(L, limits);
    R.active = splittable(R, limits);
    next[c] = L;
    next[c + 1] = R;
}

// stable partition of the events into the children's lists (left child's, then right child's, node
// after node)
__global__ void k_event_scatter(uint32_t n, EventSides sides, const U2* scan, const uint32_t* split_scan,
                                EventArrays out) {
    const EventArrays& ev = sides.ev;
    const KdNode* nodes = sides.nodes;
    for(uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const U2 f = sides(e);
        if(!f.a && !f.b) continue;
        const uint32_t node = ev.node[e];
        const KdNode& nd = nodes[node];
        const uint32_t b = nd.ev_begin, en = nd.ev_begin + nd.ev_count;
        const uint32_t c = 2 * split_scan[node];
        const uint32_t prim = ev.prim[e];
        const float pos = ev.pos[e];
        const uint8_t at = ev.at[e];
        if(f.a) {
            const uint32_t d = scan[e].a + scan[b].b;
            out.node[d] = c;
            out.prim[d] = prim;
            out.pos[d] = pos;
            out.at[d] = at;
        }
        if(f.b) {
            const uint32_t d = scan[en].a + scan[e].b;
            out.node[d] = c + 1;
            out.prim[d] = prim;
            out.pos[d] = pos;
            out.at[d] = at;
        }
    }
}

__global__ void k_prim_scatter(uint32_t n, PrimSides sides, const U2* scan, const uint32_t* split_scan,
                               uint32_t* out_prim, uint32_t* out_node) {
    const uint32_t* pe_prim = sides.pe_prim;
    const uint32_t* pe_node = sides.pe_node;
    const KdNode* nodes = sides.nodes;
    for(uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const U2 f = sides(i);
        if(!f.a && !f.b) continue;
        const uint32_t node = pe_node[i];
        const KdNode& nd = nodes[node];
        const uint32_t pb = nd.pe_begin, pn = nd.pe_begin + nd.prim_count;
        const uint32_t c = 2 * split_scan[node];
        if(f.a) {
            const uint32_t d = scan[i].a + scan[pb].b;
            out_prim[d] = pe_prim[i];
            out_node[d] = c;
        }
        if(f.b) {
            const uint32_t d = scan[pn].a + scan[i].b;
            out_prim[d] = pe_prim[i];
            out_node[d] = c + 1;
        }
    }
}

// bottom up: the cost the reference's build returns for each node, retracting splits that cost no
// less than a leaf (sah_kdtree.h:330-345), and the reachable subtree sizes
__global__ void k_retract(uint32_t k, KdRaw* raw, const KdRaw* next) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= k) return;
    KdRaw& r = raw[i];
    const float leaf_cost = static_cast<float>(r.prim_count) * kQueryCost;
    if(!r.leaf) {
        const KdRaw& L = next[r.left];
        const KdRaw& R = next[r.right];
        float p_left, p_right;
        split_probability(r.lo, r.hi, r.axis, r.split - r.lo[r.axis], r.hi[r.axis] - r.split, p_left, p_right);
        const float final_cost = kTraversalCost + p_left * L.cost + p_right * R.cost;
        if(final_cost < leaf_cost) {
            r.cost = final_cost;
            r.sub_nodes = 1 + L.sub_nodes + R.sub_nodes;
            r.sub_refs = L.sub_refs + R.sub_refs;
            return;
        }
        r.leaf = 1;
    }
    r.cost = leaf_cost;
    r.sub_nodes = 1;
    r.sub_refs = r.prim_count;
}

// top down: depth-first positions of the reachable nodes
__global__ void k_layout(uint32_t k, const KdRaw* raw, KdRaw* next) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= k) return;
    const KdRaw& r = raw[i];
    if(!r.reach || r.leaf) return;
    KdRaw& L = next[r.left];
    KdRaw& R = next[r.right];
    L.reach = R.reach = 1;
    L.out_index = r.out_index + 1;
    L.out_ref = r.out_ref;
    R.out_index = r.out_index + 1 + L.sub_nodes;
    R.out_ref = r.out_ref + L.sub_refs;
}

// packed nodes (interior: split bits, right << 2 | axis; leaf: first, count << 2 | 3) and references
__global__ void k_write(uint32_t k, const KdRaw* raw, const KdRaw* next, const uint32_t* pool, uint32_t level,
                        const uint64_t* node_base, const uint64_t* ref_base, const uint32_t* prim_base,
                        uint2* out_nodes, uint32_t* out_refs, uint32_t* depths) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= k) return;
    const KdRaw& r = raw[i];
    if(!r.reach) return;
    uint2* nodes = out_nodes + node_base[r.mesh];
    if(r.leaf) {
        nodes[r.out_index] = make_uint2(r.out_ref, (r.prim_count << 2) | kLeafTag);
        uint32_t* refs = out_refs + ref_base[r.mesh] + r.out_ref;
        const uint32_t base = prim_base[r.mesh];
        for(uint32_t j = 0; j < r.prim_count; ++j) refs[j] = pool[r.pe_begin + j] - base;
    } else {
        nodes[r.out_index] = make_uint2(__float_as_uint(r.split), (next[r.right].out_index << 2) | r.axis);
    }
    atomicMax(&depths[r.mesh], level + 1);
}

struct LevelStore {
    PBuf raw, pool;
    uint32_t k = 0;
};

}  // namespace

int build_kdtrees_device(lrt_context* ctx, const std::vector<uint32_t>& counts, const BigVec<float>& bmin,
                         const BigVec<float>& bmax, std::vector<PackedTree>& out, std::string& err) {
    cudaStream_t s = ctx->stream;
    BuildPool build_pool;
    LRT_CUDA(ctx, build_pool.create(ctx->device, s));
    struct PoolScope {
        BuildPool* saved;
        explicit PoolScope(BuildPool* p) : saved(t_pool) { t_pool = p; }
        ~PoolScope() { t_pool = saved; }
    } pool_scope(&build_pool);
    const uint32_t n_meshes = static_cast<uint32_t>(counts.size());
    uint64_t total = 0;
    for(const uint32_t c : counts) {
        if(c == 0) {
            err = "kd-tree build: empty mesh";
            return LRT_ERR_INVALID_ARGUMENT;
        }
        total += c;
    }
    if(n_meshes == 0) {
        out.clear();
        return LRT_OK;
    }
    if(bmin.size() != 3 * total || bmax.size() != 3 * total) {
        err = "kd-tree build: box arrays do not match the counts";
        return LRT_ERR_INVALID_ARGUMENT;
    }
    if(6 * total >= (1ull << 32) || n_meshes >= (1u << 20)) {
        err = "kd-tree build: more than 715M primitives or 2^20 meshes";
        return LRT_ERR_RANGE;
    }
    const uint32_t n_prims = static_cast<uint32_t>(total);

    // per mesh: root voxel, depth limit, events, first primitive (host, in the reference's order)
    std::vector<KdNode> roots(n_meshes);
    std::vector<int32_t> limits(n_meshes);
    std::vector<uint32_t> prim_base(n_meshes), prim_mesh(n_prims);
    uint64_t n_events = 0;
    {
        uint64_t first = 0;
        for(uint32_t m = 0; m < n_meshes; ++m) {
            const KdRootInfo info = kd_root_info(bmin.data() + 3 * first, bmax.data() + 3 * first, counts[m]);
            KdNode& r = roots[m];
            r = KdNode{};
            for(int a = 0; a < 3; ++a) {
                r.lo[a] = info.lo[a];
                r.hi[a] = info.hi[a];
            }
            r.ev_begin = static_cast<uint32_t>(n_events);
            r.ev_count = static_cast<uint32_t>(info.n_events);
            r.pe_begin = static_cast<uint32_t>(first);
            r.prim_count = counts[m];
            r.mesh = m;
            r.depth = 1;
            limits[m] = info.depth_limit;
            prim_base[m] = static_cast<uint32_t>(first);
            std::fill(prim_mesh.begin() + first, prim_mesh.begin() + first + counts[m], m);
            n_events += info.n_events;
            first += counts[m];
        }
    }
    const uint32_t mesh_bits = n_meshes > 1 ? 32 - __builtin_clz(n_meshes - 1) : 0;
    const int key_bits = 36 + static_cast<int>(mesh_bits);

    PBuf d_bmin, d_bmax, d_mesh, d_limits, d_err, keys, vals;
    LRT_CUDA(ctx, d_bmin.ensure(4 * bmin.size()));
    LRT_CUDA(ctx, d_bmax.ensure(4 * bmax.size()));
    LRT_CUDA(ctx, d_mesh.ensure(4ull * n_prims));
    LRT_CUDA(ctx, d_limits.ensure(4ull * n_meshes));
    LRT_CUDA(ctx, d_err.ensure(4));
    LRT_CUDA(ctx, cudaMemcpyAsync(d_bmin.ptr, bmin.data(), 4 * bmin.size(), cudaMemcpyHostToDevice, s));
    LRT_CUDA(ctx, cudaMemcpyAsync(d_bmax.ptr, bmax.data(), 4 * bmax.size(), cudaMemcpyHostToDevice, s));
    LRT_CUDA(ctx, cudaMemcpyAsync(d_mesh.ptr, prim_mesh.data(), 4ull * n_prims, cudaMemcpyHostToDevice, s));
    LRT_CUDA(ctx, cudaMemcpyAsync(d_limits.ptr, limits.data(), 4ull * n_meshes, cudaMemcpyHostToDevice, s));
    LRT_CUDA(ctx, cudaMemsetAsync(d_err.ptr, 0, 4, s));
    const float* gmin = d_bmin.as<float>();
    const float* gmax = d_bmax.as<float>();
    const int32_t* glimits = d_limits.as<int32_t>();
    uint32_t* gerr = d_err.as<uint32_t>();

    // ---- the sorted events of the roots
    ScanTemp st;
    EventBufs ev_a, ev_b;
    {
        const uint32_t slots = 6 * n_prims;
        LRT_CUDA(ctx, keys.ensure(8ull * slots));
        LRT_CUDA(ctx, vals.ensure(4ull * slots));
        k_event_keys<<<grid_of(slots), kThreads, 0, s>>>(n_prims, gmin, gmax, d_mesh.as<uint32_t>(), keys.as<uint64_t>(),
                                                         vals.as<uint32_t>(), gerr);
        SortBufs sb;
        LRT_CUDA(ctx, radix_sort(keys.as<uint64_t>(), vals.as<uint32_t>(), slots, key_bits, sb, st, s));
        LRT_CUDA(ctx, ev_a.ensure(n_events));
        k_event_decode<<<grid_of(n_events), kThreads, 0, s>>>(static_cast<uint32_t>(n_events), keys.as<uint64_t>(),
                                                               vals.as<uint32_t>(), gmin, gmax, ev_a.view());
        LRT_CUDA(ctx, cudaGetLastError());
    }
    keys.release();
    vals.release();

    // ---- level by level
    std::vector<std::unique_ptr<LevelStore>> levels;
    PBuf nodes_a, nodes_b, pe_node_a, pe_node_b, scan4, tails, axis_begin, best, plb, split_scan, ev_scan, pe_scan;
    LRT_CUDA(ctx, nodes_a.ensure(sizeof(KdNode) * std::max<size_t>(n_prims / 2 + 1024, n_meshes)));
    LRT_CUDA(ctx, cudaMemcpyAsync(nodes_a.ptr, roots.data(), sizeof(KdNode) * n_meshes, cudaMemcpyHostToDevice, s));
    k_level0_active<<<grid_each(n_meshes), kThreads, 0, s>>>(n_meshes, nodes_a.as<KdNode>(), glimits);
    levels.emplace_back(new LevelStore());
    LRT_CUDA(ctx, levels[0]->pool.ensure(4ull * n_prims));
    LRT_CUDA(ctx, pe_node_a.ensure(4ull * n_prims));
    k_level0_prims<<<grid_of(n_prims), kThreads, 0, s>>>(n_prims, d_mesh.as<uint32_t>(), levels[0]->pool.as<uint32_t>(),
                                                         pe_node_a.as<uint32_t>());
    uint32_t K = n_meshes, E = static_cast<uint32_t>(n_events), P = n_prims;
    {
        // the level buffers at once for twice the root's events (references duplicate as the tree
        // deepens); a level that needs more grows them
        const size_t e2 = 2 * n_events + 1024, p2 = 2ull * n_prims + 1024;
        const size_t k2 = std::max<size_t>(n_prims / 2 + 1024, n_meshes);
        LRT_CUDA(ctx, ev_b.ensure(e2));
        LRT_CUDA(ctx, pe_node_b.ensure(4 * p2));
        LRT_CUDA(ctx, scan4.ensure(sizeof(U4) * e2));
        LRT_CUDA(ctx, ev_scan.ensure(sizeof(U2) * e2));
        LRT_CUDA(ctx, pe_scan.ensure(sizeof(U2) * p2));
        LRT_CUDA(ctx, tails.ensure(4 * e2));
        LRT_CUDA(ctx, plb.ensure(e2));
        LRT_CUDA(ctx, nodes_b.ensure(sizeof(KdNode) * k2));
        LRT_CUDA(ctx, axis_begin.ensure(12 * k2));
        LRT_CUDA(ctx, best.ensure(8 * k2));
        LRT_CUDA(ctx, split_scan.ensure(4 * k2));
    }
    EventBufs* ev_cur = &ev_a;
    EventBufs* ev_next = &ev_b;
    PBuf* nodes_cur = &nodes_a;
    PBuf* nodes_next = &nodes_b;
    PBuf* pen_cur = &pe_node_a;
    PBuf* pen_next = &pe_node_b;
    for(uint32_t level = 0; K > 0; ++level) {
        if(level >= static_cast<uint32_t>(kMaxLevels)) {
            err = "kd-tree build: too many levels";
            return LRT_ERR_RANGE;
        }
        LevelStore& L = *levels[level];
        L.k = K;
        LRT_CUDA(ctx, L.raw.ensure(sizeof(KdRaw) * K));
        LRT_CUDA(ctx, scan4.ensure(sizeof(U4) * (E + 1ull)));
        LRT_CUDA(ctx, tails.ensure(4ull * E + 4));
        LRT_CUDA(ctx, axis_begin.ensure(12ull * K));
        LRT_CUDA(ctx, best.ensure(8ull * K));
        LRT_CUDA(ctx, plb.ensure(E + 4ull));
        LRT_CUDA(ctx, split_scan.ensure(4ull * (K + 1)));
        LRT_CUDA(ctx, ev_scan.ensure(sizeof(U2) * (E + 1ull)));
        LRT_CUDA(ctx, pe_scan.ensure(sizeof(U2) * (P + 1ull)));
        const EventArrays ev = ev_cur->view();
        KdNode* nodes = nodes_cur->as<KdNode>();
        const uint32_t* pe_prim = L.pool.as<uint32_t>();
        const uint32_t* pe_node = pen_cur->as<uint32_t>();

        LRT_CUDA(ctx, cudaMemsetAsync(best.ptr, 0xff, 8ull * K, s));
        LRT_CUDA(ctx, scan_exclusive(EventCounts{ev, nodes}, scan4.as<U4>(), E, st, s));
        if(E) {
            k_group_tails<<<grid_of(E), kThreads, 0, s>>>(E, ev, nodes, scan4.as<U4>(), tails.as<uint32_t>(),
                                                         axis_begin.as<uint32_t>());
            k_group_costs<<<grid_of(E), kThreads, 0, s>>>(E, ev, nodes, scan4.as<U4>(), tails.as<uint32_t>(),
                                                         axis_begin.as<uint32_t>(), best.as<unsigned long long>(),
                                                         plb.as<uint8_t>(), gerr);
        }
        k_node_decide<<<grid_each(K), kThreads, 0, s>>>(K, nodes, best.as<unsigned long long>(), ev, plb.as<uint8_t>(),
                                                      L.raw.as<KdRaw>(), level);
        const EventSides ev_sides{ev, nodes, gmin, gmax};
        const PrimSides pe_sides{pe_prim, pe_node, nodes, gmin, gmax};
        LRT_CUDA(ctx, scan_exclusive(SplitFlags{nodes}, split_scan.as<uint32_t>(), K, st, s));
        LRT_CUDA(ctx, scan_exclusive(ev_sides, ev_scan.as<U2>(), E, st, s));
        LRT_CUDA(ctx, scan_exclusive(pe_sides, pe_scan.as<U2>(), P, st, s));
        LRT_CUDA(ctx, cudaGetLastError());

        uint32_t n_split = 0, error = 0;
        U2 ev_total{0, 0}, pe_total{0, 0};
        LRT_CUDA(ctx, cudaMemcpyAsync(&n_split, split_scan.as<uint32_t>() + K, 4, cudaMemcpyDeviceToHost, s));
        LRT_CUDA(ctx, cudaMemcpyAsync(&ev_total, ev_scan.as<U2>() + E, sizeof(U2), cudaMemcpyDeviceToHost, s));
        LRT_CUDA(ctx, cudaMemcpyAsync(&pe_total, pe_scan.as<U2>() + P, sizeof(U2), cudaMemcpyDeviceToHost, s));
        LRT_CUDA(ctx, cudaMemcpyAsync(&error, gerr, 4, cudaMemcpyDeviceToHost, s));
        LRT_CUDA(ctx, cudaStreamSynchronize(s));
        if(error & 1u) {
            err = "kd-tree build: NaN in a primitive box";
            return LRT_ERR_INVALID_ARGUMENT;
        }
        if(error & 2u) {
            err = "kd-tree build: a split cost is NaN (degenerate voxel)";
            return LRT_ERR_RANGE;
        }
        const uint64_t K2 = 2ull * n_split;
        const uint64_t E2 = static_cast<uint64_t>(ev_total.a) + ev_total.b;
        const uint64_t P2 = static_cast<uint64_t>(pe_total.a) + pe_total.b;
        if(E2 >= (1ull << 32) || P2 >= (1ull << 32)) {
            err = "kd-tree build: more than 2^32 events or references in one level";
            return LRT_ERR_RANGE;
        }
        if(K2 == 0) break;
        levels.emplace_back(new LevelStore());
        LevelStore& N = *levels[level + 1];
        LRT_CUDA(ctx, nodes_next->ensure(sizeof(KdNode) * K2));
        LRT_CUDA(ctx, ev_next->ensure(E2));
        LRT_CUDA(ctx, N.pool.ensure(4 * P2 + 4));
        LRT_CUDA(ctx, pen_next->ensure(4 * P2 + 4));
        k_children<<<grid_each(K), kThreads, 0, s>>>(K, nodes, split_scan.as<uint32_t>(), ev_scan.as<U2>(), pe_scan.as<U2>(),
                                                   L.raw.as<KdRaw>(), nodes_next->as<KdNode>(), glimits);
        if(E) {
            k_event_scatter<<<grid_of(E), kThreads, 0, s>>>(E, ev_sides, ev_scan.as<U2>(), split_scan.as<uint32_t>(),
                                                            ev_next->view());
        }
        if(P) {
            k_prim_scatter<<<grid_of(P), kThreads, 0, s>>>(P, pe_sides, pe_scan.as<U2>(), split_scan.as<uint32_t>(),
                                                           N.pool.as<uint32_t>(), pen_next->as<uint32_t>());
        }
        LRT_CUDA(ctx, cudaGetLastError());
        std::swap(ev_cur, ev_next);
        std::swap(nodes_cur, nodes_next);
        std::swap(pen_cur, pen_next);
        K = static_cast<uint32_t>(K2);
        E = static_cast<uint32_t>(E2);
        P = static_cast<uint32_t>(P2);
    }
    // free the per-level working set before the tree passes
    for(PBuf* b : {&ev_a.node, &ev_a.prim, &ev_a.pos, &ev_a.at, &ev_b.node, &ev_b.prim, &ev_b.pos, &ev_b.at, &scan4,
                     &tails, &ev_scan, &pe_scan, &pe_node_a, &pe_node_b}) {
        b->release();
    }

    // ---- retraction and subtree sizes, bottom up; positions, top down
    const size_t n_levels = levels.size();
    for(size_t l = n_levels; l-- > 0;) {
        const KdRaw* next = l + 1 < n_levels ? levels[l + 1]->raw.as<KdRaw>() : nullptr;
        k_retract<<<grid_each(levels[l]->k), kThreads, 0, s>>>(levels[l]->k, levels[l]->raw.as<KdRaw>(), next);
    }
    for(size_t l = 0; l + 1 < n_levels; ++l) {
        k_layout<<<grid_each(levels[l]->k), kThreads, 0, s>>>(levels[l]->k, levels[l]->raw.as<KdRaw>(),
                                                           levels[l + 1]->raw.as<KdRaw>());
    }
    LRT_CUDA(ctx, cudaGetLastError());
    std::vector<KdRaw> root_raw(n_meshes);
    LRT_CUDA(ctx, cudaMemcpyAsync(root_raw.data(), levels[0]->raw.ptr, sizeof(KdRaw) * n_meshes, cudaMemcpyDeviceToHost, s));
    LRT_CUDA(ctx, cudaStreamSynchronize(s));
    std::vector<uint64_t> node_base(n_meshes + 1, 0), ref_base(n_meshes + 1, 0);
    for(uint32_t m = 0; m < n_meshes; ++m) {
        node_base[m + 1] = node_base[m] + root_raw[m].sub_nodes;
        ref_base[m + 1] = ref_base[m] + root_raw[m].sub_refs;
    }
    PBuf d_node_base, d_ref_base, d_prim_base, d_nodes, d_refs, d_depths;
    LRT_CUDA(ctx, d_node_base.ensure(8ull * n_meshes));
    LRT_CUDA(ctx, d_ref_base.ensure(8ull * n_meshes));
    LRT_CUDA(ctx, d_prim_base.ensure(4ull * n_meshes));
    LRT_CUDA(ctx, d_nodes.ensure(8 * node_base[n_meshes] + 8));
    LRT_CUDA(ctx, d_refs.ensure(4 * ref_base[n_meshes] + 4));
    LRT_CUDA(ctx, d_depths.ensure(4ull * n_meshes));
    LRT_CUDA(ctx, cudaMemcpyAsync(d_node_base.ptr, node_base.data(), 8ull * n_meshes, cudaMemcpyHostToDevice, s));
    LRT_CUDA(ctx, cudaMemcpyAsync(d_ref_base.ptr, ref_base.data(), 8ull * n_meshes, cudaMemcpyHostToDevice, s));
    LRT_CUDA(ctx, cudaMemcpyAsync(d_prim_base.ptr, prim_base.data(), 4ull * n_meshes, cudaMemcpyHostToDevice, s));
    LRT_CUDA(ctx, cudaMemsetAsync(d_depths.ptr, 0, 4ull * n_meshes, s));
    for(size_t l = 0; l < n_levels; ++l) {
        const KdRaw* next = l + 1 < n_levels ? levels[l + 1]->raw.as<KdRaw>() : nullptr;
        k_write<<<grid_each(levels[l]->k), kThreads, 0, s>>>(levels[l]->k, levels[l]->raw.as<KdRaw>(), next,
                                                          levels[l]->pool.as<uint32_t>(), static_cast<uint32_t>(l),
                                                          d_node_base.as<uint64_t>(), d_ref_base.as<uint64_t>(),
                                                          d_prim_base.as<uint32_t>(), d_nodes.as<uint2>(),
                                                          d_refs.as<uint32_t>(), d_depths.as<uint32_t>());
    }
    LRT_CUDA(ctx, cudaGetLastError());
    BigVec<uint2> all_nodes(node_base[n_meshes]);
    BigVec<uint32_t> all_refs(ref_base[n_meshes]);
    std::vector<uint32_t> depths(n_meshes);
    LRT_CUDA(ctx, cudaMemcpyAsync(all_nodes.data(), d_nodes.ptr, 8 * all_nodes.size(), cudaMemcpyDeviceToHost, s));
    LRT_CUDA(ctx, cudaMemcpyAsync(all_refs.data(), d_refs.ptr, 4 * all_refs.size(), cudaMemcpyDeviceToHost, s));
    LRT_CUDA(ctx, cudaMemcpyAsync(depths.data(), d_depths.ptr, 4ull * n_meshes, cudaMemcpyDeviceToHost, s));
    LRT_CUDA(ctx, cudaStreamSynchronize(s));
    out.assign(n_meshes, PackedTree{});
    for(uint32_t m = 0; m < n_meshes; ++m) {
        PackedTree& t = out[m];
        t.nodes.assign(all_nodes.begin() + node_base[m], all_nodes.begin() + node_base[m + 1]);
        t.refs.assign(all_refs.begin() + ref_base[m], all_refs.begin() + ref_base[m + 1]);
        t.depth = depths[m];
    }
    return LRT_OK;
}

}  // namespace lrt
