// lrt_photon_tree.cu — the photon map's kd-tree built on the GPU, identical to the reference's
// photon_map::build_range (photon_map.h:83-114): the same node order, the same photon order and the
// same split values, so that the k-nearest-photon search (photon_map.h:117-165) returns the
// reference's neighbour sets bit for bit.
//
// The reference partitions each node's range with std::nth_element (GCC's libstdc++, the standard
// library the reference is built with): introselect (Musser 1997) -- a median-of-three pivot moved
// to the range's first slot, a Hoare partition of the rest without bounds checks, recursion into the
// side that holds the n-th position, an insertion sort once at most three elements remain, and a
// heap selection once 2*floor(log2(n)) partitions have not finished the job. The arrangement it
// leaves depends on the exact sequence of swaps, and the split of a node is read from the photon at
// the middle position after both children have re-partitioned their ranges, so a tree with the
// reference's k-NN sets has to reproduce that arrangement exactly.
//
// The partition is restated for many threads. In the sequential Hoare loop the left scan stops at
// elements not below the pivot and the right scan at elements not above it; the k-th stop from the
// left swaps with the k-th stop from the right while it lies left of it. With L_k the k-th such
// element from the left and R_k the k-th from the right in the range as it was before the loop, the
// loop performs exactly the swaps (L_k, R_k) for k = 1..K, K = max over x of
// min(#L-stops before x, #R-stops at or after x), and returns min(L_{K+1}, R_K) -- each pair is a
// position the sequential scans reach before any swap changes what they read. A block computes the
// stop counts with block-wide scans, records the positions of the first K stops from each side,
// swaps the K pairs in parallel and finds the cut; pivots, the final insertion sort of at most three
// elements and the (rare) heap selection run on one thread.
//
// Build: one launch per tree level, one block per interior node of that level (larger blocks for
// larger ranges), working on the node's range in place: float4 positions carrying the photon's index,
// plus the split-axis keys of the current level. The node order of the reference's depth-first
// recursion depends only on the range sizes and is laid out on the host; the split values are read
// after the last level. The photons' other attributes are gathered into the search layout at the end.
#include <algorithm>
#include <vector>

#include "lrt_context.cuh"
#include "lrt_math.cuh"

using namespace lrt;

namespace {

constexpr float kTreeInf = __builtin_huge_valf();

struct TreeSeg {
    int32_t start, count, node, pad;
};

__device__ __forceinline__ float axis_value(const float4& p, int axis) {
    return axis == 0 ? p.x : (axis == 1 ? p.y : p.z);
}

__device__ __forceinline__ void swap_slots(float4* pos, float* key, int32_t a, int32_t b) {
    const float4 pa = pos[a];
    pos[a] = pos[b];
    pos[b] = pa;
    const float ka = key[a];
    key[a] = key[b];
    key[b] = ka;
}

// ---- the sequential pieces (one thread) ----

// the median of keys at a, b, c moved to `first` (the pivot choice of the introselect step)
__device__ void median_to_first(float4* pos, float* key, int32_t first, int32_t a, int32_t b, int32_t c) {
    const float ka = key[a], kb = key[b], kc = key[c];
    int32_t m;
    if(ka < kb) {
        m = kb < kc ? b : (ka < kc ? c : a);
    } else {
        m = ka < kc ? a : (kb < kc ? c : b);
    }
    swap_slots(pos, key, first, m);
}

// stable insertion sort of [first, last) by key (at most three elements here)
__device__ void insertion_sort(float4* pos, float* key, int32_t first, int32_t last) {
    for(int32_t i = first + 1; i < last; ++i) {
        const float4 vp = pos[i];
        const float vk = key[i];
        int32_t j = i;
        while(j > first && vk < key[j - 1]) {
            pos[j] = pos[j - 1];
            key[j] = key[j - 1];
            --j;
        }
        pos[j] = vp;
        key[j] = vk;
    }
}

// Binary max-heap on [first, first + len) by key, moved with a hole: the hole at `hole` sinks to a
// leaf, each step into the larger child (the right one unless the left one is strictly larger), then
// the value (vp, vk) rises from there while its parent's key is smaller than vk.
__device__ void heap_sift(float4* pos, float* key, int32_t first, int32_t hole, int32_t len, float4 vp, float vk) {
    const int32_t top = hole;
    int32_t child = hole;
    while(child < (len - 1) / 2) {
        child = 2 * (child + 1);
        if(key[first + child] < key[first + child - 1]) --child;
        pos[first + hole] = pos[first + child];
        key[first + hole] = key[first + child];
        hole = child;
    }
    if((len & 1) == 0 && child == (len - 2) / 2) {
        child = 2 * (child + 1);
        pos[first + hole] = pos[first + child - 1];
        key[first + hole] = key[first + child - 1];
        hole = child - 1;
    }
    int32_t parent = (hole - 1) / 2;
    while(hole > top && key[first + parent] < vk) {
        pos[first + hole] = pos[first + parent];
        key[first + hole] = key[first + parent];
        hole = parent;
        parent = (hole - 1) / 2;
    }
    pos[first + hole] = vp;
    key[first + hole] = vk;
}

// heap selection of the smallest (middle - first) keys into [first, middle), largest of them first
__device__ void heap_select(float4* pos, float* key, int32_t first, int32_t middle, int32_t last) {
    const int32_t len = middle - first;
    if(len >= 2) {
        for(int32_t parent = (len - 2) / 2;; --parent) {
            heap_sift(pos, key, first, parent, len, pos[first + parent], key[first + parent]);
            if(parent == 0) break;
        }
    }
    for(int32_t i = middle; i < last; ++i) {
        if(key[i] < key[first]) {
            const float4 vp = pos[i];
            const float vk = key[i];
            pos[i] = pos[first];
            key[i] = key[first];
            heap_sift(pos, key, first, 0, len, vp, vk);
        }
    }
}

// ---- block-wide helpers ----

// exclusive prefix of a packed pair of counters (high word: left stops, low word: right stops) over
// the block's threads in thread order; `total` gets the block's sum. ws: kThreads / 32 slots.
template <int kThreads>
__device__ __forceinline__ uint64_t block_exclusive_scan(uint64_t v, uint64_t* ws, uint64_t& total) {
    constexpr int kWarps = kThreads / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint64_t inc = v;
#pragma unroll
    for(int d = 1; d < 32; d <<= 1) {
        const uint64_t o = __shfl_up_sync(0xffffffffu, inc, d);
        if(lane >= d) inc += o;
    }
    if(kWarps == 1) {
        total = __shfl_sync(0xffffffffu, inc, 31);
        return inc - v;
    }
    if(lane == 31) ws[warp] = inc;
    __syncthreads();
    if(warp == 0) {
        uint64_t x = lane < kWarps ? ws[lane] : 0;
#pragma unroll
        for(int d = 1; d < 32; d <<= 1) {
            const uint64_t o = __shfl_up_sync(0xffffffffu, x, d);
            if(lane >= d) x += o;
        }
        if(lane < kWarps) ws[lane] = x;
    }
    __syncthreads();
    const uint64_t before = warp > 0 ? ws[warp - 1] : 0;
    total = ws[kWarps - 1];
    __syncthreads();
    return before + inc - v;
}

template <int kThreads>
__device__ __forceinline__ uint64_t block_sum(uint64_t v, uint64_t* ws) {
    uint64_t total;
    block_exclusive_scan<kThreads>(v, ws, total);
    return total;
}

template <int kThreads>
__device__ __forceinline__ int32_t block_max(int32_t v, uint64_t* ws) {
    constexpr int kWarps = kThreads / 32;
#pragma unroll
    for(int d = 16; d > 0; d >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, d));
    if(kWarps == 1) return v;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if(lane == 0) ws[warp] = static_cast<uint64_t>(static_cast<uint32_t>(v));
    __syncthreads();
    int32_t m = 0;
    for(int w = 0; w < kWarps; ++w) m = max(m, static_cast<int32_t>(static_cast<uint32_t>(ws[w])));
    __syncthreads();
    return m;
}

// min (max) over the block with std::min (std::max) semantics; the value is order-independent for the
// finite positions photons have, up to the sign of a zero, which the axis choice does not see
template <int kThreads, bool kMax>
__device__ __forceinline__ float block_extreme(float v, float* wf) {
    constexpr int kWarps = kThreads / 32;
#pragma unroll
    for(int d = 16; d > 0; d >>= 1) {
        const float o = __shfl_xor_sync(0xffffffffu, v, d);
        v = kMax ? smax(v, o) : smin(v, o);
    }
    if(kWarps == 1) return v;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if(lane == 0) wf[warp] = v;
    __syncthreads();
    float m = wf[0];
    for(int w = 1; w < kWarps; ++w) m = kMax ? smax(m, wf[w]) : smin(m, wf[w]);
    __syncthreads();
    return m;
}

// ---- one tree level ----

constexpr int kTreeV = 4;  // consecutive elements per thread in a tile

// One interior node per block: the bounds of its photons and the largest-extent axis
// (photon_map.h:94-100), the axis keys, then std::nth_element(start, start + count / 2, start + count)
// on those keys, restated as described at the top of this file. lp / rp: scratch ranks of the
// partition's stops, indexed inside the node's own range.
template <int kThreads>
__global__ void __launch_bounds__(kThreads) k_tree_level(float4* pos, float* key, int32_t* lp, int32_t* rp,
                                                          const TreeSeg* segs, PhotonNode* nodes, int depth_limit) {
    constexpr int kWarps = kThreads / 32;
    constexpr int kTile = kThreads * kTreeV;
    __shared__ uint64_t ws[kWarps > 1 ? kWarps : 1];
    __shared__ float wf[kWarps > 1 ? kWarps : 1];
    __shared__ int32_t s_first, s_last, s_lnext, s_axis;
    __shared__ float s_pivot;
    const TreeSeg sg = segs[blockIdx.x];
    const int32_t start = sg.start, end = sg.start + sg.count;

    float lo[3] = {kTreeInf, kTreeInf, kTreeInf}, hi[3] = {-kTreeInf, -kTreeInf, -kTreeInf};
    for(int32_t i = start + threadIdx.x; i < end; i += kThreads) {
        const float4 p = pos[i];
        lo[0] = smin(lo[0], p.x);
        lo[1] = smin(lo[1], p.y);
        lo[2] = smin(lo[2], p.z);
        hi[0] = smax(hi[0], p.x);
        hi[1] = smax(hi[1], p.y);
        hi[2] = smax(hi[2], p.z);
    }
#pragma unroll
    for(int a = 0; a < 3; ++a) {
        lo[a] = block_extreme<kThreads, false>(lo[a], wf);
        hi[a] = block_extreme<kThreads, true>(hi[a], wf);
    }
    if(threadIdx.x == 0) {
        const float extent[3] = {hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]};
        int axis = 0;
        if(extent[1] > extent[axis]) axis = 1;
        if(extent[2] > extent[axis]) axis = 2;
        s_axis = axis;
        nodes[sg.node].axis = axis;
    }
    __syncthreads();
    const int axis = s_axis;
    for(int32_t i = start + threadIdx.x; i < end; i += kThreads) key[i] = axis_value(pos[i], axis);
    __syncthreads();

    const int32_t nth = start + sg.count / 2;
    int32_t first = start, last = end;
    int depth = depth_limit >= 0 ? depth_limit : 2 * (31 - __clz(sg.count));
    bool selected = false;
    while(last - first > 3) {
        if(depth == 0) {
            if(threadIdx.x == 0) {
                heap_select(pos, key, first, nth + 1, last);
                swap_slots(pos, key, first, nth);
            }
            selected = true;
            break;
        }
        --depth;
        if(threadIdx.x == 0) {
            median_to_first(pos, key, first, first + 1, first + (last - first) / 2, last - 1);
            s_pivot = key[first];
            s_lnext = INT32_MAX;
        }
        __syncthreads();
        const float pivot = s_pivot;
        const int32_t f = first + 1, l = last;
        // stop counts: left stops are keys not below the pivot, right stops keys not above it
        uint64_t mine = 0;
        for(int32_t base = f; base < l; base += kTile) {
#pragma unroll
            for(int v = 0; v < kTreeV; ++v) {
                const int32_t i = base + threadIdx.x * kTreeV + v;
                if(i < l) {
                    const float k = key[i];
                    mine += (static_cast<uint64_t>(!(k < pivot)) << 32) | static_cast<uint64_t>(!(pivot < k));
                }
            }
        }
        const uint64_t tot = block_sum<kThreads>(mine, ws);
        const int32_t total_right = static_cast<int32_t>(tot & 0xffffffffu);
        // K = max over x of min(left stops before x, right stops at or after x)
        int32_t kmax = 0;
        uint64_t carry = 0;
        for(int32_t base = f; base < l; base += kTile) {
            uint64_t cnt = 0;
            float k4[kTreeV];
#pragma unroll
            for(int v = 0; v < kTreeV; ++v) {
                const int32_t i = base + threadIdx.x * kTreeV + v;
                k4[v] = i < l ? key[i] : 0.0f;
                if(i < l) cnt += (static_cast<uint64_t>(!(k4[v] < pivot)) << 32) | static_cast<uint64_t>(!(pivot < k4[v]));
            }
            uint64_t tile_total;
            uint64_t before = carry + block_exclusive_scan<kThreads>(cnt, ws, tile_total);
            carry += tile_total;
#pragma unroll
            for(int v = 0; v < kTreeV; ++v) {
                const int32_t i = base + threadIdx.x * kTreeV + v;
                if(i < l) {
                    const int32_t cl = static_cast<int32_t>(before >> 32);
                    const int32_t cr = static_cast<int32_t>(before & 0xffffffffu);
                    kmax = max(kmax, min(cl, total_right - cr));
                    before += (static_cast<uint64_t>(!(k4[v] < pivot)) << 32) | static_cast<uint64_t>(!(pivot < k4[v]));
                }
            }
        }
        const int32_t K = block_max<kThreads>(kmax, ws);
        // positions of the first K stops from each side (and of left stop K + 1)
        carry = 0;
        for(int32_t base = f; base < l; base += kTile) {
            uint64_t cnt = 0;
            float k4[kTreeV];
#pragma unroll
            for(int v = 0; v < kTreeV; ++v) {
                const int32_t i = base + threadIdx.x * kTreeV + v;
                k4[v] = i < l ? key[i] : 0.0f;
                if(i < l) cnt += (static_cast<uint64_t>(!(k4[v] < pivot)) << 32) | static_cast<uint64_t>(!(pivot < k4[v]));
            }
            uint64_t tile_total;
            uint64_t before = carry + block_exclusive_scan<kThreads>(cnt, ws, tile_total);
            carry += tile_total;
#pragma unroll
            for(int v = 0; v < kTreeV; ++v) {
                const int32_t i = base + threadIdx.x * kTreeV + v;
                if(i < l) {
                    const bool is_l = !(k4[v] < pivot), is_r = !(pivot < k4[v]);
                    const int32_t cl = static_cast<int32_t>(before >> 32);
                    const int32_t cr = static_cast<int32_t>(before & 0xffffffffu);
                    if(is_l) {
                        if(cl < K) {
                            lp[start + cl] = i;
                        } else if(cl == K) {
                            s_lnext = i;
                        }
                    }
                    if(is_r) {
                        const int32_t rank = total_right - cr;  // right stops at or after i
                        if(rank <= K) rp[start + rank - 1] = i;
                    }
                    before += (static_cast<uint64_t>(is_l) << 32) | static_cast<uint64_t>(is_r);
                }
            }
        }
        __syncthreads();
        for(int32_t k = threadIdx.x; k < K; k += kThreads) swap_slots(pos, key, lp[start + k], rp[start + k]);
        __syncthreads();
        if(threadIdx.x == 0) {
            const int32_t cut = min(s_lnext, K > 0 ? rp[start + K - 1] : l);
            s_first = cut <= nth ? cut : first;
            s_last = cut <= nth ? last : cut;
        }
        __syncthreads();
        first = s_first;
        last = s_last;
    }
    if(!selected && threadIdx.x == 0) insertion_sort(pos, key, first, last);
}

// split of every interior node: the key of the photon at its middle position once every level is done
// (photon_map.h:110 reads it after both children have been built)
__global__ void k_tree_splits(const float4* pos, const TreeSeg* segs, uint32_t n_segs, PhotonNode* nodes) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= n_segs) return;
    const TreeSeg sg = segs[i];
    PhotonNode& nd = nodes[sg.node];
    nd.split = axis_value(pos[sg.start + sg.count / 2], nd.axis);
}

__global__ void k_tree_positions(const lrt_photon* in, uint32_t n, float4* pos) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= n) return;
    pos[i] = make_float4(in[i].position[0], in[i].position[1], in[i].position[2], __uint_as_float(i));
}

// the search layout: direction + depth, normal, power of each photon in tree order
__global__ void k_tree_attrs(const lrt_photon* in, const float4* pos, uint32_t n, float4* dir, float4* nrm, float4* pw) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= n) return;
    const lrt_photon& p = in[__float_as_uint(pos[i].w)];
    dir[i] = make_float4(p.direction[0], p.direction[1], p.direction[2], __int_as_float(static_cast<int>(p.depth)));
    nrm[i] = make_float4(p.normal[0], p.normal[1], p.normal[2], 0.0f);
    pw[i] = make_float4(p.power[0], p.power[1], p.power[2], 0.0f);
}

// The reference's depth-first node order (photon_map.h:83-114): a node, its left subtree, its right
// subtree; a leaf at <= 8 photons. Interior nodes are listed per level for the level launches.
int32_t lay_out(int32_t start, int32_t count, uint32_t depth, std::vector<PhotonNode>& nodes,
                std::vector<std::vector<TreeSeg>>& levels, uint32_t& max_depth) {
    const int32_t index = static_cast<int32_t>(nodes.size());
    nodes.push_back(PhotonNode{start, count, 3, 0.0f});
    max_depth = std::max(max_depth, depth);
    if(count <= 8) return index;
    const int32_t mid = start + count / 2;
    const int32_t left = lay_out(start, mid - start, depth + 1, nodes, levels, max_depth);
    const int32_t right = lay_out(mid, start + count - mid, depth + 1, nodes, levels, max_depth);
    nodes[index] = PhotonNode{left, right, 0, 0.0f};
    if(levels.size() < depth) levels.resize(depth);
    levels[depth - 1].push_back(TreeSeg{start, count, index, 0});
    return index;
}

}  // namespace

namespace lrt {

int photon_tree_build_device(lrt_context* ctx, PhotonMap& pm, const lrt_photon* photons_dev, uint32_t n,
                             int depth_limit) {
    std::vector<PhotonNode> nodes;
    std::vector<std::vector<TreeSeg>> levels;
    nodes.reserve(n / 4 + 16);
    uint32_t max_depth = 0;
    lay_out(0, static_cast<int32_t>(n), 1, nodes, levels, max_depth);
    std::vector<TreeSeg> segs;
    std::vector<size_t> level_begin;
    for(const auto& lv : levels) {
        level_begin.push_back(segs.size());
        segs.insert(segs.end(), lv.begin(), lv.end());
    }
    level_begin.push_back(segs.size());
    cudaStream_t s = ctx->stream;
    LRT_CUDA(ctx, pm.pos.ensure(16ull * n));
    LRT_CUDA(ctx, pm.dir.ensure(16ull * n));
    LRT_CUDA(ctx, pm.nrm.ensure(16ull * n));
    LRT_CUDA(ctx, pm.pow.ensure(16ull * n));
    LRT_CUDA(ctx, pm.nodes.ensure(sizeof(PhotonNode) * nodes.size()));
    LRT_CUDA(ctx, ctx->ph_keys.ensure(4ull * n));
    LRT_CUDA(ctx, ctx->ph_vals.ensure(8ull * n));
    LRT_CUDA(ctx, ctx->ph_seg.ensure(sizeof(TreeSeg) * std::max<size_t>(1, segs.size())));
    LRT_CUDA(ctx, cudaMemcpyAsync(pm.nodes.ptr, nodes.data(), sizeof(PhotonNode) * nodes.size(), cudaMemcpyHostToDevice, s));
    if(!segs.empty()) {
        LRT_CUDA(ctx, cudaMemcpyAsync(ctx->ph_seg.ptr, segs.data(), sizeof(TreeSeg) * segs.size(), cudaMemcpyHostToDevice, s));
    }
    float4* pos = pm.pos.as<float4>();
    float* key = ctx->ph_keys.as<float>();
    int32_t* lp = ctx->ph_vals.as<int32_t>();
    int32_t* rp = lp + n;
    PhotonNode* d_nodes = pm.nodes.as<PhotonNode>();
    const TreeSeg* d_segs = ctx->ph_seg.as<TreeSeg>();
    k_tree_positions<<<(n + 255) / 256, 256, 0, s>>>(photons_dev, n, pos);
    LRT_CUDA(ctx, cudaGetLastError());
    for(size_t lv = 0; lv + 1 < level_begin.size(); ++lv) {
        const size_t b = level_begin[lv], e = level_begin[lv + 1];
        if(b == e) continue;
        const unsigned grid = static_cast<unsigned>(e - b);
        const int32_t count = segs[b].count;  // the counts of one level differ by at most one
        if(count >= 32768) {
            k_tree_level<512><<<grid, 512, 0, s>>>(pos, key, lp, rp, d_segs + b, d_nodes, depth_limit);
        } else if(count >= 2048) {
            k_tree_level<128><<<grid, 128, 0, s>>>(pos, key, lp, rp, d_segs + b, d_nodes, depth_limit);
        } else {
            k_tree_level<32><<<grid, 32, 0, s>>>(pos, key, lp, rp, d_segs + b, d_nodes, depth_limit);
        }
        LRT_CUDA(ctx, cudaGetLastError());
        ctx->stats.kernel_launches += 1;
    }
    if(!segs.empty()) {
        const uint32_t ns = static_cast<uint32_t>(segs.size());
        k_tree_splits<<<(ns + 255) / 256, 256, 0, s>>>(pos, d_segs, ns, d_nodes);
        LRT_CUDA(ctx, cudaGetLastError());
    }
    k_tree_attrs<<<(n + 255) / 256, 256, 0, s>>>(photons_dev, pos, n, pm.dir.as<float4>(), pm.nrm.as<float4>(),
                                                 pm.pow.as<float4>());
    LRT_CUDA(ctx, cudaGetLastError());
    LRT_CUDA(ctx, cudaStreamSynchronize(s));
    pm.n_nodes = static_cast<uint32_t>(nodes.size());
    pm.depth = max_depth;
    return LRT_OK;
}

}  // namespace lrt
