// lrt_photon.cu — photon tracing, the GPU-built balanced photon kd-tree and the k-nearest-photon
// gather / irradiance estimate of the LinRT photon mapper.
//
//   photon trace   photon_tracer::trace_particle (photon_tracer.h:23-96) per particle index, one
//                  thread per particle; a counting pass and a storing pass at prefix-sum offsets give
//                  the photons in particle-index order, cut exactly as photon_gather::process_result
//                  cuts them with one worker (photon_gather.h:65-101)
//   map build      the tree photon_map::build_range describes (photon_map.h:83-114): a node over
//                  [start, start+count) is a leaf when count <= 8, otherwise it splits at the median
//                  (start + count/2) on the largest-extent axis of its photons. The topology depends
//                  only on the count; the device computes, level by level, each node's bounds and
//                  axis, sorts every node range on its axis (CUB segmented radix sort) and reads the
//                  split at the median.
//   k-NN gather    photon_map::nearest/search (photon_map.h:117-165): near child first, the far child
//                  when delta^2 <= the limit taken at node entry, a max-heap of (d2, index) that pops
//                  its maximum for every candidate with d2 <= limit once full
//   irradiance     photon_map::estimate_irradiance (photon_map.h:38-70) over the neighbours in heap
//                  pop order
#include <cub/device/device_segmented_radix_sort.cuh>

#include <algorithm>
#include <cstring>
#include <thread>
#include <unordered_map>
#include <vector>

#include "lrt_context.cuh"
#include "lrt_scene.cuh"

using namespace lrt;

namespace {

// ---------------------------------------------------------------------------------------------
// photon trace

struct EmitterRay {
    Ray ray;
    f3 weight;
};

// area_emitter::sample_ray (area_emitter.h:93-122)
__device__ __forceinline__ bool area_sample_ray(const DeviceScene& s, const EmitRec& e, float sx, float sy, float dx,
                                                float dy, EmitterRay& out) {
    if(e.area <= 0.0f) return false;
    f3 p, n;
    float pdf_area = 0.0f;
    emitter_sample_position(s, e, sx, sy, p, n, pdf_area);
    if(pdf_area <= 0.0f) return false;
    const float cos_theta = sqrtf(dx);
    const float sin_theta = sqrtf(1.0f - dx);
    const float phi = 2.0f * kPi * dy;
    float sin_phi, cos_phi;
    sincos_rn(phi, sin_phi, cos_phi);
    const f3 local{cos_phi * sin_theta, sin_phi * sin_theta, cos_theta};
    const Onb frame = onb_from_normal(n);
    out.ray = Ray{p, to_world(frame, local)};
    out.weight = load3(e.radiance) * (kPi * e.area);  // power()
    return true;
}

// scene::sample_emitter_ray (scene.h:113-142)
__device__ __forceinline__ bool sample_emitter_ray(const DeviceScene& s, F2 spatial, F2 directional, EmitterRay& out) {
    if(s.emission_power <= 0.0f || s.n_emission <= 0) return false;
    const float target = spatial.x * s.emission_power;
    int32_t bin = 0;  // std::upper_bound: first bin with cdf > target
    while(bin < s.n_emission && !(target < s.emission_cdf[bin])) ++bin;
    if(bin >= s.n_emission) bin = s.n_emission - 1;
    const float prev = bin == 0 ? 0.0f : s.emission_cdf[bin - 1];
    const float span = s.emission_cdf[bin] - prev;
    if(span <= 0.0f) return false;
    const float selection_pdf = span / s.emission_power;
    const float u = (target - prev) / span;
    const EmitRec& e = s.emitters[s.emission_index[bin]];
    if(e.kind != LRT_EMITTER_AREA) return false;  // env_emitter::sample_ray returns false
    if(!area_sample_ray(s, e, u, spatial.y, directional.x, directional.y, out)) return false;
    out.weight /= selection_pdf;
    return true;
}

struct PhotonOut {
    lrt_photon* out;    // destination (nullptr: count only)
    uint64_t base;      // index of this particle's first photon in `out`
    uint64_t limit;     // photons at index >= limit are dropped
    uint32_t count;     // photons emitted by the particle
};

__device__ __forceinline__ void emit_photon(PhotonOut& o, f3 p, f3 dir, f3 n, f3 power, int depth) {
    const uint64_t slot = o.base + o.count;
    ++o.count;
    if(!o.out || slot >= o.limit) return;
    lrt_photon ph;
    store3(ph.position, p);
    store3(ph.direction, dir);
    store3(ph.normal, n);
    store3(ph.power, power);
    ph.depth = static_cast<uint32_t>(static_cast<uint16_t>(depth));
    o.out[slot] = ph;
}

// photon_tracer::trace_particle + store_if_accepted (photon_tracer.h:23-96)
__device__ void trace_particle(const DeviceScene& s, int kind, uint32_t index, int max_depth, int rr_depth,
                               PhotonOut& out) {
    const uint32_t(*table)[32] = sobol_table(s);
    Sampler smp = sampler_start(0u, index);
    // sample_emitter_ray(next_2d(), next_2d(), ...): the right argument (directional) draws first
    const F2 directional = sampler_next_2d(table, smp);
    const F2 spatial = sampler_next_2d(table, smp);
    EmitterRay er;
    if(!sample_emitter_ray(s, spatial, directional, er)) return;
    Ray current = er.ray;
    f3 throughput = mk(1.0f);
    bool delta = false;
    TraceCount cnt{0, 0};
    for(int depth = 1; !is_zero(throughput) && depth <= max_depth;) {
        HitInfo rec;
        if(!scene_hit<false>(s, current, 0.001f, kInf, rec, cnt)) break;
        const int32_t mid = s.objects[rec.object].material;
        if(mid < 0) break;
        const MatRec& mat = s.materials[mid];
        const bool smooth = (mat.flags & kDiffuse) != 0 || (mat.flags & kGlossy) != 0;
        if(smooth && depth > 1 && (kind == LRT_GATHER_CAUSTIC ? delta : !delta)) {
            emit_photon(out, rec.p, normalize(current.d), rec.normal, throughput * er.weight, depth);
        }
        const Onb basis = onb_from_normal(rec.normal);
        BsdfCtx ctx = ctx_default(LRT_MODE_IMPORTANCE);
        ctx.lobe_sample = sampler_next_1d(table, smp);
        BRec br{};
        br.wi = to_local(basis, -normalize(current.d));
        br.wo = mk(0.0f);
        br.front_face = rec.front_face;
        br.eta = 1.0f;
        const F2 u = sampler_next_2d(table, smp);
        const f3 weight = bsdf_sample(s.materials, s.tables, mid, ctx, br, u.x, u.y);
        if(is_zero(weight)) break;
        const f3 outgoing = to_world(basis, br.wo);
        const f3 incoming = to_world(basis, br.wi);
        if(dot(rec.normal, incoming) * br.wi.z <= 0.0f || dot(rec.normal, outgoing) * br.wo.z <= 0.0f) break;
        throughput *= weight;
        delta = (br.sampled_type & kSpecular) != 0;
        current = Ray{rec.p, outgoing};
        if(depth++ >= rr_depth) {
            const float survival = smin(max3(throughput), 0.95f);
            if(sampler_next_1d(table, smp) >= survival) break;
            throughput /= survival;
        }
    }
}

// one slot of max_per photons per particle (parity entry point)
__global__ void k_particles_slots(DeviceScene s, int kind, uint32_t first, uint32_t count, int max_depth, int rr_depth,
                                  uint32_t max_per, lrt_photon* out, uint32_t* counts) {
    for(uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        PhotonOut o{out, static_cast<uint64_t>(i) * max_per, static_cast<uint64_t>(i) * max_per + max_per, 0};
        trace_particle(s, kind, first + i, max_depth, rr_depth, o);
        counts[i] = o.count;
    }
}

// The gather traces each particle once: its first kStagedPhotons photons go to a staging slot of its own
// and its photon count beside them; once the host has walked the counts in particle order (the work
// items' cut and `shot`), the staged photons are copied to their places. A particle that stored more
// photons than its slot holds is traced again, straight into its place (k_particles_store_list).
constexpr uint32_t kStagedPhotons = 4;

__global__ void k_particles_trace(DeviceScene s, int kind, uint32_t first, uint32_t count, int max_depth, int rr_depth,
                                  lrt_photon* staging, uint32_t* counts) {
    for(uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        PhotonOut o{staging, static_cast<uint64_t>(i) * kStagedPhotons, static_cast<uint64_t>(i + 1) * kStagedPhotons, 0};
        trace_particle(s, kind, first + i, max_depth, rr_depth, o);
        counts[i] = o.count;
    }
}

// staged photons of particles [0, count) to out[offsets[i] ..], dropping indices >= limit; one warp per
// particle run of 32 photons would not pay: a particle has a handful
__global__ void k_particles_place(const lrt_photon* staging, const uint32_t* counts, const uint64_t* offsets,
                                  uint32_t count, uint64_t limit, lrt_photon* out) {
    for(uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        const uint32_t c = counts[i];
        if(c > kStagedPhotons) continue;  // traced again
        const uint64_t o = offsets[i];
        for(uint32_t k = 0; k < c && o + k < limit; ++k) out[o + k] = staging[static_cast<uint64_t>(i) * kStagedPhotons + k];
    }
}

// the listed particles traced again, writing at their offsets (absolute photon index), dropping indices >= limit
__global__ void k_particles_store_list(DeviceScene s, int kind, uint32_t first, const uint32_t* list, uint32_t n,
                                       int max_depth, int rr_depth, const uint64_t* offsets, uint64_t limit,
                                       lrt_photon* out) {
    for(uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        const uint32_t i = list[j];
        PhotonOut o{out, offsets[i], limit, 0};
        trace_particle(s, kind, first + i, max_depth, rr_depth, o);
    }
}

// ---------------------------------------------------------------------------------------------
// photon map build, reference-identical (host): photon_map::build_range (photon_map.h:83-114) with the
// same std::nth_element. The split of a node is read from photons[mid] after both children have been
// built, i.e. after the right child has re-partitioned its range, exactly as the reference does; that
// value is generally not the median the node was partitioned on, and the search inherits the effect.
struct HostPhoton {
    float p[3];
    uint32_t index;
};

int32_t build_range_host(std::vector<HostPhoton>& ph, int32_t start, int32_t count, std::vector<PhotonNode>& nodes,
                         uint32_t depth, uint32_t& max_depth) {
    const int32_t index = static_cast<int32_t>(nodes.size());
    nodes.push_back(PhotonNode{start, count, 3, 0.0f});
    max_depth = std::max(max_depth, depth);
    if(count <= 8) return index;
    float lo[3] = {kInf, kInf, kInf}, hi[3] = {-kInf, -kInf, -kInf};
    for(int32_t i = 0; i < count; ++i) {
        for(int a = 0; a < 3; ++a) {
            lo[a] = smin(lo[a], ph[start + i].p[a]);
            hi[a] = smax(hi[a], ph[start + i].p[a]);
        }
    }
    const float extent[3] = {hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]};
    int axis = 0;
    if(extent[1] > extent[axis]) axis = 1;
    if(extent[2] > extent[axis]) axis = 2;
    const int32_t mid = start + count / 2;
    std::nth_element(ph.begin() + start, ph.begin() + mid, ph.begin() + start + count,
                     [axis](const HostPhoton& a, const HostPhoton& b) { return a.p[axis] < b.p[axis]; });
    const int32_t left = build_range_host(ph, start, mid - start, nodes, depth + 1, max_depth);
    const int32_t right = build_range_host(ph, mid, start + count - mid, nodes, depth + 1, max_depth);
    nodes[index] = PhotonNode{left, right, axis, ph[mid].p[axis]};
    return index;
}

// Nodes of the subtree over `count` photons (a leaf at <= 8): the tree's shape depends on counts only.
int32_t subtree_nodes(int32_t count, std::unordered_map<int32_t, int32_t>& memo) {
    if(count <= 8) return 1;
    const auto it = memo.find(count);
    if(it != memo.end()) return it->second;
    const int32_t n = 1 + subtree_nodes(count / 2, memo) + subtree_nodes(count - count / 2, memo);
    memo[count] = n;
    return n;
}

// build_range_host on several host threads: a node's nth_element runs before its children, which
// work on disjoint ranges and write their nodes at the places the depth-first order gives them, so
// the tree (photon order, nodes, splits) is the serial one.
void build_range_parallel(std::vector<HostPhoton>& ph, int32_t start, int32_t count, PhotonNode* nodes,
                          int32_t index, uint32_t depth, uint32_t& max_depth, int spawn_levels,
                          std::unordered_map<int32_t, int32_t>& memo) {
    if(spawn_levels <= 0 || count <= 8) {
        std::vector<PhotonNode> local;
        uint32_t md = depth;
        build_range_host(ph, start, count, local, depth, md);
        for(size_t i = 0; i < local.size(); ++i) {  // shift the subtree's child links to its place
            PhotonNode nd = local[i];
            if(nd.axis != 3) {
                nd.a += index;
                nd.b += index;
            }
            nodes[index + i] = nd;
        }
        max_depth = std::max(max_depth, md);
        return;
    }
    float lo[3] = {kInf, kInf, kInf}, hi[3] = {-kInf, -kInf, -kInf};
    for(int32_t i = 0; i < count; ++i) {
        for(int a = 0; a < 3; ++a) {
            lo[a] = smin(lo[a], ph[start + i].p[a]);
            hi[a] = smax(hi[a], ph[start + i].p[a]);
        }
    }
    const float extent[3] = {hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]};
    int axis = 0;
    if(extent[1] > extent[axis]) axis = 1;
    if(extent[2] > extent[axis]) axis = 2;
    const int32_t mid = start + count / 2;
    std::nth_element(ph.begin() + start, ph.begin() + mid, ph.begin() + start + count,
                     [axis](const HostPhoton& a, const HostPhoton& b) { return a.p[axis] < b.p[axis]; });
    const int32_t left = index + 1;
    const int32_t right = left + subtree_nodes(mid - start, memo);
    max_depth = std::max(max_depth, depth);
    uint32_t md_left = depth, md_right = depth;
    std::unordered_map<int32_t, int32_t> memo_left = memo;  // each thread its own cache
    std::thread t([&]() {
        build_range_parallel(ph, start, mid - start, nodes, left, depth + 1, md_left, spawn_levels - 1, memo_left);
    });
    build_range_parallel(ph, mid, start + count - mid, nodes, right, depth + 1, md_right, spawn_levels - 1, memo);
    t.join();
    max_depth = std::max(max_depth, std::max(md_left, md_right));
    nodes[index] = PhotonNode{left, right, axis, ph[mid].p[axis]};
}

__global__ void k_photon_gather_attrs(const lrt_photon* in, const uint32_t* order, uint32_t n, float4* pos, float4* dir,
                                      float4* nrm, float4* pw) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= n) return;
    const uint32_t src = order[i];
    const lrt_photon& p = in[src];
    pos[i] = make_float4(p.position[0], p.position[1], p.position[2], __uint_as_float(src));
    dir[i] = make_float4(p.direction[0], p.direction[1], p.direction[2], __int_as_float(static_cast<int>(p.depth)));
    nrm[i] = make_float4(p.normal[0], p.normal[1], p.normal[2], 0.0f);
    pw[i] = make_float4(p.power[0], p.power[1], p.power[2], 0.0f);
}

// ---------------------------------------------------------------------------------------------
// k-NN gather

struct MapView {
    const float4* pos;
    const float4* dir;
    const float4* nrm;
    const float4* pw;
    const PhotonNode* nodes;
    uint32_t n;
    float scale;
};

// (d2, index) pairs compared as std::pair
__device__ __forceinline__ bool pair_less(float da, uint32_t ia, float db, uint32_t ib) {
    return da < db || (!(db < da) && ia < ib);
}

// The k nearest photons found so far: a max-heap of (d2 bits, index) pairs under pair_less. Element j of
// a thread's heap sits at e[j * stride]: a local array (stride 1), or the thread's column of a shared
// array interleaved across the block (stride = threads per block), where the threads of a warp at the
// same heap position touch consecutive words and the heap stays on chip (a local heap of 1 KB per
// thread is far beyond what L1 holds for a full SM).
struct KnnHeap {
    uint2* e;
    uint32_t stride;
    uint32_t size;

    __device__ __forceinline__ uint2 at(uint32_t j) const { return e[j * stride]; }
    __device__ __forceinline__ void put(uint32_t j, uint2 v) { e[j * stride] = v; }
    __device__ __forceinline__ float top_d() const { return __uint_as_float(e[0].x); }
    __device__ __forceinline__ uint32_t top_i() const { return e[0].y; }

    __device__ __forceinline__ void pop() {  // remove the maximum
        --size;
        if(size == 0) return;
        const uint2 last = at(size);
        const float dl = __uint_as_float(last.x);
        uint32_t k = 0;
        while(true) {
            uint32_t c = 2 * k + 1;
            if(c >= size) break;
            uint2 cv = at(c);
            if(c + 1 < size) {
                const uint2 c2 = at(c + 1);
                if(pair_less(__uint_as_float(cv.x), cv.y, __uint_as_float(c2.x), c2.y)) {
                    ++c;
                    cv = c2;
                }
            }
            if(!pair_less(dl, last.y, __uint_as_float(cv.x), cv.y)) break;
            put(k, cv);
            k = c;
        }
        put(k, last);
    }
    __device__ __forceinline__ void push(float dv, uint32_t iv) {
        uint32_t k = size++;
        while(k > 0) {
            const uint32_t parent = (k - 1) / 2;
            const uint2 pv = at(parent);
            if(!pair_less(__uint_as_float(pv.x), pv.y, dv, iv)) break;
            put(k, pv);
            k = parent;
        }
        put(k, make_uint2(__float_as_uint(dv), iv));
    }
};

// threads per block of the kernels that keep their heaps in shared memory: kCap heap entries of 8 bytes
// per thread, 32 KB per block (kCap = 0: heaps in local memory, the library's usual block)
template <uint32_t kCap>
struct HeapBlock {
    static constexpr int kThreads = kCap == 0 ? kBlock : static_cast<int>(4096 / kCap);
};

// per-query work of a k-NN search (algorithmic-bytes accounting); compiled out unless requested
struct KnnCount {
    uint32_t nodes;
    uint32_t tested;
};

template <bool kCount = false>
__device__ __forceinline__ void knn_search(const MapView& m, f3 point, float r2, uint32_t k, KnnHeap& heap,
                                           KnnCount* cnt = nullptr) {
    heap.size = 0;
    if(m.n == 0 || k == 0) return;
    int32_t stack[64];
    int top = 0;
    stack[top++] = 0;
    while(top > 0) {
        const PhotonNode nd = m.nodes[stack[--top]];
        if(kCount) ++cnt->nodes;
        float limit = r2;
        if(heap.size == k) limit = smin(limit, heap.top_d());
        if(nd.axis == 3) {
            for(int32_t j = 0; j < nd.b; ++j) {
                const uint32_t pi = static_cast<uint32_t>(nd.a + j);
                if(kCount) ++cnt->tested;
                const float4 p4 = __ldg(m.pos + pi);
                const float distance = length_squared(f3{p4.x, p4.y, p4.z} - point);
                if(distance > limit) continue;
                if(heap.size == k) heap.pop();
                heap.push(distance, pi);
                if(heap.size == k) limit = smin(r2, heap.top_d());
            }
            continue;
        }
        const float delta = comp(point, nd.axis) - nd.split;
        const int32_t near = delta <= 0.0f ? nd.a : nd.b;
        const int32_t far = delta <= 0.0f ? nd.b : nd.a;
        if(delta * delta <= limit && top < 64) stack[top++] = far;
        if(top < 64) stack[top++] = near;
    }
}

__global__ void __launch_bounds__(kBlock) k_knn(MapView m, const float* points, uint32_t n, float r2, uint32_t k,
                                                uint32_t* idx_out, float* d2_out, uint32_t* cnt_out) {
    for(uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        uint2 heap_store[kMaxKnn];
        KnnHeap heap{heap_store, 1u, 0u};
        knn_search(m, load3(points + 3ull * q), r2, k, heap);
        const uint32_t found = heap.size;
        cnt_out[q] = found;
        for(uint32_t j = 0; j < found; ++j) {  // max-heap pop order
            idx_out[static_cast<size_t>(q) * k + j] = __float_as_uint(m.pos[heap.top_i()].w);
            d2_out[static_cast<size_t>(q) * k + j] = heap.top_d();
            heap.pop();
        }
    }
}

// photon_map::estimate_irradiance (photon_map.h:38-70), neighbours in heap pop order
template <bool kCount = false>
__device__ __forceinline__ f3 estimate_irradiance(const MapView& m, f3 point, f3 normal, float radius, int32_t max_depth,
                                                 uint32_t k, KnnHeap& heap, KnnCount* cnt = nullptr,
                                                 uint32_t* found = nullptr) {
    f3 sum = mk(0.0f);
    if(m.n == 0 || radius <= 0.0f || k == 0) return sum;
    const float squared_radius = radius * radius;
    knn_search<kCount>(m, point, squared_radius, k, heap, cnt);
    if(kCount) *found += heap.size;
    const float inverse_squared_radius = 1.0f / squared_radius;
    while(heap.size > 0) {
        const uint32_t pi = heap.top_i();
        const float d2 = heap.top_d();
        heap.pop();
        const float4 dir = m.dir[pi];
        if(__float_as_int(dir.w) > max_depth) continue;
        const float4 pn = m.nrm[pi];
        const f3 photon_normal{pn.x, pn.y, pn.z};
        const f3 incoming = -f3{dir.x, dir.y, dir.z};
        const float incoming_dot_photon = dot(photon_normal, incoming);
        const float incoming_dot_shading = dot(normal, incoming);
        if(incoming_dot_shading <= 0.0f || dot(photon_normal, normal) <= 1e-1f || incoming_dot_photon <= 1e-2f) {
            continue;
        }
        const float square = 1.0f - d2 * inverse_squared_radius;
        const float weight = (incoming_dot_shading / incoming_dot_photon) * (square * square);
        const float4 pw = m.pw[pi];
        sum += f3{pw.x, pw.y, pw.z} * fabsf(weight);
    }
    return sum * (m.scale * 3.0f * (1.0f / kPi) * inverse_squared_radius);
}

// one query per thread; kCount adds the queries' nodes, photons tested and photons found to work[0..3]
// kCap > 0: heaps of kCap entries in shared memory (k <= kCap); 0: in local memory
template <bool kCount, uint32_t kCap>
__global__ void __launch_bounds__(HeapBlock<kCap>::kThreads) k_irradiance(MapView m, const float* points,
                                                                         const float* normals, uint32_t n, float radius,
                                                                         int32_t max_depth, uint32_t k, float* rgb,
                                                                         unsigned long long* work) {
    constexpr int kThreads = HeapBlock<kCap>::kThreads;
    __shared__ uint2 shared_heaps[kCap == 0 ? 1 : kCap * kThreads];
    uint2 local_heap[kCap == 0 ? kMaxKnn : 1];
    KnnCount cnt{0, 0};
    uint32_t found = 0, queries = 0;
    for(uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        KnnHeap heap = kCap == 0 ? KnnHeap{local_heap, 1u, 0u}
                                 : KnnHeap{shared_heaps + threadIdx.x, static_cast<uint32_t>(kThreads), 0u};
        store3(rgb + 3ull * q, estimate_irradiance<kCount>(m, load3(points + 3ull * q), load3(normals + 3ull * q),
                                                           radius, max_depth, k, heap, &cnt, &found));
        ++queries;
    }
    if(kCount) {
        add_count(&work[0], queries);
        add_count(&work[1], cnt.nodes);
        add_count(&work[2], cnt.tested);
        add_count(&work[3], found);
    }
}

// ---------------------------------------------------------------------------------------------
// photon-map eye pass: photon_integrator::li and its helpers (photon_integrator.h:39-296) with the
// recursion as an explicit per-thread stack of frames. Frames run in the reference's depth-first
// order, so every camera sample draws its sampler dimensions in the reference's order. A frame's
// contributions are added to the sample's radiance times the product of the weights on the way down
// (the reference multiplies the child's returned radiance instead: same terms, other rounding).

constexpr int kEyeFrames = 128;  // one frame per recursion level: max_depth <= 128
enum EyeStage : uint8_t { kEyeStart = 0, kEyeSpecular = 1, kEyeEmitters = 2, kEyeBsdf = 3, kEyeLookup = 4 };

struct EyeFrame {
    f3 ro, rd;       // the ray li was called with
    f3 p, n;         // its hit
    f3 tp;           // weight of this frame's radiance in the camera sample
    int32_t obj;     // hit object, -1 on a miss
    int16_t depth;
    int16_t iter;
    uint8_t stage;
    uint8_t evaluated;
    uint8_t emission;
    uint8_t front_face;
};

struct EyeParams {
    MapView global, caustic;
    float global_radius, caustic_radius;
    int32_t max_depth, max_specular_depth, direct_samples, glossy_samples;
    uint32_t lookup_size;
};

struct EyeCounts {
    int emitter, bsdf;
    float emitter_weight, bsdf_weight;
};

__device__ __forceinline__ EyeCounts eye_counts(const EyeParams& ep, int depth, bool diffuse) {
    EyeCounts c{1, 1, 1.0f, 1.0f};  // photon_integrator.h:287-296
    if(depth == 1) {
        c.emitter = ep.direct_samples;
        c.bsdf = diffuse ? ep.direct_samples : ep.glossy_samples;
        c.emitter_weight = 1.0f / static_cast<float>(c.emitter);
        c.bsdf_weight = 1.0f / static_cast<float>(c.bsdf);
    }
    return c;
}

__device__ f3 eye_sample(const DeviceScene& s, const EyeParams& ep, Sampler& smp, Ray camera, EyeFrame* st, KnnHeap& heap,
                         int* overflow) {
    const uint32_t(*table)[32] = sobol_table(s);
    constexpr uint32_t kSmooth = kDiffuse | kGlossy;
    TraceCount cnt{0, 0};
    f3 L = mk(0.0f);
    int top = 0;
    st[0] = EyeFrame{camera.o, camera.d, mk(0.0f), mk(0.0f), mk(1.0f), -1, 1, 0, kEyeStart, 0, 1, 0};
    while(top >= 0) {
        EyeFrame& F = st[top];
        const int32_t mid = F.obj >= 0 ? s.objects[F.obj].material : -1;
        if(F.stage == kEyeStart) {
            if(!F.evaluated) {
                HitInfo h;
                if(scene_hit<false>(s, Ray{F.ro, F.rd}, 0.001f, kInf, h, cnt)) {
                    F.obj = h.object;
                    F.p = h.p;
                    F.n = h.normal;
                    F.front_face = h.front_face ? 1 : 0;
                } else {
                    F.obj = -1;
                }
                F.evaluated = 1;
            }
            if(F.obj < 0) {
                if(F.emission) L += F.tp * eval_environment(s, F.rd);
                --top;
                continue;
            }
            const ObjRec& o = s.objects[F.obj];
            if(F.emission && o.emitter >= 0 && F.front_face) {
                L += F.tp * area_emitted(s.emitters[o.emitter], F.n, -normalize(F.rd));
            }
            const int32_t m = o.material;
            if(F.depth >= ep.max_depth || m < 0) {
                --top;
                continue;
            }
            const uint32_t flags = s.materials[m].flags;
            const bool diffuse = (flags & (kDiffuse | kGlossy | kSpecular)) == kDiffuse;
            if(diffuse && dot(F.n, F.rd) < 0.0f) {  // photon lookups (photon_integrator.h:95-106)
                const int photon_depth = ep.max_depth - F.depth;
                const f3 reflectance = bsdf_diffuse_reflectance(s.materials, m) * (1.0f / kPi);
                if(ep.global.n > 0) {
                    L += F.tp * (estimate_irradiance(ep.global, F.p, F.n, ep.global_radius, photon_depth, ep.lookup_size,
                                                     heap) * reflectance);
                }
                if(ep.caustic.n > 0) {
                    L += F.tp * (estimate_irradiance(ep.caustic, F.p, F.n, ep.caustic_radius, photon_depth,
                                                     ep.lookup_size, heap) * reflectance);
                }
            }
            F.stage = kEyeSpecular;
            F.iter = 0;
            continue;
        }
        const uint32_t flags = s.materials[mid].flags;
        const bool diffuse = (flags & (kDiffuse | kGlossy | kSpecular)) == kDiffuse;
        const bool specular = (flags & kSpecular) != 0;
        const bool smooth = (flags & kSmooth) != 0;
        const bool exhaustive = specular && F.depth < ep.max_specular_depth;
        const Onb basis = onb_from_normal(F.n);
        BRec rec{};
        rec.wi = to_local(basis, -normalize(F.rd));
        rec.wo = mk(0.0f);
        rec.front_face = F.front_face != 0;
        rec.eta = 1.0f;
        if(F.stage == kEyeSpecular) {  // specular_lobes (photon_integrator.h:126-155)
            bool pushed = false;
            if(exhaustive) {
                const int count = s.materials[mid].component_count;
                while(F.iter < count) {
                    const int c = F.iter++;
                    if((bsdf_component_flags(s.materials, mid, c) & kSpecular) == 0) continue;
                    BsdfCtx ctx = ctx_default(LRT_MODE_RADIANCE);
                    ctx.component = c;
                    BRec r = rec;
                    const f3 w = bsdf_sample(s.materials, s.tables, mid, ctx, r, 0.5f, 0.5f);
                    if(is_zero(w)) continue;
                    if(top + 1 >= kEyeFrames) {
                        *overflow = 1;
                        continue;
                    }
                    st[top + 1] = EyeFrame{F.p, to_world(basis, r.wo), mk(0.0f), mk(0.0f), F.tp * w, -1,
                                           static_cast<int16_t>(F.depth + 1), 0, kEyeStart, 0, 1, 0};
                    ++top;
                    pushed = true;
                    break;
                }
            }
            if(pushed) continue;
            F.stage = kEyeEmitters;
        }
        if(F.stage == kEyeEmitters) {  // emitter_samples (photon_integrator.h:157-217)
            if(smooth) {
                const EyeCounts counts = eye_counts(ep, F.depth, diffuse);
                for(int i = 0; i < counts.emitter; ++i) {
                    const F2 u = sampler_next_2d(table, smp);
                    DirectSample light{};
                    light.distance = kInf;
                    if(!sample_emitter_direction(s, F.p, u.x, u.y, light)) continue;
                    const f3 shadow_origin = F.p + F.n * 1e-4f;
                    f3 shadow_dir = light.direction;
                    float tmax = kInf;
                    if(!isinf(light.distance)) {
                        const f3 to_light = light.point - shadow_origin;
                        const float distance = length(to_light);
                        if(distance < 1e-6f) continue;
                        shadow_dir = to_light / distance;
                        tmax = distance * (1.0f - 1e-4f);
                    }
                    BRec r = rec;
                    r.wo = to_local(basis, shadow_dir);
                    BsdfCtx ctx = ctx_default(LRT_MODE_RADIANCE);
                    if(!specular || exhaustive) ctx.type_mask = kSmooth;
                    const f3 value = bsdf_eval(s.materials, s.tables, mid, ctx, r, kSolidAngle);
                    if(is_zero(value)) continue;
                    if(scene_occluded<false>(s, Ray{shadow_origin, shadow_dir}, 0.001f, tmax, light.emitter, cnt)) continue;
                    const float light_pdf = pdf_emitter_direction(s, F.p, shadow_dir);
                    const float bsdf_pdf_v = bsdf_pdf(s.materials, s.tables, mid, ctx, r, kSolidAngle);
                    if(light_pdf <= 0.0f) continue;
                    const float weight = power_heuristic(light_pdf * static_cast<float>(counts.emitter),
                                                         bsdf_pdf_v * static_cast<float>(counts.bsdf)) * counts.emitter_weight;
                    L += F.tp * (value * light.radiance * (weight / light_pdf));
                }
            }
            F.stage = kEyeBsdf;
            F.iter = 0;
        }
        // bsdf_samples (photon_integrator.h:219-277)
        const bool sample_direct = smooth || (specular && !exhaustive);
        const bool sample_indirect = !diffuse && (smooth || (specular && !exhaustive));
        bool pushed = false;
        if(sample_direct || sample_indirect) {
            const EyeCounts counts = eye_counts(ep, F.depth, diffuse);
            while(F.iter < counts.bsdf) {
                ++F.iter;
                BsdfCtx ctx = ctx_default(LRT_MODE_RADIANCE);
                ctx.lobe_sample = sampler_next_1d(table, smp);
                if(!specular || exhaustive) ctx.type_mask = kSmooth;
                BRec r = rec;
                const F2 u = sampler_next_2d(table, smp);
                const f3 weight = bsdf_sample(s.materials, s.tables, mid, ctx, r, u.x, u.y);
                if(is_zero(weight) || r.pdf <= 0.0f) continue;
                const Ray scattered{F.p, to_world(basis, r.wo)};
                HitInfo occluder;
                const bool hit = scene_hit<false>(s, scattered, 0.001f, kInf, occluder, cnt);
                if(sample_direct) {
                    f3 emission = mk(0.0f);
                    float light_pdf = 0.0f;
                    if(hit) {
                        const ObjRec& oo = s.objects[occluder.object];
                        if(oo.emitter >= 0 && occluder.front_face) {
                            emission = area_emitted(s.emitters[oo.emitter], occluder.normal, -normalize(scattered.d));
                            light_pdf = pdf_emitter_direction(s, F.p, scattered.d);
                        }
                    } else {
                        emission = eval_environment(s, scattered.d);
                        light_pdf = pdf_emitter_direction(s, F.p, scattered.d);
                    }
                    if(!is_zero(emission)) {
                        const float mis = power_heuristic(r.pdf * static_cast<float>(counts.bsdf),
                                                          light_pdf * static_cast<float>(counts.emitter)) * counts.bsdf_weight;
                        L += F.tp * (emission * weight * mis);
                    }
                }
                if(sample_indirect) {
                    if(top + 1 >= kEyeFrames) {
                        *overflow = 1;
                        continue;
                    }
                    EyeFrame child{scattered.o, scattered.d, occluder.p, occluder.normal, F.tp * weight * counts.bsdf_weight,
                                   hit ? occluder.object : -1, static_cast<int16_t>(F.depth + 1), 0, kEyeStart, 1, 0,
                                   static_cast<uint8_t>(hit && occluder.front_face ? 1 : 0)};
                    st[top + 1] = child;
                    ++top;
                    pushed = true;
                    break;
                }
            }
        }
        if(!pushed) --top;
    }
    return L;
}

__global__ void __launch_bounds__(kBlock) k_photon_eye(DeviceScene s, EyeParams ep, uint32_t width, uint32_t height,
                                                       uint32_t pixel_begin, uint32_t n_pixels, uint32_t sample_begin,
                                                       uint32_t n_samples, float4* L_out, int* overflow) {
    EyeFrame frames[kEyeFrames];
    uint2 heap_store[kMaxKnn];
    KnnHeap heap{heap_store, 1u, 0u};
    const uint32_t n = n_pixels * n_samples;
    for(uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x; slot < n; slot += gridDim.x * blockDim.x) {
        const uint32_t pix = pixel_begin + slot / n_samples;
        const uint32_t sample = sample_begin + slot % n_samples;
        Sampler smp = sampler_start(pix, sample);
        const F2 off = sampler_next_2d(sobol_table(s), smp);
        const float u = (static_cast<float>(pix % width) + off.x) / static_cast<float>(width - 1);
        const float v = (static_cast<float>(pix / width) + off.y) / static_cast<float>(height - 1);
        const f3 L = eye_sample(s, ep, smp, camera_ray(s.cam, u, v), frames, heap, overflow);
        L_out[slot] = make_float4(L.x, L.y, L.z, 0.0f);
    }
}

// ---- persistent eye pass ----
//
// The same depth-first walk as eye_sample, cut at every ray query so that the rays of a warp's lanes
// are traced together: each lane runs its walk until it needs a ray (the first hit of a frame, an NEE
// shadow ray, a BSDF sample's ray), then all lanes advance their traversals one unit at a time
// (trav_step, the persistent traversal of the path tracer), and a lane whose ray is done resumes its
// walk with the result; a lane whose camera sample is done takes the next one. Samples, sampler
// draws, rays and additions to L are those of eye_sample, in the same order.
enum EyeQueryKind : uint8_t { kQueryNone = 0, kQueryHit = 1, kQueryShadow = 2, kQueryBsdf = 3, kQueryIrradiance = 4 };

// A ray query of the wavefront eye pass, in device memory with its result. A lane's walk issues the
// shadow rays of a frame's emitter samples, and the rays of its BSDF samples when they do not recurse,
// as one batch of up to kEyeBatch queries: their sampler draws happen in order when they are issued,
// none depends on another's result, and the results are applied in issue order, so the radiance sums
// are those of one query at a time. A frame's own ray and a BSDF sample that recurses go alone.
constexpr uint32_t kEyeBatch = 16;

// A photon lookup (kQueryIrradiance) uses the record as: o = (point, radius), d = (normal, -), a =
// (diffuse reflectance / pi, -), b = (frame weight, -), light = map (0 global, 1 caustic), any_mode =
// photon depth limit; the estimate comes back in (closest, u, v).
struct EyeQuery {
    float4 o;          // origin, t_min
    float4 d;          // direction, t_max
    float4 a;          // shadow: what L gains when the light is visible; BSDF sample: weight (xyz), pdf (w)
    float4 b;          // photon lookup: the frame's weight
    int32_t kind;      // EyeQueryKind
    int32_t light;     // shadow: the light
    int32_t any_mode;
    int32_t best;      // result: the traversal's best object (-1 none), closest t, the hit's u, v, reference
    float closest;
    float u, v;
    uint32_t ref;
};

// where eye_advance puts its queries: q == nullptr -- one query at a time, into the lane and `ts`
struct EyeBatch {
    EyeQuery* q;
    uint32_t n;
};

struct EyeLane {
    Sampler smp;
    f3 L;
    int top;
    uint32_t slot;
    uint8_t query;
    f3 qa;           // shadow: what L gains when the light is visible; BSDF sample: its weight
    float qpdf;      // BSDF sample: its pdf
    int32_t qlight;  // shadow: the light
};

struct EyeFlags {
    bool diffuse, specular, smooth, exhaustive;
};

__device__ __forceinline__ EyeFlags eye_flags(const DeviceScene& s, const EyeParams& ep, int32_t mid, int depth) {
    const uint32_t flags = s.materials[mid].flags;
    EyeFlags f;
    f.diffuse = (flags & (kDiffuse | kGlossy | kSpecular)) == kDiffuse;
    f.specular = (flags & kSpecular) != 0;
    f.smooth = (flags & (kDiffuse | kGlossy)) != 0;
    f.exhaustive = f.specular && depth < ep.max_specular_depth;
    return f;
}

// Issues a query: without a batch, into the lane and ts (the walk then stops); with one, appended to it.
// Returns true when the walk must stop here: always without a batch; with one, when the query must go
// alone (its result decides what the walk does next) or the batch is full.
__device__ __forceinline__ bool eye_issue(EyeLane& ln, TravState& ts, EyeBatch& b, uint8_t kind, const Ray& r,
                                          float t_max, bool any_mode, f3 qa, float qpdf, int32_t qlight, bool alone) {
    if(!b.q) {
        ln.query = kind;
        ln.qa = qa;
        ln.qpdf = qpdf;
        ln.qlight = qlight;
        trav_begin(ts, r, 0.001f, t_max, any_mode);
        return true;
    }
    EyeQuery& Q = b.q[b.n++];
    Q.o = make_float4(r.o.x, r.o.y, r.o.z, 0.001f);
    Q.d = make_float4(r.d.x, r.d.y, r.d.z, t_max);
    Q.a = make_float4(qa.x, qa.y, qa.z, qpdf);
    Q.kind = kind;
    Q.light = qlight;
    Q.any_mode = any_mode ? 1 : 0;
    return alone || b.n == kEyeBatch;
}

// Advances the lane's walk until it issues a ray query (true; ts holds the ray, or the batch its queries)
// or finishes its sample.
__device__ bool eye_advance(const DeviceScene& s, const EyeParams& ep, EyeLane& ln, EyeFrame* st, KnnHeap& heap,
                            int* overflow, TravState& ts, int frame_limit, EyeBatch& batch) {
    const uint32_t(*table)[32] = sobol_table(s);
    constexpr uint32_t kSmooth = kDiffuse | kGlossy;
    while(ln.top >= 0) {
        EyeFrame& F = st[ln.top];
        if(F.stage == kEyeStart) {
            if(!F.evaluated) {
                eye_issue(ln, ts, batch, kQueryHit, Ray{F.ro, F.rd}, kInf, false, mk(0.0f), 0.0f, -1, true);
                return true;
            }
            if(F.obj < 0) {
                if(F.emission) ln.L += F.tp * eval_environment(s, F.rd);
                --ln.top;
                continue;
            }
            const ObjRec& o = s.objects[F.obj];
            if(F.emission && o.emitter >= 0 && F.front_face) {
                ln.L += F.tp * area_emitted(s.emitters[o.emitter], F.n, -normalize(F.rd));
            }
            const int32_t m = o.material;
            if(F.depth >= ep.max_depth || m < 0) {
                --ln.top;
                continue;
            }
            const uint32_t flags = s.materials[m].flags;
            const bool diffuse = (flags & (kDiffuse | kGlossy | kSpecular)) == kDiffuse;
            if(diffuse && dot(F.n, F.rd) < 0.0f && batch.q) {  // the lookups go into the batch
                F.stage = kEyeLookup;
                continue;
            }
            if(diffuse && dot(F.n, F.rd) < 0.0f) {  // photon lookups (photon_integrator.h:95-106)
                const int photon_depth = ep.max_depth - F.depth;
                const f3 reflectance = bsdf_diffuse_reflectance(s.materials, m) * (1.0f / kPi);
                if(ep.global.n > 0) {
                    ln.L += F.tp * (estimate_irradiance(ep.global, F.p, F.n, ep.global_radius, photon_depth, ep.lookup_size,
                                                        heap) * reflectance);
                }
                if(ep.caustic.n > 0) {
                    ln.L += F.tp * (estimate_irradiance(ep.caustic, F.p, F.n, ep.caustic_radius, photon_depth,
                                                        ep.lookup_size, heap) * reflectance);
                }
            }
            F.stage = kEyeSpecular;
            F.iter = 0;
            continue;
        }
        if(F.stage == kEyeLookup) {  // the photon lookups as queries of the batch, global map first
            const int32_t m = s.objects[F.obj].material;
            const int photon_depth = ep.max_depth - F.depth;
            const f3 reflectance = bsdf_diffuse_reflectance(s.materials, m) * (1.0f / kPi);
            if(!batch.q) {  // a walk continued one query at a time (the wave's tail): the lookups inline
                if(ep.global.n > 0) {
                    ln.L += F.tp * (estimate_irradiance(ep.global, F.p, F.n, ep.global_radius, photon_depth, ep.lookup_size,
                                                        heap) * reflectance);
                }
                if(ep.caustic.n > 0) {
                    ln.L += F.tp * (estimate_irradiance(ep.caustic, F.p, F.n, ep.caustic_radius, photon_depth,
                                                        ep.lookup_size, heap) * reflectance);
                }
                F.stage = kEyeSpecular;
                F.iter = 0;
                continue;
            }
            const int need = (ep.global.n > 0 ? 1 : 0) + (ep.caustic.n > 0 ? 1 : 0);
            if(batch.n + need > kEyeBatch) return true;  // the batch is not empty: resume here
            for(int map = 0; map < 2; ++map) {
                if((map == 0 ? ep.global.n : ep.caustic.n) == 0) continue;
                EyeQuery& Q = batch.q[batch.n++];
                Q.o = make_float4(F.p.x, F.p.y, F.p.z, map == 0 ? ep.global_radius : ep.caustic_radius);
                Q.d = make_float4(F.n.x, F.n.y, F.n.z, 0.0f);
                Q.a = make_float4(reflectance.x, reflectance.y, reflectance.z, 0.0f);
                Q.b = make_float4(F.tp.x, F.tp.y, F.tp.z, 0.0f);
                Q.kind = kQueryIrradiance;
                Q.light = map;
                Q.any_mode = photon_depth;
            }
            F.stage = kEyeSpecular;
            F.iter = 0;
            if(batch.n == kEyeBatch) return true;  // full: the walk resumes at the specular lobes
            continue;
        }
        const int32_t mid = s.objects[F.obj].material;
        const EyeFlags fl = eye_flags(s, ep, mid, F.depth);
        const Onb basis = onb_from_normal(F.n);
        BRec rec{};
        rec.wi = to_local(basis, -normalize(F.rd));
        rec.wo = mk(0.0f);
        rec.front_face = F.front_face != 0;
        rec.eta = 1.0f;
        if(F.stage == kEyeSpecular) {  // specular_lobes (photon_integrator.h:126-155)
            bool pushed = false;
            if(fl.exhaustive) {
                const int count = s.materials[mid].component_count;
                while(F.iter < count) {
                    const int c = F.iter++;
                    if((bsdf_component_flags(s.materials, mid, c) & kSpecular) == 0) continue;
                    BsdfCtx ctx = ctx_default(LRT_MODE_RADIANCE);
                    ctx.component = c;
                    BRec r = rec;
                    const f3 w = bsdf_sample(s.materials, s.tables, mid, ctx, r, 0.5f, 0.5f);
                    if(is_zero(w)) continue;
                    if(ln.top + 1 >= frame_limit) {
                        *overflow = 1;
                        continue;
                    }
                    st[ln.top + 1] = EyeFrame{F.p, to_world(basis, r.wo), mk(0.0f), mk(0.0f), F.tp * w, -1,
                                              static_cast<int16_t>(F.depth + 1), 0, kEyeStart, 0, 1, 0};
                    ++ln.top;
                    pushed = true;
                    break;
                }
            }
            if(pushed) continue;
            F.stage = kEyeEmitters;
            F.iter = 0;
        }
        if(F.stage == kEyeEmitters) {  // emitter_samples (photon_integrator.h:157-217), one shadow ray per visit
            if(fl.smooth) {
                const EyeCounts counts = eye_counts(ep, F.depth, fl.diffuse);
                while(F.iter < counts.emitter) {
                    ++F.iter;
                    const F2 u = sampler_next_2d(table, ln.smp);
                    DirectSample light{};
                    light.distance = kInf;
                    if(!sample_emitter_direction(s, F.p, u.x, u.y, light)) continue;
                    const f3 shadow_origin = F.p + F.n * 1e-4f;
                    f3 shadow_dir = light.direction;
                    float tmax = kInf;
                    if(!isinf(light.distance)) {
                        const f3 to_light = light.point - shadow_origin;
                        const float distance = length(to_light);
                        if(distance < 1e-6f) continue;
                        shadow_dir = to_light / distance;
                        tmax = distance * (1.0f - 1e-4f);
                    }
                    BRec r = rec;
                    r.wo = to_local(basis, shadow_dir);
                    BsdfCtx ctx = ctx_default(LRT_MODE_RADIANCE);
                    if(!fl.specular || fl.exhaustive) ctx.type_mask = kSmooth;
                    const f3 value = bsdf_eval(s.materials, s.tables, mid, ctx, r, kSolidAngle);
                    if(is_zero(value)) continue;
                    // the pdfs do not depend on the shadow ray's outcome; a sample they reject adds nothing
                    const float light_pdf = pdf_emitter_direction(s, F.p, shadow_dir);
                    const float bsdf_pdf_v = bsdf_pdf(s.materials, s.tables, mid, ctx, r, kSolidAngle);
                    if(light_pdf <= 0.0f) continue;
                    const float weight = power_heuristic(light_pdf * static_cast<float>(counts.emitter),
                                                         bsdf_pdf_v * static_cast<float>(counts.bsdf)) * counts.emitter_weight;
                    const Ray sr{shadow_origin, shadow_dir};
                    bool any_mode = true;
                    const EmitRec& e = s.emitters[light.emitter];
                    if(e.kind == LRT_EMITTER_AREA) {  // scene_occluded's rule
                        any_mode = !light_shape_reachable(s, s.objects[e.object], sr, 0.001f, tmax);
                    }
                    if(eye_issue(ln, ts, batch, kQueryShadow, sr, tmax, any_mode,
                                 F.tp * (value * light.radiance * (weight / light_pdf)), 0.0f, light.emitter, false)) {
                        return true;
                    }
                }
                if(batch.n > 0) return true;
            }
            F.stage = kEyeBsdf;
            F.iter = 0;
        }
        // bsdf_samples (photon_integrator.h:219-277), one ray per visit
        const bool sample_direct = fl.smooth || (fl.specular && !fl.exhaustive);
        const bool sample_indirect = !fl.diffuse && (fl.smooth || (fl.specular && !fl.exhaustive));
        if(sample_direct || sample_indirect) {
            const EyeCounts counts = eye_counts(ep, F.depth, fl.diffuse);
            while(F.iter < counts.bsdf) {
                ++F.iter;
                BsdfCtx ctx = ctx_default(LRT_MODE_RADIANCE);
                ctx.lobe_sample = sampler_next_1d(table, ln.smp);
                if(!fl.specular || fl.exhaustive) ctx.type_mask = kSmooth;
                BRec r = rec;
                const F2 u = sampler_next_2d(table, ln.smp);
                const f3 weight = bsdf_sample(s.materials, s.tables, mid, ctx, r, u.x, u.y);
                if(is_zero(weight) || r.pdf <= 0.0f) continue;
                if(eye_issue(ln, ts, batch, kQueryBsdf, Ray{F.p, to_world(basis, r.wo)}, kInf, false, weight, r.pdf,
                             -1, sample_indirect)) {
                    return true;
                }
            }
            if(batch.n > 0) return true;
        }
        --ln.top;
    }
    return false;
}

// Hands a finished ray query's result to the lane's walk.
__device__ void eye_resume(const DeviceScene& s, const EyeParams& ep, EyeLane& ln, EyeFrame* st, int* overflow,
                           const TravState& ts, int frame_limit) {
    EyeFrame& F = st[ln.top];
    if(ln.query == kQueryHit) {
        if(ts.best >= 0) {
            HitInfo h;
            hit_record_of(s, ts.r, ts.best, ts.closest_so_far, ts.best_mesh, h);
            F.obj = h.object;
            F.p = h.p;
            F.n = h.normal;
            F.front_face = h.front_face ? 1 : 0;
        } else {
            F.obj = -1;
        }
        F.evaluated = 1;
    } else if(ln.query == kQueryShadow) {
        const bool blocked = ts.any_mode ? ts.best >= 0 : (ts.best >= 0 && s.objects[ts.best].emitter != ln.qlight);
        if(!blocked) ln.L += ln.qa;
    } else if(ln.query == kQueryBsdf) {
        const int32_t mid = s.objects[F.obj].material;
        const EyeFlags fl = eye_flags(s, ep, mid, F.depth);
        const EyeCounts counts = eye_counts(ep, F.depth, fl.diffuse);
        const bool sample_direct = fl.smooth || (fl.specular && !fl.exhaustive);
        const bool sample_indirect = !fl.diffuse && (fl.smooth || (fl.specular && !fl.exhaustive));
        const bool hit = ts.best >= 0;
        HitInfo occluder{};
        if(hit) hit_record_of(s, ts.r, ts.best, ts.closest_so_far, ts.best_mesh, occluder);
        const f3 weight = ln.qa;
        if(sample_direct) {
            f3 emission = mk(0.0f);
            float light_pdf = 0.0f;
            if(hit) {
                const ObjRec& oo = s.objects[occluder.object];
                if(oo.emitter >= 0 && occluder.front_face) {
                    emission = area_emitted(s.emitters[oo.emitter], occluder.normal, -normalize(ts.r.d));
                    light_pdf = pdf_emitter_direction(s, F.p, ts.r.d);
                }
            } else {
                emission = eval_environment(s, ts.r.d);
                light_pdf = pdf_emitter_direction(s, F.p, ts.r.d);
            }
            if(!is_zero(emission)) {
                const float mis = power_heuristic(ln.qpdf * static_cast<float>(counts.bsdf),
                                                  light_pdf * static_cast<float>(counts.emitter)) * counts.bsdf_weight;
                ln.L += F.tp * (emission * weight * mis);
            }
        }
        if(sample_indirect) {
            if(ln.top + 1 >= frame_limit) {
                *overflow = 1;
            } else {
                st[ln.top + 1] = EyeFrame{ts.r.o, ts.r.d, occluder.p, occluder.normal, F.tp * weight * counts.bsdf_weight,
                                          hit ? occluder.object : -1, static_cast<int16_t>(F.depth + 1), 0, kEyeStart, 1,
                                          0, static_cast<uint8_t>(hit && occluder.front_face ? 1 : 0)};
                ++ln.top;
            }
        }
    }
    ln.query = kQueryNone;
}

__global__ void __launch_bounds__(kBlock) k_photon_eye_persistent(DeviceScene s, EyeParams ep, uint32_t width,
                                                                  uint32_t height, uint32_t pixel_begin,
                                                                  uint32_t n_pixels, uint32_t sample_begin,
                                                                  uint32_t n_samples, float4* L_out, int* overflow,
                                                                  uint32_t* fetch) {
    EyeFrame frames[kEyeFrames];
    uint2 heap_store[kMaxKnn];
    KnnHeap heap{heap_store, 1u, 0u};
    TravItem stack[kStackSize];
    int32_t tl_stack[kTlasStack];
    TravState ts;
    EyeLane ln;
    TraceCount cnt{0, 0};
    const uint32_t n = n_pixels * n_samples;
    bool have = false, tracing = false, done = false;
    while(true) {
        while(!tracing && !done) {
            if(!have) {
                const uint32_t i = atomicAdd(fetch, 1u);
                if(i >= n) {
                    done = true;
                    break;
                }
                const uint32_t pix = pixel_begin + i / n_samples;
                const uint32_t sample = sample_begin + i % n_samples;
                ln.smp = sampler_start(pix, sample);
                const F2 off = sampler_next_2d(sobol_table(s), ln.smp);
                const float u = (static_cast<float>(pix % width) + off.x) / static_cast<float>(width - 1);
                const float v = (static_cast<float>(pix / width) + off.y) / static_cast<float>(height - 1);
                const Ray camera = camera_ray(s.cam, u, v);
                frames[0] = EyeFrame{camera.o, camera.d, mk(0.0f), mk(0.0f), mk(1.0f), -1, 1, 0, kEyeStart, 0, 1, 0};
                ln.top = 0;
                ln.L = mk(0.0f);
                ln.slot = i;
                ln.query = kQueryNone;
                have = true;
            }
            EyeBatch one{nullptr, 0};
            if(eye_advance(s, ep, ln, frames, heap, overflow, ts, kEyeFrames, one)) {
                tracing = true;
            } else {
                L_out[ln.slot] = make_float4(ln.L.x, ln.L.y, ln.L.z, 0.0f);
                have = false;
            }
        }
        if(__all_sync(0xffffffffu, done)) break;
        if(tracing && trav_step<false>(s, ts, stack, tl_stack, cnt)) {
            tracing = false;
            eye_resume(s, ep, ln, frames, overflow, ts, kEyeFrames);
        }
    }
}

// ---- wavefront eye pass ----
//
// Camera samples in flight live in slots in device memory: the walk's frames, the lane record, the
// pending ray query and its result. Each iteration k_eye_shade resumes every slot whose ray was traced
// and advances it to its next query (a finished sample writes its radiance and the slot starts the
// next sample of the wave), queueing the slot; k_eye_trace then traces the queue with the persistent
// traversal. Every sample's walk is the sequential program of eye_sample: the same draws, rays and
// additions in the same order.
enum EyeSlotState : uint32_t { kSlotIdle = 0, kSlotTracing = 1, kSlotDone = 2 };

struct EyeSlot {
    EyeLane ln;
    uint32_t state;
    uint32_t nq;  // queries of the slot's batch in flight
};

struct EyeWave {
    EyeSlot* slots;
    EyeFrame* frames;      // frame_limit frames per slot
    EyeQuery* queries;     // kEyeBatch per slot
    uint32_t* queue;       // queries to trace (slot * kEyeBatch + index)
    uint32_t* lookups;     // photon lookups (slot * kEyeBatch + index)
    uint32_t* counters;    // [0] queue length, [1] next sample, [2] trace fetch, [3] lookups, [4] slots in
                           // `order`, [5] order valid, [8, 8 + kEyeKeys) slots per key, then the key cursors
    uint32_t* order;       // the slots to shade next round, grouped by key (when counters[5] is set)
    uint32_t* slot_key;    // each slot's key for the grouping
    float4* L_out;
    int* overflow;
    uint32_t n_slots;
    uint32_t n_total;      // samples of the wave
    int frame_limit;
    uint32_t width, height, pixel_begin, n_samples, sample_begin;
};

// A slot's finished batch handed to its walk, in issue order: a photon lookup adds tp * (estimate *
// reflectance) to L as the walk would have, a ray query goes through eye_resume.
__device__ __forceinline__ void eye_apply_batch(const DeviceScene& s, const EyeParams& ep, EyeLane& ln, EyeFrame* st,
                                                const EyeQuery* queries, uint32_t nq, int* overflow, int frame_limit) {
    for(uint32_t q = 0; q < nq; ++q) {
        const EyeQuery& Q = queries[q];
        if(Q.kind == kQueryIrradiance) {
            ln.L += f3{Q.b.x, Q.b.y, Q.b.z} * (f3{Q.closest, Q.u, Q.v} * f3{Q.a.x, Q.a.y, Q.a.z});
            continue;
        }
        ln.query = static_cast<uint8_t>(Q.kind);
        ln.qa = f3{Q.a.x, Q.a.y, Q.a.z};
        ln.qpdf = Q.a.w;
        ln.qlight = Q.light;
        TravState ts;
        ts.r = Ray{f3{Q.o.x, Q.o.y, Q.o.z}, f3{Q.d.x, Q.d.y, Q.d.z}};
        ts.any_mode = Q.any_mode != 0;
        ts.best = Q.best;
        ts.closest_so_far = Q.closest;
        ts.best_mesh = MeshHit{Q.closest, Q.u, Q.v, Q.ref};
        eye_resume(s, ep, ln, st, overflow, ts, frame_limit);
    }
}

// Slots waiting for their batch are shaded grouped by the surface their walk resumes on: the key is
// 2 + the material type of the object the batch's last hit or BSDF ray found, or of the current frame's
// object for a batch of shadow rays and lookups (0: nothing hit, 1: no material). Warps then run one
// material's code, as the path tracer's per-key shading does; each slot's walk is unchanged.
constexpr int kEyeKeys = 10;
constexpr int kEyeKeyCounts = 8;  // counters[8..] per-key counts, then per-key cursors

__device__ __forceinline__ int eye_slot_key(const DeviceScene& s, const EyeSlot& S, const EyeFrame* st,
                                            const EyeQuery* queries) {
    int32_t obj = st[S.ln.top].obj;
    if(S.nq > 0) {
        const EyeQuery& Q = queries[S.nq - 1];
        if(Q.kind == kQueryHit || Q.kind == kQueryBsdf) obj = Q.best;
    }
    if(obj < 0) return 0;
    const int32_t m = s.objects[obj].material;
    return m < 0 ? 1 : 2 + static_cast<int>(s.materials[m].type);
}

__global__ void __launch_bounds__(kBlock) k_eye_order_count(DeviceScene s, EyeWave w) {
    for(uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x; slot < w.n_slots; slot += gridDim.x * blockDim.x) {
        const EyeSlot& S = w.slots[slot];
        if(S.state != kSlotTracing) continue;
        const int key = eye_slot_key(s, S, w.frames + static_cast<size_t>(slot) * w.frame_limit,
                                     w.queries + static_cast<size_t>(slot) * kEyeBatch);
        w.slot_key[slot] = static_cast<uint32_t>(key);
        warp_append_keyed(w.counters + kEyeKeyCounts, key);
    }
}

__global__ void __launch_bounds__(kBlock) k_eye_order_scatter(EyeWave w) {
    __shared__ uint32_t prefix[kEyeKeys + 1];
    if(threadIdx.x == 0) {
        uint32_t acc = 0;
        for(int k = 0; k < kEyeKeys; ++k) {
            prefix[k] = acc;
            acc += w.counters[kEyeKeyCounts + k];
        }
        prefix[kEyeKeys] = acc;
        if(blockIdx.x == 0) {
            w.counters[4] = acc;
            w.counters[5] = 1;
        }
    }
    __syncthreads();
    for(uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x; slot < w.n_slots; slot += gridDim.x * blockDim.x) {
        if(w.slots[slot].state != kSlotTracing) continue;
        const int key = static_cast<int>(w.slot_key[slot]);
        w.order[prefix[key] + warp_append_keyed(w.counters + kEyeKeyCounts + kEyeKeys, key)] = slot;
    }
}

__global__ void __launch_bounds__(kBlock) k_eye_shade(DeviceScene s, EyeParams ep, EyeWave w) {
    uint2 heap_store[kMaxKnn];
    KnnHeap heap{heap_store, 1u, 0u};
    const bool ordered = w.counters[5] != 0;
    const uint32_t n = ordered ? w.counters[4] : w.n_slots;
    for(uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t slot = ordered ? w.order[i] : i;
        EyeSlot& S = w.slots[slot];
        if(S.state == kSlotDone) continue;
        EyeFrame* st = w.frames + static_cast<size_t>(slot) * w.frame_limit;
        EyeQuery* queries = w.queries + static_cast<size_t>(slot) * kEyeBatch;
        EyeLane ln = S.ln;
        bool have = false;
        if(S.state == kSlotTracing) {
            eye_apply_batch(s, ep, ln, st, queries, S.nq, w.overflow, w.frame_limit);
            have = true;
        }
        uint32_t state = kSlotDone, nq = 0;
        while(true) {
            if(!have) {
                const uint32_t i = atomicAdd(&w.counters[1], 1u);
                if(i >= w.n_total) break;
                const uint32_t pix = w.pixel_begin + i / w.n_samples;
                const uint32_t sample = w.sample_begin + i % w.n_samples;
                ln.smp = sampler_start(pix, sample);
                const F2 off = sampler_next_2d(sobol_table(s), ln.smp);
                const float u = (static_cast<float>(pix % w.width) + off.x) / static_cast<float>(w.width - 1);
                const float v = (static_cast<float>(pix / w.width) + off.y) / static_cast<float>(w.height - 1);
                const Ray camera = camera_ray(s.cam, u, v);
                st[0] = EyeFrame{camera.o, camera.d, mk(0.0f), mk(0.0f), mk(1.0f), -1, 1, 0, kEyeStart, 0, 1, 0};
                ln.top = 0;
                ln.L = mk(0.0f);
                ln.slot = i;
                ln.query = kQueryNone;
                have = true;
            }
            TravState ts;
            EyeBatch batch{queries, 0};
            if(eye_advance(s, ep, ln, st, heap, w.overflow, ts, w.frame_limit, batch)) {
                state = kSlotTracing;
                nq = batch.n;
                uint32_t n_lookups = 0;
                for(uint32_t q = 0; q < nq; ++q) n_lookups += queries[q].kind == kQueryIrradiance ? 1u : 0u;
                const uint32_t tbase = nq > n_lookups ? atomicAdd(&w.counters[0], nq - n_lookups) : 0u;
                const uint32_t kbase = n_lookups > 0 ? atomicAdd(&w.counters[3], n_lookups) : 0u;
                for(uint32_t q = 0, t = 0, k = 0; q < nq; ++q) {
                    if(queries[q].kind == kQueryIrradiance) {
                        w.lookups[kbase + k++] = slot * kEyeBatch + q;
                    } else {
                        w.queue[tbase + t++] = slot * kEyeBatch + q;
                    }
                }
                break;
            }
            w.L_out[ln.slot] = make_float4(ln.L.x, ln.L.y, ln.L.z, 0.0f);
            have = false;
        }
        S.ln = ln;
        S.state = state;
        S.nq = nq;
    }
}

// the queued queries with the persistent traversal (closest hit, or any hit for occlusion without a
// reachable light); results written beside each query
__global__ void __launch_bounds__(kBlock) k_eye_trace(DeviceScene s, EyeWave w) {
    const uint32_t n = w.counters[0];
    TravItem stack[kStackSize];
    int32_t tl_stack[kTlasStack];
    TravState st;
    TraceCount cnt{0, 0};
    bool active = false, exhausted = n == 0;
    uint32_t entry = 0;
    while(true) {
        if(!exhausted && __popc(__ballot_sync(0xffffffffu, !active)) >= 16) {  // refill half-idle warps
            const uint32_t i = warp_fetch(&w.counters[2], !active, n, exhausted);
            if(!active && i < n) {
                entry = w.queue[i];
                const EyeQuery& Q = w.queries[entry];
                trav_begin(st, Ray{f3{Q.o.x, Q.o.y, Q.o.z}, f3{Q.d.x, Q.d.y, Q.d.z}}, Q.o.w, Q.d.w, Q.any_mode != 0);
                active = true;
            }
        }
        if(!__any_sync(0xffffffffu, active)) break;
        if(active && trav_step<false>(s, st, stack, tl_stack, cnt)) {
            EyeQuery& Q = w.queries[entry];
            Q.best = st.best;
            Q.closest = st.closest_so_far;
            Q.u = st.best_mesh.u;
            Q.v = st.best_mesh.v;
            Q.ref = st.best_mesh.ref;
            active = false;
        }
    }
}

// The wave's tail: once no sample is left to start and few slots still have queries, each remaining slot
// applies its finished batch and runs the rest of its walk alone, one query at a time traced in place
// (the persistent form's step), so that the last, deepest walks do not each cost a round of three
// launches per query. The walk, its draws and its additions are those of the other forms.
__global__ void __launch_bounds__(kBlock) k_eye_finish(DeviceScene s, EyeParams ep, EyeWave w) {
    uint2 heap_store[kMaxKnn];
    KnnHeap heap{heap_store, 1u, 0u};
    TravItem stack[kStackSize];
    int32_t tl_stack[kTlasStack];
    TraceCount cnt{0, 0};
    for(uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x; slot < w.n_slots; slot += gridDim.x * blockDim.x) {
        EyeSlot& S = w.slots[slot];
        if(S.state != kSlotTracing) continue;
        EyeFrame* st = w.frames + static_cast<size_t>(slot) * w.frame_limit;
        EyeLane ln = S.ln;
        eye_apply_batch(s, ep, ln, st, w.queries + static_cast<size_t>(slot) * kEyeBatch, S.nq, w.overflow,
                        w.frame_limit);
        while(true) {
            TravState ts;
            EyeBatch one{nullptr, 0};
            if(!eye_advance(s, ep, ln, st, heap, w.overflow, ts, w.frame_limit, one)) break;
            while(!trav_step<false>(s, ts, stack, tl_stack, cnt)) {
            }
            eye_resume(s, ep, ln, st, w.overflow, ts, w.frame_limit);
        }
        w.L_out[ln.slot] = make_float4(ln.L.x, ln.L.y, ln.L.z, 0.0f);
        S.ln = ln;
        S.state = kSlotDone;
        S.nq = 0;
    }
}

// the queued photon lookups, one per thread (photon_map::estimate_irradiance); the estimate is written
// beside each query
template <uint32_t kCap>
__global__ void __launch_bounds__(HeapBlock<kCap>::kThreads) k_eye_lookup(EyeParams ep, EyeWave w) {
    constexpr int kThreads = HeapBlock<kCap>::kThreads;
    __shared__ uint2 shared_heaps[kCap == 0 ? 1 : kCap * kThreads];
    uint2 local_heap[kCap == 0 ? kMaxKnn : 1];
    KnnHeap heap = kCap == 0 ? KnnHeap{local_heap, 1u, 0u}
                             : KnnHeap{shared_heaps + threadIdx.x, static_cast<uint32_t>(kThreads), 0u};
    const uint32_t n = w.counters[3];
    for(uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        EyeQuery& Q = w.queries[w.lookups[i]];
        const f3 E = estimate_irradiance(Q.light == 0 ? ep.global : ep.caustic, f3{Q.o.x, Q.o.y, Q.o.z},
                                         f3{Q.d.x, Q.d.y, Q.d.z}, Q.o.w, Q.any_mode, ep.lookup_size, heap);
        Q.closest = E.x;
        Q.u = E.y;
        Q.v = E.z;
    }
}

__global__ void k_photon_eye_accumulate(const float4* L, uint32_t pixel_begin, uint32_t n_pixels, uint32_t n_samples,
                                        uint32_t spp, float* sum, int first, int last, float* rgb) {
    const uint32_t pl = blockIdx.x * blockDim.x + threadIdx.x;
    if(pl >= n_pixels) return;
    f3 acc = first ? mk(0.0f) : load3(sum + 3ull * pl);
    for(uint32_t s = 0; s < n_samples; ++s) {
        const float4 v = L[static_cast<size_t>(pl) * n_samples + s];
        acc += f3{v.x, v.y, v.z};
    }
    if(last) {
        store3(rgb + 3ull * (pixel_begin + pl), acc / static_cast<float>(spp));
    } else {
        store3(sum + 3ull * pl, acc);
    }
}

MapView view_of(const PhotonMap& pm) {
    return MapView{pm.pos.as<float4>(), pm.dir.as<float4>(), pm.nrm.as<float4>(), pm.pow.as<float4>(),
                   pm.nodes.as<PhotonNode>(), pm.n, pm.scale};
}

bool unsuccessful(uint64_t needed, uint64_t stored, uint64_t shot) {
    return stored < needed && (stored == 0 || stored < shot / 1024);
}

}  // namespace

extern "C" {

int lrt_photon_trace_particles(lrt_context* ctx, int32_t kind, uint32_t first, uint32_t count, int32_t max_depth,
                               int32_t rr_depth, uint32_t max_per, lrt_photon* photons_out, uint32_t* counts_out) {
    if(!ctx) return LRT_ERR_INVALID_ARGUMENT;
    if(!ctx->has_scene) return fail(ctx, LRT_ERR_NO_SCENE, "no scene uploaded");
    if(count == 0) return LRT_OK;
    if(!photons_out || !counts_out || max_per == 0 || (kind != LRT_GATHER_SURFACE && kind != LRT_GATHER_CAUSTIC)) {
        return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "bad photon trace arguments");
    }
    const size_t pb = sizeof(lrt_photon) * static_cast<size_t>(count) * max_per, cb = 4ull * count;
    LRT_CUDA(ctx, ctx->ph_out.ensure(pb));
    LRT_CUDA(ctx, ctx->ph_counts.ensure(cb));
    LRT_CUDA(ctx, cudaMemsetAsync(ctx->ph_out.ptr, 0, pb, ctx->stream));
    k_particles_slots<<<blocks_for(count), kBlock, 0, ctx->stream>>>(ctx->ds, kind, first, count, max_depth, rr_depth,
                                                                    max_per, ctx->ph_out.as<lrt_photon>(),
                                                                    ctx->ph_counts.as<uint32_t>());
    LRT_CUDA(ctx, cudaGetLastError());
    LRT_CUDA(ctx, cudaMemcpyAsync(photons_out, ctx->ph_out.ptr, pb, cudaMemcpyDeviceToHost, ctx->stream));
    LRT_CUDA(ctx, cudaMemcpyAsync(counts_out, ctx->ph_counts.ptr, cb, cudaMemcpyDeviceToHost, ctx->stream));
    LRT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return LRT_OK;
}

}  // extern "C"

namespace {

// photon_gather::run; photons_out == nullptr leaves the photons in ctx->ph_out (device)
int photon_trace_impl(lrt_context* ctx, int32_t kind, uint32_t requested, int32_t max_depth, int32_t rr_depth,
                      lrt_photon* photons_out, uint32_t* n_out, uint64_t* shot_out) {
    if(!ctx) return LRT_ERR_INVALID_ARGUMENT;
    if(!ctx->has_scene) return fail(ctx, LRT_ERR_NO_SCENE, "no scene uploaded");
    if(!n_out || !shot_out || (kind != LRT_GATHER_SURFACE && kind != LRT_GATHER_CAUSTIC)) {
        return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "bad photon trace arguments");
    }
    *n_out = 0;
    *shot_out = 0;
    if(requested == 0 || max_depth < 1) return LRT_OK;  // photon_gather.h:20-22
    // work items of `granularity` particles as with one worker (photon_gather.h:26-28)
    const uint64_t granularity = std::max<uint64_t>(1, requested / 16);
    const uint64_t batches_per_launch = std::max<uint64_t>(1, (1ull << 21) / granularity);
    const uint64_t chunk = std::min<uint64_t>(granularity * batches_per_launch, 1ull << 24);
    LRT_CUDA(ctx, ctx->ph_out.ensure(sizeof(lrt_photon) * static_cast<size_t>(requested)));
    LRT_CUDA(ctx, ctx->ph_counts.ensure(4 * chunk));
    LRT_CUDA(ctx, ctx->ph_offsets.ensure(8 * chunk + 4 * chunk));
    LRT_CUDA(ctx, ctx->ph_stage.ensure(sizeof(lrt_photon) * kStagedPhotons * chunk));
    std::vector<uint32_t> counts(chunk);
    std::vector<uint64_t> offsets(chunk);
    std::vector<uint32_t> again;
    uint64_t stored = 0, shot = 0, returned = 0, next = 0;
    bool done = false;
    const int grid = grid_for(ctx, (const void*)k_particles_trace, kBlock);
    uint32_t* d_again = reinterpret_cast<uint32_t*>(ctx->ph_offsets.as<uint64_t>() + chunk);
    while(!done) {
        if(next + chunk > 0xffffffffull) return fail(ctx, LRT_ERR_RANGE, "particle index space exhausted");
        const uint32_t first = static_cast<uint32_t>(next);
        const uint32_t n = static_cast<uint32_t>(chunk);
        k_particles_trace<<<grid, kBlock, 0, ctx->stream>>>(ctx->ds, kind, first, n, max_depth, rr_depth,
                                                            ctx->ph_stage.as<lrt_photon>(), ctx->ph_counts.as<uint32_t>());
        LRT_CUDA(ctx, cudaGetLastError());
        LRT_CUDA(ctx, cudaMemcpyAsync(counts.data(), ctx->ph_counts.ptr, 4 * chunk, cudaMemcpyDeviceToHost, ctx->stream));
        LRT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        // walk the work items in order: generate_work's stop test, then process_result's cut
        uint64_t taken = 0;  // particles of this launch that store
        for(uint64_t b = 0; b < batches_per_launch && !done; ++b) {
            if(returned >= requested || (shot > 100000 && unsuccessful(requested, stored, shot))) {
                done = true;
                break;
            }
            uint64_t counted = 0, batch_photons = 0;
            bool full = false;
            for(uint64_t j = 0; j < granularity; ++j) {
                const uint64_t i = b * granularity + j;
                batch_photons += counts[i];
                offsets[i] = stored;
                if(full) continue;
                ++counted;
                if(counts[i] > 0 && stored >= requested) {
                    full = true;
                    continue;
                }
                const uint64_t room = requested - stored;
                if(counts[i] > room) {
                    stored = requested;
                    full = true;
                } else {
                    stored += counts[i];
                }
                taken = i + 1;
            }
            shot += counted;
            returned += batch_photons;
        }
        if(taken > 0) {
            LRT_CUDA(ctx, cudaMemcpyAsync(ctx->ph_offsets.ptr, offsets.data(), 8 * taken, cudaMemcpyHostToDevice, ctx->stream));
            k_particles_place<<<blocks_for(static_cast<uint32_t>(taken)), kBlock, 0, ctx->stream>>>(
                ctx->ph_stage.as<lrt_photon>(), ctx->ph_counts.as<uint32_t>(), ctx->ph_offsets.as<uint64_t>(),
                static_cast<uint32_t>(taken), requested, ctx->ph_out.as<lrt_photon>());
            LRT_CUDA(ctx, cudaGetLastError());
            again.clear();
            for(uint64_t i = 0; i < taken; ++i) {
                if(counts[i] > kStagedPhotons && offsets[i] < requested) again.push_back(static_cast<uint32_t>(i));
            }
            if(!again.empty()) {
                const uint32_t na = static_cast<uint32_t>(again.size());
                LRT_CUDA(ctx, cudaMemcpyAsync(d_again, again.data(), 4ull * na, cudaMemcpyHostToDevice, ctx->stream));
                k_particles_store_list<<<blocks_for(na), kBlock, 0, ctx->stream>>>(
                    ctx->ds, kind, first, d_again, na, max_depth, rr_depth, ctx->ph_offsets.as<uint64_t>(), requested,
                    ctx->ph_out.as<lrt_photon>());
                LRT_CUDA(ctx, cudaGetLastError());
            }
            LRT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        }
        next += chunk;
    }
    if(stored > 0 && photons_out) {
        LRT_CUDA(ctx, cudaMemcpyAsync(photons_out, ctx->ph_out.ptr, sizeof(lrt_photon) * stored, cudaMemcpyDeviceToHost,
                                      ctx->stream));
        LRT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    }
    *n_out = static_cast<uint32_t>(stored);
    *shot_out = shot;
    return LRT_OK;
}

// photon_map::build (photon_map.h:26-33) of photons given on the host or (photons_dev) on the device
int photon_map_build_impl(lrt_context* ctx, int32_t map, const lrt_photon* photons, const lrt_photon* photons_dev,
                          uint32_t n, float scale) {
    if(!ctx) return LRT_ERR_INVALID_ARGUMENT;
    if(map < 0 || map >= kMaxPhotonMaps) return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "photon map id out of range");
    if(n > 0 && !photons && !photons_dev) return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "null photons");
    if(n >= (1u << 30)) return fail(ctx, LRT_ERR_RANGE, "too many photons");
    LRT_CUDA(ctx, cudaSetDevice(ctx->device));
    PhotonMap& pm = ctx->maps[map];
    pm.n = n;
    pm.scale = scale;
    pm.n_nodes = 0;
    if(n == 0) return LRT_OK;
    cudaStream_t s = ctx->stream;
    std::vector<lrt_photon> host_copy;
    if(!ctx->photon_tree_device && !photons) {
        host_copy.resize(n);
        LRT_CUDA(ctx, cudaMemcpyAsync(host_copy.data(), photons_dev, sizeof(lrt_photon) * static_cast<size_t>(n),
                                      cudaMemcpyDeviceToHost, s));
        LRT_CUDA(ctx, cudaStreamSynchronize(s));
        photons = host_copy.data();
    }
    if(!ctx->photon_tree_device) {  // the same tree built on the host cores with std::nth_element itself
        std::vector<HostPhoton> ph(n);
        for(uint32_t i = 0; i < n; ++i) {
            ph[i] = HostPhoton{{photons[i].position[0], photons[i].position[1], photons[i].position[2]}, i};
        }
        std::unordered_map<int32_t, int32_t> memo;
        std::vector<PhotonNode> nodes(subtree_nodes(static_cast<int32_t>(n), memo));
        uint32_t max_depth = 0;
        const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
        int levels = 0;
        while((1u << (levels + 1)) <= hw && levels < 6) ++levels;
        build_range_parallel(ph, 0, static_cast<int32_t>(n), nodes.data(), 0, 1, max_depth, n >= (1u << 16) ? levels : 0,
                             memo);
        std::vector<uint32_t> order(n);
        for(uint32_t i = 0; i < n; ++i) order[i] = ph[i].index;
        LRT_CUDA(ctx, pm.pos.ensure(16ull * n));
        LRT_CUDA(ctx, pm.dir.ensure(16ull * n));
        LRT_CUDA(ctx, pm.nrm.ensure(16ull * n));
        LRT_CUDA(ctx, pm.pow.ensure(16ull * n));
        LRT_CUDA(ctx, pm.nodes.ensure(sizeof(PhotonNode) * nodes.size()));
        LRT_CUDA(ctx, ctx->ph_tmp.ensure(sizeof(lrt_photon) * static_cast<size_t>(n)));
        LRT_CUDA(ctx, ctx->ph_vals.ensure(4ull * n));
        LRT_CUDA(ctx, cudaMemcpyAsync(ctx->ph_tmp.ptr, photons, sizeof(lrt_photon) * static_cast<size_t>(n),
                                      cudaMemcpyHostToDevice, s));
        LRT_CUDA(ctx, cudaMemcpyAsync(ctx->ph_vals.ptr, order.data(), 4ull * n, cudaMemcpyHostToDevice, s));
        LRT_CUDA(ctx, cudaMemcpyAsync(pm.nodes.ptr, nodes.data(), sizeof(PhotonNode) * nodes.size(), cudaMemcpyHostToDevice, s));
        k_photon_gather_attrs<<<blocks_for(n), kBlock, 0, s>>>(ctx->ph_tmp.as<lrt_photon>(), ctx->ph_vals.as<uint32_t>(), n,
                                                               pm.pos.as<float4>(), pm.dir.as<float4>(), pm.nrm.as<float4>(),
                                                               pm.pow.as<float4>());
        LRT_CUDA(ctx, cudaGetLastError());
        LRT_CUDA(ctx, cudaStreamSynchronize(s));
        pm.n_nodes = static_cast<uint32_t>(nodes.size());
        pm.depth = max_depth;
        return LRT_OK;
    }
    if(!photons_dev) {
        LRT_CUDA(ctx, ctx->ph_tmp.ensure(sizeof(lrt_photon) * static_cast<size_t>(n)));
        LRT_CUDA(ctx, cudaMemcpyAsync(ctx->ph_tmp.ptr, photons, sizeof(lrt_photon) * static_cast<size_t>(n),
                                      cudaMemcpyHostToDevice, s));
        photons_dev = ctx->ph_tmp.as<lrt_photon>();
    }
    return photon_tree_build_device(ctx, pm, photons_dev, n, ctx->photon_tree_depth_limit);
}

}  // namespace

extern "C" {

int lrt_photon_trace(lrt_context* ctx, int32_t kind, uint32_t requested, int32_t max_depth, int32_t rr_depth,
                     lrt_photon* photons_out, uint32_t* n_out, uint64_t* shot_out) {
    if(ctx && requested > 0 && max_depth >= 1 && !photons_out) {
        return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "null photon buffer");
    }
    return photon_trace_impl(ctx, kind, requested, max_depth, rr_depth, photons_out, n_out, shot_out);
}

int lrt_photon_map_build(lrt_context* ctx, int32_t map, const lrt_photon* photons, uint32_t n, float scale) {
    if(ctx && n > 0 && !photons) return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "null photons");
    return photon_map_build_impl(ctx, map, photons, nullptr, n, scale);
}

int lrt_photon_map_tree(lrt_context* ctx, int32_t map, uint32_t* order, int32_t* nodes, uint64_t max_nodes,
                        uint32_t* n_nodes) {
    if(!ctx) return LRT_ERR_INVALID_ARGUMENT;
    if(map < 0 || map >= kMaxPhotonMaps || !n_nodes) return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "bad photon map query");
    const PhotonMap& pm = ctx->maps[map];
    *n_nodes = pm.n_nodes;
    if(pm.n == 0) return LRT_OK;
    if(!order || !nodes || max_nodes < pm.n_nodes) return fail(ctx, LRT_ERR_RANGE, "photon map tree: output too small");
    LRT_CUDA(ctx, cudaSetDevice(ctx->device));
    std::vector<float4> pos(pm.n);
    LRT_CUDA(ctx, cudaMemcpyAsync(pos.data(), pm.pos.ptr, 16ull * pm.n, cudaMemcpyDeviceToHost, ctx->stream));
    static_assert(sizeof(PhotonNode) == 16, "4 words per node");
    LRT_CUDA(ctx, cudaMemcpyAsync(nodes, pm.nodes.ptr, sizeof(PhotonNode) * pm.n_nodes, cudaMemcpyDeviceToHost, ctx->stream));
    LRT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    for(uint32_t i = 0; i < pm.n; ++i) {
        uint32_t bits;
        std::memcpy(&bits, &pos[i].w, 4);
        order[i] = bits;
    }
    return LRT_OK;
}

int lrt_photon_knn(lrt_context* ctx, int32_t map, const float* points, uint32_t n, float r2, uint32_t k,
                   uint32_t* idx_out, float* d2_out, uint32_t* count_out) {
    if(!ctx) return LRT_ERR_INVALID_ARGUMENT;
    if(map < 0 || map >= kMaxPhotonMaps) return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "photon map id out of range");
    if(k > kMaxKnn) return fail(ctx, LRT_ERR_RANGE, "k must be at most %u", kMaxKnn);
    if(n == 0) return LRT_OK;
    if(!points || !idx_out || !d2_out || !count_out) return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "null buffer");
    const size_t pb = 12ull * n, ib = 4ull * n * k, cb = 4ull * n;
    LRT_CUDA(ctx, ctx->scratch_a.ensure(pb + 2 * ib + cb));
    char* base = ctx->scratch_a.as<char>();
    LRT_CUDA(ctx, cudaMemcpyAsync(base, points, pb, cudaMemcpyHostToDevice, ctx->stream));
    uint32_t* di = reinterpret_cast<uint32_t*>(base + pb);
    float* dd = reinterpret_cast<float*>(base + pb + ib);
    uint32_t* dc = reinterpret_cast<uint32_t*>(base + pb + 2 * ib);
    const int grid = grid_for(ctx, (const void*)k_knn, kBlock);
    k_knn<<<grid, kBlock, 0, ctx->stream>>>(view_of(ctx->maps[map]), reinterpret_cast<float*>(base), n, r2, k, di, dd, dc);
    LRT_CUDA(ctx, cudaGetLastError());
    LRT_CUDA(ctx, cudaMemcpyAsync(idx_out, di, ib, cudaMemcpyDeviceToHost, ctx->stream));
    LRT_CUDA(ctx, cudaMemcpyAsync(d2_out, dd, ib, cudaMemcpyDeviceToHost, ctx->stream));
    LRT_CUDA(ctx, cudaMemcpyAsync(count_out, dc, cb, cudaMemcpyDeviceToHost, ctx->stream));
    LRT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return LRT_OK;
}

}  // extern "C"

namespace {

// the irradiance queries on device buffers; with count_work their k-NN work goes into the stats
// k_irradiance with the heap placement the option knn_shared_heap and k call for
template <bool kCount>
int irradiance_kernel(lrt_context* ctx, const MapView& view, const float* points, const float* normals, uint32_t n,
                      float radius, int32_t max_depth, uint32_t k, float* rgb, unsigned long long* work) {
    // shared-memory heaps only for k <= 64: a 128-entry heap leaves 32 threads per 32 KB block, 7 warps
    // per SM, and ran slower than local heaps (the large scene's eye pass, k = 100: 2.37 against 2.08 s)
    if(ctx->knn_shared_heap && k <= 64) {
        const int grid = grid_for(ctx, (const void*)k_irradiance<kCount, 64>, HeapBlock<64>::kThreads);
        k_irradiance<kCount, 64><<<grid, HeapBlock<64>::kThreads, 0, ctx->stream>>>(view, points, normals, n, radius,
                                                                                   max_depth, k, rgb, work);
    } else {
        const int grid = grid_for(ctx, (const void*)k_irradiance<kCount, 0>, HeapBlock<0>::kThreads);
        k_irradiance<kCount, 0><<<grid, HeapBlock<0>::kThreads, 0, ctx->stream>>>(view, points, normals, n, radius,
                                                                                 max_depth, k, rgb, work);
    }
    LRT_CUDA(ctx, cudaGetLastError());
    ctx->stats.kernel_launches += 1;
    return LRT_OK;
}

int irradiance_launch(lrt_context* ctx, int32_t map, const float* points, const float* normals, uint32_t n,
                      float radius, int32_t max_depth, uint32_t k, float* rgb) {
    const MapView view = view_of(ctx->maps[map]);
    if(!ctx->count_work) return irradiance_kernel<false>(ctx, view, points, normals, n, radius, max_depth, k, rgb, nullptr);
    LRT_CUDA(ctx, ctx->knn_work.ensure(4 * sizeof(unsigned long long)));
    unsigned long long* work = ctx->knn_work.as<unsigned long long>();
    LRT_CUDA(ctx, cudaMemsetAsync(work, 0, 4 * sizeof(unsigned long long), ctx->stream));
    const int st = irradiance_kernel<true>(ctx, view, points, normals, n, radius, max_depth, k, rgb, work);
    if(st != LRT_OK) return st;
    unsigned long long h[4];
    LRT_CUDA(ctx, cudaMemcpyAsync(h, work, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
    LRT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    ctx->stats.knn_queries += h[0];
    ctx->stats.knn_nodes_visited += h[1];
    ctx->stats.knn_photons_tested += h[2];
    ctx->stats.knn_photons_found += h[3];
    return LRT_OK;
}

int irradiance_check(lrt_context* ctx, int32_t map, uint32_t k) {
    if(map < 0 || map >= kMaxPhotonMaps) return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "photon map id out of range");
    if(k > kMaxKnn) return fail(ctx, LRT_ERR_RANGE, "k must be at most %u", kMaxKnn);
    return LRT_OK;
}

}  // namespace

extern "C" {

int lrt_photon_irradiance_dev(lrt_context* ctx, int32_t map, const float* points_dev, const float* normals_dev,
                              uint32_t n, float radius, int32_t max_depth, uint32_t k, float* rgb_dev) {
    if(!ctx) return LRT_ERR_INVALID_ARGUMENT;
    const int st = irradiance_check(ctx, map, k);
    if(st != LRT_OK) return st;
    if(n == 0) return LRT_OK;
    if(!points_dev || !normals_dev || !rgb_dev) return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "null buffer");
    LRT_CUDA(ctx, cudaSetDevice(ctx->device));
    return irradiance_launch(ctx, map, points_dev, normals_dev, n, radius, max_depth, k, rgb_dev);
}

int lrt_photon_irradiance(lrt_context* ctx, int32_t map, const float* points, const float* normals, uint32_t n,
                          float radius, int32_t max_depth, uint32_t k, float* rgb_out) {
    if(!ctx) return LRT_ERR_INVALID_ARGUMENT;
    const int st = irradiance_check(ctx, map, k);
    if(st != LRT_OK) return st;
    if(n == 0) return LRT_OK;
    if(!points || !normals || !rgb_out) return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "null buffer");
    LRT_CUDA(ctx, cudaSetDevice(ctx->device));
    const size_t pb = 12ull * n;
    LRT_CUDA(ctx, ctx->scratch_a.ensure(3 * pb));
    float* base = ctx->scratch_a.as<float>();
    LRT_CUDA(ctx, cudaMemcpyAsync(base, points, pb, cudaMemcpyHostToDevice, ctx->stream));
    LRT_CUDA(ctx, cudaMemcpyAsync(base + 3ull * n, normals, pb, cudaMemcpyHostToDevice, ctx->stream));
    const int r = irradiance_launch(ctx, map, base, base + 3ull * n, n, radius, max_depth, k, base + 6ull * n);
    if(r != LRT_OK) return r;
    LRT_CUDA(ctx, cudaMemcpyAsync(rgb_out, base + 6ull * n, pb, cudaMemcpyDeviceToHost, ctx->stream));
    LRT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return LRT_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------
// eye pass + preprocess entry points

namespace {

MapView view_or_empty(lrt_context* ctx, int32_t map) {
    if(map < 0 || map >= kMaxPhotonMaps) return MapView{nullptr, nullptr, nullptr, nullptr, nullptr, 0, 1.0f};
    return view_of(ctx->maps[map]);
}

int photon_render_impl(lrt_context* ctx, const lrt_render_params* p, const lrt_photon_render_params* pp, float* rgb_dev) {
    if(!ctx->has_scene) return fail(ctx, LRT_ERR_NO_SCENE, "no scene uploaded");
    if(!p || !pp || p->width < 2 || p->height < 2 || p->spp == 0) {
        return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "render parameters out of range");
    }
    if(pp->lookup_size > kMaxKnn) return fail(ctx, LRT_ERR_RANGE, "lookup_size must be at most %u", kMaxKnn);
    if(pp->max_depth < 1 || pp->max_depth > kEyeFrames || pp->direct_samples < 1 || pp->glossy_samples < 1) {
        return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "photon render parameters out of range");
    }
    const uint32_t row_begin = p->row_end > p->row_begin ? p->row_begin : 0u;
    const uint32_t row_end = p->row_end > p->row_begin ? std::min(p->row_end, p->height) : p->height;
    if(row_begin >= row_end) return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "empty row range");
    EyeParams ep;
    ep.global = view_or_empty(ctx, pp->global_map);
    ep.caustic = view_or_empty(ctx, pp->caustic_map);
    ep.global_radius = pp->global_radius;
    ep.caustic_radius = pp->caustic_radius;
    ep.max_depth = pp->max_depth;
    ep.max_specular_depth = pp->max_specular_depth;
    ep.direct_samples = pp->direct_samples;
    ep.glossy_samples = pp->glossy_samples;
    ep.lookup_size = pp->lookup_size;
    const uint32_t cap = 1u << 20;
    LRT_CUDA(ctx, ctx->ph_eye.ensure(16ull * cap + 12ull * cap + 64));
    float4* L = ctx->ph_eye.as<float4>();
    float* sum = reinterpret_cast<float*>(L + cap);
    int* overflow = reinterpret_cast<int*>(L + cap) + 3 * cap;
    uint32_t* fetch = reinterpret_cast<uint32_t*>(overflow + 4);
    LRT_CUDA(ctx, cudaMemsetAsync(overflow, 0, 4, ctx->stream));
    const int mode = ctx->photon_eye_kernel;
    const bool persistent = mode == 1;
    const int grid = grid_for(ctx, persistent ? (const void*)k_photon_eye_persistent : (const void*)k_photon_eye, kBlock);
    // wavefront slots: frames up to max_depth deep (a child is pushed only below max_depth)
    const int frame_limit = pp->max_depth;
    const uint64_t slot_bytes = sizeof(EyeSlot) + sizeof(EyeFrame) * static_cast<uint64_t>(frame_limit) +
                                (sizeof(EyeQuery) + 4) * kEyeBatch;
    // up to 2^20 slots within a budget of the option photon_eye_slot_mb (8 GB by default): with the
    // reference's 128-deep walks a slot holds ~11 KB of frames, and more slots in flight mean fewer
    // rounds for the same samples
    // rounds for the same samples; never more slots than the render has samples
    const uint64_t slot_budget = static_cast<uint64_t>(ctx->photon_eye_slot_mb) << 20;
    const uint64_t render_samples = static_cast<uint64_t>(row_end - row_begin) * p->width * p->spp;
    const uint32_t n_slots = static_cast<uint32_t>(std::max<uint64_t>(
        1, std::min<uint64_t>(render_samples, std::max<uint64_t>(1024, std::min<uint64_t>(1u << 20, slot_budget / slot_bytes)))));
    EyeWave w{};
    if(mode == 2) {
        LRT_CUDA(ctx, ctx->eye_slots.ensure(sizeof(EyeSlot) * n_slots));
        LRT_CUDA(ctx, ctx->eye_frames.ensure(sizeof(EyeFrame) * static_cast<size_t>(n_slots) * frame_limit));
        LRT_CUDA(ctx, ctx->eye_queue.ensure(8ull * kEyeBatch * n_slots + 256 + 8ull * n_slots));
        LRT_CUDA(ctx, ctx->eye_queries.ensure(sizeof(EyeQuery) * kEyeBatch * static_cast<size_t>(n_slots)));
        w.slots = ctx->eye_slots.as<EyeSlot>();
        w.frames = ctx->eye_frames.as<EyeFrame>();
        w.queries = ctx->eye_queries.as<EyeQuery>();
        w.queue = ctx->eye_queue.as<uint32_t>();
        w.counters = w.queue + static_cast<size_t>(kEyeBatch) * n_slots;
        w.lookups = w.counters + 64;
        w.order = w.lookups + static_cast<size_t>(kEyeBatch) * n_slots;
        w.slot_key = w.order + n_slots;
        w.L_out = L;
        w.overflow = overflow;
        w.frame_limit = frame_limit;
        w.width = p->width;
        w.height = p->height;
    }
    const int g_shade = grid_for(ctx, (const void*)k_eye_shade, kBlock);
    const int g_trace = grid_for(ctx, (const void*)k_eye_trace, kBlock);
    // photon lookups: heaps in shared memory for k <= 64 (option knn_shared_heap), else in local memory
    const uint32_t heap_cap = ctx->knn_shared_heap && pp->lookup_size <= 64 ? 64u : 0u;
    const void* lookup_kernel = heap_cap == 0 ? (const void*)k_eye_lookup<0> : (const void*)k_eye_lookup<64>;
    const int lookup_threads = heap_cap == 0 ? HeapBlock<0>::kThreads : HeapBlock<64>::kThreads;
    const int g_lookup = grid_for(ctx, lookup_kernel, lookup_threads);
    const int g_finish = grid_for(ctx, (const void*)k_eye_finish, kBlock);
    const int g_order = grid_for(ctx, (const void*)k_eye_order_count, kBlock);
    const uint32_t spp = p->spp;
    // the wavefront form keeps refilling its slots from one large pool of samples, so that the slow drain
    // of the longest walks happens once per pool rather than once per 2^20 samples
    const uint32_t wave_cap = mode == 2 ? (1u << 26) : cap;
    const uint32_t samples_per_wave = std::min(spp, wave_cap);
    const uint32_t pixels_per_wave = std::max(1u, wave_cap / samples_per_wave);
    const uint32_t pix0 = row_begin * p->width, pix1 = row_end * p->width;
    if(mode == 2) {
        const uint64_t pool = std::min<uint64_t>(wave_cap, static_cast<uint64_t>(pix1 - pix0) * spp);
        const uint64_t pixels = std::min<uint64_t>(pixels_per_wave, pix1 - pix0);
        LRT_CUDA(ctx, ctx->eye_L.ensure(16 * pool + 12 * pixels));
        L = ctx->eye_L.as<float4>();
        sum = reinterpret_cast<float*>(L + pool);
        w.L_out = L;
    }
    for(uint32_t pb = pix0; pb < pix1; pb += pixels_per_wave) {
        const uint32_t np = std::min(pixels_per_wave, pix1 - pb);
        for(uint32_t sb = 0; sb < spp; sb += samples_per_wave) {
            const uint32_t ns = std::min(samples_per_wave, spp - sb);
            if(mode == 2) {
                w.n_total = np * ns;
                w.n_slots = std::min(n_slots, w.n_total);
                w.pixel_begin = pb;
                w.n_samples = ns;
                w.sample_begin = p->sample_offset + sb;
                LRT_CUDA(ctx, cudaMemsetAsync(w.slots, 0, sizeof(EyeSlot) * w.n_slots, ctx->stream));
                LRT_CUDA(ctx, cudaMemsetAsync(w.counters, 0, 256, ctx->stream));
                // rounds of (advance every slot to its next query, trace the queued queries), kEyeRounds at a
                // time without a host round trip: the trace kernel reads the queue length on the device, and
                // rounds past the last query find every slot done and launch no work. The host reads the
                // last round's queue length after each batch: zero means every sample is finished.
                constexpr int kEyeRounds = 16;
                while(true) {
                    for(int r = 0; r < kEyeRounds; ++r) {
                        LRT_CUDA(ctx, cudaMemsetAsync(w.counters, 0, 4, ctx->stream));
                        LRT_CUDA(ctx, cudaMemsetAsync(w.counters + 2, 0, 8, ctx->stream));
                        k_eye_shade<<<g_shade, kBlock, 0, ctx->stream>>>(ctx->ds, ep, w);
                        k_eye_trace<<<g_trace, kBlock, 0, ctx->stream>>>(ctx->ds, w);
                        if(heap_cap == 0) {
                            k_eye_lookup<0><<<g_lookup, lookup_threads, 0, ctx->stream>>>(ep, w);
                        } else {
                            k_eye_lookup<64><<<g_lookup, lookup_threads, 0, ctx->stream>>>(ep, w);
                        }
                        if(ctx->photon_eye_sort) {  // next round's shading order, grouped by key
                            LRT_CUDA(ctx, cudaMemsetAsync(w.counters + kEyeKeyCounts, 0, 8 * kEyeKeys, ctx->stream));
                            k_eye_order_count<<<g_order, kBlock, 0, ctx->stream>>>(ctx->ds, w);
                            k_eye_order_scatter<<<g_order, kBlock, 0, ctx->stream>>>(w);
                        }
                    }
                    ctx->stats.kernel_launches += (ctx->photon_eye_sort ? 5 : 3) * kEyeRounds;
                    uint32_t queued[4] = {0, 0, 0, 0};
                    LRT_CUDA(ctx, cudaMemcpyAsync(queued, w.counters, 16, cudaMemcpyDeviceToHost, ctx->stream));
                    LRT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
                    if(queued[0] == 0 && queued[3] == 0) break;
                    // the tail: every sample started and few queries left -- finish the walks in place
                    if(queued[1] >= w.n_total && queued[0] + queued[3] <= ctx->photon_eye_tail) {
                        k_eye_finish<<<g_finish, kBlock, 0, ctx->stream>>>(ctx->ds, ep, w);
                        LRT_CUDA(ctx, cudaGetLastError());
                        ctx->stats.kernel_launches += 1;
                        break;
                    }
                }
            } else if(persistent) {
                LRT_CUDA(ctx, cudaMemsetAsync(fetch, 0, 4, ctx->stream));
                k_photon_eye_persistent<<<grid, kBlock, 0, ctx->stream>>>(ctx->ds, ep, p->width, p->height, pb, np,
                                                                          p->sample_offset + sb, ns, L, overflow, fetch);
            } else {
                k_photon_eye<<<grid, kBlock, 0, ctx->stream>>>(ctx->ds, ep, p->width, p->height, pb, np,
                                                               p->sample_offset + sb, ns, L, overflow);
            }
            k_photon_eye_accumulate<<<blocks_for(np), kBlock, 0, ctx->stream>>>(L, pb, np, ns, spp, sum, sb == 0 ? 1 : 0,
                                                                                sb + ns >= spp ? 1 : 0, rgb_dev);
            LRT_CUDA(ctx, cudaGetLastError());
            ctx->stats.kernel_launches += mode == 2 ? 1 : 2;
        }
    }
    int h_overflow = 0;
    LRT_CUDA(ctx, cudaMemcpyAsync(&h_overflow, overflow, 4, cudaMemcpyDeviceToHost, ctx->stream));
    LRT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    ctx->stats.paths += static_cast<uint64_t>(pix1 - pix0) * spp;
    if(h_overflow) return fail(ctx, LRT_ERR_RANGE, "photon eye pass: recursion deeper than %d levels", kEyeFrames);
    return LRT_OK;
}

}  // namespace

extern "C" {

int lrt_render_photon_dev(lrt_context* ctx, const lrt_render_params* params, const lrt_photon_render_params* pp,
                          float* rgb_dev) {
    if(!ctx) return LRT_ERR_INVALID_ARGUMENT;
    if(!rgb_dev) return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "null output");
    LRT_CUDA(ctx, cudaSetDevice(ctx->device));
    return photon_render_impl(ctx, params, pp, rgb_dev);
}

int lrt_render_photon(lrt_context* ctx, const lrt_render_params* params, const lrt_photon_render_params* pp, float* rgb) {
    if(!ctx) return LRT_ERR_INVALID_ARGUMENT;
    if(!rgb || !params) return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "null argument");
    LRT_CUDA(ctx, cudaSetDevice(ctx->device));
    const size_t bytes = sizeof(float) * 3 * static_cast<size_t>(params->width) * params->height;
    LRT_CUDA(ctx, ctx->out_rgb.ensure(bytes));
    LRT_CUDA(ctx, cudaMemsetAsync(ctx->out_rgb.ptr, 0, bytes, ctx->stream));
    const int st = photon_render_impl(ctx, params, pp, ctx->out_rgb.as<float>());
    if(st != LRT_OK) return st;
    LRT_CUDA(ctx, cudaMemcpyAsync(rgb, ctx->out_rgb.ptr, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    LRT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return LRT_OK;
}

// photon_integrator::preprocess (photon_integrator.h:15-37): radii from the scene's bounding sphere
// (capped at radius_cap), the global gather, the caustic gather when the scene has a specular BSDF, and
// a map for each gather that reached its request (maps 0 and 1).
int lrt_photon_preprocess(lrt_context* ctx, uint32_t global_photons, uint32_t caustic_photons, int32_t max_depth,
                          int32_t rr_depth, float radius_cap, lrt_photon_render_params* out, uint64_t* shots) {
    if(!ctx || !out) return LRT_ERR_INVALID_ARGUMENT;
    if(!ctx->has_scene) return fail(ctx, LRT_ERR_NO_SCENE, "no scene uploaded");
    const float radius = ctx->host.bounding_radius;
    out->global_radius = smin(radius_cap, 0.05f * radius);
    out->caustic_radius = smin(radius_cap, 0.0125f * radius);
    out->global_map = -1;
    out->caustic_map = -1;
    const uint32_t requested[2] = {global_photons, ctx->host.has_delta_bsdf ? caustic_photons : 0u};
    const int32_t kinds[2] = {LRT_GATHER_SURFACE, LRT_GATHER_CAUSTIC};
    for(int m = 0; m < 2; ++m) {
        if(shots) shots[m] = 0;
        if(requested[m] == 0) continue;
        uint32_t n = 0;
        uint64_t shot = 0;
        // the photons stay on the device (ctx->ph_out) for the map build
        int st = photon_trace_impl(ctx, kinds[m], requested[m], max_depth - 1, rr_depth, nullptr, &n, &shot);
        if(st != LRT_OK) return st;
        if(shots) shots[m] = shot;
        if(n != requested[m]) continue;  // not full: the reference leaves the map empty
        st = photon_map_build_impl(ctx, m, nullptr, ctx->ph_out.as<lrt_photon>(), n, 1.0f / static_cast<float>(shot));
        if(st != LRT_OK) return st;
        if(m == 0) {
            out->global_map = 0;
        } else {
            out->caustic_map = 1;
        }
    }
    return LRT_OK;
}

}  // extern "C"
