// lrt_api.cu — liblrt: context, scene upload, parity kernels and the wavefront path tracer, behind
// the C ABI of include/lrt.h. sm_100a only; no CPU fallback: every entry point that computes runs its
// CUDA kernels or returns an error.
//
// Wavefront path tracer (one render = a sequence of waves; a wave = all samples of a pixel range):
//   raygen      camera rays of every (pixel, sample) slot of the wave        main.cpp:121-132
//   extend      closest hit of every active path + append to the shading      path_integrator.h:31
//               queue of its material type (warp-aggregated match/ballot)
//   shade       miss/emission + MIS, NEE light sample + BSDF eval/pdf (emits  path_integrator.h:32-166
//               a shadow ray), BSDF sample, Russian roulette; survivors are
//               compacted into the next queue
//   shadow      closest-emitter query of each shadow ray; unoccluded rays add path_integrator.h:113-125
//               their precomputed NEE contribution
//   accumulate  per-pixel sum over the wave's samples in sample order         main.cpp:133-136
// Every stage reads its queue length on the device, so the grid sizes are fixed (SM count x resident
// blocks, grid-stride loops) and no host round trip happens inside a wave.
#include <algorithm>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "lrt_adjoint.cuh"
#include "lrt_context.cuh"
#include "lrt_scene.cuh"

using namespace lrt;

namespace lrt {

int job_records(lrt_context* ctx, const lrt_job_desc* jobs, uint32_t n_jobs, std::vector<JobRec>& recs,
                unsigned long long& total, unsigned long long& out_floats) {
    recs.resize(n_jobs);
    total = 0;
    out_floats = 0;
    for(uint32_t i = 0; i < n_jobs; ++i) {
        const lrt_job_desc& j = jobs[i];
        if(j.width < 2 || j.height < 2 || j.spp == 0) return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "job %u: bad size", i);
        if(static_cast<uint64_t>(j.width) * j.height > 0x3fffffffull) return fail(ctx, LRT_ERR_RANGE, "job %u: image too large", i);
        if(j.override_object >= ctx->ds.n_objects || j.override_material >= ctx->ds.n_materials ||
           (j.override_object >= 0 && j.override_material < 0)) {
            return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "job %u: material override out of range", i);
        }
        JobRec& r = recs[i];
        r.cam = camera_from_desc(j.camera);
        r.width = j.width;
        r.height = j.height;
        r.spp = j.spp;
        r.sample_offset = j.sample_offset;
        r.override_obj = j.override_object;
        r.override_mat = j.override_object >= 0 ? j.override_material : -1;
        r.path_begin = total;
        r.out_offset = j.output_offset;
        total += static_cast<unsigned long long>(j.width) * j.height * j.spp;
        out_floats = std::max<unsigned long long>(out_floats, j.output_offset + 3ull * j.width * j.height);
    }
    return LRT_OK;
}

}  // namespace lrt

namespace {

template <typename V>
cudaError_t upload(DevBuf& buf, const V& v, cudaStream_t s, uint64_t& bytes) {
    using T = typename V::value_type;
    const size_t n = std::max<size_t>(1, v.size()) * sizeof(T);
    cudaError_t e = buf.ensure(n);
    if(e != cudaSuccess) return e;
    if(!v.empty()) {
        e = cudaMemcpyAsync(buf.ptr, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s);
        bytes += v.size() * sizeof(T);
    }
    return e;
}

// ================================ parity kernels ================================

__global__ void k_trace(DeviceScene s, const lrt_ray* rays, uint32_t n, lrt_hit* hits) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= n) return;
    const lrt_ray in = rays[i];
    const Ray r{load3(in.origin), load3(in.direction)};
    HitInfo h;
    TraceCount cnt{0, 0};
    lrt_hit out;
    memset(&out, 0, sizeof(out));
    out.object = -1;
    out.prim = -1;
    if(scene_hit<false>(s, r, in.t_min, in.t_max, h, cnt)) {
        out.t = h.t;
        out.object = h.object;
        out.prim = h.prim;
        out.front_face = h.front_face ? 1 : 0;
        store3(out.p, h.p);
        store3(out.normal, h.normal);
    }
    hits[i] = out;
}

// shadow-ray occlusion as the path tracer evaluates it (early-exit any-hit unless the light is reachable)
__global__ void k_occluded(DeviceScene s, const lrt_ray* rays, uint32_t n, int32_t light, uint8_t* out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= n) return;
    const lrt_ray in = rays[i];
    TraceCount cnt{0, 0};
    out[i] = scene_occluded<false>(s, Ray{load3(in.origin), load3(in.direction)}, in.t_min, in.t_max, light, cnt) ? 1 : 0;
}

__global__ void k_bsdf(DeviceScene s, int32_t mid, const lrt_bsdf_query* q, uint32_t n, lrt_bsdf_result* out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= n) return;
    const lrt_bsdf_query in = q[i];
    const BsdfCtx c{in.mode, in.type_mask, in.component, in.lobe_sample};
    BRec r{};
    r.wi = load3(in.wi);
    r.wo = mk(0.0f);
    r.front_face = in.front_face != 0;
    const f3 w = bsdf_sample(s.materials, s.tables, mid, c, r, in.u[0], in.u[1]);
    lrt_bsdf_result o;
    store3(o.sample_weight, w);
    store3(o.sample_wo, r.wo);
    o.sample_pdf = r.pdf;
    o.sample_eta = r.eta;
    o.sampled_type = r.sampled_type;
    o.sampled_component = r.sampled_component;
    BRec e{};
    e.wi = load3(in.wi);
    e.wo = load3(in.wo);
    e.front_face = in.front_face != 0;
    e.eta = 1.0f;
    const int meas = in.measure == LRT_MEASURE_DISCRETE ? kDiscrete : kSolidAngle;
    store3(o.eval, bsdf_eval(s.materials, s.tables, mid, c, e, meas));
    o.pdf = bsdf_pdf(s.materials, s.tables, mid, c, e, meas);
    out[i] = o;
}

__global__ void k_sky(DeviceScene s, const float* dirs, uint32_t n, float* rgb) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= n) return;
    store3(rgb + 3ull * i, eval_environment(s, load3(dirs + 3ull * i)));
}

__global__ void k_sampler(const uint32_t* table, const uint32_t* ps, uint32_t n, uint32_t dims, float* out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= n) return;
    const uint32_t(*t)[32] = reinterpret_cast<const uint32_t(*)[32]>(table);
    Sampler smp = sampler_start(ps[2 * i], ps[2 * i + 1]);
    for(uint32_t d = 0; d < dims; ++d) out[static_cast<size_t>(i) * dims + d] = sampler_next_1d(t, smp);
}

// emitter sampling parity: same record layout as the reference harness (16 floats)
__global__ void k_emitter(DeviceScene s, const float* points, const float* u2, const float* dirs, uint32_t n, float* out,
                          float* pdf_out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= n) return;
    const f3 p = load3(points + 3ull * i);
    DirectSample ds{};
    ds.distance = kInf;
    const bool ok = sample_emitter_direction(s, p, u2[2 * i], u2[2 * i + 1], ds);
    float* o = out + 16ull * i;
    o[0] = ok ? 1.0f : 0.0f;
    store3(o + 1, ds.direction);
    store3(o + 4, ds.point);
    o[7] = o[8] = o[9] = 0.0f;
    o[10] = ds.pdf;
    o[11] = ds.distance;
    store3(o + 12, ds.radiance);
    o[15] = ok ? static_cast<float>(ds.emitter) : -1.0f;
    pdf_out[i] = pdf_emitter_direction(s, p, load3(dirs + 3ull * i));
}

__global__ void k_camera(DeviceScene s, uint32_t width, uint32_t height, const uint32_t* ps, uint32_t n, lrt_ray* rays) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= n) return;
    const uint32_t pixel = ps[2 * i];
    Sampler smp = sampler_start(pixel, ps[2 * i + 1]);
    const F2 off = sampler_next_2d(sobol_table(s), smp);
    const float u = (static_cast<float>(pixel % width) + off.x) / static_cast<float>(width - 1);
    const float v = (static_cast<float>(pixel / width) + off.y) / static_cast<float>(height - 1);
    const Ray r = camera_ray(s.cam, u, v);
    lrt_ray out;
    store3(out.origin, r.o);
    store3(out.direction, r.d);
    out.t_min = 0.001f;
    out.t_max = kInf;
    rays[i] = out;
}

// ================================ wavefront path tracer ================================

struct WaveArgs {
    DeviceScene s;
    float4* o;       // ray origin
    float4* d;       // ray direction
    float4* tp;      // throughput rgb, eta
    float4* L;       // radiance rgb
    float2* misc;    // solid-angle pdf, have_pdf (0/1)
    uint2* id;       // pixel index, sample index
    float4* hit_p;   // hit point, object index bits
    float4* hit_n;   // shading normal, front_face
    uint32_t* q0;    // active queue (even bounces read q0)
    uint32_t* q1;
    uint32_t* keyed; // kKeys segments of `capacity`
    float4* sh_o;    // shadow origin, tmax
    float4* sh_d;    // shadow direction, light index bits
    float4* sh_c;    // contribution rgb, path id bits (a sky sample: the contribution before its radiance)
    float* sh_s;     // a sky sample: the factor w / light_pdf applied after the radiance
    BounceCounters* counters;
    unsigned long long* work;  // [0] nodes, [1] triangles, [2] shading events, [3] extension rays, [4] shadow rays
    float* sum;      // per-pixel running sums (3 floats per pixel of the wave)
    uint32_t capacity;
    uint32_t width, height;
    uint32_t pixel_begin;    // first pixel of the wave (row-major over the image)
    uint32_t n_pixels;
    uint32_t sample_begin;   // first sample index of the wave
    uint32_t n_samples;      // samples per pixel in this wave
    int32_t max_depth, rr_depth;
    // batched jobs (null for single-image renders)
    const JobRec* jobs;
    uint32_t n_jobs;
    uint32_t* path_job;             // job of each slot
    unsigned long long* wave_base;  // first batch path of the current wave (device, advanced per wave)
    unsigned long long total_paths;
    float* batch_out;
    float* batch_sums;              // running per-pixel sums where a pixel spans waves
    uint32_t pixel_tile;            // path order within a job: bands of this many rows, column by column
    // path-replay adjoint (null for renders)
    const float* adjoint;           // dLoss/dimage, batch output layout
    DiffDev diff;
    uint32_t adj_kmax;              // groups per material at most
    uint32_t* adj_vmask;            // per slot: depths whose sampled direction carries a derivative record
    int32_t* adj_vmid;              // [depth][capacity] material of that record
    float4* adj_lsnap;              // [depth][capacity] radiance gathered through depth (incl. its NEE)
    float4* adj_dlog;               // [depth][kmax][capacity] dE/E of the sampled direction per group
    int32_t* adj_sh_mid;            // [2 capacity] material of each shadow ray's vertex, -1 none
    uint8_t* adj_sh_vis;            // [2 capacity] shadow ray unoccluded
    float4* adj_sh_prod;            // [kmax][2 capacity] adjoint x dNEE per group
    double* adj_grad;
};

// the material of object `obj` for path `pid`: a batch job may replace one object's material
__device__ __forceinline__ int32_t effective_material(const WaveArgs& a, uint32_t pid, int32_t obj) {
    int32_t m = a.s.objects[obj].material;
    if(a.jobs) {
        const JobRec& j = a.jobs[a.path_job[pid]];
        if(obj == j.override_obj) m = j.override_mat;
    }
    return m;
}

__global__ void __launch_bounds__(kBlock) k_raygen(WaveArgs a) {
    const uint32_t n = a.n_pixels * a.n_samples;
    for(uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x; slot < n; slot += gridDim.x * blockDim.x) {
        const uint32_t pix = a.pixel_begin + slot / a.n_samples;
        const uint32_t sample = a.sample_begin + slot % a.n_samples;
        Sampler smp = sampler_start(pix, sample);
        const F2 off = sampler_next_2d(sobol_table(a.s), smp);
        const float u = (static_cast<float>(pix % a.width) + off.x) / static_cast<float>(a.width - 1);
        const float v = (static_cast<float>(pix / a.width) + off.y) / static_cast<float>(a.height - 1);
        const Ray r = camera_ray(a.s.cam, u, v);
        a.o[slot] = make_float4(r.o.x, r.o.y, r.o.z, 0.0f);
        a.d[slot] = make_float4(r.d.x, r.d.y, r.d.z, 0.0f);
        a.tp[slot] = make_float4(1.0f, 1.0f, 1.0f, 1.0f);
        a.L[slot] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        a.misc[slot] = make_float2(0.0f, 0.0f);
        a.id[slot] = make_uint2(pix, sample);
        const int seg = heavy_key(a.s, r, 0.001f, kInf);
        a.q0[static_cast<size_t>(seg) * a.capacity + warp_append_keyed(a.counters[0].active, seg)] = slot;
    }
}

// ---- persistent traversal: every lane keeps a ray and idle lanes take new ones from the queue inside
// the traversal loop (ray replacement), so a warp's lanes stay busy while its rays need very different
// numbers of nodes: occlusion rays are fetched as soon as a lane is idle, closest-hit rays once three
// quarters of the warp are (a fetch, one atomic and the new rays' loads, stalls the warp's busy lanes
// too: on the seven-material step's extension rays 12 idle lanes gave 210 ms, 16 205 ms, 20 201 ms,
// 24 200 ms). The per-ray work is the state machine of trav_step.


// closest hits of the active queue; writes the raw result (t, u, v, object) and the leaf reference
constexpr int kRefillLanes = 24;  // idle lanes of a warp before k_extend_persistent fetches new rays

template <bool kCount>
__global__ void __launch_bounds__(kBlock, 8) k_extend_persistent(WaveArgs a, int depth) {
    const uint32_t* queue = (depth & 1) ? a.q1 : a.q0;
    BounceCounters& bc = a.counters[depth];
    const uint32_t n0 = bc.active[0];
    const uint32_t n = n0 + bc.active[1];
    TravItem stack[kStackSize];
    int32_t tl_stack[kTlasStack];
    TravState st;
    TraceCount cnt{0, 0};
    uint32_t rays = 0;
    bool active = false, exhausted = n == 0;
    uint32_t pid = 0;
    while(true) {
        // refill only once half the warp is idle: a fetch per finished ray costs more than the idle lanes
        if(!exhausted && __popc(__ballot_sync(0xffffffffu, !active)) >= kRefillLanes) {
            const uint32_t i = warp_fetch(&bc.pad[0], !active, n, exhausted);
            if(!active && i < n) {
                pid = i < n0 ? queue[i] : queue[a.capacity + (i - n0)];
                const float4 o = a.o[pid];
                const float4 d = a.d[pid];
                trav_begin(st, Ray{f3{o.x, o.y, o.z}, f3{d.x, d.y, d.z}}, 0.001f, kInf, false);
                active = true;
                ++rays;
            }
        }
        if(!__any_sync(0xffffffffu, active)) break;
        if(active && trav_step<kCount>(a.s, st, stack, tl_stack, cnt)) {
            a.hit_p[pid] = make_float4(st.closest_so_far, st.best_mesh.u, st.best_mesh.v, __int_as_float(st.best));
            a.hit_n[pid] = make_float4(__uint_as_float(st.best_mesh.ref), 0.0f, 0.0f, 0.0f);
            active = false;
        }
    }
    if(kCount) {
        add_count(&a.work[0], cnt.nodes);
        add_count(&a.work[1], cnt.tris);
        add_count(&a.work[3], rays);
        if(blockIdx.x == 0 && threadIdx.x == 0 && depth < LRT_MAX_STAT_DEPTH) {
            atomicAdd(&a.work[8 + depth], static_cast<unsigned long long>(n));
        }
    }
}

// the material-type shading queues of the raw results, in queue order; each shading kernel computes the
// full hit record of its own hits (hit_p / hit_n keep the raw result: t, u, v, object; leaf reference)
__global__ void __launch_bounds__(kBlock) k_hitrec(WaveArgs a, int depth) {
    const uint32_t* queue = (depth & 1) ? a.q1 : a.q0;
    BounceCounters& bc = a.counters[depth];
    const uint32_t n0 = bc.active[0];
    const uint32_t n = n0 + bc.active[1];
    for(uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t pid = i < n0 ? queue[i] : queue[a.capacity + (i - n0)];
        const float4 raw = a.hit_p[pid];
        const int32_t best = __float_as_int(raw.w);
        int key = 0;
        if(best >= 0) {
            const int32_t mat = effective_material(a, pid, best);
            key = mat < 0 ? 1 : 2 + a.s.materials[mat].type;
        }
        const uint32_t slot = warp_append_keyed(bc.key_count, key);
        a.keyed[static_cast<size_t>(key) * a.capacity + slot] = pid;
    }
}

// A shadow record's light index carries two flags: a sky sample whose radiance waits for the ray's
// visibility, and that ray found unoccluded. The shading kernels sample the sky's direction only; the
// FP64 sky model (env_emitter::eval) then runs in k_shadow_sky for the unoccluded rays alone, and the
// contribution is ((throughput * f) * radiance) * (w / light_pdf), the expression of path_integrator.h:118.
constexpr int32_t kShadowSkyDeferred = 1 << 30;
constexpr int32_t kShadowSkyVisible = 1 << 29;
constexpr int32_t kShadowLightMask = kShadowSkyVisible - 1;

__global__ void __launch_bounds__(kBlock) k_shadow_sky(WaveArgs a, int depth) {
    const BounceCounters& bc = a.counters[depth];
    const uint32_t n0 = bc.shadow[0];
    const uint32_t n = n0 + bc.shadow[1];
    for(uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const size_t k = i < n0 ? i : a.capacity + (i - n0);
        const float4 d = a.sh_d[k];
        const int32_t bits = __float_as_int(d.w);
        if((bits & (kShadowSkyDeferred | kShadowSkyVisible)) != (kShadowSkyDeferred | kShadowSkyVisible)) continue;
        const f3 radiance = env_eval(a.s.emitters[bits & kShadowLightMask], f3{d.x, d.y, d.z});
        const float4 c = a.sh_c[k];
        const f3 contrib = f3{c.x, c.y, c.z} * radiance * a.sh_s[k];
        const uint32_t p = __float_as_uint(c.w);
        float4 L = a.L[p];
        L.x += contrib.x;
        L.y += contrib.y;
        L.z += contrib.z;
        a.L[p] = L;
    }
}

// shadow rays with ray replacement: any-hit unless the light's own shape is reachable (then the
// closest hit decides, scene_occluded)
template <bool kCount, bool kVis = false>
__global__ void __launch_bounds__(kBlock, 8) k_shadow_persistent(WaveArgs a, int depth) {
    BounceCounters& bc = a.counters[depth];
    const uint32_t n0 = bc.shadow[0];
    const uint32_t n = n0 + bc.shadow[1];
    TravItem stack[kStackSize];
    int32_t tl_stack[kTlasStack];
    TravState st;
    TraceCount cnt{0, 0};
    uint32_t rays = 0;
    bool active = false, exhausted = n == 0;
    size_t k = 0;
    int32_t light = 0;
    while(true) {
        if(!exhausted && __any_sync(0xffffffffu, !active)) {
            const uint32_t i = warp_fetch(&bc.pad[1], !active, n, exhausted);
            if(!active && i < n) {
                k = i < n0 ? i : a.capacity + (i - n0);
                const float4 o = a.sh_o[k], d = a.sh_d[k];
                light = __float_as_int(d.w) & kShadowLightMask;
                const Ray r{f3{o.x, o.y, o.z}, f3{d.x, d.y, d.z}};
                bool any_mode = true;
                const EmitRec& e = a.s.emitters[light];
                if(e.kind == LRT_EMITTER_AREA) any_mode = !light_shape_reachable(a.s, a.s.objects[e.object], r, 0.001f, o.w);
                trav_begin(st, r, 0.001f, o.w, any_mode);
                active = true;
                ++rays;
            }
        }
        if(!__any_sync(0xffffffffu, active)) break;
        if(active && trav_step<kCount, true>(a.s, st, stack, tl_stack, cnt)) {
            const bool blocked = st.any_mode ? st.best >= 0 : (st.best >= 0 && a.s.objects[st.best].emitter != light);
            if(kVis) a.adj_sh_vis[k] = blocked ? 0 : 1;
            const int32_t bits = __float_as_int(a.sh_d[k].w);
            if(!blocked && (bits & kShadowSkyDeferred)) {  // k_shadow_sky adds it with the sky's radiance
                reinterpret_cast<int32_t*>(a.sh_d + k)[3] = bits | kShadowSkyVisible;
            } else if(!blocked) {
                const float4 c = a.sh_c[k];
                const uint32_t p = __float_as_uint(c.w);
                float4 L = a.L[p];
                L.x += c.x;
                L.y += c.y;
                L.z += c.z;
                a.L[p] = L;
            }
            active = false;
        }
    }
    if(kCount) {
        add_count(&a.work[5], cnt.nodes);
        add_count(&a.work[6], cnt.tris);
        add_count(&a.work[4], rays);
    }
}

// one bounce of shading; kAdj adds the adjoint's derivative records (sampled direction, NEE)
// kKey < 0: every shading key's segment in one launch; kKey >= 0: that key's segment only (0 misses,
// 1 hits without a BSDF, 2 + t materials of type t), with only that type's BSDF code compiled in
template <bool kAdj, int kKey = -1>
__device__ __forceinline__ void shade_wave(const WaveArgs& a, int depth, uint32_t* prefix) {
    constexpr int kType = kKey >= 2 ? kKey - 2 : -1;
    constexpr bool kMeshLights = kKey < 0;  // the per-key kernels run only on scenes without mesh lights
    constexpr bool kDeferSky = !kAdj;       // the adjoint needs the sky radiance of every NEE sample here
    BounceCounters& bc = a.counters[depth];
    if(kKey < 0 && threadIdx.x == 0) {
        uint32_t acc = 0;
        for(int k = 0; k < kKeys; ++k) {
            prefix[k] = acc;
            acc += bc.key_count[k];
        }
        prefix[kKeys] = acc;
    }
    if(kKey < 0) __syncthreads();
    const uint32_t total = kKey < 0 ? prefix[kKeys] : bc.key_count[kKey < 0 ? 0 : kKey];
    uint32_t* next = (depth & 1) ? a.q0 : a.q1;
    BounceCounters& nc = a.counters[depth + 1];
    const DeviceScene& s = a.s;
    uint32_t shading = 0;
    for(uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        int key = kKey;
        uint32_t pid;
        if(kKey < 0) {
            key = 0;
            while(key + 1 < kKeys && prefix[key + 1] <= i) ++key;
            pid = a.keyed[static_cast<size_t>(key) * a.capacity + (i - prefix[key])];
        } else {
            pid = a.keyed[static_cast<size_t>(key) * a.capacity + i];
        }
        const float4 o4 = a.o[pid], d4 = a.d[pid], tp4 = a.tp[pid], L4 = a.L[pid];
        const float2 misc = a.misc[pid];
        const f3 ro{o4.x, o4.y, o4.z};
        const f3 rd{d4.x, d4.y, d4.z};
        f3 throughput{tp4.x, tp4.y, tp4.z};
        float eta = tp4.w;
        f3 result{L4.x, L4.y, L4.z};
        const bool have_pdf = misc.y != 0.0f;
        const float sa_pdf = misc.x;
        f3 delta = mk(0.0f);
        if(kAdj) {  // this path's share of dLoss/dimage; the radiance gathered through the previous depth
            const JobRec& job = a.jobs[a.path_job[pid]];
            delta = load3(a.adjoint + job.out_offset + 3ull * a.id[pid].x) / static_cast<float>(job.spp);
            if(depth > 0) a.adj_lsnap[static_cast<size_t>(depth - 1) * a.capacity + pid] = L4;
        }

        if(key == 0) {  // miss: environment + MIS (path_integrator.h:32-45); rec.p of a miss is (0,0,0)
            const f3 Le = eval_environment(s, rd);
            if(!have_pdf) {
                result += throughput * Le;
            } else {
                const float light_pdf = pdf_emitter_direction<kMeshLights>(s, mk(0.0f), rd);
                const float w = power_heuristic(sa_pdf, light_pdf);
                result += throughput * w * Le;
            }
            a.L[pid] = make_float4(result.x, result.y, result.z, 0.0f);
            continue;
        }
        // the hit record of the raw closest hit (hittable_list::hit's record)
        const float4 raw = a.hit_p[pid];
        HitInfo hrec;
        hit_record_of(s, Ray{ro, rd}, __float_as_int(raw.w), raw.x,
                      MeshHit{raw.x, raw.y, raw.z, __float_as_uint(a.hit_n[pid].x)}, hrec);
        const f3 p = hrec.p;
        const f3 normal = hrec.normal;
        const bool front_face = hrec.front_face;
        const ObjRec& obj = s.objects[hrec.object];
        if(obj.emitter >= 0 && front_face) {  // path_integrator.h:47-59
            const f3 outgoing = -normalize(rd);
            const f3 Le = area_emitted(s.emitters[obj.emitter], normal, outgoing);
            if(!is_zero(Le)) {
                if(!have_pdf) {
                    result += throughput * Le;
                } else {
                    const float light_pdf = pdf_emitter_direction<kMeshLights>(s, ro, rd);
                    const float w = power_heuristic(sa_pdf, light_pdf);
                    result += throughput * w * Le;
                }
            }
        }
        if(key == 1) {
            a.L[pid] = make_float4(result.x, result.y, result.z, 0.0f);
            continue;
        }
        ++shading;
        const int32_t mid = effective_material(a, pid, hrec.object);
        const Onb basis = onb_from_normal(normal);
        BRec rec{};
        rec.wi = to_local(basis, -normalize(rd));
        rec.wo = mk(0.0f);
        rec.front_face = front_face;
        rec.eta = 1.0f;
        const uint2 ident = a.id[pid];
        Sampler smp = sampler_start(ident.x, ident.y);
        smp.dimension = 2u + 6u * static_cast<uint32_t>(depth);
        // path_integrator.h:80-83: light (2), lobe (1), bsdf (2), roulette (1)
        const F2 light_uv = sampler_next_2d(sobol_table(s), smp);
        BsdfCtx ctx = ctx_default(LRT_MODE_RADIANCE);
        ctx.lobe_sample = sampler_next_1d(sobol_table(s), smp);
        const F2 bsdf_uv = sampler_next_2d(sobol_table(s), smp);
        const float rr_u = sampler_next_1d(sobol_table(s), smp);

        const MatRec& mat = s.materials[mid];
        if((mat.flags & (kDiffuse | kGlossy)) != 0) {  // NEE (path_integrator.h:86-128)
            DirectSample light{};
            light.distance = kInf;
            if(sample_emitter_direction<kMeshLights, !kDeferSky>(s, p, light_uv.x, light_uv.y, light)) {
                const bool sky = kDeferSky && s.emitters[light.emitter].kind == LRT_EMITTER_ENV;
                const f3 shadow_origin = p + normal * 1e-4f;
                f3 shadow_dir = light.direction;
                float tmax = kInf;
                bool have_target = true;
                if(!isinf(light.distance)) {
                    const f3 to_light = light.point - shadow_origin;
                    const float dist = length(to_light);
                    if(dist < 1e-6f) {
                        have_target = false;
                    } else {
                        shadow_dir = to_light / dist;
                        tmax = dist * (1.0f - 1e-4f);
                    }
                }
                if(have_target) {
                    rec.wo = to_local(basis, shadow_dir);
                    const f3 f_cos = bsdf_eval_t<kType>(s.materials, s.tables, mid, ctx, rec, kSolidAngle);
                    if(!is_zero(f_cos)) {
                        const float bsdf_pdf_v = bsdf_pdf_t<kType>(s.materials, s.tables, mid, ctx, rec, kSolidAngle);
                        const float light_pdf = pdf_emitter_direction<kMeshLights>(s, p, shadow_dir);
                        if(light_pdf > 0.0f) {
                            const float w = power_heuristic(light_pdf, bsdf_pdf_v);
                            // a sky sample leaves radiance and w / light_pdf to k_shadow_sky
                            const f3 contrib = sky ? throughput * f_cos
                                                   : throughput * f_cos * light.radiance * (w / light_pdf);
                            const int seg = heavy_key(s, Ray{shadow_origin, shadow_dir}, 0.001f, tmax);
                            const size_t si = static_cast<size_t>(seg) * a.capacity + warp_append_keyed(bc.shadow, seg);
                            a.sh_o[si] = make_float4(shadow_origin.x, shadow_origin.y, shadow_origin.z, tmax);
                            a.sh_d[si] = make_float4(shadow_dir.x, shadow_dir.y, shadow_dir.z,
                                                     __int_as_float(light.emitter | (sky ? kShadowSkyDeferred : 0)));
                            a.sh_c[si] = make_float4(contrib.x, contrib.y, contrib.z, __uint_as_float(pid));
                            if(sky) a.sh_s[si] = w / light_pdf;
                            if(kAdj) {  // delta x dNEE per group, kept until the shadow ray's visibility is known
                                int32_t smid = -1;
                                if(!is_zero(delta)) {
                                    const f3 scale = delta * (throughput * light.radiance * (w / light_pdf));
                                    const int32_t ab = a.diff.aff_begin[mid];
                                    const int32_t an = a.diff.aff_begin[mid + 1] - ab;
                                    for(int32_t k = 0; k < an; ++k) {
                                        const f3 v = scale * group_d_eval(a.diff, mid, ctx, rec, a.diff.aff_list[ab + k]);
                                        a.adj_sh_prod[static_cast<size_t>(k) * 2 * a.capacity + si] =
                                            make_float4(v.x, v.y, v.z, 0.0f);
                                    }
                                    if(an > 0) smid = mid;
                                }
                                a.adj_sh_mid[si] = smid;
                            }
                        }
                    }
                }
            }
        }
        if(depth == a.max_depth - 1) {
            a.L[pid] = make_float4(result.x, result.y, result.z, 0.0f);
            continue;
        }
        const f3 weight = bsdf_sample_t<kType>(s.materials, s.tables, mid, ctx, rec, bsdf_uv.x, bsdf_uv.y);
        bool alive = !is_zero(weight);
        f3 new_dir = rd;
        if(alive) {
            new_dir = to_world(basis, rec.wo);
            throughput *= weight;
            eta *= rec.eta;
            if(depth >= a.rr_depth) {
                const float q = smin(max3(throughput) * eta * eta, 0.95f);
                if(rr_u >= q) {
                    alive = false;
                } else {
                    throughput /= q;
                }
            }
        }
        a.L[pid] = make_float4(result.x, result.y, result.z, 0.0f);
        if(alive) {
            const bool have = measure_of(rec.sampled_type) == kSolidAngle && rec.pdf > 0.0f;
            a.o[pid] = make_float4(p.x, p.y, p.z, 0.0f);
            a.d[pid] = make_float4(new_dir.x, new_dir.y, new_dir.z, 0.0f);
            a.tp[pid] = make_float4(throughput.x, throughput.y, throughput.z, eta);
            a.misc[pid] = make_float2(rec.pdf, have ? 1.0f : 0.0f);
            const int seg = heavy_key(s, Ray{p, new_dir}, 0.001f, kInf);
            next[static_cast<size_t>(seg) * a.capacity + warp_append_keyed(nc.active, seg)] = pid;
            if(kAdj && !is_zero(delta)) {
                // dE/E of the sampled direction per group (E in the sampled lobe's measure); its suffix is
                // known at the end of the wave
                const int32_t ab = a.diff.aff_begin[mid];
                const int32_t an = a.diff.aff_begin[mid + 1] - ab;
                if(an > 0) {
                    const int meas = measure_of(rec.sampled_type);
                    const BsdfCtx ectx = sampled_value_ctx(ctx, rec);
                    const f3 e0 = bsdf_eval(s.materials, s.tables, mid, ectx, rec, meas);
                    for(int32_t k = 0; k < an; ++k) {
                        const f3 de = group_d_eval(a.diff, mid, ectx, rec, a.diff.aff_list[ab + k], meas);
                        a.adj_dlog[(static_cast<size_t>(depth) * a.adj_kmax + k) * a.capacity + pid] =
                            make_float4(safe_ratio(de.x, e0.x), safe_ratio(de.y, e0.y), safe_ratio(de.z, e0.z), 0.0f);
                    }
                    a.adj_vmid[static_cast<size_t>(depth) * a.capacity + pid] = mid;
                    a.adj_vmask[pid] |= 1u << depth;
                }
            }
        }
    }
    if(a.work) add_count(&a.work[2], shading);
}

__global__ void __launch_bounds__(kBlock) k_shade(WaveArgs a, int depth) {
    __shared__ uint32_t prefix[kKeys + 1];
    shade_wave<false>(a, depth, prefix);
}

__global__ void __launch_bounds__(kBlock) k_shade_adj(WaveArgs a, int depth) {
    __shared__ uint32_t prefix[kKeys + 1];
    shade_wave<true>(a, depth, prefix);
}

// The forward kernels are held to 80 registers (6 resident blocks per SM): misses, hits without a BSDF,
// the diffuse and the dielectric/plastic materials fit without spills; the rough conductor and the two
// coatings spill a little, and still gain more from the occupancy than they lose (the seven-material
// step's shading 80.4 -> 76.7 ms against 4 blocks per SM for the materials). The adjoint kernels keep
// 4 blocks per SM (128 registers); with no floor they grew to 162-172 registers and slowed by 14%.
template <int kKey, bool kAdj = false>
__global__ void __launch_bounds__(kBlock, kAdj ? 4 : 6) k_shade_key(WaveArgs a, int depth) {
    shade_wave<kAdj, kKey>(a, depth, nullptr);
}

// the shading launches of one bounce: one kernel per key present in the scene, or the all-keys kernel
struct ShadeLaunch {
    uint32_t keys = 0;  // bit k: launch k_shade_key<k>; 0: launch k_shade
    int grid[kKeys + 1] = {};
};

template <bool kAdj>
const void* shade_kernel_of(int key) {
    switch(key) {
    case 0: return reinterpret_cast<const void*>(&k_shade_key<0, kAdj>);
    case 1: return reinterpret_cast<const void*>(&k_shade_key<1, kAdj>);
    case 2: return reinterpret_cast<const void*>(&k_shade_key<2, kAdj>);
    case 3: return reinterpret_cast<const void*>(&k_shade_key<3, kAdj>);
    case 4: return reinterpret_cast<const void*>(&k_shade_key<4, kAdj>);
    case 5: return reinterpret_cast<const void*>(&k_shade_key<5, kAdj>);
    case 6: return reinterpret_cast<const void*>(&k_shade_key<6, kAdj>);
    case 7: return reinterpret_cast<const void*>(&k_shade_key<7, kAdj>);
    case 8: return reinterpret_cast<const void*>(&k_shade_key<8, kAdj>);
    default: return reinterpret_cast<const void*>(&k_shade_key<9, kAdj>);
    }
}
static_assert(kKeys == 10, "one shading kernel per key");

template <bool kAdj = false>
ShadeLaunch shade_launch(lrt_context* ctx) {
    ShadeLaunch l;
    if(!ctx->shade_per_key || ctx->has_mesh_lights) {
        l.grid[kKeys] = grid_for(ctx, kAdj ? (const void*)k_shade_adj : (const void*)k_shade, kBlock);
        return l;
    }
    l.keys = ctx->shade_keys;
    for(int k = 0; k < kKeys; ++k) {
        if(l.keys >> k & 1u) l.grid[k] = grid_for(ctx, shade_kernel_of<kAdj>(k), kBlock);
    }
    return l;
}

template <bool kAdj = false>
void launch_shade(const ShadeLaunch& l, const WaveArgs& a, int depth, cudaStream_t st) {
    if(!l.keys) {
        if(kAdj) {
            k_shade_adj<<<l.grid[kKeys], kBlock, 0, st>>>(a, depth);
        } else {
            k_shade<<<l.grid[kKeys], kBlock, 0, st>>>(a, depth);
        }
        return;
    }
    if(l.keys & (1u << 0)) k_shade_key<0, kAdj><<<l.grid[0], kBlock, 0, st>>>(a, depth);
    if(l.keys & (1u << 1)) k_shade_key<1, kAdj><<<l.grid[1], kBlock, 0, st>>>(a, depth);
    if(l.keys & (1u << 2)) k_shade_key<2, kAdj><<<l.grid[2], kBlock, 0, st>>>(a, depth);
    if(l.keys & (1u << 3)) k_shade_key<3, kAdj><<<l.grid[3], kBlock, 0, st>>>(a, depth);
    if(l.keys & (1u << 4)) k_shade_key<4, kAdj><<<l.grid[4], kBlock, 0, st>>>(a, depth);
    if(l.keys & (1u << 5)) k_shade_key<5, kAdj><<<l.grid[5], kBlock, 0, st>>>(a, depth);
    if(l.keys & (1u << 6)) k_shade_key<6, kAdj><<<l.grid[6], kBlock, 0, st>>>(a, depth);
    if(l.keys & (1u << 7)) k_shade_key<7, kAdj><<<l.grid[7], kBlock, 0, st>>>(a, depth);
    if(l.keys & (1u << 8)) k_shade_key<8, kAdj><<<l.grid[8], kBlock, 0, st>>>(a, depth);
    if(l.keys & (1u << 9)) k_shade_key<9, kAdj><<<l.grid[9], kBlock, 0, st>>>(a, depth);
}

uint32_t shade_launch_count(const ShadeLaunch& l) { return l.keys ? static_cast<uint32_t>(__builtin_popcount(l.keys)) : 1u; }

// adjoint: the NEE derivatives of the shadow rays of one depth that reached their light
__global__ void __launch_bounds__(kBlock) k_adj_nee(WaveArgs a, int depth) {
    __shared__ float acc[LRT_MAX_DIFF_PARAMS];
    for(uint32_t j = threadIdx.x; j < a.diff.n_params; j += blockDim.x) acc[j] = 0.0f;
    __syncthreads();
    const uint32_t n0 = a.counters[depth].shadow[0];
    const uint32_t n = n0 + a.counters[depth].shadow[1];
    for(uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const size_t k = i < n0 ? i : a.capacity + (i - n0);
        const int32_t mid = a.adj_sh_mid[k];
        if(mid < 0 || !a.adj_sh_vis[k]) continue;
        const int32_t ab = a.diff.aff_begin[mid];
        const int32_t an = a.diff.aff_begin[mid + 1] - ab;
        for(int32_t g = 0; g < an; ++g) {
            const float4 v = a.adj_sh_prod[static_cast<size_t>(g) * 2 * a.capacity + k];
            add_group<true>(a.diff, acc, a.diff.aff_list[ab + g], f3{v.x, v.y, v.z});
        }
    }
    __syncthreads();
    for(uint32_t j = threadIdx.x; j < a.diff.n_params; j += blockDim.x) {
        if(acc[j] != 0.0f) atomicAdd(a.adj_grad + j, static_cast<double>(acc[j]));
    }
}

// sum the wave's samples per pixel in sample order; the last wave of a pixel divides by spp
__global__ void __launch_bounds__(kBlock) k_accumulate(WaveArgs a, float* rgb, uint32_t spp, int first_wave,
                                                       int last_wave) {
    for(uint32_t pl = blockIdx.x * blockDim.x + threadIdx.x; pl < a.n_pixels; pl += gridDim.x * blockDim.x) {
        f3 acc = first_wave ? mk(0.0f) : load3(a.sum + 3ull * pl);
        for(uint32_t s = 0; s < a.n_samples; ++s) {
            const float4 L = a.L[static_cast<size_t>(pl) * a.n_samples + s];
            acc += f3{L.x, L.y, L.z};
        }
        if(last_wave) {
            store3(rgb + 3ull * (a.pixel_begin + pl), acc / static_cast<float>(spp));
        } else {
            store3(a.sum + 3ull * pl, acc);
        }
    }
}

// ---- batched jobs ----

__device__ __forceinline__ uint32_t wave_slots(const WaveArgs& a) {
    const unsigned long long base = *a.wave_base;
    if(base >= a.total_paths) return 0u;
    const unsigned long long left = a.total_paths - base;
    return left < a.capacity ? static_cast<uint32_t>(left) : a.capacity;
}

// camera rays of the batch paths [wave_base, wave_base + capacity)
__global__ void __launch_bounds__(kBlock) k_raygen_batch(WaveArgs a) {
    const unsigned long long base = *a.wave_base;
    const uint32_t n = wave_slots(a);
    for(uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x; slot < n; slot += gridDim.x * blockDim.x) {
        const unsigned long long g = base + slot;
        uint32_t lo = 0, hi = a.n_jobs;  // last job with path_begin <= g
        while(hi - lo > 1) {
            const uint32_t mid = (lo + hi) / 2;
            if(a.jobs[mid].path_begin <= g) {
                lo = mid;
            } else {
                hi = mid;
            }
        }
        const JobRec& job = a.jobs[lo];
        const unsigned long long local = g - job.path_begin;
        const uint32_t q = static_cast<uint32_t>(local / job.spp);  // the job's q-th pixel in path order
        uint32_t pix = q;
        if(a.pixel_tile > 1) {  // bands of pixel_tile rows, each band column by column
            const uint32_t band = q / (a.pixel_tile * job.width);
            const uint32_t y0 = band * a.pixel_tile;
            const uint32_t bh = min(a.pixel_tile, job.height - y0);
            const uint32_t r = q - y0 * job.width;
            pix = (y0 + r % bh) * job.width + r / bh;
        }
        const uint32_t sample = job.sample_offset + static_cast<uint32_t>(local % job.spp);
        Sampler smp = sampler_start(pix, sample);
        const F2 off = sampler_next_2d(sobol_table(a.s), smp);
        const float u = (static_cast<float>(pix % job.width) + off.x) / static_cast<float>(job.width - 1);
        const float v = (static_cast<float>(pix / job.width) + off.y) / static_cast<float>(job.height - 1);
        const Ray r = camera_ray(job.cam, u, v);
        a.o[slot] = make_float4(r.o.x, r.o.y, r.o.z, 0.0f);
        a.d[slot] = make_float4(r.d.x, r.d.y, r.d.z, 0.0f);
        a.tp[slot] = make_float4(1.0f, 1.0f, 1.0f, 1.0f);
        a.L[slot] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        a.misc[slot] = make_float2(0.0f, 0.0f);
        a.id[slot] = make_uint2(pix, sample);
        a.path_job[slot] = lo;
        const int seg = heavy_key(a.s, r, 0.001f, kInf);
        a.q0[static_cast<size_t>(seg) * a.capacity + warp_append_keyed(a.counters[0].active, seg)] = slot;
    }
}

// per pixel run of the wave (consecutive slots of one job pixel), in sample order: the run's sum joins
// the pixel's running sum; the run holding the pixel's last sample writes sum / spp
__global__ void __launch_bounds__(kBlock) k_accumulate_batch(WaveArgs a) {
    const uint32_t n = wave_slots(a);
    for(uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x; slot < n; slot += gridDim.x * blockDim.x) {
        const uint32_t job_i = a.path_job[slot];
        const uint2 ident = a.id[slot];
        if(slot > 0 && a.path_job[slot - 1] == job_i && a.id[slot - 1].x == ident.x) continue;
        const JobRec& job = a.jobs[job_i];
        const unsigned long long px = job.out_offset + 3ull * ident.x;
        f3 acc = ident.y == job.sample_offset ? mk(0.0f) : load3(a.batch_sums + px);
        uint32_t k = slot;
        uint32_t last_sample = ident.y;
        while(k < n && a.path_job[k] == job_i && a.id[k].x == ident.x) {
            const float4 L = a.L[k];
            acc += f3{L.x, L.y, L.z};
            last_sample = a.id[k].y;
            ++k;
        }
        if(last_sample == job.sample_offset + job.spp - 1) {
            store3(a.batch_out + px, acc / static_cast<float>(job.spp));
        } else {
            store3(a.batch_sums + px, acc);
        }
    }
}

__global__ void k_wave_advance(WaveArgs a) {
    if(blockIdx.x == 0 && threadIdx.x == 0) *a.wave_base += a.capacity;
}

// adjoint, once per wave after its last depth: every derivative record of a sampled direction times
// what the path gathered after that depth (its final radiance minus the radiance through the depth)
__global__ void __launch_bounds__(kBlock) k_adj_suffix(WaveArgs a) {
    __shared__ float acc[LRT_MAX_DIFF_PARAMS];
    for(uint32_t j = threadIdx.x; j < a.diff.n_params; j += blockDim.x) acc[j] = 0.0f;
    __syncthreads();
    const uint32_t n = wave_slots(a);
    for(uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x; slot < n; slot += gridDim.x * blockDim.x) {
        uint32_t mask = a.adj_vmask[slot];
        if(mask == 0) continue;
        const JobRec& job = a.jobs[a.path_job[slot]];
        const f3 delta = load3(a.adjoint + job.out_offset + 3ull * a.id[slot].x) / static_cast<float>(job.spp);
        const float4 L = a.L[slot];
        while(mask != 0) {
            const int d = __ffs(mask) - 1;
            mask &= mask - 1;
            const float4 before = a.adj_lsnap[static_cast<size_t>(d) * a.capacity + slot];
            const f3 w = delta * f3{L.x - before.x, L.y - before.y, L.z - before.z};
            const int32_t mid = a.adj_vmid[static_cast<size_t>(d) * a.capacity + slot];
            const int32_t ab = a.diff.aff_begin[mid];
            const int32_t an = a.diff.aff_begin[mid + 1] - ab;
            for(int32_t g = 0; g < an; ++g) {
                const float4 v = a.adj_dlog[(static_cast<size_t>(d) * a.adj_kmax + g) * a.capacity + slot];
                add_group<true>(a.diff, acc, a.diff.aff_list[ab + g], w * f3{v.x, v.y, v.z});
            }
        }
    }
    __syncthreads();
    for(uint32_t j = threadIdx.x; j < a.diff.n_params; j += blockDim.x) {
        if(acc[j] != 0.0f) atomicAdd(a.adj_grad + j, static_cast<double>(acc[j]));
    }
}

// Default paths per wave. A forward wave holds about 250 bytes of state per path, so 2^24 paths (one
// 512x512 frame at 64 spp) take 4 GB; fewer, larger waves leave less of each bounce to the tail of its
// persistent kernel. An adjoint path also keeps records for every bounce and material group, so its
// waves stay at 2^21 paths.
constexpr uint32_t kForwardWaveCapacity = 1u << 24;
constexpr uint32_t kAdjointWaveCapacity = 1u << 21;

// slots of the wave that renders `paths` paths: the configured capacity, never more than the call needs
uint32_t wave_slots(const lrt_context* ctx, unsigned long long paths, bool adjoint) {
    const uint32_t cap = ctx->wave_capacity ? ctx->wave_capacity : adjoint ? kAdjointWaveCapacity : kForwardWaveCapacity;
    return static_cast<uint32_t>(std::max<unsigned long long>(1, std::min<unsigned long long>(cap, paths)));
}

int ensure_wave(lrt_context* ctx, uint32_t cap) {
    WaveState& w = ctx->wave;
    if(w.capacity >= cap) return LRT_OK;
    const size_t c = cap;
    LRT_CUDA(ctx, w.o.ensure(c * 16));
    LRT_CUDA(ctx, w.d.ensure(c * 16));
    LRT_CUDA(ctx, w.tp.ensure(c * 16));
    LRT_CUDA(ctx, w.L.ensure(c * 16));
    LRT_CUDA(ctx, w.misc.ensure(c * 8));
    LRT_CUDA(ctx, w.id.ensure(c * 8));
    LRT_CUDA(ctx, w.hit_p.ensure(c * 16));
    LRT_CUDA(ctx, w.hit_n.ensure(c * 16));
    LRT_CUDA(ctx, w.q0.ensure(c * 8));
    LRT_CUDA(ctx, w.q1.ensure(c * 8));
    LRT_CUDA(ctx, w.keyed.ensure(c * 4 * kKeys));
    LRT_CUDA(ctx, w.sh_o.ensure(c * 32));
    LRT_CUDA(ctx, w.sh_d.ensure(c * 32));
    LRT_CUDA(ctx, w.sh_c.ensure(c * 32));
    LRT_CUDA(ctx, w.sh_s.ensure(c * 8));
    LRT_CUDA(ctx, w.sum.ensure(c * 12));
    w.capacity = cap;
    return LRT_OK;
}

void record_stage(lrt_context* ctx, int stage, bool begin) {
    if(!ctx->stage_timing) return;
    cudaEvent_t ev;
    if(cudaEventCreate(&ev) != cudaSuccess) return;
    cudaEventRecord(ev, ctx->stream);
    ctx->events.push_back(ev);
    ctx->event_stage.push_back(begin ? stage : -1 - stage);
}

void collect_stage_times(lrt_context* ctx) {
    for(size_t i = 0; i + 1 < ctx->events.size(); i += 2) {
        float ms = 0.0f;
        if(cudaEventElapsedTime(&ms, ctx->events[i], ctx->events[i + 1]) == cudaSuccess) {
            const int stage = ctx->event_stage[i];
            if(stage >= 0 && stage < LRT_STAGE_COUNT) {
                ctx->stats.stage_ms[stage] += ms;
                ctx->stats.stage_launches[stage] += 1;
            }
        }
    }
    for(cudaEvent_t e : ctx->events) cudaEventDestroy(e);
    ctx->events.clear();
    ctx->event_stage.clear();
}

// The wave plan of one render -- the pixel range [pix0, pix1) x the sample range, at most `cap` slots
// per wave -- and its launches: ray generation, per bounce extend, hit records, shading and shadow rays,
// then the accumulation. Shared by lrt_render(_dev) and the allocation-free entry point, which differ
// only in where the wave's arrays live; `stages` records the stage events of the option stage_timing.
int run_render_waves(lrt_context* ctx, WaveArgs& a, const lrt_render_params* p, uint32_t pix0, uint32_t pix1,
                     uint32_t cap, size_t counters_bytes, bool cnt, bool stages, float* rgb_dev, uint64_t& launches) {
    const int g_raygen = grid_for(ctx, (const void*)k_raygen, kBlock);
    const int g_extend =
        grid_for(ctx, cnt ? (const void*)k_extend_persistent<true> : (const void*)k_extend_persistent<false>, kBlock);
    const int g_hitrec = grid_for(ctx, (const void*)k_hitrec, kBlock);
    const ShadeLaunch shade = shade_launch(ctx);
    const int g_shadow =
        grid_for(ctx, cnt ? (const void*)k_shadow_persistent<true> : (const void*)k_shadow_persistent<false>, kBlock);
    const int g_accum = grid_for(ctx, (const void*)k_accumulate, kBlock);
    const int g_sky = grid_for(ctx, (const void*)k_shadow_sky, kBlock);
    auto stage = [&](int which, bool begin) {
        if(stages) record_stage(ctx, which, begin);
    };
    const uint32_t spp = p->spp;
    const uint32_t samples_per_wave = std::min(spp, cap);
    const uint32_t pixels_per_wave = std::max(1u, cap / samples_per_wave);
    for(uint32_t pb = pix0; pb < pix1; pb += pixels_per_wave) {
        const uint32_t np = std::min(pixels_per_wave, pix1 - pb);
        for(uint32_t sb = 0; sb < spp; sb += samples_per_wave) {
            const uint32_t ns = std::min(samples_per_wave, spp - sb);
            a.pixel_begin = pb;
            a.n_pixels = np;
            a.sample_begin = p->sample_offset + sb;
            a.n_samples = ns;
            LRT_CUDA(ctx, cudaMemsetAsync(a.counters, 0, counters_bytes, ctx->stream));
            stage(LRT_STAGE_RAYGEN, true);
            k_raygen<<<g_raygen, kBlock, 0, ctx->stream>>>(a);
            stage(LRT_STAGE_RAYGEN, false);
            launches += 1;
            for(int depth = 0; depth < p->max_depth; ++depth) {
                stage(LRT_STAGE_EXTEND, true);
                if(cnt) {
                    k_extend_persistent<true><<<g_extend, kBlock, 0, ctx->stream>>>(a, depth);
                } else {
                    k_extend_persistent<false><<<g_extend, kBlock, 0, ctx->stream>>>(a, depth);
                }
                stage(LRT_STAGE_EXTEND, false);
                stage(LRT_STAGE_SORT, true);
                k_hitrec<<<g_hitrec, kBlock, 0, ctx->stream>>>(a, depth);
                stage(LRT_STAGE_SORT, false);
                stage(LRT_STAGE_SHADE, true);
                launch_shade(shade, a, depth, ctx->stream);
                stage(LRT_STAGE_SHADE, false);
                stage(LRT_STAGE_SHADOW, true);
                if(cnt) {
                    k_shadow_persistent<true><<<g_shadow, kBlock, 0, ctx->stream>>>(a, depth);
                } else {
                    k_shadow_persistent<false><<<g_shadow, kBlock, 0, ctx->stream>>>(a, depth);
                }
                if(ctx->has_sky) k_shadow_sky<<<g_sky, kBlock, 0, ctx->stream>>>(a, depth);
                stage(LRT_STAGE_SHADOW, false);
                launches += 3 + shade_launch_count(shade) + (ctx->has_sky ? 1 : 0);
            }
            stage(LRT_STAGE_ACCUM, true);
            k_accumulate<<<g_accum, kBlock, 0, ctx->stream>>>(a, rgb_dev, spp, sb == 0 ? 1 : 0, sb + ns >= spp ? 1 : 0);
            stage(LRT_STAGE_ACCUM, false);
            launches += 1;
            LRT_CUDA(ctx, cudaGetLastError());
        }
    }
    return LRT_OK;
}

int render_impl(lrt_context* ctx, const lrt_render_params* p, float* rgb_dev) {
    if(!ctx->has_scene) return fail(ctx, LRT_ERR_NO_SCENE, "no scene uploaded");
    if(!p || p->width < 2 || p->height < 2 || p->spp == 0 || p->max_depth < 1 || p->max_depth > 1024) {
        return fail(ctx, LRT_ERR_INVALID_ARGUMENT,
                    "render parameters out of range (width, height >= 2; spp >= 1; 1 <= max_depth <= 1024)");
    }
    const uint32_t row_begin = p->row_end > p->row_begin ? p->row_begin : 0u;
    const uint32_t row_end = p->row_end > p->row_begin ? std::min(p->row_end, p->height) : p->height;
    if(row_begin >= row_end) return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "empty row range");
    if(static_cast<uint64_t>(p->width) * p->height > 0x3fffffffull) return fail(ctx, LRT_ERR_RANGE, "image too large");
    const uint32_t cap = wave_slots(ctx, static_cast<unsigned long long>(row_end - row_begin) * p->width * p->spp, false);
    int st = ensure_wave(ctx, cap);
    if(st != LRT_OK) return st;
    const size_t counters_bytes = sizeof(BounceCounters) * (p->max_depth + 1);
    LRT_CUDA(ctx, ctx->counters.ensure(counters_bytes));
    WaveState& w = ctx->wave;
    WaveArgs a{};
    a.s = ctx->ds;
    a.o = w.o.as<float4>();
    a.d = w.d.as<float4>();
    a.tp = w.tp.as<float4>();
    a.L = w.L.as<float4>();
    a.misc = w.misc.as<float2>();
    a.id = w.id.as<uint2>();
    a.hit_p = w.hit_p.as<float4>();
    a.hit_n = w.hit_n.as<float4>();
    a.q0 = w.q0.as<uint32_t>();
    a.q1 = w.q1.as<uint32_t>();
    a.keyed = w.keyed.as<uint32_t>();
    a.sh_o = w.sh_o.as<float4>();
    a.sh_d = w.sh_d.as<float4>();
    a.sh_c = w.sh_c.as<float4>();
    a.sh_s = w.sh_s.as<float>();
    a.counters = ctx->counters.as<BounceCounters>();
    a.sum = w.sum.as<float>();
    a.capacity = cap;
    a.width = p->width;
    a.height = p->height;
    a.max_depth = p->max_depth;
    a.rr_depth = p->rr_depth;
    unsigned long long* work = nullptr;
    constexpr size_t kWorkBytes = 8 * (8 + LRT_MAX_STAT_DEPTH);
    if(ctx->count_work) {
        LRT_CUDA(ctx, ctx->scratch_b.ensure(kWorkBytes));
        work = ctx->scratch_b.as<unsigned long long>();
        LRT_CUDA(ctx, cudaMemsetAsync(work, 0, kWorkBytes, ctx->stream));
    }
    a.work = work;

    const bool cnt = ctx->count_work;
    const uint32_t pix0 = row_begin * p->width;
    const uint32_t pix1 = row_end * p->width;
    const uint32_t spp = p->spp;
    uint64_t launches = 0;
    st = run_render_waves(ctx, a, p, pix0, pix1, cap, counters_bytes, cnt, true, rgb_dev, launches);
    if(st != LRT_OK) return st;
    ctx->stats.paths += static_cast<uint64_t>(pix1 - pix0) * spp;
    ctx->stats.kernel_launches += launches;
    if(ctx->stage_timing || cnt) {
        LRT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        collect_stage_times(ctx);
        if(cnt) {
            unsigned long long h[8 + LRT_MAX_STAT_DEPTH];
            LRT_CUDA(ctx, cudaMemcpy(h, work, sizeof(h), cudaMemcpyDeviceToHost));
            for(int d = 0; d < LRT_MAX_STAT_DEPTH; ++d) ctx->stats.rays_at_depth[d] += h[8 + d];
            ctx->stats.nodes_visited += h[0];
            ctx->stats.triangles_tested += h[1];
            ctx->stats.shading_events += h[2];
            ctx->stats.extension_rays += h[3];
            ctx->stats.shadow_rays += h[4];
            ctx->stats.shadow_nodes_visited += h[5];
            ctx->stats.shadow_triangles_tested += h[6];
        }
    }
    return LRT_OK;
}


// The launch sequence of one wave of a batch (also what the CUDA graph holds).
void launch_batch_wave(lrt_context* ctx, const WaveArgs& a, size_t counters_bytes, int g_raygen, int g_extend,
                       int g_hitrec, const ShadeLaunch& shade, int g_shadow, int g_accum) {
    cudaMemsetAsync(a.counters, 0, counters_bytes, ctx->stream);
    k_raygen_batch<<<g_raygen, kBlock, 0, ctx->stream>>>(a);
    for(int depth = 0; depth < a.max_depth; ++depth) {
        k_extend_persistent<false><<<g_extend, kBlock, 0, ctx->stream>>>(a, depth);
        k_hitrec<<<g_hitrec, kBlock, 0, ctx->stream>>>(a, depth);
        launch_shade(shade, a, depth, ctx->stream);
        k_shadow_persistent<false><<<g_shadow, kBlock, 0, ctx->stream>>>(a, depth);
        if(ctx->has_sky) k_shadow_sky<<<g_shadow, kBlock, 0, ctx->stream>>>(a, depth);
    }
    k_accumulate_batch<<<g_accum, kBlock, 0, ctx->stream>>>(a);
    k_wave_advance<<<1, 32, 0, ctx->stream>>>(a);
}

// the wave state, counters and job table of a batch of paths (jobs already validated)
int batch_wave_args(lrt_context* ctx, const std::vector<JobRec>& recs, unsigned long long total, int32_t max_depth,
                    int32_t rr_depth, bool adjoint, WaveArgs& a) {
    const uint32_t cap = wave_slots(ctx, total, adjoint);
    const uint32_t n_jobs = static_cast<uint32_t>(recs.size());
    int st = ensure_wave(ctx, cap);
    if(st != LRT_OK) return st;
    const size_t counters_bytes = sizeof(BounceCounters) * (max_depth + 1);
    LRT_CUDA(ctx, ctx->counters.ensure(counters_bytes));
    LRT_CUDA(ctx, ctx->batch_jobs.ensure(sizeof(JobRec) * n_jobs));
    LRT_CUDA(ctx, ctx->batch_path_job.ensure(4ull * cap));
    LRT_CUDA(ctx, ctx->batch_cursor.ensure(8));
    LRT_CUDA(ctx, cudaMemcpyAsync(ctx->batch_jobs.ptr, recs.data(), sizeof(JobRec) * n_jobs, cudaMemcpyHostToDevice,
                                  ctx->stream));
    LRT_CUDA(ctx, cudaMemsetAsync(ctx->batch_cursor.ptr, 0, 8, ctx->stream));
    WaveState& w = ctx->wave;
    a = WaveArgs{};
    a.s = ctx->ds;
    a.o = w.o.as<float4>();
    a.d = w.d.as<float4>();
    a.tp = w.tp.as<float4>();
    a.L = w.L.as<float4>();
    a.misc = w.misc.as<float2>();
    a.id = w.id.as<uint2>();
    a.hit_p = w.hit_p.as<float4>();
    a.hit_n = w.hit_n.as<float4>();
    a.q0 = w.q0.as<uint32_t>();
    a.q1 = w.q1.as<uint32_t>();
    a.keyed = w.keyed.as<uint32_t>();
    a.sh_o = w.sh_o.as<float4>();
    a.sh_d = w.sh_d.as<float4>();
    a.sh_c = w.sh_c.as<float4>();
    a.sh_s = w.sh_s.as<float>();
    a.counters = ctx->counters.as<BounceCounters>();
    a.sum = w.sum.as<float>();
    a.capacity = cap;
    a.max_depth = max_depth;
    a.rr_depth = rr_depth;
    a.work = nullptr;
    a.jobs = ctx->batch_jobs.as<JobRec>();
    a.n_jobs = n_jobs;
    a.path_job = ctx->batch_path_job.as<uint32_t>();
    a.wave_base = ctx->batch_cursor.as<unsigned long long>();
    a.total_paths = total;
    a.pixel_tile = ctx->pixel_tile;
    return LRT_OK;
}

// replays `launch_one` (the launch sequence of one wave, which advances the device cursor) `waves`
// times: captured once into a CUDA graph, or launched directly when the batch_graph option is off
template <typename F>
int run_waves(lrt_context* ctx, unsigned long long waves, F launch_one) {
    if(ctx->batch_graph) {
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        LRT_CUDA(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
        launch_one();
        const cudaError_t ce = cudaStreamEndCapture(ctx->stream, &graph);
        if(ce != cudaSuccess) return fail(ctx, LRT_ERR_CUDA, "graph capture: %s", cudaGetErrorString(ce));
        const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
        if(ie != cudaSuccess) {
            cudaGraphDestroy(graph);
            return fail(ctx, LRT_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(ie));
        }
        cudaError_t le = cudaSuccess;
        for(unsigned long long i = 0; i < waves && le == cudaSuccess; ++i) le = cudaGraphLaunch(exec, ctx->stream);
        cudaGraphExecDestroy(exec);
        cudaGraphDestroy(graph);
        if(le != cudaSuccess) return fail(ctx, LRT_ERR_CUDA, "graph launch: %s", cudaGetErrorString(le));
    } else {
        for(unsigned long long i = 0; i < waves; ++i) launch_one();
        LRT_CUDA(ctx, cudaGetLastError());
    }
    return LRT_OK;
}

int render_batch_impl(lrt_context* ctx, const lrt_job_desc* jobs, uint32_t n_jobs, int32_t max_depth, int32_t rr_depth,
                      float* rgb_dev) {
    if(!ctx->has_scene) return fail(ctx, LRT_ERR_NO_SCENE, "no scene uploaded");
    if(n_jobs == 0) return LRT_OK;
    if(!jobs || !rgb_dev) return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "null argument");
    if(max_depth < 1 || max_depth > 1024) return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "max_depth out of range");
    std::vector<JobRec> recs;
    unsigned long long total = 0, out_floats = 0;
    const int jst = job_records(ctx, jobs, n_jobs, recs, total, out_floats);
    if(jst != LRT_OK) return jst;
    if(ctx->batch_queue) return render_batch_queue(ctx, recs, total, max_depth, rr_depth, rgb_dev);
    WaveArgs a;
    const int st = batch_wave_args(ctx, recs, total, max_depth, rr_depth, false, a);
    if(st != LRT_OK) return st;
    LRT_CUDA(ctx, ctx->batch_sums.ensure(4ull * out_floats));
    a.batch_out = rgb_dev;
    a.batch_sums = ctx->batch_sums.as<float>();
    const size_t counters_bytes = sizeof(BounceCounters) * (max_depth + 1);
    const int g_raygen = grid_for(ctx, (const void*)k_raygen_batch, kBlock);
    const int g_extend = grid_for(ctx, (const void*)k_extend_persistent<false>, kBlock);
    const int g_hitrec = grid_for(ctx, (const void*)k_hitrec, kBlock);
    const ShadeLaunch shade = shade_launch(ctx);
    const int g_shadow = grid_for(ctx, (const void*)k_shadow_persistent<false>, kBlock);
    const int g_accum = grid_for(ctx, (const void*)k_accumulate_batch, kBlock);
    const unsigned long long waves = (total + a.capacity - 1) / a.capacity;
    const uint64_t per_wave = 3 + (3ull + shade_launch_count(shade) + (ctx->has_sky ? 1 : 0)) * max_depth;
    const int rst = run_waves(ctx, waves, [&]() {
        launch_batch_wave(ctx, a, counters_bytes, g_raygen, g_extend, g_hitrec, shade, g_shadow, g_accum);
    });
    if(rst != LRT_OK) return rst;
    ctx->stats.paths += total;
    ctx->stats.kernel_launches += waves * per_wave;
    return LRT_OK;
}

}  // namespace


namespace lrt {

int adjoint_wavefront(lrt_context* ctx, const std::vector<JobRec>& recs, unsigned long long total, int32_t max_depth,
                      int32_t rr_depth, const float* adjoint_dev, double* grad_dev) {
    WaveArgs a;
    const int st = batch_wave_args(ctx, recs, total, max_depth, rr_depth, true, a);
    if(st != LRT_OK) return st;
    const size_t cap = a.capacity;
    const uint32_t kmax = std::max<uint32_t>(1, ctx->diff_kmax);
    LRT_CUDA(ctx, ctx->adj_vmask.ensure(4 * cap));
    LRT_CUDA(ctx, ctx->adj_vmid.ensure(4 * cap * max_depth));
    LRT_CUDA(ctx, ctx->adj_lsnap.ensure(16 * cap * max_depth));
    LRT_CUDA(ctx, ctx->adj_dlog.ensure(16 * cap * max_depth * kmax));
    LRT_CUDA(ctx, ctx->adj_sh_mid.ensure(4 * 2 * cap));
    LRT_CUDA(ctx, ctx->adj_sh_vis.ensure(2 * cap));
    LRT_CUDA(ctx, ctx->adj_sh_prod.ensure(16 * 2 * cap * kmax));
    a.adjoint = adjoint_dev;
    a.diff = diff_dev(ctx);
    a.adj_kmax = kmax;
    a.adj_vmask = ctx->adj_vmask.as<uint32_t>();
    a.adj_vmid = ctx->adj_vmid.as<int32_t>();
    a.adj_lsnap = ctx->adj_lsnap.as<float4>();
    a.adj_dlog = ctx->adj_dlog.as<float4>();
    a.adj_sh_mid = ctx->adj_sh_mid.as<int32_t>();
    a.adj_sh_vis = ctx->adj_sh_vis.as<uint8_t>();
    a.adj_sh_prod = ctx->adj_sh_prod.as<float4>();
    a.adj_grad = grad_dev;
    const size_t counters_bytes = sizeof(BounceCounters) * (max_depth + 1);
    const int g_raygen = grid_for(ctx, (const void*)k_raygen_batch, kBlock);
    const int g_extend = grid_for(ctx, (const void*)k_extend_persistent<false>, kBlock);
    const int g_hitrec = grid_for(ctx, (const void*)k_hitrec, kBlock);
    const ShadeLaunch shade = shade_launch<true>(ctx);
    const int g_shadow = grid_for(ctx, (const void*)k_shadow_persistent<false, true>, kBlock);
    const int g_nee = grid_for(ctx, (const void*)k_adj_nee, kBlock);
    const int g_suffix = grid_for(ctx, (const void*)k_adj_suffix, kBlock);
    cudaStream_t sm = ctx->stream;
    const unsigned long long waves = (total + cap - 1) / cap;
    const int rst = run_waves(ctx, waves, [&]() {
        cudaMemsetAsync(a.counters, 0, counters_bytes, sm);
        cudaMemsetAsync(a.adj_vmask, 0, 4 * cap, sm);
        k_raygen_batch<<<g_raygen, kBlock, 0, sm>>>(a);
        for(int depth = 0; depth < max_depth; ++depth) {
            k_extend_persistent<false><<<g_extend, kBlock, 0, sm>>>(a, depth);
            k_hitrec<<<g_hitrec, kBlock, 0, sm>>>(a, depth);
            launch_shade<true>(shade, a, depth, sm);
            k_shadow_persistent<false, true><<<g_shadow, kBlock, 0, sm>>>(a, depth);
            k_adj_nee<<<g_nee, kBlock, 0, sm>>>(a, depth);
        }
        k_adj_suffix<<<g_suffix, kBlock, 0, sm>>>(a);
        k_wave_advance<<<1, 32, 0, sm>>>(a);
    });
    if(rst != LRT_OK) return rst;
    ctx->stats.paths += total;
    ctx->stats.kernel_launches += waves * (3 + (4ull + shade_launch_count(shade)) * max_depth);
    return LRT_OK;
}

}  // namespace lrt
// ======================================= C ABI =======================================

extern "C" {

const char* lrt_status_string(int status) {
    switch(status) {
    case LRT_OK: return "LRT_OK";
    case LRT_ERR_INVALID_ARGUMENT: return "LRT_ERR_INVALID_ARGUMENT";
    case LRT_ERR_CUDA: return "LRT_ERR_CUDA";
    case LRT_ERR_OUT_OF_MEMORY: return "LRT_ERR_OUT_OF_MEMORY";
    case LRT_ERR_IO: return "LRT_ERR_IO";
    case LRT_ERR_RANGE: return "LRT_ERR_RANGE";
    case LRT_ERR_NO_SCENE: return "LRT_ERR_NO_SCENE";
    case LRT_ERR_NO_DEVICE: return "LRT_ERR_NO_DEVICE";
    default: return "LRT_ERR_UNKNOWN";
    }
}

int lrt_create(int device, void* cuda_stream, lrt_context** out) {
    if(!out) return LRT_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    int count = 0;
    if(cudaGetDeviceCount(&count) != cudaSuccess || count <= 0) {
        cudaGetLastError();
        return LRT_ERR_NO_DEVICE;
    }
    if(device < 0 || device >= count) return LRT_ERR_INVALID_ARGUMENT;
    auto ctx = std::make_unique<lrt_context>();
    ctx->device = device;
    if(cudaSetDevice(device) != cudaSuccess) return LRT_ERR_CUDA;
    cudaDeviceProp prop;
    if(cudaGetDeviceProperties(&prop, device) != cudaSuccess) return LRT_ERR_CUDA;
    if(prop.major < 10) return LRT_ERR_NO_DEVICE;  // built for sm_100a only
    ctx->sm_count = prop.multiProcessorCount;
    if(cuda_stream) {
        ctx->stream = static_cast<cudaStream_t>(cuda_stream);
    } else {
        if(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) return LRT_ERR_CUDA;
        ctx->own_stream = true;
    }
    uint32_t table[kSobolDims][32];
    sobol_direction_table(table);
    if(ctx->sobol.ensure(sizeof(table)) != cudaSuccess) return LRT_ERR_OUT_OF_MEMORY;
    if(cudaMemcpy(ctx->sobol.ptr, table, sizeof(table), cudaMemcpyHostToDevice) != cudaSuccess) return LRT_ERR_CUDA;
    *out = ctx.release();
    return LRT_OK;
}

int lrt_destroy(lrt_context* ctx) {
    if(!ctx) return LRT_OK;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    for(cudaEvent_t e : ctx->events) cudaEventDestroy(e);
    if(ctx->own_stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return LRT_OK;
}

const char* lrt_last_error(const lrt_context* ctx) { return ctx ? ctx->error.c_str() : "null context"; }

int lrt_rough_transmittance_slice(const char* ggx_path, float eta, float alpha, float* table_out, float* diffuse_out) {
    if(!ggx_path || !table_out || !diffuse_out) return LRT_ERR_INVALID_ARGUMENT;
    std::string err;
    return rough_transmittance_slice(ggx_path, eta, alpha, table_out, diffuse_out, err);
}

float lrt_fresnel_diffuse_reflectance(float eta) { return fresnel_diffuse_reflectance(eta); }

int lrt_hosek_state(const float* sun_direction, float turbidity, float albedo, double* config, double* radiance) {
    if(!sun_direction || !config || !radiance) return LRT_ERR_INVALID_ARGUMENT;
    std::string err;
    double cfg[3][9], rad[3];
    const int st = hosek_state(sun_direction, turbidity, albedo, cfg, rad, err);
    if(st != LRT_OK) return st;
    for(int c = 0; c < 3; ++c) {
        for(int k = 0; k < 9; ++k) config[9 * c + k] = cfg[c][k];
        radiance[c] = rad[c];
    }
    return LRT_OK;
}

int lrt_load_obj(const char* path, uint32_t* n_vertices, uint32_t* n_indices, float* positions,
                 uint32_t vertex_capacity, uint32_t* indices, float* corner_normals, uint32_t index_capacity) {
    if(!path || !n_vertices || !n_indices) return LRT_ERR_INVALID_ARGUMENT;
    std::vector<float> pos, nrm;
    std::vector<uint32_t> idx;
    std::string err;
    const int st = load_obj(path, pos, idx, nrm, err);
    if(st != LRT_OK) return st;
    if(pos.size() / 3 > 0xffffffffull || idx.size() > 0xffffffffull) return LRT_ERR_RANGE;
    *n_vertices = static_cast<uint32_t>(pos.size() / 3);
    *n_indices = static_cast<uint32_t>(idx.size());
    if(!positions && !indices && !corner_normals) return LRT_OK;
    if(!positions || !indices || !corner_normals) return LRT_ERR_INVALID_ARGUMENT;
    if(vertex_capacity < *n_vertices || index_capacity < *n_indices) return LRT_ERR_RANGE;
    memcpy(positions, pos.data(), pos.size() * sizeof(float));
    memcpy(indices, idx.data(), idx.size() * sizeof(uint32_t));
    memcpy(corner_normals, nrm.data(), nrm.size() * sizeof(float));
    return LRT_OK;
}

int lrt_rough_transmittance_eta_slice(const char* ggx_path, float eta, float* sliced_table, float* sliced_diffuse,
                                      uint32_t capacity, uint32_t* n_alpha_out, float* alpha_range_out) {
    if(!ggx_path || !n_alpha_out || !alpha_range_out) return LRT_ERR_INVALID_ARGUMENT;
    std::string err;
    std::vector<float> t, d;
    float lo = 0.0f, hi = 0.0f;
    const int st = rough_transmittance_eta(ggx_path, eta, t, d, lo, hi, err);
    if(st != LRT_OK) return st;
    *n_alpha_out = static_cast<uint32_t>(d.size());
    alpha_range_out[0] = lo;
    alpha_range_out[1] = hi;
    if(d.size() > capacity) return LRT_ERR_RANGE;
    if(!sliced_table || !sliced_diffuse) return LRT_ERR_INVALID_ARGUMENT;
    memcpy(sliced_table, t.data(), t.size() * sizeof(float));
    memcpy(sliced_diffuse, d.data(), d.size() * sizeof(float));
    return LRT_OK;
}

int lrt_rough_transmittance_at_alpha(const float* sliced_table, const float* sliced_diffuse, uint32_t n_alpha,
                                     const float* alpha_range, float alpha, float* table_out, float* diffuse_out) {
    if(!sliced_table || !sliced_diffuse || !alpha_range || !table_out || !diffuse_out) return LRT_ERR_INVALID_ARGUMENT;
    std::string err;
    return rough_transmittance_alpha(sliced_table, sliced_diffuse, n_alpha, alpha_range[0], alpha_range[1], alpha,
                                     table_out, diffuse_out, err);
}

int lrt_kdtree_build(const float* bmin, const float* bmax, uint32_t n, uint32_t* nodes_out, uint32_t max_nodes,
                     uint32_t* refs_out, uint32_t max_refs, uint32_t* n_nodes, uint32_t* n_refs, uint32_t* depth) {
    if((n && (!bmin || !bmax)) || !n_nodes || !n_refs) return LRT_ERR_INVALID_ARGUMENT;
    PackedTree t;
    build_kdtree(bmin, bmax, n, t);
    *n_nodes = static_cast<uint32_t>(t.nodes.size());
    *n_refs = static_cast<uint32_t>(t.refs.size());
    if(depth) *depth = t.depth;
    if(t.nodes.size() > max_nodes || t.refs.size() > max_refs || !nodes_out || (!refs_out && !t.refs.empty())) {
        return LRT_ERR_RANGE;
    }
    for(size_t i = 0; i < t.nodes.size(); ++i) {
        nodes_out[2 * i] = t.nodes[i].x;
        nodes_out[2 * i + 1] = t.nodes[i].y;
    }
    std::copy(t.refs.begin(), t.refs.end(), refs_out);
    return LRT_OK;
}

int lrt_kdtree_build_device(lrt_context* ctx, uint32_t n_meshes, const uint32_t* counts, const float* bmin,
                            const float* bmax, uint32_t* nodes_out, uint64_t max_nodes, uint32_t* refs_out,
                            uint64_t max_refs, uint32_t* node_counts, uint32_t* ref_counts, uint32_t* depths,
                            uint64_t* total_nodes, uint64_t* total_refs) {
    if(!ctx) return LRT_ERR_INVALID_ARGUMENT;
    if((n_meshes && !counts) || !total_nodes || !total_refs) return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "null argument");
    if(n_meshes == 0) {  // nothing to build, nothing written
        *total_nodes = 0;
        *total_refs = 0;
        return LRT_OK;
    }
    LRT_CUDA(ctx, cudaSetDevice(ctx->device));
    uint64_t n = 0;
    for(uint32_t m = 0; m < n_meshes; ++m) {
        if(counts[m] == 0) return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "mesh %u has no primitives", m);
        n += counts[m];
    }
    if(n && (!bmin || !bmax)) return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "null boxes");
    std::vector<uint32_t> cv(counts, counts + n_meshes);
    BigVec<float> lo(bmin, bmin + 3 * n), hi(bmax, bmax + 3 * n);
    std::vector<PackedTree> trees;
    std::string err;
    const int st = build_kdtrees_device(ctx, cv, lo, hi, trees, err);
    if(st != LRT_OK) return err.empty() ? st : fail(ctx, st, "%s", err.c_str());
    uint64_t tn = 0, tr = 0;
    for(const PackedTree& t : trees) {
        tn += t.nodes.size();
        tr += t.refs.size();
    }
    *total_nodes = tn;
    *total_refs = tr;
    if(tn > max_nodes || tr > max_refs || !nodes_out || (tr && !refs_out) || (n_meshes && (!node_counts || !ref_counts))) {
        return fail(ctx, LRT_ERR_RANGE, "output arrays too small: %llu nodes, %llu references needed",
                    static_cast<unsigned long long>(tn), static_cast<unsigned long long>(tr));
    }
    uint64_t on = 0, orf = 0;
    for(uint32_t m = 0; m < n_meshes; ++m) {
        const PackedTree& t = trees[m];
        for(size_t i = 0; i < t.nodes.size(); ++i) {
            nodes_out[2 * (on + i)] = t.nodes[i].x;
            nodes_out[2 * (on + i) + 1] = t.nodes[i].y;
        }
        std::copy(t.refs.begin(), t.refs.end(), refs_out + orf);
        node_counts[m] = static_cast<uint32_t>(t.nodes.size());
        ref_counts[m] = static_cast<uint32_t>(t.refs.size());
        if(depths) depths[m] = t.depth;
        on += t.nodes.size();
        orf += t.refs.size();
    }
    return LRT_OK;
}

int lrt_scene_upload(lrt_context* ctx, const lrt_scene_desc* desc) {
    if(!ctx) return LRT_ERR_INVALID_ARGUMENT;
    LRT_CUDA(ctx, cudaSetDevice(ctx->device));
    ctx->has_scene = false;
    ctx->diff_params = 0;
    std::string err;
    const KdBatchBuilder device_kd = [ctx](const std::vector<uint32_t>& counts, const BigVec<float>& bmin,
                                           const BigVec<float>& bmax, std::vector<PackedTree>& trees,
                                           std::string& e) {
        const int r = build_kdtrees_device(ctx, counts, bmin, bmax, trees, e);
        if(r != LRT_OK && e.empty()) e = ctx->error;
        return r;
    };
    // the GPU build pays a few milliseconds of fixed cost per tree level; below 2^15 triangles the host
    // build is as fast
    uint64_t n_tris = 0;
    for(uint32_t i = 0; desc && desc->objects && i < desc->n_objects; ++i) {
        if(desc->objects[i].kind == LRT_OBJECT_MESH) n_tris += desc->objects[i].n_indices / 3;
    }
    const bool device_trees = ctx->kd_build_device == 1 || (ctx->kd_build_device == 2 && n_tris >= (1u << 15));
    const int st = build_host_scene(desc, ctx->host, err, device_trees ? &device_kd : nullptr);
    if(st != LRT_OK) return fail(ctx, st, "%s", err.c_str());
    HostScene& h = ctx->host;
    uint64_t bytes = 0;
    cudaStream_t s = ctx->stream;
    LRT_CUDA(ctx, upload(ctx->nodes, h.nodes, s, bytes));
    LRT_CUDA(ctx, upload(ctx->tris, h.tris, s, bytes));
    LRT_CUDA(ctx, upload(ctx->ref_prim, h.ref_prim, s, bytes));
    LRT_CUDA(ctx, upload(ctx->normals, h.normals, s, bytes));
    LRT_CUDA(ctx, upload(ctx->objects, h.objects, s, bytes));
    LRT_CUDA(ctx, upload(ctx->materials, h.materials, s, bytes));
    LRT_CUDA(ctx, upload(ctx->tables, h.tables, s, bytes));
    LRT_CUDA(ctx, upload(ctx->emitters, h.emitters, s, bytes));
    // emission CDF (floats) followed by its emitter indices
    std::vector<float> emission(h.emission_cdf);
    emission.resize(2 * h.emission_cdf.size() + 1);
    for(size_t i = 0; i < h.emission_index.size(); ++i) {
        memcpy(&emission[h.emission_cdf.size() + i], &h.emission_index[i], 4);
    }
    LRT_CUDA(ctx, upload(ctx->emission, emission, s, bytes));
    LRT_CUDA(ctx, upload(ctx->tlas, h.tlas, s, bytes));
    LRT_CUDA(ctx, upload(ctx->tlas_objs, h.tlas_objs, s, bytes));
    LRT_CUDA(ctx, upload(ctx->light_cdf, h.light_cdf, s, bytes));
    LRT_CUDA(ctx, upload(ctx->light_tri, h.light_tri, s, bytes));
    LRT_CUDA(ctx, cudaStreamSynchronize(s));
    DeviceScene& ds = ctx->ds;
    ds.nodes = ctx->nodes.as<uint2>();
    ds.tris = ctx->tris.as<float4>();
    ds.ref_prim = ctx->ref_prim.as<uint32_t>();
    ds.normals = ctx->normals.as<float4>();
    ds.objects = ctx->objects.as<ObjRec>();
    ds.materials = ctx->materials.as<MatRec>();
    ds.tables = ctx->tables.as<float>();
    ds.emitters = ctx->emitters.as<EmitRec>();
    ds.sobol = ctx->sobol.as<uint32_t>();
    ds.emission_cdf = ctx->emission.as<float>();
    ds.emission_index = reinterpret_cast<const int32_t*>(ctx->emission.as<float>() + h.emission_cdf.size());
    ds.light_cdf = ctx->light_cdf.as<float>();
    ds.light_tri = ctx->light_tri.as<float4>();
    ds.n_objects = static_cast<int32_t>(h.objects.size());
    ds.n_materials = static_cast<int32_t>(h.materials.size());
    ds.n_emitters = static_cast<int32_t>(h.emitters.size());
    ds.n_infinite = h.n_infinite;
    ds.n_emission = static_cast<int32_t>(h.emission_cdf.size());
    ds.emission_power = h.emission_power;
    ds.n_heavy = h.n_heavy;
    for(int i = 0; i < 4; ++i) ds.heavy[i] = h.heavy[i];
    ds.cam = h.cam;
    ds.tlas = ctx->tlas.as<float4>();
    ds.tlas_objs = ctx->tlas_objs.as<int32_t>();
    ds.n_tlas = ctx->object_bvh ? static_cast<int32_t>(h.tlas.size() / 2) : 0;
    // shading keys a hit can carry: misses, hits without a BSDF, and 2 + each material type present
    ctx->shade_keys = 3u;
    for(const MatRec& m : h.materials) ctx->shade_keys |= 1u << (2 + m.type);
    ctx->has_sky = false;
    for(const EmitRec& e : h.emitters) ctx->has_sky |= e.kind == LRT_EMITTER_ENV;
    ctx->has_mesh_lights = false;
    for(const EmitRec& e : h.emitters) {
        ctx->has_mesh_lights |= e.kind == LRT_EMITTER_AREA && e.shape == LRT_OBJECT_MESH;
    }
    ctx->scene_bytes = bytes;
    ctx->has_scene = true;
    return LRT_OK;
}

uint64_t lrt_scene_device_bytes(const lrt_context* ctx) { return ctx ? ctx->scene_bytes : 0; }

uint64_t lrt_device_allocations(void) { return g_device_allocations.load(); }

int lrt_scene_set_camera_frame(lrt_context* ctx, const float* origin, const float* lower_left_corner,
                               const float* horizontal, const float* vertical) {
    if(!ctx) return LRT_ERR_INVALID_ARGUMENT;
    if(!origin || !lower_left_corner || !horizontal || !vertical) {
        return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "camera frame: null vector");
    }
    if(!ctx->has_scene) return fail(ctx, LRT_ERR_NO_SCENE, "no scene uploaded");
    CamRec cam{};
    for(int i = 0; i < 3; ++i) {
        cam.origin[i] = origin[i];
        cam.llc[i] = lower_left_corner[i];
        cam.horizontal[i] = horizontal[i];
        cam.vertical[i] = vertical[i];
    }
    ctx->host.cam = cam;
    ctx->ds.cam = cam;
    return LRT_OK;
}

int lrt_mesh_tree_info(const lrt_context* ctx, uint32_t object, uint32_t* nodes, uint32_t* refs, uint32_t* depth) {
    if(!ctx || !ctx->has_scene || object >= ctx->host.mesh_info.size()) return LRT_ERR_INVALID_ARGUMENT;
    const MeshTreeInfo& m = ctx->host.mesh_info[object];
    if(nodes) *nodes = m.nodes;
    if(refs) *refs = m.refs;
    if(depth) *depth = m.depth;
    return LRT_OK;
}

int lrt_trace_dev(lrt_context* ctx, const lrt_ray* rays_dev, uint32_t n, lrt_hit* hits_dev) {
    if(!ctx) return LRT_ERR_INVALID_ARGUMENT;
    if(!ctx->has_scene) return fail(ctx, LRT_ERR_NO_SCENE, "no scene uploaded");
    if(n == 0) return LRT_OK;
    if(!rays_dev || !hits_dev) return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "null buffer");
    k_trace<<<blocks_for(n), kBlock, 0, ctx->stream>>>(ctx->ds, rays_dev, n, hits_dev);
    LRT_CUDA(ctx, cudaGetLastError());
    return LRT_OK;
}

int lrt_trace(lrt_context* ctx, const lrt_ray* rays, uint32_t n, lrt_hit* hits) {
    if(!ctx) return LRT_ERR_INVALID_ARGUMENT;
    if(n == 0) return LRT_OK;
    if(!rays || !hits) return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "null buffer");
    LRT_CUDA(ctx, ctx->scratch_a.ensure(sizeof(lrt_ray) * static_cast<size_t>(n) + sizeof(lrt_hit) * static_cast<size_t>(n)));
    lrt_ray* dr = ctx->scratch_a.as<lrt_ray>();
    lrt_hit* dh = reinterpret_cast<lrt_hit*>(dr + n);
    LRT_CUDA(ctx, cudaMemcpyAsync(dr, rays, sizeof(lrt_ray) * n, cudaMemcpyHostToDevice, ctx->stream));
    const int st = lrt_trace_dev(ctx, dr, n, dh);
    if(st != LRT_OK) return st;
    LRT_CUDA(ctx, cudaMemcpyAsync(hits, dh, sizeof(lrt_hit) * n, cudaMemcpyDeviceToHost, ctx->stream));
    LRT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return LRT_OK;
}

int lrt_occluded(lrt_context* ctx, const lrt_ray* rays, uint32_t n, int32_t light, uint8_t* blocked) {
    if(!ctx) return LRT_ERR_INVALID_ARGUMENT;
    if(!ctx->has_scene) return fail(ctx, LRT_ERR_NO_SCENE, "no scene uploaded");
    if(light < 0 || light >= ctx->ds.n_emitters) return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "emitter out of range");
    if(n == 0) return LRT_OK;
    if(!rays || !blocked) return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "null buffer");
    const size_t rb = sizeof(lrt_ray) * static_cast<size_t>(n);
    LRT_CUDA(ctx, ctx->scratch_a.ensure(rb + n));
    char* base = ctx->scratch_a.as<char>();
    LRT_CUDA(ctx, cudaMemcpyAsync(base, rays, rb, cudaMemcpyHostToDevice, ctx->stream));
    k_occluded<<<blocks_for(n), kBlock, 0, ctx->stream>>>(ctx->ds, reinterpret_cast<lrt_ray*>(base), n, light,
                                                          reinterpret_cast<uint8_t*>(base + rb));
    LRT_CUDA(ctx, cudaGetLastError());
    LRT_CUDA(ctx, cudaMemcpyAsync(blocked, base + rb, n, cudaMemcpyDeviceToHost, ctx->stream));
    LRT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return LRT_OK;
}

int lrt_bsdf_evaluate(lrt_context* ctx, int32_t material, const lrt_bsdf_query* q, uint32_t n, lrt_bsdf_result* out) {
    if(!ctx) return LRT_ERR_INVALID_ARGUMENT;
    if(!ctx->has_scene) return fail(ctx, LRT_ERR_NO_SCENE, "no scene uploaded");
    if(material < 0 || material >= ctx->ds.n_materials) return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "material out of range");
    if(n == 0) return LRT_OK;
    if(!q || !out) return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "null buffer");
    const size_t qb = sizeof(lrt_bsdf_query) * n, rb = sizeof(lrt_bsdf_result) * n;
    LRT_CUDA(ctx, ctx->scratch_a.ensure(qb + rb));
    char* base = ctx->scratch_a.as<char>();
    LRT_CUDA(ctx, cudaMemcpyAsync(base, q, qb, cudaMemcpyHostToDevice, ctx->stream));
    k_bsdf<<<blocks_for(n), kBlock, 0, ctx->stream>>>(ctx->ds, material, reinterpret_cast<lrt_bsdf_query*>(base), n,
                                                      reinterpret_cast<lrt_bsdf_result*>(base + qb));
    LRT_CUDA(ctx, cudaGetLastError());
    LRT_CUDA(ctx, cudaMemcpyAsync(out, base + qb, rb, cudaMemcpyDeviceToHost, ctx->stream));
    LRT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return LRT_OK;
}

int lrt_sky_eval(lrt_context* ctx, const float* directions, uint32_t n, float* rgb) {
    if(!ctx) return LRT_ERR_INVALID_ARGUMENT;
    if(!ctx->has_scene) return fail(ctx, LRT_ERR_NO_SCENE, "no scene uploaded");
    if(n == 0) return LRT_OK;
    if(!directions || !rgb) return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "null buffer");
    const size_t b = sizeof(float) * 3 * n;
    LRT_CUDA(ctx, ctx->scratch_a.ensure(2 * b));
    float* base = ctx->scratch_a.as<float>();
    LRT_CUDA(ctx, cudaMemcpyAsync(base, directions, b, cudaMemcpyHostToDevice, ctx->stream));
    k_sky<<<blocks_for(n), kBlock, 0, ctx->stream>>>(ctx->ds, base, n, base + 3ull * n);
    LRT_CUDA(ctx, cudaGetLastError());
    LRT_CUDA(ctx, cudaMemcpyAsync(rgb, base + 3ull * n, b, cudaMemcpyDeviceToHost, ctx->stream));
    LRT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return LRT_OK;
}

int lrt_sampler_values(lrt_context* ctx, const uint32_t* pixel_sample, uint32_t n, uint32_t n_dims, float* values) {
    if(!ctx) return LRT_ERR_INVALID_ARGUMENT;
    if(n == 0 || n_dims == 0) return LRT_OK;
    if(!pixel_sample || !values) return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "null buffer");
    const size_t ib = sizeof(uint32_t) * 2 * n, ob = sizeof(float) * static_cast<size_t>(n) * n_dims;
    LRT_CUDA(ctx, ctx->scratch_a.ensure(ib + ob));
    char* base = ctx->scratch_a.as<char>();
    LRT_CUDA(ctx, cudaMemcpyAsync(base, pixel_sample, ib, cudaMemcpyHostToDevice, ctx->stream));
    k_sampler<<<blocks_for(n), kBlock, 0, ctx->stream>>>(ctx->sobol.as<uint32_t>(), reinterpret_cast<uint32_t*>(base), n,
                                                         n_dims, reinterpret_cast<float*>(base + ib));
    LRT_CUDA(ctx, cudaGetLastError());
    LRT_CUDA(ctx, cudaMemcpyAsync(values, base + ib, ob, cudaMemcpyDeviceToHost, ctx->stream));
    LRT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return LRT_OK;
}

int lrt_emitter_query(lrt_context* ctx, const float* points, const float* u2, const float* dirs, uint32_t n,
                      float* sample_out, float* pdf_out) {
    if(!ctx) return LRT_ERR_INVALID_ARGUMENT;
    if(!ctx->has_scene) return fail(ctx, LRT_ERR_NO_SCENE, "no scene uploaded");
    if(n == 0) return LRT_OK;
    if(!points || !u2 || !dirs || !sample_out || !pdf_out) return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "null buffer");
    const size_t pb = 12ull * n, ub = 8ull * n, ob = 64ull * n, fb = 4ull * n;
    LRT_CUDA(ctx, ctx->scratch_a.ensure(2 * pb + ub + ob + fb));
    char* base = ctx->scratch_a.as<char>();
    LRT_CUDA(ctx, cudaMemcpyAsync(base, points, pb, cudaMemcpyHostToDevice, ctx->stream));
    LRT_CUDA(ctx, cudaMemcpyAsync(base + pb, dirs, pb, cudaMemcpyHostToDevice, ctx->stream));
    LRT_CUDA(ctx, cudaMemcpyAsync(base + 2 * pb, u2, ub, cudaMemcpyHostToDevice, ctx->stream));
    float* o = reinterpret_cast<float*>(base + 2 * pb + ub);
    float* pdf = reinterpret_cast<float*>(base + 2 * pb + ub + ob);
    k_emitter<<<blocks_for(n), kBlock, 0, ctx->stream>>>(ctx->ds, reinterpret_cast<float*>(base),
                                                         reinterpret_cast<float*>(base + 2 * pb),
                                                         reinterpret_cast<float*>(base + pb), n, o, pdf);
    LRT_CUDA(ctx, cudaGetLastError());
    LRT_CUDA(ctx, cudaMemcpyAsync(sample_out, o, ob, cudaMemcpyDeviceToHost, ctx->stream));
    LRT_CUDA(ctx, cudaMemcpyAsync(pdf_out, pdf, fb, cudaMemcpyDeviceToHost, ctx->stream));
    LRT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return LRT_OK;
}

int lrt_camera_rays(lrt_context* ctx, uint32_t width, uint32_t height, const uint32_t* pixel_sample, uint32_t n,
                    lrt_ray* rays) {
    if(!ctx) return LRT_ERR_INVALID_ARGUMENT;
    if(!ctx->has_scene) return fail(ctx, LRT_ERR_NO_SCENE, "no scene uploaded");
    if(n == 0) return LRT_OK;
    if(!pixel_sample || !rays || width < 2 || height < 2) return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "bad arguments");
    const size_t ib = 8ull * n, ob = sizeof(lrt_ray) * n;
    LRT_CUDA(ctx, ctx->scratch_a.ensure(ib + ob));
    char* base = ctx->scratch_a.as<char>();
    LRT_CUDA(ctx, cudaMemcpyAsync(base, pixel_sample, ib, cudaMemcpyHostToDevice, ctx->stream));
    k_camera<<<blocks_for(n), kBlock, 0, ctx->stream>>>(ctx->ds, width, height, reinterpret_cast<uint32_t*>(base), n,
                                                        reinterpret_cast<lrt_ray*>(base + ib));
    LRT_CUDA(ctx, cudaGetLastError());
    LRT_CUDA(ctx, cudaMemcpyAsync(rays, base + ib, ob, cudaMemcpyDeviceToHost, ctx->stream));
    LRT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return LRT_OK;
}

int lrt_render_dev(lrt_context* ctx, const lrt_render_params* params, float* rgb_dev) {
    if(!ctx) return LRT_ERR_INVALID_ARGUMENT;
    if(!rgb_dev) return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "null output");
    LRT_CUDA(ctx, cudaSetDevice(ctx->device));
    return render_impl(ctx, params, rgb_dev);
}

int lrt_render(lrt_context* ctx, const lrt_render_params* params, float* rgb) {
    if(!ctx) return LRT_ERR_INVALID_ARGUMENT;
    if(!rgb || !params) return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "null argument");
    LRT_CUDA(ctx, cudaSetDevice(ctx->device));
    const size_t bytes = sizeof(float) * 3 * static_cast<size_t>(params->width) * params->height;
    LRT_CUDA(ctx, ctx->out_rgb.ensure(bytes));
    LRT_CUDA(ctx, cudaMemsetAsync(ctx->out_rgb.ptr, 0, bytes, ctx->stream));
    const int st = render_impl(ctx, params, ctx->out_rgb.as<float>());
    if(st != LRT_OK) return st;
    LRT_CUDA(ctx, cudaMemcpyAsync(rgb, ctx->out_rgb.ptr, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    LRT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return LRT_OK;
}

int lrt_render_batch_dev(lrt_context* ctx, const lrt_job_desc* jobs, uint32_t n_jobs, int32_t max_depth, int32_t rr_depth,
                         float* rgb_dev) {
    if(!ctx) return LRT_ERR_INVALID_ARGUMENT;
    LRT_CUDA(ctx, cudaSetDevice(ctx->device));
    return render_batch_impl(ctx, jobs, n_jobs, max_depth, rr_depth, rgb_dev);
}

int lrt_render_batch(lrt_context* ctx, const lrt_job_desc* jobs, uint32_t n_jobs, int32_t max_depth, int32_t rr_depth,
                     float* rgb) {
    if(!ctx) return LRT_ERR_INVALID_ARGUMENT;
    if(n_jobs == 0) return LRT_OK;
    if(!jobs || !rgb) return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "null argument");
    LRT_CUDA(ctx, cudaSetDevice(ctx->device));
    unsigned long long floats = 0;
    for(uint32_t i = 0; i < n_jobs; ++i) {
        floats = std::max<unsigned long long>(floats, jobs[i].output_offset + 3ull * jobs[i].width * jobs[i].height);
    }
    LRT_CUDA(ctx, ctx->batch_out.ensure(4ull * floats));
    LRT_CUDA(ctx, cudaMemsetAsync(ctx->batch_out.ptr, 0, 4ull * floats, ctx->stream));
    const int st = render_batch_impl(ctx, jobs, n_jobs, max_depth, rr_depth, ctx->batch_out.as<float>());
    if(st != LRT_OK) return st;
    LRT_CUDA(ctx, cudaMemcpyAsync(rgb, ctx->batch_out.ptr, 4ull * floats, cudaMemcpyDeviceToHost, ctx->stream));
    LRT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return LRT_OK;
}

int lrt_render_stats_get(lrt_context* ctx, lrt_render_stats* out) {
    if(!ctx || !out) return LRT_ERR_INVALID_ARGUMENT;
    *out = ctx->stats;
    return LRT_OK;
}

int lrt_render_stats_reset(lrt_context* ctx) {
    if(!ctx) return LRT_ERR_INVALID_ARGUMENT;
    ctx->stats = lrt_render_stats{};
    return LRT_OK;
}

int lrt_set_option(lrt_context* ctx, const char* name, int64_t value) {
    if(!ctx || !name) return LRT_ERR_INVALID_ARGUMENT;
    if(strcmp(name, "stage_timing") == 0) {
        ctx->stage_timing = value != 0;
    } else if(strcmp(name, "count_work") == 0) {
        ctx->count_work = value != 0;
    } else if(strcmp(name, "batch_graph") == 0) {
        ctx->batch_graph = value != 0;
    } else if(strcmp(name, "adjoint_megakernel") == 0) {
        ctx->adjoint_megakernel = value != 0;
    } else if(strcmp(name, "photon_eye_kernel") == 0) {
        if(value < 0 || value > 2) return fail(ctx, LRT_ERR_RANGE, "photon_eye_kernel must be 0, 1 or 2");
        ctx->photon_eye_kernel = static_cast<int>(value);
    } else if(strcmp(name, "shade_per_key") == 0) {
        ctx->shade_per_key = value != 0;
    } else if(strcmp(name, "kd_build_device") == 0) {
        if(value < 0 || value > 2) return fail(ctx, LRT_ERR_RANGE, "kd_build_device must be 0, 1 or 2");
        ctx->kd_build_device = static_cast<int>(value);
    } else if(strcmp(name, "object_bvh") == 0) {
        ctx->object_bvh = value != 0;
        if(ctx->has_scene) ctx->ds.n_tlas = ctx->object_bvh ? static_cast<int32_t>(ctx->host.tlas.size() / 2) : 0;
    } else if(strcmp(name, "blocks_per_sm") == 0) {
        if(value < 0 || value > 32) return fail(ctx, LRT_ERR_RANGE, "blocks_per_sm must be in [0, 32]");
        ctx->blocks_per_sm_cap = static_cast<uint32_t>(value);
    } else if(strcmp(name, "pixel_tile") == 0) {
        if(value < 1 || value > 64) return fail(ctx, LRT_ERR_RANGE, "pixel_tile must be in [1, 64]");
        ctx->pixel_tile = static_cast<uint32_t>(value);
    } else if(strcmp(name, "photon_tree_device") == 0) {
        ctx->photon_tree_device = value != 0;
    } else if(strcmp(name, "photon_eye_slot_mb") == 0) {
        ctx->photon_eye_slot_mb = static_cast<uint64_t>(std::max<int64_t>(16, std::min<int64_t>(value, 1ll << 20)));
    } else if(strcmp(name, "photon_eye_sort") == 0) {
        ctx->photon_eye_sort = value != 0;
    } else if(strcmp(name, "photon_eye_tail") == 0) {
        ctx->photon_eye_tail = static_cast<uint32_t>(std::max<int64_t>(0, std::min<int64_t>(value, 1ll << 30)));
    } else if(strcmp(name, "knn_shared_heap") == 0) {
        ctx->knn_shared_heap = value != 0;
    } else if(strcmp(name, "batch_queue") == 0) {
        ctx->batch_queue = value != 0;
    } else if(strcmp(name, "photon_tree_depth_limit") == 0) {
        ctx->photon_tree_depth_limit = value < 0 ? -1 : static_cast<int>(std::min<int64_t>(value, 64));
    } else if(strcmp(name, "wave_capacity") == 0) {
        if(value != 0 && (value < 1024 || value > (1ll << 26))) {
            return fail(ctx, LRT_ERR_RANGE, "wave_capacity must be 0 (the defaults) or in [1024, 2^26]");
        }
        ctx->wave_capacity = static_cast<uint32_t>(value);
    } else {
        return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "unknown option %s", name);
    }
    return LRT_OK;
}

}  // extern "C"

// ================================ allocation-free render ================================
//
// lrt_render_dev_noalloc renders with the same kernels as lrt_render_dev, but its wavefront state lives
// in one fixed device array of this file instead of memory the library allocates. It serves callers
// that cannot let a library call cudaMalloc: a cudaMalloc may synchronise the whole device (a stall a
// frame loop sharing the GPU with other streams cannot take), and it fails in processes whose device
// memory is already committed -- to a framework's caching allocator, or to a fixed budget reserved at
// start-up. Those callers pass their own output buffer and keep the scene uploaded beforehand.
//
// The array is a file-scope __device__ variable: every GPU that loads this library holds its
// kNoAllocScratchBytes until the process exits. Its name is a host-side stand-in in host code, so the
// device address is looked up once per device with cudaGetSymbolAddress (on the entry point's first
// call on that device, with that device current); make that first call before any stream capture.
// All calls on a device share the array and it keeps the last call's contents: the counters are
// cleared at every wave, and calls that overlap on the GPU (two streams, two threads) race on it.
namespace {

constexpr size_t kNoAllocScratchBytes = 32ull << 20;  // 32 MiB
constexpr int kNoAllocMaxDepth = 64;                  // counters for at most this many bounces
constexpr int kNoAllocMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_noalloc_mutex;
unsigned char* g_noalloc_base[kNoAllocMaxDevices] = {nullptr};

// bytes of wavefront state per path slot: o, d, tp, L, hit_p, hit_n, sh_o, sh_d, sh_c (float4 each),
// sh_s (float), misc (float2), id (uint2), two queues, kKeys shading segments and the per-pixel sum
// (3 floats); the shadow arrays have two entries per slot
constexpr size_t kNoAllocSlotBytes = 6 * 16 + 3 * 32 + 2 * 4 + 8 + 8 + 2 * 8 + kKeys * 4 + 12;
constexpr size_t kNoAllocHeaderBytes = (sizeof(BounceCounters) * (kNoAllocMaxDepth + 1) + 255) / 256 * 256;
constexpr uint32_t kNoAllocCapacity =
    static_cast<uint32_t>((kNoAllocScratchBytes - kNoAllocHeaderBytes - 17 * 256) / kNoAllocSlotBytes);

int noalloc_scratch(lrt_context* ctx, unsigned char** base) {
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if(ctx->device < 0 || ctx->device >= kNoAllocMaxDevices) {
        return fail(ctx, LRT_ERR_RANGE, "allocation-free render supports device ordinals below %d", kNoAllocMaxDevices);
    }
    // The address is looked up again on every call outside stream capture (cheap, host side), so that a
    // device reset that recreated the primary context between calls cannot leave a stale address; inside
    // a capture the address of the last call outside one is used.
    cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
    if(cudaStreamIsCapturing(ctx->stream, &capture) != cudaSuccess) capture = cudaStreamCaptureStatusNone;
    if(!g_noalloc_base[ctx->device] || capture == cudaStreamCaptureStatusNone) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if(e != cudaSuccess || !p) {
            return fail(ctx, LRT_ERR_CUDA, "cudaGetSymbolAddress(scratch) on device %d: %s", ctx->device,
                        cudaGetErrorString(e));
        }
        g_noalloc_base[ctx->device] = static_cast<unsigned char*>(p);
    }
    *base = g_noalloc_base[ctx->device];
    return LRT_OK;
}

}  // namespace

extern "C" int lrt_render_dev_noalloc(lrt_context* ctx, const lrt_render_params* p, float* rgb_dev) {
    if(!ctx) return LRT_ERR_INVALID_ARGUMENT;
    if(!rgb_dev || !p) return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "null argument");
    if(!ctx->has_scene) return fail(ctx, LRT_ERR_NO_SCENE, "no scene uploaded");
    if(p->width < 2 || p->height < 2 || p->spp == 0 || p->max_depth < 1) {
        return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "render parameters out of range (width, height >= 2; spp, max_depth >= 1)");
    }
    if(p->max_depth > kNoAllocMaxDepth) {
        return fail(ctx, LRT_ERR_RANGE, "allocation-free render: max_depth %d exceeds its maximum of %d", p->max_depth,
                    kNoAllocMaxDepth);
    }
    if(static_cast<uint64_t>(p->width) * p->height > 0x3fffffffull) return fail(ctx, LRT_ERR_RANGE, "image too large");
    const uint32_t row_begin = p->row_end > p->row_begin ? p->row_begin : 0u;
    const uint32_t row_end = p->row_end > p->row_begin ? std::min(p->row_end, p->height) : p->height;
    if(row_begin >= row_end) return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "empty row range");
    LRT_CUDA(ctx, cudaSetDevice(ctx->device));
    unsigned char* base = nullptr;
    const int st = noalloc_scratch(ctx, &base);
    if(st != LRT_OK) return st;

    // carve the fixed array: counters, then each slot array on a 256-byte boundary
    const uint32_t cap = kNoAllocCapacity;
    size_t off = kNoAllocHeaderBytes;
    auto take = [&](size_t bytes) {
        unsigned char* q = base + off;
        off += (bytes + 255) / 256 * 256;
        return q;
    };
    WaveArgs a{};
    a.s = ctx->ds;
    a.counters = reinterpret_cast<BounceCounters*>(base);
    a.o = reinterpret_cast<float4*>(take(16ull * cap));
    a.d = reinterpret_cast<float4*>(take(16ull * cap));
    a.tp = reinterpret_cast<float4*>(take(16ull * cap));
    a.L = reinterpret_cast<float4*>(take(16ull * cap));
    a.hit_p = reinterpret_cast<float4*>(take(16ull * cap));
    a.hit_n = reinterpret_cast<float4*>(take(16ull * cap));
    a.sh_o = reinterpret_cast<float4*>(take(32ull * cap));
    a.sh_d = reinterpret_cast<float4*>(take(32ull * cap));
    a.sh_c = reinterpret_cast<float4*>(take(32ull * cap));
    a.sh_s = reinterpret_cast<float*>(take(8ull * cap));
    a.misc = reinterpret_cast<float2*>(take(8ull * cap));
    a.id = reinterpret_cast<uint2*>(take(8ull * cap));
    a.q0 = reinterpret_cast<uint32_t*>(take(8ull * cap));
    a.q1 = reinterpret_cast<uint32_t*>(take(8ull * cap));
    a.keyed = reinterpret_cast<uint32_t*>(take(4ull * cap * kKeys));
    a.sum = reinterpret_cast<float*>(take(12ull * cap));
    if(off > kNoAllocScratchBytes) return fail(ctx, LRT_ERR_RANGE, "allocation-free render: scratch layout overflow");
    a.work = nullptr;
    a.capacity = cap;
    a.width = p->width;
    a.height = p->height;
    a.max_depth = p->max_depth;
    a.rr_depth = p->rr_depth;
    const size_t counters_bytes = sizeof(BounceCounters) * (p->max_depth + 1);

    const uint32_t spp = p->spp;
    const uint32_t pix0 = row_begin * p->width;
    const uint32_t pix1 = row_end * p->width;
    uint64_t launches = 0;
    const int rst = run_render_waves(ctx, a, p, pix0, pix1, cap, counters_bytes, false, false, rgb_dev, launches);
    if(rst != LRT_OK) return rst;
    ctx->stats.paths += static_cast<uint64_t>(pix1 - pix0) * spp;
    ctx->stats.kernel_launches += launches;
    return LRT_OK;
}
