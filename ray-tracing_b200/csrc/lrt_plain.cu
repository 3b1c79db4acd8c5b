// lrt_plain.cu — the plain GPU path tracer: one kernel launch per job, one thread per pixel, each
// thread running the reference's render loop (main.cpp:121-136: samples in order, the whole path of a
// sample in registers, path_integrator::li of path_integrator.h:23-166 with closest-hit traversal,
// emission + MIS, NEE with its shadow ray, BSDF sampling and Russian roulette) — a megakernel with no
// queues, no sorting and no persistence.
//
// It is the comparison point for the wavefront renderer and the batched renderer: it draws the same
// samples in the same order and makes the same floating-point operations per path, so its images are
// bit-identical to theirs, and its throughput is what a direct CUDA port of the reference loop gets.
#include <algorithm>
#include <vector>

#include "lrt_bsdf.cuh"
#include "lrt_context.cuh"
#include "lrt_scene.cuh"

using namespace lrt;

namespace {

struct PlainArgs {
    DeviceScene s;
    const JobRec* job;
    float* out;  // the job's image (3 floats per pixel)
    int32_t max_depth, rr_depth;
};

// One pixel of one job: its spp samples in order through path_integrator::li, the mean into out.
__device__ __forceinline__ void plain_pixel(const DeviceScene& s, const JobRec& job, uint32_t pix, int32_t max_depth,
                                            int32_t rr_depth, float* out) {
    TraceCount cnt{0, 0};
    f3 acc = mk(0.0f);
    for(uint32_t k = 0; k < job.spp; ++k) {
        const uint32_t sample = job.sample_offset + k;
        Sampler cam_smp = sampler_start(pix, sample);
        const F2 off = sampler_next_2d(sobol_table(s), cam_smp);
        const float u = (static_cast<float>(pix % job.width) + off.x) / static_cast<float>(job.width - 1);
        const float v = (static_cast<float>(pix / job.width) + off.y) / static_cast<float>(job.height - 1);
        Ray ray = camera_ray(job.cam, u, v);
        f3 result = mk(0.0f);
        f3 throughput = mk(1.0f);
        float eta = 1.0f;
        bool have_pdf = false;
        float sa_pdf = 0.0f;
        for(int depth = 0; depth < max_depth; ++depth) {
            HitInfo h;
            if(!scene_hit<false>(s, ray, 0.001f, kInf, h, cnt)) {  // path_integrator.h:32-45
                const f3 Le = eval_environment(s, ray.d);
                if(!have_pdf) {
                    result += throughput * Le;
                } else {
                    const float light_pdf = pdf_emitter_direction(s, mk(0.0f), ray.d);
                    result += throughput * power_heuristic(sa_pdf, light_pdf) * Le;
                }
                break;
            }
            const ObjRec& obj = s.objects[h.object];
            if(obj.emitter >= 0 && h.front_face) {  // path_integrator.h:47-59
                const f3 Le = area_emitted(s.emitters[obj.emitter], h.normal, -normalize(ray.d));
                if(!is_zero(Le)) {
                    if(!have_pdf) {
                        result += throughput * Le;
                    } else {
                        const float light_pdf = pdf_emitter_direction(s, ray.o, ray.d);
                        result += throughput * power_heuristic(sa_pdf, light_pdf) * Le;
                    }
                }
            }
            int32_t mid = obj.material;
            if(h.object == job.override_obj) mid = job.override_mat;
            if(mid < 0) break;
            const Onb basis = onb_from_normal(h.normal);
            BRec rec{};
            rec.wi = to_local(basis, -normalize(ray.d));
            rec.wo = mk(0.0f);
            rec.front_face = h.front_face;
            rec.eta = 1.0f;
            Sampler smp = sampler_start(pix, sample);
            smp.dimension = 2u + 6u * static_cast<uint32_t>(depth);
            const F2 light_uv = sampler_next_2d(sobol_table(s), smp);
            BsdfCtx bctx = ctx_default(LRT_MODE_RADIANCE);
            bctx.lobe_sample = sampler_next_1d(sobol_table(s), smp);
            const F2 bsdf_uv = sampler_next_2d(sobol_table(s), smp);
            const float rr_u = sampler_next_1d(sobol_table(s), smp);
            const MatRec& mat = s.materials[mid];
            if((mat.flags & (kDiffuse | kGlossy)) != 0) {  // NEE (path_integrator.h:86-128)
                DirectSample light{};
                light.distance = kInf;
                if(sample_emitter_direction(s, h.p, light_uv.x, light_uv.y, light)) {
                    const f3 shadow_origin = h.p + h.normal * 1e-4f;
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
                        const f3 f_cos = bsdf_eval(s.materials, s.tables, mid, bctx, rec, kSolidAngle);
                        if(!is_zero(f_cos)) {
                            const float bsdf_pdf_v = bsdf_pdf(s.materials, s.tables, mid, bctx, rec, kSolidAngle);
                            const float light_pdf = pdf_emitter_direction(s, h.p, shadow_dir);
                            if(light_pdf > 0.0f) {
                                const float w = power_heuristic(light_pdf, bsdf_pdf_v);
                                const f3 contrib = throughput * f_cos * light.radiance * (w / light_pdf);
                                if(!scene_occluded<false>(s, Ray{shadow_origin, shadow_dir}, 0.001f, tmax,
                                                          light.emitter, cnt)) {
                                    result += contrib;
                                }
                            }
                        }
                    }
                }
            }
            if(depth == max_depth - 1) break;
            const f3 weight = bsdf_sample(s.materials, s.tables, mid, bctx, rec, bsdf_uv.x, bsdf_uv.y);
            if(is_zero(weight)) break;
            const f3 new_dir = to_world(basis, rec.wo);
            throughput *= weight;
            eta *= rec.eta;
            if(depth >= rr_depth) {
                const float q = smin(max3(throughput) * eta * eta, 0.95f);
                if(rr_u >= q) break;
                throughput /= q;
            }
            have_pdf = measure_of(rec.sampled_type) == kSolidAngle && rec.pdf > 0.0f;
            sa_pdf = rec.pdf;
            ray = Ray{h.p, new_dir};
        }
        acc += result;
    }
    store3(out + 3ull * pix, acc / static_cast<float>(job.spp));
}

__global__ void __launch_bounds__(kBlock) k_pt_plain(PlainArgs a) {
    const JobRec& job = *a.job;
    const uint32_t n_pixels = job.width * job.height;
    for(uint32_t pix = blockIdx.x * blockDim.x + threadIdx.x; pix < n_pixels; pix += gridDim.x * blockDim.x) {
        plain_pixel(a.s, job, pix, a.max_depth, a.rr_depth, a.out);
    }
}

// ---- batched jobs as one persistent launch over a device queue of (job, tile) items ----
//
// Each warp takes the next item from the queue (one atomic per warp): a tile of 32 consecutive pixels of
// one job, which its lanes render with plain_pixel. Items are ordered costliest job first (by spp), so the
// longest tiles start early and the launch's tail is made of cheap ones. Every pixel's samples, draws and
// arithmetic are those of k_pt_plain, so the images are the per-job launches' bit for bit.
constexpr uint32_t kQueueTile = 32;

struct QueueArgs {
    DeviceScene s;
    const JobRec* jobs;
    const uint2* items;  // (job, first pixel of the tile)
    uint32_t n_items;
    uint32_t* cursor;
    float* out;          // the batch's output; each job's image at its out_offset
    int32_t max_depth, rr_depth;
};

__global__ void __launch_bounds__(kBlock) k_pt_queue(QueueArgs a) {
    const int lane = threadIdx.x & 31;
    while(true) {
        uint32_t item = 0;
        if(lane == 0) item = atomicAdd(a.cursor, 1u);
        item = __shfl_sync(0xffffffffu, item, 0);
        if(item >= a.n_items) break;
        const uint2 it = a.items[item];
        const JobRec& job = a.jobs[it.x];
        const uint32_t pix = it.y + static_cast<uint32_t>(lane);
        if(pix < job.width * job.height) {
            plain_pixel(a.s, job, pix, a.max_depth, a.rr_depth, a.out + job.out_offset);
        }
        __syncwarp();
    }
}

}  // namespace

namespace lrt {

int render_batch_queue(lrt_context* ctx, const std::vector<JobRec>& recs, unsigned long long total, int32_t max_depth,
                       int32_t rr_depth, float* rgb_dev) {
    const uint32_t n_jobs = static_cast<uint32_t>(recs.size());
    std::vector<uint32_t> by_cost(n_jobs);
    for(uint32_t i = 0; i < n_jobs; ++i) by_cost[i] = i;
    std::stable_sort(by_cost.begin(), by_cost.end(), [&](uint32_t x, uint32_t y) { return recs[x].spp > recs[y].spp; });
    std::vector<uint2> items;
    for(const uint32_t j : by_cost) {
        const uint32_t n = recs[j].width * recs[j].height;
        for(uint32_t p = 0; p < n; p += kQueueTile) items.push_back(make_uint2(j, p));
    }
    const size_t job_bytes = (sizeof(JobRec) * n_jobs + 255) / 256 * 256;
    const size_t item_bytes = sizeof(uint2) * items.size();
    LRT_CUDA(ctx, ctx->batch_jobs.ensure(job_bytes + item_bytes + 16));
    char* base = ctx->batch_jobs.as<char>();
    LRT_CUDA(ctx, cudaMemcpyAsync(base, recs.data(), sizeof(JobRec) * n_jobs, cudaMemcpyHostToDevice, ctx->stream));
    LRT_CUDA(ctx, cudaMemcpyAsync(base + job_bytes, items.data(), item_bytes, cudaMemcpyHostToDevice, ctx->stream));
    uint32_t* cursor = reinterpret_cast<uint32_t*>(base + job_bytes + item_bytes);
    LRT_CUDA(ctx, cudaMemsetAsync(cursor, 0, 4, ctx->stream));
    QueueArgs a{};
    a.s = ctx->ds;
    a.jobs = reinterpret_cast<const JobRec*>(base);
    a.items = reinterpret_cast<const uint2*>(base + job_bytes);
    a.n_items = static_cast<uint32_t>(items.size());
    a.cursor = cursor;
    a.out = rgb_dev;
    a.max_depth = max_depth;
    a.rr_depth = rr_depth;
    k_pt_queue<<<grid_for(ctx, (const void*)k_pt_queue, kBlock), kBlock, 0, ctx->stream>>>(a);
    LRT_CUDA(ctx, cudaGetLastError());
    ctx->stats.paths += total;
    ctx->stats.kernel_launches += 1;
    return LRT_OK;
}

}  // namespace lrt

extern "C" {

int lrt_render_plain_dev(lrt_context* ctx, const lrt_job_desc* jobs, uint32_t n_jobs, int32_t max_depth, int32_t rr_depth,
                         float* rgb_dev) {
    if(!ctx) return LRT_ERR_INVALID_ARGUMENT;
    if(!ctx->has_scene) return fail(ctx, LRT_ERR_NO_SCENE, "no scene uploaded");
    if(n_jobs == 0) return LRT_OK;
    if(!jobs || !rgb_dev) return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "null argument");
    if(max_depth < 1 || max_depth > 1024) return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "max_depth out of range");
    LRT_CUDA(ctx, cudaSetDevice(ctx->device));
    std::vector<JobRec> recs;
    unsigned long long total = 0, out_floats = 0;
    const int st = job_records(ctx, jobs, n_jobs, recs, total, out_floats);
    if(st != LRT_OK) return st;
    LRT_CUDA(ctx, ctx->batch_jobs.ensure(sizeof(JobRec) * n_jobs));
    LRT_CUDA(ctx, cudaMemcpyAsync(ctx->batch_jobs.ptr, recs.data(), sizeof(JobRec) * n_jobs, cudaMemcpyHostToDevice,
                                  ctx->stream));
    PlainArgs a{};
    a.s = ctx->ds;
    a.max_depth = max_depth;
    a.rr_depth = rr_depth;
    for(uint32_t i = 0; i < n_jobs; ++i) {
        a.job = ctx->batch_jobs.as<JobRec>() + i;
        a.out = rgb_dev + recs[i].out_offset;
        const uint32_t blocks = blocks_for(recs[i].width * recs[i].height);
        k_pt_plain<<<blocks, kBlock, 0, ctx->stream>>>(a);
    }
    LRT_CUDA(ctx, cudaGetLastError());
    ctx->stats.paths += total;
    ctx->stats.kernel_launches += n_jobs;
    return LRT_OK;
}

int lrt_render_plain(lrt_context* ctx, const lrt_job_desc* jobs, uint32_t n_jobs, int32_t max_depth, int32_t rr_depth,
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
    const int st = lrt_render_plain_dev(ctx, jobs, n_jobs, max_depth, rr_depth, ctx->batch_out.as<float>());
    if(st != LRT_OK) return st;
    LRT_CUDA(ctx, cudaMemcpyAsync(rgb, ctx->batch_out.ptr, 4ull * floats, cudaMemcpyDeviceToHost, ctx->stream));
    LRT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return LRT_OK;
}

}  // extern "C"
