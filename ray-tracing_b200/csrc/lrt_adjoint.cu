// lrt_adjoint.cu — differentiation of the path tracer with respect to material parameters by
// path-replay backpropagation, and the host side of its setup (material updates, perturbed records).
//
// Estimator. A path's radiance is L = sum_d c_d, where c_d is what depth d adds (the emission or sky
// radiance reached at d and the NEE contribution made at d), each carrying the throughput of the
// vertices before it. Under detached sampling (sampled directions, lobe choices, roulette and MIS
// weights held fixed), a parameter moves L only through BSDF values:
//   dL = sum_d [ dNEE_d  +  (sum_{d' > d} c_d') * dE_d(wo_d) / E_d(wo_d) ]
// where E_d is the BSDF value (f * cos) of vertex d at its sampled direction wo_d (zero for delta
// lobes, whose values carry no parameter), and dNEE_d is the NEE term with its BSDF value replaced by
// the value's derivative. The kernel replays each path once from its sampler state — the same
// samples, rays and operations as the renderers — keeping c_d and dE_d/E_d of the parameters that
// move vertex d's material in local arrays, then sums the suffix products backwards. The BSDF
// derivative is the central difference of the packed +step / -step material records of a parameter
// group, so every material type (and the rough-transmittance tables of rough plastic and rough
// coating) is covered by the BSDF code the renderer runs; one pair of evaluations serves the three
// channel parameters of an albedo, eta or k, since channel c of a BSDF value moves only with channel c
// of those. Per-thread sums are warp-reduced before one double atomic per parameter and warp.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "lrt_adjoint.cuh"
#include "lrt_bsdf.cuh"
#include "lrt_context.cuh"
#include "lrt_scene.cuh"

using namespace lrt;

namespace {

constexpr int kMaxParams = LRT_MAX_DIFF_PARAMS;
constexpr int kMaxAff = LRT_MAX_GROUPS_PER_MATERIAL;
constexpr int kMaxAdjDepth = LRT_MAX_ADJOINT_DEPTH;

struct AdjArgs {
    DeviceScene s;
    DiffDev d;
    const JobRec* jobs;
    uint32_t n_jobs;
    unsigned long long total_paths;
    const float* adjoint;  // dLoss/dimage, batch output layout
    int32_t max_depth, rr_depth;
    double* grad;
};

__global__ void __launch_bounds__(kBlock) k_adjoint(AdjArgs a) {
    float g[kMaxParams];
    for(uint32_t j = 0; j < a.d.n_params; ++j) g[j] = 0.0f;
    f3 vc[kMaxAdjDepth];
    f3 vd[kMaxAdjDepth][kMaxAff];
    int32_t vmid[kMaxAdjDepth];
    int32_t vn[kMaxAdjDepth];
    const DeviceScene& s = a.s;
    TraceCount cnt{0, 0};
    const unsigned long long stride = static_cast<unsigned long long>(gridDim.x) * blockDim.x;
    for(unsigned long long gp = blockIdx.x * blockDim.x + threadIdx.x; gp < a.total_paths; gp += stride) {
        uint32_t lo = 0, hi = a.n_jobs;  // last job with path_begin <= gp
        while(hi - lo > 1) {
            const uint32_t mid = (lo + hi) / 2;
            if(a.jobs[mid].path_begin <= gp) {
                lo = mid;
            } else {
                hi = mid;
            }
        }
        const JobRec& job = a.jobs[lo];
        const unsigned long long local = gp - job.path_begin;
        const uint32_t pix = static_cast<uint32_t>(local / job.spp);
        const uint32_t sample = job.sample_offset + static_cast<uint32_t>(local % job.spp);
        const f3 delta = load3(a.adjoint + job.out_offset + 3ull * pix) / static_cast<float>(job.spp);
        if(is_zero(delta)) continue;

        Sampler cam_smp = sampler_start(pix, sample);
        const F2 off = sampler_next_2d(sobol_table(s), cam_smp);
        const float u = (static_cast<float>(pix % job.width) + off.x) / static_cast<float>(job.width - 1);
        const float v = (static_cast<float>(pix / job.width) + off.y) / static_cast<float>(job.height - 1);
        Ray ray = camera_ray(job.cam, u, v);
        f3 throughput = mk(1.0f);
        float eta = 1.0f;
        bool have_pdf = false;
        float sa_pdf = 0.0f;
        int n_vertices = 0;
        for(int depth = 0; depth < a.max_depth; ++depth) {
            f3 c = mk(0.0f);
            vn[depth] = 0;
            vmid[depth] = -1;
            n_vertices = depth + 1;
            HitInfo h;
            if(!scene_hit<false>(s, ray, 0.001f, kInf, h, cnt)) {  // path_integrator.h:32-45
                const f3 Le = eval_environment(s, ray.d);
                if(!have_pdf) {
                    c += throughput * Le;
                } else {
                    const float light_pdf = pdf_emitter_direction(s, mk(0.0f), ray.d);
                    c += throughput * power_heuristic(sa_pdf, light_pdf) * Le;
                }
                vc[depth] = c;
                break;
            }
            const ObjRec& obj = s.objects[h.object];
            if(obj.emitter >= 0 && h.front_face) {  // path_integrator.h:47-59
                const f3 Le = area_emitted(s.emitters[obj.emitter], h.normal, -normalize(ray.d));
                if(!is_zero(Le)) {
                    if(!have_pdf) {
                        c += throughput * Le;
                    } else {
                        const float light_pdf = pdf_emitter_direction(s, ray.o, ray.d);
                        c += throughput * power_heuristic(sa_pdf, light_pdf) * Le;
                    }
                }
            }
            int32_t mid = obj.material;
            if(h.object == job.override_obj) mid = job.override_mat;
            if(mid < 0) {
                vc[depth] = c;
                break;
            }
            const int32_t ab = a.d.aff_begin[mid];
            const int32_t an = a.d.aff_begin[mid + 1] - ab;
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
                                if(!scene_occluded<false>(s, Ray{shadow_origin, shadow_dir}, 0.001f, tmax,
                                                          light.emitter, cnt)) {
                                    c += throughput * f_cos * light.radiance * (w / light_pdf);
                                    const f3 scale = delta * (throughput * light.radiance * (w / light_pdf));
                                    for(int32_t k = 0; k < an; ++k) {
                                        const int32_t grp = a.d.aff_list[ab + k];
                                        add_group<false>(a.d, g, grp, scale * group_d_eval(a.d, mid, bctx, rec, grp));
                                    }
                                }
                            }
                        }
                    }
                }
            }
            vc[depth] = c;
            if(depth == a.max_depth - 1) break;
            const f3 weight = bsdf_sample(s.materials, s.tables, mid, bctx, rec, bsdf_uv.x, bsdf_uv.y);
            if(is_zero(weight)) break;
            if(an > 0) {
                const int meas = measure_of(rec.sampled_type);
                const BsdfCtx ectx = sampled_value_ctx(bctx, rec);
                const f3 e0 = bsdf_eval(s.materials, s.tables, mid, ectx, rec, meas);
                for(int32_t k = 0; k < an; ++k) {
                    const f3 de = group_d_eval(a.d, mid, ectx, rec, a.d.aff_list[ab + k], meas);
                    vd[depth][k] = f3{safe_ratio(de.x, e0.x), safe_ratio(de.y, e0.y), safe_ratio(de.z, e0.z)};
                }
                vn[depth] = an;
                vmid[depth] = mid;
            }
            const f3 new_dir = to_world(basis, rec.wo);
            throughput *= weight;
            eta *= rec.eta;
            if(depth >= a.rr_depth) {
                const float q = smin(max3(throughput) * eta * eta, 0.95f);
                if(rr_u >= q) break;
                throughput /= q;
            }
            have_pdf = measure_of(rec.sampled_type) == kSolidAngle && rec.pdf > 0.0f;
            sa_pdf = rec.pdf;
            ray = Ray{h.p, new_dir};
        }
        // suffix sums: the sampled direction of depth d carries everything added after d
        f3 suffix = mk(0.0f);
        for(int d = n_vertices - 1; d >= 0; --d) {
            if(vn[d] > 0) {
                const f3 ds = delta * suffix;
                const int32_t ab = a.d.aff_begin[vmid[d]];
                for(int32_t k = 0; k < vn[d]; ++k) add_group<false>(a.d, g, a.d.aff_list[ab + k], ds * vd[d][k]);
            }
            suffix += vc[d];
        }
    }
    for(uint32_t j = 0; j < a.d.n_params; ++j) {
        float x = g[j];
        for(int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if(lane_id() == 0 && x != 0.0f) atomicAdd(a.grad + j, static_cast<double>(x));
    }
}

template <typename T>
cudaError_t put(DevBuf& buf, const std::vector<T>& v, cudaStream_t s) {
    const size_t n = std::max<size_t>(1, v.size()) * sizeof(T);
    cudaError_t e = buf.ensure(n);
    if(e != cudaSuccess || v.empty()) return e;
    return cudaMemcpyAsync(buf.ptr, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s);
}

bool same_structure(const MatRec& a, const MatRec& b) {
    return a.type == b.type && a.nested == b.nested && a.flags == b.flags && a.component_count == b.component_count &&
           (a.table >= 0) == (b.table >= 0);
}

// record r (tables r_tables) differs from the scene's record base (tables compared by content)
bool record_differs(const MatRec& r, const float* r_tables, const MatRec& base, const float* base_tables) {
    MatRec x = r, y = base;
    x.table = y.table = 0;
    if(memcmp(&x, &y, sizeof(MatRec)) != 0) return true;
    if(r.table >= 0) {
        return memcmp(r_tables + static_cast<size_t>(r.table) * LRT_TRANS_SAMPLES,
                      base_tables + static_cast<size_t>(base.table) * LRT_TRANS_SAMPLES,
                      sizeof(float) * LRT_TRANS_SAMPLES) != 0;
    }
    return false;
}

}  // namespace

extern "C" {

int lrt_scene_update_materials(lrt_context* ctx, const lrt_material_desc* materials, uint32_t n_materials) {
    if(!ctx) return LRT_ERR_INVALID_ARGUMENT;
    if(!ctx->has_scene) return fail(ctx, LRT_ERR_NO_SCENE, "no scene uploaded");
    if(n_materials != ctx->host.materials.size()) {
        return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "material count %u differs from the scene's %zu", n_materials,
                    ctx->host.materials.size());
    }
    LRT_CUDA(ctx, cudaSetDevice(ctx->device));
    std::vector<MatRec> recs;
    std::vector<float> tables;
    std::string err;
    const int st = pack_materials(materials, n_materials, recs, tables, err);
    if(st != LRT_OK) return fail(ctx, st, "%s", err.c_str());
    for(uint32_t i = 0; i < n_materials; ++i) {
        if(!same_structure(recs[i], ctx->host.materials[i])) {
            return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "material %u: type, nesting or BSDF flags changed", i);
        }
    }
    if(tables.empty()) tables.assign(LRT_TRANS_SAMPLES, 0.0f);
    ctx->diff_params = 0;
    LRT_CUDA(ctx, put(ctx->materials, recs, ctx->stream));
    LRT_CUDA(ctx, put(ctx->tables, tables, ctx->stream));
    LRT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    ctx->host.materials.swap(recs);
    ctx->host.tables.swap(tables);
    ctx->ds.materials = ctx->materials.as<MatRec>();
    ctx->ds.tables = ctx->tables.as<float>();
    return LRT_OK;
}

int lrt_diff_setup(lrt_context* ctx, uint32_t n_groups, const float* steps, const lrt_material_desc* plus,
                   const lrt_material_desc* minus, uint32_t n_params, const lrt_diff_param* params) {
    if(!ctx) return LRT_ERR_INVALID_ARGUMENT;
    if(!ctx->has_scene) return fail(ctx, LRT_ERR_NO_SCENE, "no scene uploaded");
    ctx->diff_params = 0;
    ctx->diff_groups = 0;
    if(n_params == 0 || n_params > kMaxParams) {
        return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "n_params must be in [1, %d]", kMaxParams);
    }
    if(n_groups == 0 || n_groups > n_params) return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "n_groups must be in [1, n_params]");
    if(!steps || !plus || !minus || !params) return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "null argument");
    LRT_CUDA(ctx, cudaSetDevice(ctx->device));
    // parameters per group: channels 0..2 at most once each, or one scalar (-1) alone
    std::vector<std::vector<int32_t>> members(n_groups);
    for(uint32_t j = 0; j < n_params; ++j) {
        const lrt_diff_param& p = params[j];
        if(p.group >= n_groups || p.channel < -1 || p.channel > 2) {
            return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "parameter %u: group or channel out of range", j);
        }
        for(int32_t e : members[p.group]) {
            const int ch = (e & 3) - 1;
            if(ch < 0 || p.channel < 0 || ch == p.channel) {
                return fail(ctx, LRT_ERR_INVALID_ARGUMENT,
                            "parameter %u: a group holds one scalar parameter or distinct channels", j);
            }
        }
        members[p.group].push_back(static_cast<int32_t>(j << 2) | (p.channel + 1));
    }
    std::vector<int32_t> group_begin(n_groups + 1, 0), group_params;
    for(uint32_t gi = 0; gi < n_groups; ++gi) {
        if(members[gi].empty()) return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "group %u has no parameter", gi);
        group_begin[gi] = static_cast<int32_t>(group_params.size());
        group_params.insert(group_params.end(), members[gi].begin(), members[gi].end());
    }
    group_begin[n_groups] = static_cast<int32_t>(group_params.size());

    const std::vector<MatRec>& base = ctx->host.materials;
    const std::vector<float>& base_tables = ctx->host.tables;
    const uint32_t nm = static_cast<uint32_t>(base.size());
    std::vector<MatRec> all;
    std::vector<float> tables;
    std::vector<float> inv2step(n_groups);
    std::vector<std::vector<uint8_t>> affected(nm, std::vector<uint8_t>(n_groups, 0));
    all.reserve(2ull * n_groups * nm);
    for(uint32_t j = 0; j < n_groups; ++j) {
        if(!(steps[j] > 0.0f) || !std::isfinite(steps[j])) {
            return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "group %u: step must be positive", j);
        }
        inv2step[j] = 1.0f / (2.0f * steps[j]);
        for(int sign = 0; sign < 2; ++sign) {
            const lrt_material_desc* list = (sign == 0 ? plus : minus) + static_cast<size_t>(j) * nm;
            std::vector<MatRec> recs;
            std::vector<float> tabs;
            std::string err;
            const int st = pack_materials(list, nm, recs, tabs, err);
            if(st != LRT_OK) return fail(ctx, st, "group %u: %s", j, err.c_str());
            const int32_t offset = static_cast<int32_t>(tables.size() / LRT_TRANS_SAMPLES);
            for(uint32_t i = 0; i < nm; ++i) {
                if(!same_structure(recs[i], base[i])) {
                    return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "group %u: material %u changes type, nesting or flags", j, i);
                }
                if(record_differs(recs[i], tabs.data(), base[i], base_tables.data())) affected[i][j] = 1;
                if(recs[i].table >= 0) recs[i].table += offset;
            }
            tables.insert(tables.end(), tabs.begin(), tabs.end());
            all.insert(all.end(), recs.begin(), recs.end());
        }
    }
    // a coating moves with the groups of its nested material (nested index < coating index)
    for(uint32_t i = 0; i < nm; ++i) {
        if(base[i].nested >= 0) {
            for(uint32_t j = 0; j < n_groups; ++j) affected[i][j] |= affected[base[i].nested][j];
        }
    }
    std::vector<int32_t> aff_begin(nm + 1, 0), aff_list;
    for(uint32_t i = 0; i < nm; ++i) {
        aff_begin[i] = static_cast<int32_t>(aff_list.size());
        for(uint32_t j = 0; j < n_groups; ++j) {
            if(affected[i][j]) aff_list.push_back(static_cast<int32_t>(j));
        }
        if(aff_list.size() - aff_begin[i] > static_cast<size_t>(kMaxAff)) {
            return fail(ctx, LRT_ERR_RANGE, "material %u depends on more than %d groups", i, kMaxAff);
        }
    }
    aff_begin[nm] = static_cast<int32_t>(aff_list.size());
    uint32_t kmax = 0;
    for(uint32_t i = 0; i < nm; ++i) kmax = std::max<uint32_t>(kmax, aff_begin[i + 1] - aff_begin[i]);
    if(tables.empty()) tables.assign(LRT_TRANS_SAMPLES, 0.0f);
    LRT_CUDA(ctx, put(ctx->diff_mats, all, ctx->stream));
    LRT_CUDA(ctx, put(ctx->diff_tables, tables, ctx->stream));
    LRT_CUDA(ctx, put(ctx->diff_inv2step, inv2step, ctx->stream));
    LRT_CUDA(ctx, put(ctx->diff_aff_begin, aff_begin, ctx->stream));
    LRT_CUDA(ctx, put(ctx->diff_aff_list, aff_list, ctx->stream));
    LRT_CUDA(ctx, put(ctx->diff_group_begin, group_begin, ctx->stream));
    LRT_CUDA(ctx, put(ctx->diff_group_params, group_params, ctx->stream));
    LRT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    ctx->diff_params = n_params;
    ctx->diff_groups = n_groups;
    ctx->diff_kmax = kmax;
    return LRT_OK;
}

int lrt_render_adjoint_dev(lrt_context* ctx, const lrt_job_desc* jobs, uint32_t n_jobs, int32_t max_depth,
                           int32_t rr_depth, const float* adjoint_dev, double* grad_dev) {
    if(!ctx) return LRT_ERR_INVALID_ARGUMENT;
    if(!ctx->has_scene) return fail(ctx, LRT_ERR_NO_SCENE, "no scene uploaded");
    if(ctx->diff_params == 0) return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "no lrt_diff_setup for the current materials");
    if(n_jobs == 0) return LRT_OK;
    if(!jobs || !adjoint_dev || !grad_dev) return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "null argument");
    if(max_depth < 1 || max_depth > kMaxAdjDepth) {
        return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "max_depth must be in [1, %d] for the adjoint", kMaxAdjDepth);
    }
    LRT_CUDA(ctx, cudaSetDevice(ctx->device));
    std::vector<JobRec> recs;
    unsigned long long total = 0, out_floats = 0;
    const int st = job_records(ctx, jobs, n_jobs, recs, total, out_floats);
    if(st != LRT_OK) return st;
    if(!ctx->adjoint_megakernel) return adjoint_wavefront(ctx, recs, total, max_depth, rr_depth, adjoint_dev, grad_dev);
    LRT_CUDA(ctx, ctx->batch_jobs.ensure(sizeof(JobRec) * n_jobs));
    LRT_CUDA(ctx, cudaMemcpyAsync(ctx->batch_jobs.ptr, recs.data(), sizeof(JobRec) * n_jobs, cudaMemcpyHostToDevice,
                                  ctx->stream));
    AdjArgs a{};
    a.s = ctx->ds;
    a.jobs = ctx->batch_jobs.as<JobRec>();
    a.n_jobs = n_jobs;
    a.total_paths = total;
    a.adjoint = adjoint_dev;
    a.d = diff_dev(ctx);
    a.max_depth = max_depth;
    a.rr_depth = rr_depth;
    a.grad = grad_dev;
    k_adjoint<<<grid_for(ctx, (const void*)k_adjoint, kBlock), kBlock, 0, ctx->stream>>>(a);
    LRT_CUDA(ctx, cudaGetLastError());
    ctx->stats.paths += total;
    ctx->stats.kernel_launches += 1;
    return LRT_OK;
}

int lrt_render_adjoint(lrt_context* ctx, const lrt_job_desc* jobs, uint32_t n_jobs, int32_t max_depth,
                       int32_t rr_depth, const float* adjoint, double* grad) {
    if(!ctx) return LRT_ERR_INVALID_ARGUMENT;
    if(n_jobs == 0) return LRT_OK;
    if(!jobs || !adjoint || !grad) return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "null argument");
    if(ctx->diff_params == 0) return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "no lrt_diff_setup for the current materials");
    LRT_CUDA(ctx, cudaSetDevice(ctx->device));
    unsigned long long floats = 0;
    for(uint32_t i = 0; i < n_jobs; ++i) {
        floats = std::max<unsigned long long>(floats, jobs[i].output_offset + 3ull * jobs[i].width * jobs[i].height);
    }
    const uint32_t np = ctx->diff_params;
    LRT_CUDA(ctx, ctx->diff_adjoint.ensure(4ull * floats));
    LRT_CUDA(ctx, ctx->diff_grad.ensure(8ull * np));
    LRT_CUDA(ctx, cudaMemcpyAsync(ctx->diff_adjoint.ptr, adjoint, 4ull * floats, cudaMemcpyHostToDevice, ctx->stream));
    LRT_CUDA(ctx, cudaMemsetAsync(ctx->diff_grad.ptr, 0, 8ull * np, ctx->stream));
    const int st = lrt_render_adjoint_dev(ctx, jobs, n_jobs, max_depth, rr_depth, ctx->diff_adjoint.as<float>(),
                                          ctx->diff_grad.as<double>());
    if(st != LRT_OK) return st;
    std::vector<double> g(np);
    LRT_CUDA(ctx, cudaMemcpyAsync(g.data(), ctx->diff_grad.ptr, 8ull * np, cudaMemcpyDeviceToHost, ctx->stream));
    LRT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    for(uint32_t j = 0; j < np; ++j) grad[j] += g[j];
    return LRT_OK;
}

}  // extern "C"
