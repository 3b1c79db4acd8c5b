// lrt_adjoint.cuh — device pieces of the path-replay adjoint shared by its megakernel and its
// wavefront form: the parameter groups' perturbed material records and the accumulation of a
// group's derivative into its parameters.
#pragma once

#include "lrt_bsdf.cuh"
#include "lrt_context.cuh"

namespace lrt {

struct DiffDev {
    const MatRec* pert;           // 2 * n_groups lists of n_materials records: [2g] +step, [2g+1] -step
    const float* pert_tables;
    const float* inv2step;        // per group: 1 / (2 step_g)
    const int32_t* aff_begin;     // per material: the groups that move it are aff_list[aff_begin[m] .. aff_begin[m+1])
    const int32_t* aff_list;
    const int32_t* group_begin;   // per group: its parameters are group_params[group_begin[g] .. group_begin[g+1])
    const int32_t* group_params;  // (parameter << 2) | (channel + 1)
    uint32_t n_params;
    int32_t n_materials;
};

inline DiffDev diff_dev(const lrt_context* ctx) {
    DiffDev d{};
    d.pert = ctx->diff_mats.as<MatRec>();
    d.pert_tables = ctx->diff_tables.as<float>();
    d.inv2step = ctx->diff_inv2step.as<float>();
    d.aff_begin = ctx->diff_aff_begin.as<int32_t>();
    d.aff_list = ctx->diff_aff_list.as<int32_t>();
    d.group_begin = ctx->diff_group_begin.as<int32_t>();
    d.group_params = ctx->diff_group_params.as<int32_t>();
    d.n_params = ctx->diff_params;
    d.n_materials = ctx->ds.n_materials;
    return d;
}

// The adjoint on the wavefront pipeline (lrt_api.cu): the batch's paths in waves through the
// persistent traversal kernels, with per-depth derivative records and a suffix pass per wave.
int adjoint_wavefront(lrt_context* ctx, const std::vector<JobRec>& recs, unsigned long long total, int32_t max_depth,
                      int32_t rr_depth, const float* adjoint_dev, double* grad_dev);

#ifdef __CUDACC__
// d(f cos)/d(group) at rec in measure `meas`: the central difference of the group's packed records (kept
// out of line, one copy of the BSDF dispatch for every call site)
static __device__ __noinline__ f3 d_eval(const MatRec* plus, const MatRec* minus, const float* tables, float inv2step,
                                  int32_t mid, const BsdfCtx& c, const BRec& rec, int meas) {
    const f3 ep = bsdf_eval(plus, tables, mid, c, rec, meas);
    const f3 em = bsdf_eval(minus, tables, mid, c, rec, meas);
    return (ep - em) * inv2step;
}

__device__ __forceinline__ f3 group_d_eval(const DiffDev& d, int32_t mid, const BsdfCtx& c, const BRec& rec, int32_t grp,
                                           int meas = kSolidAngle) {
    const MatRec* plus = d.pert + static_cast<size_t>(2 * grp) * d.n_materials;
    return d_eval(plus, plus + d.n_materials, d.pert_tables, d.inv2step[grp], mid, c, rec, meas);
}

// The BSDF value a sampled direction's path weight carries (weight = value / sampling probability): in
// solid angle, the whole BSDF at wo; for a delta lobe, the discrete value of the sampled component alone
// (the evaluation context restricted to it), since several delta components can share a direction (a
// coating's mirror reflection and its nested material's refracted mirror reflection).
__device__ __forceinline__ BsdfCtx sampled_value_ctx(const BsdfCtx& c, const BRec& rec) {
    BsdfCtx e = c;
    if(measure_of(rec.sampled_type) == kDiscrete) e.component = rec.sampled_component;
    return e;
}

__device__ __forceinline__ float rgb_channel(f3 v, int c) { return c == 0 ? v.x : (c == 1 ? v.y : v.z); }

// adds a group's per-channel products to its parameters: a channel parameter takes its channel, a
// scalar parameter the sum of the three (kShared: atomically into shared memory)
template <bool kShared>
__device__ __forceinline__ void add_group(const DiffDev& d, float* acc, int32_t grp, f3 prod) {
    for(int32_t i = d.group_begin[grp]; i < d.group_begin[grp + 1]; ++i) {
        const int32_t e = d.group_params[i];
        const int ch = (e & 3) - 1;
        const float v = ch < 0 ? (prod.x + prod.y) + prod.z : rgb_channel(prod, ch);
        if(kShared) {
            atomicAdd(acc + (e >> 2), v);
        } else {
            acc[e >> 2] += v;
        }
    }
}

__device__ __forceinline__ float safe_ratio(float num, float den) { return den != 0.0f ? num / den : 0.0f; }
#endif

}  // namespace lrt
