// lrt_bsdf.cuh — the eight LinRT BSDFs as device functions over MatRec records.
//
// Each function restates its reference counterpart operation by operation (file:line in the
// comments); nothing is dispatched virtually: a switch on MatRec::type selects the BSDF, and the two
// coatings call the base switch for their nested BSDF (one level of nesting).
#pragma once

#include "lrt_math.cuh"
#include "lrt_types.h"
#include "../../include/lrt.h"

namespace lrt {

constexpr uint32_t kDiffuse = LRT_BSDF_DIFFUSE, kSpecular = LRT_BSDF_SPECULAR, kReflective = LRT_BSDF_REFLECTIVE;
constexpr uint32_t kGlossy = LRT_BSDF_GLOSSY, kMetallic = LRT_BSDF_METALLIC, kDielectric = LRT_BSDF_DIELECTRIC;
constexpr uint32_t kRefractive = LRT_BSDF_REFRACTIVE;
constexpr int kSolidAngle = LRT_MEASURE_SOLID_ANGLE;
constexpr int kDiscrete = LRT_MEASURE_DISCRETE;
constexpr float kDeltaEpsilon = 1e-3f;  // src/core/core.h:14

struct BsdfCtx {
    int32_t mode;          // LRT_MODE_*
    uint32_t type_mask;
    int32_t component;
    float lobe_sample;
};

LRT_HD BsdfCtx ctx_default(int mode) { return BsdfCtx{mode, 0xffffffffu, -1, 0.0f}; }

struct BRec {
    f3 wi;
    f3 wo;
    float eta;
    float pdf;
    uint32_t sampled_type;
    int32_t sampled_component;
    bool front_face;
};

LRT_HD int measure_of(uint32_t sampled_type) { return (sampled_type & kSpecular) != 0 ? kDiscrete : kSolidAngle; }

// ---- helpers: src/material/func/frame.h ----
LRT_HD bool delta_aligned(f3 sampled, f3 wo) { return fabsf(dot(sampled, wo) - 1.0f) < kDeltaEpsilon; }
LRT_HD f3 reflect(f3 w, f3 n) { return 2.0f * dot(w, n) * n - w; }
LRT_HD f3 refract(f3 wi, f3 n, float cos_theta_t, float eta_i, float eta_t) {
    const float scale = eta_i / eta_t;
    return n * (scale * dot(wi, n) - cos_theta_t) - wi * scale;
}

// ---- GGX: src/material/func/microfacet.h:16-77 (alpha already clamped to >= 1e-4) ----
LRT_HD float ggx_D(float alpha, f3 m) {
    if(m.z <= 0.0f) return 0.0f;
    const float alpha2 = alpha * alpha;
    const float temp = (m.x * m.x + m.y * m.y) / alpha2 + m.z * m.z;
    return 1.0f / (kPi * alpha2 * temp * temp);
}
LRT_HD float ggx_G1(float alpha, f3 v, f3 m) {
    const float cos_v = fabsf(v.z);
    if(cos_v < 1e-6f || dot(v, m) * v.z <= 0.0f) return 0.0f;
    const float tan_theta_alpha_2 = (alpha * alpha) * (v.x * v.x + v.y * v.y) / (v.z * v.z);
    const float lambda = 0.5f * (-1.0f + sqrtf(1.0f + tan_theta_alpha_2));
    return 1.0f / (1.0f + lambda);
}
LRT_HD float ggx_G(float alpha, f3 wi, f3 wo, f3 m) { return ggx_G1(alpha, wi, m) * ggx_G1(alpha, wo, m); }
LRT_HD float ggx_pdf(float alpha, f3 wi, f3 m) {
    if(wi.z <= 1e-6f) return 0.0f;
    return ggx_G1(alpha, wi, m) * smax(0.0f, dot(wi, m)) * ggx_D(alpha, m) / wi.z;
}
LRT_HD f3 ggx_sample(float alpha, f3 wi, float ux, float uy) {
    const f3 vh = normalize(f3{alpha * wi.x, alpha * wi.y, wi.z});
    const float lensq = vh.x * vh.x + vh.y * vh.y;
    const f3 t1 = lensq > 0.0f ? f3{-vh.y, vh.x, 0.0f} / sqrtf(lensq) : f3{1.0f, 0.0f, 0.0f};
    const f3 t2 = cross(vh, t1);
    const float r = sqrtf(ux);
    const float phi = 2.0f * kPi * uy;
    float sin_phi, cos_phi;
    sincos_rn(phi, sin_phi, cos_phi);
    const float disk_x = r * cos_phi;
    float disk_y = r * sin_phi;
    const float stretch = 0.5f * (1.0f + vh.z);
    disk_y = (1.0f - stretch) * sqrtf(smax(0.0f, 1.0f - disk_x * disk_x)) + stretch * disk_y;
    const f3 nh = disk_x * t1 + disk_y * t2 + sqrtf(smax(0.0f, 1.0f - disk_x * disk_x - disk_y * disk_y)) * vh;
    return normalize(f3{alpha * nh.x, alpha * nh.y, smax(0.0f, nh.z)});
}

// ---- Fresnel: src/material/func/fresnel.h ----

// Conductor Fresnel with the complex index eta + i k (fresnel.h:43-56). Products and sums are the
// float operations std::complex<float> performs; complex division and square root are evaluated in
// double and rounded once (the reference's library routines are at least that accurate).
struct c32 {
    float re, im;
};
LRT_HD c32 cmul(c32 a, c32 b) { return c32{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
LRT_HD c32 cdiv(c32 a, c32 b) {
    const double ar = a.re, ai = a.im, br = b.re, bi = b.im;
    const double den = br * br + bi * bi;
    return c32{static_cast<float>((ar * br + ai * bi) / den), static_cast<float>((ai * br - ar * bi) / den)};
}
LRT_HD c32 csqrt_(c32 z) {
    const double x = z.re, y = z.im;
    if(x == 0.0 && y == 0.0) return c32{0.0f, z.im};
    const double r = hypot(x, y);
    if(x >= 0.0) {
        const double t = sqrt(0.5 * (r + x));
        return c32{static_cast<float>(t), static_cast<float>(y / (2.0 * t))};
    }
    const double t = sqrt(0.5 * (r - x));
    return c32{static_cast<float>(fabs(y) / (2.0 * t)), static_cast<float>(copysign(t, y))};
}
LRT_HD float cnorm(c32 z) { return z.re * z.re + z.im * z.im; }

LRT_HD float fresnel_conductor1(float cos_theta_i, float eta, float k) {
    cos_theta_i = sclamp(cos_theta_i, 0.0f, 1.0f);
    const c32 ior{eta, k};
    const float sin2_theta_i = 1.0f - cos_theta_i * cos_theta_i;
    const c32 sin2_theta_t = cdiv(c32{sin2_theta_i, 0.0f}, cmul(ior, ior));
    const c32 cos_theta_t = csqrt_(c32{1.0f - sin2_theta_t.re, 0.0f - sin2_theta_t.im});
    const c32 ior_c{ior.re * cos_theta_i, ior.im * cos_theta_i};
    const c32 r_parallel = cdiv(c32{ior_c.re - cos_theta_t.re, ior_c.im - cos_theta_t.im},
                                c32{ior_c.re + cos_theta_t.re, ior_c.im + cos_theta_t.im});
    const c32 ior_t = cmul(ior, cos_theta_t);
    const c32 r_perpendicular = cdiv(c32{cos_theta_i - ior_t.re, -ior_t.im}, c32{cos_theta_i + ior_t.re, ior_t.im});
    return 0.5f * (cnorm(r_parallel) + cnorm(r_perpendicular));
}
LRT_HD f3 fresnel_conductor(float cos_theta_i, const float* eta, const float* k) {
    return f3{fresnel_conductor1(cos_theta_i, eta[0], k[0]), fresnel_conductor1(cos_theta_i, eta[1], k[1]),
              fresnel_conductor1(cos_theta_i, eta[2], k[2])};
}

struct DielFresnel {
    float reflectance;
    float cos_theta_t;
};
// fresnel.h:72-95
LRT_HD DielFresnel fresnel_dielectric(float cos_theta_i, float eta_i, float eta_t) {
    DielFresnel r{1.0f, 0.0f};
    if(eta_i <= 0.0f || eta_t <= 0.0f) return r;
    cos_theta_i = sclamp(cos_theta_i, 0.0f, 1.0f);
    const float sin2_i = 1.0f - cos_theta_i * cos_theta_i;
    const float scale = eta_i / eta_t;
    const float sin2_t = scale * scale * sin2_i;
    if(sin2_t > 1.0f) return r;
    r.cos_theta_t = sqrtf(1.0f - sin2_t);
    const float r_perp = (eta_i * cos_theta_i - eta_t * r.cos_theta_t) / (eta_i * cos_theta_i + eta_t * r.cos_theta_t);
    const float r_parl = (eta_t * cos_theta_i - eta_i * r.cos_theta_t) / (eta_t * cos_theta_i + eta_i * r.cos_theta_t);
    r.reflectance = 0.5f * (r_perp * r_perp + r_parl * r_parl);
    return r;
}
// fresnelDielectricExt, fresnel.h:99-119
LRT_HD float fresnel_dielectric_ext(float cos_theta_i, float& cos_theta_t, float eta) {
    if(eta == 1.0f) {
        cos_theta_t = -cos_theta_i;
        return 0.0f;
    }
    const float scale = cos_theta_i > 0.0f ? (1.0f / eta) : eta;
    const float cos_theta_t_sqr = 1.0f - (1.0f - cos_theta_i * cos_theta_i) * (scale * scale);
    if(cos_theta_t_sqr <= 0.0f) {
        cos_theta_t = 0.0f;
        return 1.0f;
    }
    const float cos_i = fabsf(cos_theta_i);
    const float cos_t = sqrtf(cos_theta_t_sqr);
    const float rs = (cos_i - eta * cos_t) / (cos_i + eta * cos_t);
    const float rp = (eta * cos_i - cos_t) / (eta * cos_i + cos_t);
    cos_theta_t = cos_theta_i > 0.0f ? -cos_t : cos_t;
    return 0.5f * (rs * rs + rp * rp);
}
LRT_HD float fresnel_dielectric_ext(float cos_theta_i, float eta) {
    float c = 0.0f;
    return fresnel_dielectric_ext(cos_theta_i, c, eta);
}

// ---- rough transmittance 1-D lookup: rough_transmittance.h:26-34 + catmull_rom.h:10-34 ----
LRT_HD float cubic_interp_1d(float x, const float* values, uint32_t size) {
    if(!(x >= 0.0f && x <= 1.0f)) return 0.0f;
    float t = ((x - 0.0f) * static_cast<float>(size - 1)) / (1.0f - 0.0f);
    uint32_t k = static_cast<uint32_t>(t);
    if(k > size - 2) k = size - 2;
    const float f0 = values[k];
    const float f1 = values[k + 1];
    const float d0 = k > 0 ? 0.5f * (values[k + 1] - values[k - 1]) : (values[k + 1] - values[k]);
    const float d1 = (k + 2 < size) ? 0.5f * (values[k + 2] - values[k]) : (values[k + 1] - values[k]);
    t -= static_cast<float>(k);
    const float t2 = t * t;
    const float t3 = t2 * t;
    return (2.0f * t3 - 3.0f * t2 + 1.0f) * f0 + (-2.0f * t3 + 3.0f * t2) * f1 + (t3 - 2.0f * t2 + t) * d0 +
           (t3 - t2) * d1;
}
LRT_HD float trans_eval(const float* table, float cos_theta) {
    if(!(cos_theta >= 0.0f)) return 0.0f;
    const float warped = quartic_root_rn(cos_theta);
    return sclamp(cubic_interp_1d(warped, table, LRT_TRANS_SAMPLES), 0.0f, 1.0f);
}

LRT_HD f3 cosine_hemisphere(float ux, float uy, float& pdf) {
    const float cos_theta = sqrtf(ux);
    const float sin_theta = sqrtf(1.0f - ux);
    const float phi = 2.0f * kPi * uy;
    pdf = cos_theta / kPi;
    float sin_phi, cos_phi;
    sincos_rn(phi, sin_phi, cos_phi);
    return f3{cos_phi * sin_theta, sin_phi * sin_theta, cos_theta};
}

LRT_HD void rec_reset(BRec& r) {
    r.pdf = 0.0f;
    r.eta = 1.0f;
    r.sampled_type = 0u;
    r.sampled_component = -1;
}

// ================= diffuse_bsdf.h:18-72 =================
LRT_HD f3 diffuse_sample(const MatRec& m, const BsdfCtx& c, BRec& r, float ux, float uy) {
    constexpr uint32_t lobe = kDiffuse | kReflective;
    rec_reset(r);
    if(!(c.type_mask & lobe)) return mk(0.0f);
    if(c.component != -1 && c.component != 0) return mk(0.0f);
    if(r.wi.z <= 0.0f) return mk(0.0f);
    const float cos_theta = sqrtf(ux);
    const float sin_theta = sqrtf(1.0f - ux);
    const float phi = 2.0f * kPi * uy;
    float sin_phi, cos_phi;
    sincos_rn(phi, sin_phi, cos_phi);
    r.wo = f3{cos_phi * sin_theta, sin_phi * sin_theta, cos_theta};
    r.pdf = cos_theta / kPi;
    r.sampled_type = lobe;
    r.sampled_component = 0;
    return load3(m.diffuse);
}
LRT_HD bool diffuse_ok(const BsdfCtx& c, const BRec& r, int meas) {
    constexpr uint32_t lobe = kDiffuse | kReflective;
    if(meas != kSolidAngle) return false;
    if(!(c.type_mask & lobe)) return false;
    if(c.component != -1 && c.component != 0) return false;
    if(r.wi.z <= 0.0f || r.wo.z <= 0.0f) return false;
    return true;
}
LRT_HD f3 diffuse_eval(const MatRec& m, const BsdfCtx& c, const BRec& r, int meas) {
    if(!diffuse_ok(c, r, meas)) return mk(0.0f);
    return load3(m.diffuse) * (r.wo.z / kPi);
}
LRT_HD float diffuse_pdf(const MatRec&, const BsdfCtx& c, const BRec& r, int meas) {
    if(!diffuse_ok(c, r, meas)) return 0.0f;
    return r.wo.z / kPi;
}

// ================= rough_conductor_bsdf.h:28-128 =================
struct ValPdf {
    f3 value;
    float pdf;
};
LRT_HD ValPdf conductor_eval_and_pdf(const MatRec& m, f3 wi, f3 wo) {
    if(wi.z <= 1e-6f || wo.z <= 1e-6f) return ValPdf{mk(0.0f), 0.0f};
    const f3 half = wi + wo;
    if(length_squared(half) <= 1e-12f) return ValPdf{mk(0.0f), 0.0f};
    const f3 mh = normalize(half);
    const float wi_dot_m = dot(wi, mh);
    if(mh.z <= 0.0f || wi_dot_m <= 0.0f) return ValPdf{mk(0.0f), 0.0f};
    const float d = ggx_D(m.dist_alpha, mh);
    const float g = ggx_G(m.dist_alpha, wi, wo, mh);
    const f3 fresnel = fresnel_conductor(wi_dot_m, m.cond_eta, m.cond_k) * load3(m.spec_refl);
    const f3 value = fresnel * (d * g / (4.0f * wi.z));
    const float pdf_m = ggx_pdf(m.dist_alpha, wi, mh);
    return ValPdf{value, pdf_m / (4.0f * wi_dot_m)};
}
LRT_HD bool conductor_allowed(const MatRec& m, const BsdfCtx& c) {
    if((c.type_mask & m.flags) == 0) return false;
    if(c.component != -1 && c.component != 0) return false;
    return true;
}
LRT_HD f3 conductor_sample(const MatRec& m, const BsdfCtx& c, BRec& r, float ux, float uy) {
    rec_reset(r);
    if(!conductor_allowed(m, c)) return mk(0.0f);
    if(r.wi.z < 0.0f) return mk(0.0f);
    if(m.alpha <= 0.0f) {
        r.wo = f3{-r.wi.x, -r.wi.y, r.wi.z};
        r.sampled_type = m.flags;
        r.sampled_component = 0;
        r.pdf = 1.0f;
        return fresnel_conductor(r.wi.z, m.cond_eta, m.cond_k) * load3(m.spec_refl);
    }
    const f3 mh = ggx_sample(m.dist_alpha, r.wi, ux, uy);
    const float wi_dot_m = dot(r.wi, mh);
    if(mh.z <= 0.0f || wi_dot_m <= 0.0f) return mk(0.0f);
    r.wo = reflect(r.wi, mh);
    if(r.wo.z <= 0.0f) return mk(0.0f);
    const ValPdf lv = conductor_eval_and_pdf(m, r.wi, r.wo);
    if(lv.pdf <= 0.0f) return mk(0.0f);
    r.pdf = lv.pdf;
    r.sampled_type = m.flags;
    r.sampled_component = 0;
    return lv.value / lv.pdf;
}
LRT_HD f3 conductor_eval(const MatRec& m, const BsdfCtx& c, const BRec& r, int meas) {
    if(!conductor_allowed(m, c)) return mk(0.0f);
    if(m.alpha <= 0.0f) {
        if(meas != kDiscrete || r.wo.z <= 0.0f || !delta_aligned(f3{-r.wi.x, -r.wi.y, r.wi.z}, r.wo)) return mk(0.0f);
        return fresnel_conductor(r.wi.z, m.cond_eta, m.cond_k) * load3(m.spec_refl);
    }
    if(meas != kSolidAngle) return mk(0.0f);
    return conductor_eval_and_pdf(m, r.wi, r.wo).value;
}
LRT_HD float conductor_pdf(const MatRec& m, const BsdfCtx& c, const BRec& r, int meas) {
    if(!conductor_allowed(m, c)) return 0.0f;
    if(m.alpha <= 0.0f) {
        if(meas != kDiscrete || r.wo.z <= 0.0f || !delta_aligned(f3{-r.wi.x, -r.wi.y, r.wi.z}, r.wo)) return 0.0f;
        return 1.0f;
    }
    if(meas != kSolidAngle) return 0.0f;
    return conductor_eval_and_pdf(m, r.wi, r.wo).pdf;
}

// ================= dielectric_bsdf.h:31-157 =================
constexpr uint32_t kDielRefl = kSpecular | kReflective | kDielectric;
constexpr uint32_t kDielTrans = kSpecular | kRefractive | kDielectric;
LRT_HD f3 dielectric_sample(const MatRec& m, const BsdfCtx& c, BRec& r, float ux, float) {
    rec_reset(r);
    if(r.wi.z <= 0.0f) return mk(0.0f);
    const bool allow_r = (c.type_mask & kDielRefl) != 0 && (c.component == -1 || c.component == 0);
    const bool allow_t = (c.type_mask & kDielTrans) != 0 && (c.component == -1 || c.component == 1);
    if(!allow_r && !allow_t) return mk(0.0f);
    const float eta_i = r.front_face ? m.ext_ior : m.int_ior;
    const float eta_t = r.front_face ? m.int_ior : m.ext_ior;
    const DielFresnel f = fresnel_dielectric(r.wi.z, eta_i, eta_t);
    const bool reflect_path = allow_r && (!allow_t || ux < f.reflectance);
    if(reflect_path) {
        r.wo = reflect(r.wi, f3{0.0f, 0.0f, 1.0f});
        r.sampled_type = kDielRefl;
        r.sampled_component = 0;
        r.pdf = allow_t ? f.reflectance : 1.0f;
        return allow_t ? load3(m.spec_refl) : load3(m.spec_refl) * f.reflectance;
    }
    if(f.reflectance >= 1.0f) return mk(0.0f);
    r.wo = refract(r.wi, f3{0.0f, 0.0f, 1.0f}, f.cos_theta_t, eta_i, eta_t);
    r.eta = eta_i / eta_t;
    r.sampled_type = kDielTrans;
    r.sampled_component = 1;
    r.pdf = allow_r ? (1.0f - f.reflectance) : 1.0f;
    f3 weight = load3(m.spec_trans);
    if(!allow_r) weight *= 1.0f - f.reflectance;
    if(c.mode == LRT_MODE_RADIANCE) weight *= r.eta * r.eta;
    return weight;
}
LRT_HD f3 dielectric_eval(const MatRec& m, const BsdfCtx& c, const BRec& r, int meas) {
    if(meas != kDiscrete || r.wi.z <= 0.0f) return mk(0.0f);
    const bool allow_r = (c.type_mask & kDielRefl) != 0 && (c.component == -1 || c.component == 0);
    const bool allow_t = (c.type_mask & kDielTrans) != 0 && (c.component == -1 || c.component == 1);
    const float eta_i = r.front_face ? m.ext_ior : m.int_ior;
    const float eta_t = r.front_face ? m.int_ior : m.ext_ior;
    const DielFresnel f = fresnel_dielectric(r.wi.z, eta_i, eta_t);
    if(r.wi.z * r.wo.z >= 0.0f) {
        if(!allow_r || !delta_aligned(reflect(r.wi, f3{0.0f, 0.0f, 1.0f}), r.wo)) return mk(0.0f);
        return load3(m.spec_refl) * f.reflectance;
    }
    if(!allow_t || f.reflectance >= 1.0f) return mk(0.0f);
    const f3 transmitted = refract(r.wi, f3{0.0f, 0.0f, 1.0f}, f.cos_theta_t, eta_i, eta_t);
    if(!delta_aligned(transmitted, r.wo)) return mk(0.0f);
    f3 value = load3(m.spec_trans) * (1.0f - f.reflectance);
    if(c.mode == LRT_MODE_RADIANCE) {
        const float eta = eta_i / eta_t;
        value *= eta * eta;
    }
    return value;
}
LRT_HD float dielectric_pdf(const MatRec& m, const BsdfCtx& c, const BRec& r, int meas) {
    if(meas != kDiscrete || r.wi.z <= 0.0f) return 0.0f;
    const bool allow_r = (c.type_mask & kDielRefl) != 0 && (c.component == -1 || c.component == 0);
    const bool allow_t = (c.type_mask & kDielTrans) != 0 && (c.component == -1 || c.component == 1);
    const float eta_i = r.front_face ? m.ext_ior : m.int_ior;
    const float eta_t = r.front_face ? m.int_ior : m.ext_ior;
    const DielFresnel f = fresnel_dielectric(r.wi.z, eta_i, eta_t);
    if(r.wi.z * r.wo.z >= 0.0f) {
        if(!allow_r || !delta_aligned(reflect(r.wi, f3{0.0f, 0.0f, 1.0f}), r.wo)) return 0.0f;
        return allow_t ? f.reflectance : 1.0f;
    }
    if(!allow_t || f.reflectance >= 1.0f) return 0.0f;
    const f3 transmitted = refract(r.wi, f3{0.0f, 0.0f, 1.0f}, f.cos_theta_t, eta_i, eta_t);
    if(!delta_aligned(transmitted, r.wo)) return 0.0f;
    return allow_r ? (1.0f - f.reflectance) : 1.0f;
}

// ================= rough_dielectric_bsdf.h:28-197 =================
constexpr uint32_t kRDielRefl = kGlossy | kReflective | kDielectric;
constexpr uint32_t kRDielTrans = kGlossy | kRefractive | kDielectric;
LRT_HD bool rdiel_refl_allowed(const BsdfCtx& c) {
    return (c.type_mask & kRDielRefl) != 0 && (c.component == -1 || c.component == 0);
}
LRT_HD bool rdiel_trans_allowed(const BsdfCtx& c) {
    return (c.type_mask & kRDielTrans) != 0 && (c.component == -1 || c.component == 1);
}
LRT_HD ValPdf rdiel_eval_reflection(const MatRec& m, const BsdfCtx& c, f3 wi, f3 wo, float eta_i, float eta_t,
                                    bool both) {
    if(!rdiel_refl_allowed(c) || wi.z <= 1e-6f || wo.z <= 1e-6f) return ValPdf{mk(0.0f), 0.0f};
    f3 mh = wi + wo;
    if(length_squared(mh) <= 1e-12f) return ValPdf{mk(0.0f), 0.0f};
    mh = normalize(mh);
    if(mh.z < 0.0f) mh = -mh;
    const float wi_dot_m = dot(wi, mh);
    if(wi_dot_m <= 0.0f) return ValPdf{mk(0.0f), 0.0f};
    const float fresnel = fresnel_dielectric(wi_dot_m, eta_i, eta_t).reflectance;
    const float d = ggx_D(m.dist_alpha, mh);
    const float g = ggx_G(m.dist_alpha, wi, wo, mh);
    const float pdf_m = ggx_pdf(m.dist_alpha, wi, mh);
    const float lobe = both ? fresnel : 1.0f;
    const float value = fresnel * d * g / (4.0f * wi.z);
    const float pdf_wo = pdf_m * lobe / (4.0f * wi_dot_m);
    return ValPdf{mk(value), pdf_wo};
}
LRT_HD ValPdf rdiel_eval_transmission(const MatRec& m, const BsdfCtx& c, f3 wi, f3 wo, float eta_i, float eta_t,
                                      bool both) {
    if(!rdiel_trans_allowed(c) || wi.z <= 1e-6f || wo.z >= -1e-6f || eta_t <= 0.0f) return ValPdf{mk(0.0f), 0.0f};
    f3 mh = -(eta_i * wi + eta_t * wo);
    if(length_squared(mh) <= 1e-12f) return ValPdf{mk(0.0f), 0.0f};
    mh = normalize(mh);
    if(mh.z < 0.0f) mh = -mh;
    const float wi_dot_m = dot(wi, mh);
    const float wo_dot_m = dot(wo, mh);
    if(wi_dot_m <= 0.0f) return ValPdf{mk(0.0f), 0.0f};
    const float fresnel = fresnel_dielectric(wi_dot_m, eta_i, eta_t).reflectance;
    const float denom = eta_i * wi_dot_m + eta_t * wo_dot_m;
    if(fresnel >= 1.0f || denom * denom <= 1e-12f) return ValPdf{mk(0.0f), 0.0f};
    const float d = ggx_D(m.dist_alpha, mh);
    const float g = ggx_G(m.dist_alpha, wi, wo, mh);
    const float pdf_m = ggx_pdf(m.dist_alpha, wi, mh);
    const float abs_wo_m = fabsf(wo_dot_m);
    const float eta_scale = c.mode == LRT_MODE_RADIANCE ? eta_i : eta_t;
    const float lobe = both ? (1.0f - fresnel) : 1.0f;
    const float value = (1.0f - fresnel) * d * g * wi_dot_m * abs_wo_m * eta_scale * eta_scale / (wi.z * denom * denom);
    const float pdf_wo = pdf_m * lobe * (eta_t * eta_t) * abs_wo_m / (denom * denom);
    return ValPdf{mk(value), pdf_wo};
}
LRT_HD ValPdf rdiel_eval_and_pdf(const MatRec& m, const BsdfCtx& c, const BRec& r) {
    if(r.wi.z <= 1e-6f || fabsf(r.wo.z) <= 1e-6f) return ValPdf{mk(0.0f), 0.0f};
    const float eta_i = r.front_face ? m.ext_ior : m.int_ior;
    const float eta_t = r.front_face ? m.int_ior : m.ext_ior;
    const bool both = rdiel_refl_allowed(c) && rdiel_trans_allowed(c);
    if(r.wi.z * r.wo.z > 0.0f) return rdiel_eval_reflection(m, c, r.wi, r.wo, eta_i, eta_t, both);
    return rdiel_eval_transmission(m, c, r.wi, r.wo, eta_i, eta_t, both);
}
LRT_HD f3 rdiel_sample(const MatRec& m, const BsdfCtx& c, BRec& r, float ux, float uy) {
    rec_reset(r);
    if(r.wi.z <= 0.0f) return mk(0.0f);
    const bool allow_r = rdiel_refl_allowed(c);
    const bool allow_t = rdiel_trans_allowed(c);
    if(!allow_r && !allow_t) return mk(0.0f);
    const float eta_i = r.front_face ? m.ext_ior : m.int_ior;
    const float eta_t = r.front_face ? m.int_ior : m.ext_ior;
    const f3 mh = ggx_sample(m.dist_alpha, r.wi, ux, uy);
    const float wi_dot_m = dot(r.wi, mh);
    if(mh.z <= 0.0f || wi_dot_m <= 0.0f) return mk(0.0f);
    const DielFresnel f = fresnel_dielectric(wi_dot_m, eta_i, eta_t);
    const bool both = allow_r && allow_t;
    const bool reflect_path = allow_r && (!allow_t || c.lobe_sample < f.reflectance);
    if(reflect_path) {
        r.wo = reflect(r.wi, mh);
        if(r.wo.z <= 0.0f) return mk(0.0f);
        const ValPdf lv = rdiel_eval_reflection(m, c, r.wi, r.wo, eta_i, eta_t, both);
        if(lv.pdf <= 0.0f) return mk(0.0f);
        r.pdf = lv.pdf;
        r.sampled_type = kRDielRefl;
        r.sampled_component = 0;
        return load3(m.spec_refl) * (lv.value / lv.pdf);
    }
    if(f.cos_theta_t <= 0.0f) return mk(0.0f);
    r.wo = refract(r.wi, mh, f.cos_theta_t, eta_i, eta_t);
    if(r.wo.z >= 0.0f) return mk(0.0f);
    r.eta = eta_i / eta_t;
    const ValPdf lv = rdiel_eval_transmission(m, c, r.wi, r.wo, eta_i, eta_t, both);
    if(lv.pdf <= 0.0f) return mk(0.0f);
    r.pdf = lv.pdf;
    r.sampled_type = kRDielTrans;
    r.sampled_component = 1;
    return load3(m.spec_trans) * (lv.value / lv.pdf);
}
LRT_HD f3 rdiel_eval(const MatRec& m, const BsdfCtx& c, const BRec& r, int meas) {
    if(meas != kSolidAngle) return mk(0.0f);
    return rdiel_eval_and_pdf(m, c, r).value;
}
LRT_HD float rdiel_pdf(const MatRec& m, const BsdfCtx& c, const BRec& r, int meas) {
    if(meas != kSolidAngle) return 0.0f;
    return rdiel_eval_and_pdf(m, c, r).pdf;
}

// ================= plastic_bsdf.h:41-191 =================
constexpr uint32_t kPlasticSpec = kSpecular | kReflective | kDielectric;
constexpr uint32_t kPlasticDiff = kDiffuse | kReflective;
LRT_HD float plastic_lobe_probability(const MatRec& m, float fresnel_i) {
    const float specular = fresnel_i * m.specular_sampling_weight;
    const float diffuse = (1.0f - fresnel_i) * (1.0f - m.specular_sampling_weight);
    return specular / (specular + diffuse);
}
LRT_HD f3 scaled_diffuse(const MatRec& m, float fdr) {
    if(m.nonlinear) {
        return f3{m.diffuse[0] / (1.0f - m.diffuse[0] * fdr), m.diffuse[1] / (1.0f - m.diffuse[1] * fdr),
                  m.diffuse[2] / (1.0f - m.diffuse[2] * fdr)};
    }
    return load3(m.diffuse) / (1.0f - fdr);
}
LRT_HD f3 plastic_diffuse_weight(const MatRec& m, float fi, float fo) {
    return scaled_diffuse(m, m.fdr) * (m.inv_eta * (1.0f - fi) * (1.0f - fo));
}
LRT_HD f3 plastic_sample(const MatRec& m, const BsdfCtx& c, BRec& r, float ux, float uy) {
    rec_reset(r);
    const bool allow_s = (c.type_mask & kPlasticSpec) != 0 && (c.component == -1 || c.component == 0);
    const bool allow_d = (c.type_mask & kPlasticDiff) != 0 && (c.component == -1 || c.component == 1);
    if((!allow_s && !allow_d) || r.wi.z <= 0.0f) return mk(0.0f);
    const float fi = fresnel_dielectric_ext(r.wi.z, m.eta);
    if(allow_s && allow_d) {
        const float prob = plastic_lobe_probability(m, fi);
        if(ux < prob) {
            r.wo = reflect(r.wi, f3{0.0f, 0.0f, 1.0f});
            r.sampled_type = kPlasticSpec;
            r.sampled_component = 0;
            r.pdf = prob;
            return load3(m.spec_refl) * (fi / prob);
        }
        float dpdf = 0.0f;
        r.wo = cosine_hemisphere((ux - prob) / (1.0f - prob), uy, dpdf);
        r.pdf = (1.0f - prob) * dpdf;
        r.sampled_type = kPlasticDiff;
        r.sampled_component = 1;
        const float fo = fresnel_dielectric_ext(r.wo.z, m.eta);
        return plastic_diffuse_weight(m, fi, fo) / (1.0f - prob);
    }
    if(allow_s) {
        r.wo = reflect(r.wi, f3{0.0f, 0.0f, 1.0f});
        r.sampled_type = kPlasticSpec;
        r.sampled_component = 0;
        r.pdf = 1.0f;
        return load3(m.spec_refl) * fi;
    }
    float dpdf = 0.0f;
    r.wo = cosine_hemisphere(ux, uy, dpdf);
    r.pdf = dpdf;
    r.sampled_type = kPlasticDiff;
    r.sampled_component = 1;
    const float fo = fresnel_dielectric_ext(r.wo.z, m.eta);
    return plastic_diffuse_weight(m, fi, fo);
}
LRT_HD f3 plastic_eval(const MatRec& m, const BsdfCtx& c, const BRec& r, int meas) {
    const bool allow_s = (c.type_mask & kPlasticSpec) != 0 && (c.component == -1 || c.component == 0);
    const bool allow_d = (c.type_mask & kPlasticDiff) != 0 && (c.component == -1 || c.component == 1);
    if(r.wi.z <= 0.0f) return mk(0.0f);
    if(meas == kDiscrete) {
        if(!allow_s || !delta_aligned(reflect(r.wi, f3{0.0f, 0.0f, 1.0f}), r.wo)) return mk(0.0f);
        return load3(m.spec_refl) * fresnel_dielectric_ext(r.wi.z, m.eta);
    }
    if(meas != kSolidAngle || !allow_d || r.wo.z <= 0.0f) return mk(0.0f);
    const float fi = fresnel_dielectric_ext(r.wi.z, m.eta);
    const float fo = fresnel_dielectric_ext(r.wo.z, m.eta);
    return plastic_diffuse_weight(m, fi, fo) * (r.wo.z / kPi);
}
LRT_HD float plastic_pdf(const MatRec& m, const BsdfCtx& c, const BRec& r, int meas) {
    const bool allow_s = (c.type_mask & kPlasticSpec) != 0 && (c.component == -1 || c.component == 0);
    const bool allow_d = (c.type_mask & kPlasticDiff) != 0 && (c.component == -1 || c.component == 1);
    if(r.wi.z <= 0.0f) return 0.0f;
    if(meas == kDiscrete) {
        if(!allow_s || !delta_aligned(reflect(r.wi, f3{0.0f, 0.0f, 1.0f}), r.wo)) return 0.0f;
        return allow_d ? plastic_lobe_probability(m, fresnel_dielectric_ext(r.wi.z, m.eta)) : 1.0f;
    }
    if(meas != kSolidAngle || !allow_d || r.wo.z <= 0.0f) return 0.0f;
    float prob_s = 0.0f;
    if(allow_s) prob_s = plastic_lobe_probability(m, fresnel_dielectric_ext(r.wi.z, m.eta));
    return (r.wo.z / kPi) * (1.0f - prob_s);
}

// ================= rough_plastic_bsdf.h:45-175 =================
constexpr uint32_t kRPlasticGlossy = kGlossy | kReflective | kDielectric;
LRT_HD float rplastic_glossy_probability(const MatRec& m, const float* table, float cos_theta_i) {
    const float reflectance = 1.0f - trans_eval(table, cos_theta_i);
    const float glossy = reflectance * m.specular_sampling_weight;
    const float diffuse = (1.0f - reflectance) * (1.0f - m.specular_sampling_weight);
    return glossy / (glossy + diffuse);
}
LRT_HD f3 rplastic_eval(const MatRec& m, const float* table, const BsdfCtx& c, const BRec& r, int meas) {
    if(meas != kSolidAngle) return mk(0.0f);
    const bool allow_g = (c.type_mask & kRPlasticGlossy) != 0 && (c.component == -1 || c.component == 0);
    const bool allow_d = (c.type_mask & kPlasticDiff) != 0 && (c.component == -1 || c.component == 1);
    if(r.wi.z <= 0.0f || r.wo.z <= 0.0f || (!allow_g && !allow_d)) return mk(0.0f);
    f3 result = mk(0.0f);
    if(allow_g) {
        const f3 half = normalize(r.wi + r.wo);
        const float d = ggx_D(m.dist_alpha, half);
        const float fresnel = fresnel_dielectric_ext(dot(r.wi, half), m.eta);
        const float g = ggx_G(m.dist_alpha, r.wi, r.wo, half);
        result += load3(m.spec_refl) * (fresnel * d * g / (4.0f * r.wi.z));
    }
    if(allow_d) {
        const float t12 = trans_eval(table, r.wi.z);
        const float t21 = trans_eval(table, r.wo.z);
        const float fdr = 1.0f - m.fdr;
        result += scaled_diffuse(m, fdr) * ((r.wo.z / kPi) * t12 * t21 * m.inv_eta);
    }
    return result;
}
LRT_HD float rplastic_pdf(const MatRec& m, const float* table, const BsdfCtx& c, const BRec& r, int meas) {
    if(meas != kSolidAngle) return 0.0f;
    const bool allow_g = (c.type_mask & kRPlasticGlossy) != 0 && (c.component == -1 || c.component == 0);
    const bool allow_d = (c.type_mask & kPlasticDiff) != 0 && (c.component == -1 || c.component == 1);
    if(r.wi.z <= 0.0f || r.wo.z <= 0.0f || (!allow_g && !allow_d)) return 0.0f;
    float prob_g = 1.0f, prob_d = 1.0f;
    if(allow_g && allow_d) {
        prob_g = rplastic_glossy_probability(m, table, r.wi.z);
        prob_d = 1.0f - prob_g;
    }
    float density = 0.0f;
    if(allow_g) {
        const f3 half = normalize(r.wi + r.wo);
        const float dwh_dwo = 1.0f / (4.0f * dot(r.wo, half));
        density += ggx_pdf(m.dist_alpha, r.wi, half) * dwh_dwo * prob_g;
    }
    if(allow_d) density += prob_d * (r.wo.z / kPi);
    return density;
}
LRT_HD f3 rplastic_sample(const MatRec& m, const float* table, const BsdfCtx& c, BRec& r, float ux, float uy) {
    rec_reset(r);
    const bool allow_g = (c.type_mask & kRPlasticGlossy) != 0 && (c.component == -1 || c.component == 0);
    const bool allow_d = (c.type_mask & kPlasticDiff) != 0 && (c.component == -1 || c.component == 1);
    if((!allow_g && !allow_d) || r.wi.z <= 0.0f) return mk(0.0f);
    float lx = ux, ly = uy;
    bool chose_glossy = allow_g;
    if(allow_g && allow_d) {
        const float prob = rplastic_glossy_probability(m, table, r.wi.z);
        if(ly < prob) {
            ly /= prob;
        } else {
            ly = (ly - prob) / (1.0f - prob);
            chose_glossy = false;
        }
    }
    if(chose_glossy) {
        const f3 mh = ggx_sample(m.dist_alpha, r.wi, lx, ly);
        r.wo = reflect(r.wi, mh);
        r.sampled_type = kRPlasticGlossy;
        r.sampled_component = 0;
        if(r.wo.z <= 0.0f) return mk(0.0f);
    } else {
        float cpdf = 0.0f;
        r.wo = cosine_hemisphere(lx, ly, cpdf);
        r.sampled_type = kPlasticDiff;
        r.sampled_component = 1;
    }
    const float density = rplastic_pdf(m, table, c, r, kSolidAngle);
    if(density == 0.0f) return mk(0.0f);
    r.pdf = density;
    return rplastic_eval(m, table, c, r, kSolidAngle) / density;
}

// ================= base dispatch (non-coating BSDFs) =================
LRT_HD const float* mat_table(const float* tables, const MatRec& m) {
    return m.table >= 0 ? tables + static_cast<size_t>(m.table) * LRT_TRANS_SAMPLES : nullptr;
}
LRT_HD f3 base_sample(const MatRec& m, const float* tables, const BsdfCtx& c, BRec& r, float ux, float uy) {
    switch(m.type) {
    case LRT_DIFFUSE: return diffuse_sample(m, c, r, ux, uy);
    case LRT_ROUGH_CONDUCTOR: return conductor_sample(m, c, r, ux, uy);
    case LRT_DIELECTRIC: return dielectric_sample(m, c, r, ux, uy);
    case LRT_ROUGH_DIELECTRIC: return rdiel_sample(m, c, r, ux, uy);
    case LRT_PLASTIC: return plastic_sample(m, c, r, ux, uy);
    case LRT_ROUGH_PLASTIC: return rplastic_sample(m, mat_table(tables, m), c, r, ux, uy);
    default: rec_reset(r); return mk(0.0f);
    }
}
LRT_HD f3 base_eval(const MatRec& m, const float* tables, const BsdfCtx& c, const BRec& r, int meas) {
    switch(m.type) {
    case LRT_DIFFUSE: return diffuse_eval(m, c, r, meas);
    case LRT_ROUGH_CONDUCTOR: return conductor_eval(m, c, r, meas);
    case LRT_DIELECTRIC: return dielectric_eval(m, c, r, meas);
    case LRT_ROUGH_DIELECTRIC: return rdiel_eval(m, c, r, meas);
    case LRT_PLASTIC: return plastic_eval(m, c, r, meas);
    case LRT_ROUGH_PLASTIC: return rplastic_eval(m, mat_table(tables, m), c, r, meas);
    default: return mk(0.0f);
    }
}
LRT_HD float base_pdf(const MatRec& m, const float* tables, const BsdfCtx& c, const BRec& r, int meas) {
    switch(m.type) {
    case LRT_DIFFUSE: return diffuse_pdf(m, c, r, meas);
    case LRT_ROUGH_CONDUCTOR: return conductor_pdf(m, c, r, meas);
    case LRT_DIELECTRIC: return dielectric_pdf(m, c, r, meas);
    case LRT_ROUGH_DIELECTRIC: return rdiel_pdf(m, c, r, meas);
    case LRT_PLASTIC: return plastic_pdf(m, c, r, meas);
    case LRT_ROUGH_PLASTIC: return rplastic_pdf(m, mat_table(tables, m), c, r, meas);
    default: return 0.0f;
    }
}

// ================= coating helpers: src/material/func/coating_layer.h =================
struct Refracted {
    f3 direction;
    float reflectance;
};
LRT_HD Refracted coating_refract_in(f3 wi, float eta, float inv_eta) {
    float cos_t = 0.0f;
    Refracted r;
    r.reflectance = fresnel_dielectric_ext(fabsf(wi.z), cos_t, eta);
    r.direction = f3{inv_eta * wi.x, inv_eta * wi.y, -signum(wi.z) * cos_t};
    return r;
}
LRT_HD Refracted coating_refract_out(f3 wi, float eta, float inv_eta) {
    float cos_t = 0.0f;
    Refracted r;
    r.reflectance = fresnel_dielectric_ext(fabsf(wi.z), cos_t, inv_eta);
    r.direction = f3{eta * wi.x, eta * wi.y, -signum(wi.z) * cos_t};
    return r;
}
LRT_HD f3 coating_refract_to(bool interior, f3 wi, float eta, float inv_eta) {
    const float scale = interior ? inv_eta : eta;
    const float sin_theta_t2 = scale * scale * (wi.x * wi.x + wi.y * wi.y);
    if(sin_theta_t2 >= 1.0f) return mk(0.0f);
    const float cos_theta_t = sqrtf(1.0f - sin_theta_t2);
    return f3{scale * wi.x, scale * wi.y, wi.z > 0.0f ? cos_theta_t : -cos_theta_t};
}
LRT_HD float coating_solid_angle_factor(float inv_eta, f3 wo, f3 wo_inner) { return inv_eta * inv_eta * wo.z / wo_inner.z; }
LRT_HD f3 coating_absorption(const MatRec& m, f3 wi_inner, f3 wo_inner) {
    if(m.sigma_zero) return mk(1.0f);
    const float path_length = (1.0f / fabsf(wi_inner.z)) + (1.0f / fabsf(wo_inner.z));
    const f3 exponent = load3(m.sigma_a) * (-m.thickness * path_length);
    return f3{exp_rn(exponent.x), exp_rn(exponent.y), exp_rn(exponent.z)};
}
LRT_HD float coating_specular_probability(float reflectance, float ssw) {
    const float specular = reflectance * ssw;
    const float nested = (1.0f - reflectance) * (1.0f - ssw);
    return specular / (specular + nested);
}

// ================= coating_bsdf.h:45-177 =================
constexpr uint32_t kCoatSpec = kSpecular | kReflective | kDielectric;
LRT_HD bool coat_spec_allowed(const MatRec& m, const BsdfCtx& c) {
    return (c.type_mask & kCoatSpec) != 0 && (c.component == -1 || c.component == m.specular_component);
}
LRT_HD bool coat_nested_allowed(const MatRec& m, const MatRec& n, const BsdfCtx& c) {
    return (c.type_mask & n.flags) != 0 && (c.component == -1 || c.component < m.specular_component);
}
LRT_HD f3 coating_sample(const MatRec& m, const MatRec& n, const float* tables, const BsdfCtx& c, BRec& r, float ux,
                         float uy) {
    rec_reset(r);
    const bool allow_s = coat_spec_allowed(m, c);
    const bool allow_n = coat_nested_allowed(m, n, c);
    if(!allow_s && !allow_n) return mk(0.0f);
    const Refracted incoming = coating_refract_in(r.wi, m.eta, m.inv_eta);
    const float prob = coating_specular_probability(incoming.reflectance, m.specular_sampling_weight);
    float lx = ux;
    const float ly = uy;
    bool chose_specular = allow_s;
    if(allow_s && allow_n) {
        if(lx < prob) {
            lx /= prob;
        } else {
            lx = (lx - prob) / (1.0f - prob);
            chose_specular = false;
        }
    }
    if(chose_specular) {
        r.wo = f3{-r.wi.x, -r.wi.y, r.wi.z};
        r.sampled_type = kCoatSpec;
        r.sampled_component = m.specular_component;
        r.pdf = allow_n ? prob : 1.0f;
        return load3(m.spec_refl) * (incoming.reflectance / r.pdf);
    }
    if(incoming.reflectance == 1.0f) return mk(0.0f);
    const f3 wi_outer = r.wi;
    r.wi = incoming.direction;
    f3 weight = base_sample(n, tables, c, r, lx, ly);
    const f3 wo_inner = r.wo;
    r.wi = wi_outer;
    if(is_zero(weight)) return mk(0.0f);
    const Refracted outgoing = coating_refract_out(wo_inner, m.eta, m.inv_eta);
    r.wo = outgoing.direction;
    if(outgoing.reflectance == 1.0f) return mk(0.0f);
    weight *= coating_absorption(m, incoming.direction, wo_inner);
    weight *= (1.0f - incoming.reflectance) * (1.0f - outgoing.reflectance);
    if(allow_s) {
        r.pdf *= 1.0f - prob;
        weight /= 1.0f - prob;
    }
    if(measure_of(r.sampled_type) == kSolidAngle) r.pdf *= coating_solid_angle_factor(m.inv_eta, r.wo, wo_inner);
    return weight;
}
LRT_HD f3 coating_eval(const MatRec& m, const MatRec& n, const float* tables, const BsdfCtx& c, const BRec& r, int meas) {
    const bool allow_s = coat_spec_allowed(m, c);
    const bool allow_n = coat_nested_allowed(m, n, c);
    if(meas == kDiscrete && allow_s && delta_aligned(f3{-r.wi.x, -r.wi.y, r.wi.z}, r.wo)) {
        return load3(m.spec_refl) * fresnel_dielectric_ext(fabsf(r.wi.z), m.eta);
    }
    if(!allow_n) return mk(0.0f);
    const Refracted incoming = coating_refract_in(r.wi, m.eta, m.inv_eta);
    const Refracted outgoing = coating_refract_in(r.wo, m.eta, m.inv_eta);
    if(incoming.reflectance == 1.0f || outgoing.reflectance == 1.0f) return mk(0.0f);
    BRec inner = r;
    inner.wi = incoming.direction;
    inner.wo = outgoing.direction;
    f3 result = base_eval(n, tables, c, inner, meas) * ((1.0f - incoming.reflectance) * (1.0f - outgoing.reflectance));
    result *= coating_absorption(m, incoming.direction, outgoing.direction);
    if(meas == kSolidAngle) result *= coating_solid_angle_factor(m.inv_eta, r.wo, outgoing.direction);
    return result;
}
LRT_HD float coating_pdf(const MatRec& m, const MatRec& n, const float* tables, const BsdfCtx& c, const BRec& r, int meas) {
    const bool allow_s = coat_spec_allowed(m, c);
    const bool allow_n = coat_nested_allowed(m, n, c);
    const Refracted incoming = coating_refract_in(r.wi, m.eta, m.inv_eta);
    if(meas == kDiscrete && allow_s && delta_aligned(f3{-r.wi.x, -r.wi.y, r.wi.z}, r.wo)) {
        return allow_n ? coating_specular_probability(incoming.reflectance, m.specular_sampling_weight) : 1.0f;
    }
    if(!allow_n) return 0.0f;
    const Refracted outgoing = coating_refract_in(r.wo, m.eta, m.inv_eta);
    if(incoming.reflectance == 1.0f || outgoing.reflectance == 1.0f) return 0.0f;
    BRec inner = r;
    inner.wi = incoming.direction;
    inner.wo = outgoing.direction;
    float density = base_pdf(n, tables, c, inner, meas);
    if(meas == kSolidAngle) density *= coating_solid_angle_factor(m.inv_eta, r.wo, outgoing.direction);
    if(allow_s) density *= 1.0f - coating_specular_probability(incoming.reflectance, m.specular_sampling_weight);
    return density;
}

// ================= rough_coating_bsdf.h:51-217 =================
constexpr uint32_t kRCoatSpec = kGlossy | kReflective | kDielectric;
LRT_HD bool rcoat_spec_component_allowed(const MatRec& m, const BsdfCtx& c) {
    return (c.type_mask & kRCoatSpec) != 0 && (c.component == -1 || c.component == m.specular_component);
}
LRT_HD float rcoat_specular_probability(const MatRec& m, const float* table, float cos_theta_i) {
    return coating_specular_probability(1.0f - trans_eval(table, fabsf(cos_theta_i)), m.specular_sampling_weight);
}
LRT_HD f3 rcoat_nested_eval(const MatRec& m, const MatRec& n, const float* tables, const float* table,
                            const BsdfCtx& c, const BRec& r, int meas) {
    BRec inner = r;
    inner.wi = coating_refract_to(true, r.wi, m.eta, m.inv_eta);
    inner.wo = coating_refract_to(true, r.wo, m.eta, m.inv_eta);
    if(is_zero(inner.wi) || is_zero(inner.wo)) return mk(0.0f);
    f3 result = base_eval(n, tables, c, inner, meas) * trans_eval(table, fabsf(r.wi.z)) * trans_eval(table, fabsf(r.wo.z));
    result *= coating_absorption(m, inner.wi, inner.wo);
    if(meas == kSolidAngle) result *= coating_solid_angle_factor(m.inv_eta, r.wo, inner.wo);
    return result;
}
LRT_HD float rcoat_nested_pdf(const MatRec& m, const MatRec& n, const float* tables, const BsdfCtx& c, const BRec& r,
                              int meas) {
    BRec inner = r;
    inner.wi = coating_refract_to(true, r.wi, m.eta, m.inv_eta);
    inner.wo = coating_refract_to(true, r.wo, m.eta, m.inv_eta);
    if(is_zero(inner.wi) || is_zero(inner.wo)) return 0.0f;
    float density = base_pdf(n, tables, c, inner, meas);
    if(meas == kSolidAngle) density *= coating_solid_angle_factor(m.inv_eta, r.wo, inner.wo);
    return density;
}
LRT_HD f3 rcoat_eval(const MatRec& m, const MatRec& n, const float* tables, const BsdfCtx& c, const BRec& r, int meas) {
    const float* table = mat_table(tables, m);
    const bool allow_n = coat_nested_allowed(m, n, c);
    const bool allow_s = rcoat_spec_component_allowed(m, c) && meas == kSolidAngle;
    f3 result = mk(0.0f);
    if(allow_s && r.wo.z * r.wi.z > 0.0f) {
        f3 half = r.wi + r.wo;
        if(length_squared(half) > 1e-12f) {
            half = normalize(half) * signum(r.wo.z);
            const float d = ggx_D(m.dist_alpha, half);
            const float fresnel = fresnel_dielectric_ext(fabsf(dot(r.wi, half)), m.eta);
            const float g = ggx_G(m.dist_alpha, r.wi, r.wo, half);
            result += load3(m.spec_refl) * (fresnel * d * g / (4.0f * fabsf(r.wi.z)));
        }
    }
    if(allow_n) result += rcoat_nested_eval(m, n, tables, table, c, r, meas);
    return result;
}
LRT_HD float rcoat_pdf(const MatRec& m, const MatRec& n, const float* tables, const BsdfCtx& c, const BRec& r, int meas) {
    const float* table = mat_table(tables, m);
    const bool allow_n = coat_nested_allowed(m, n, c);
    const bool allow_s = rcoat_spec_component_allowed(m, c) && meas == kSolidAngle;
    float prob_s = 1.0f, prob_n = 1.0f;
    if(allow_s && allow_n) {
        prob_s = rcoat_specular_probability(m, table, r.wi.z);
        prob_n = 1.0f - prob_s;
    }
    float density = 0.0f;
    if(allow_s && r.wo.z * r.wi.z > 0.0f) {
        f3 half = r.wi + r.wo;
        if(length_squared(half) > 1e-12f) {
            half = normalize(half) * signum(r.wo.z);
            const float dwh_dwo = 1.0f / (4.0f * fabsf(dot(r.wo, half)));
            density += ggx_pdf(m.dist_alpha, r.wi, half) * dwh_dwo * prob_s;
        }
    }
    if(allow_n) density += rcoat_nested_pdf(m, n, tables, c, r, meas) * prob_n;
    return density;
}
LRT_HD f3 rcoat_sample(const MatRec& m, const MatRec& n, const float* tables, const BsdfCtx& c, BRec& r, float ux,
                       float uy) {
    rec_reset(r);
    const float* table = mat_table(tables, m);
    const bool allow_s = rcoat_spec_component_allowed(m, c);
    const bool allow_n = coat_nested_allowed(m, n, c);
    if(!allow_s && !allow_n) return mk(0.0f);
    const float lx = ux;
    float ly = uy;
    bool chose_specular = allow_s;
    if(allow_s && allow_n) {
        const float prob = rcoat_specular_probability(m, table, r.wi.z);
        if(ly < prob) {
            ly /= prob;
        } else {
            ly = (ly - prob) / (1.0f - prob);
            chose_specular = false;
        }
    }
    if(chose_specular) {
        const f3 mh = ggx_sample(m.dist_alpha, r.wi, lx, ly);
        r.wo = reflect(r.wi, mh);
        r.sampled_type = kRCoatSpec;
        r.sampled_component = m.specular_component;
        r.eta = 1.0f;
        if(r.wo.z * r.wi.z <= 0.0f) return mk(0.0f);
    } else {
        const f3 wi_outer = r.wi;
        r.wi = coating_refract_to(true, wi_outer, m.eta, m.inv_eta);
        const f3 weight = base_sample(n, tables, c, r, lx, ly);
        r.wi = wi_outer;
        if(is_zero(weight)) return mk(0.0f);
        r.wo = coating_refract_to(false, r.wo, m.eta, m.inv_eta);
        if(is_zero(r.wo)) return mk(0.0f);
    }
    const int meas = measure_of(r.sampled_type);
    const float density = rcoat_pdf(m, n, tables, c, r, meas);
    if(density == 0.0f) return mk(0.0f);
    r.pdf = density;
    return rcoat_eval(m, n, tables, c, r, meas) / density;
}

// bsdf::component_flags (bsdf.h:62 default; dielectric_bsdf.h:25-27; plastic_bsdf.h:37-39;
// rough_plastic_bsdf.h:41-43; coating_bsdf.h:39-41; rough_coating_bsdf.h:45-47)
LRT_HD uint32_t base_component_flags(const MatRec& m, int component) {
    switch(m.type) {
    case LRT_DIELECTRIC: return component == 0 ? kDielRefl : kDielTrans;
    case LRT_PLASTIC: return component == 0 ? kPlasticSpec : kPlasticDiff;
    case LRT_ROUGH_PLASTIC: return component == 0 ? kRPlasticGlossy : kPlasticDiff;
    default: return m.flags;
    }
}
LRT_HD uint32_t bsdf_component_flags(const MatRec* mats, int32_t mid, int component) {
    const MatRec& m = mats[mid];
    if(m.type == LRT_COATING) return component == m.specular_component ? kCoatSpec : base_component_flags(mats[m.nested], component);
    if(m.type == LRT_ROUGH_COATING) {
        return component == m.specular_component ? kRCoatSpec : base_component_flags(mats[m.nested], component);
    }
    return base_component_flags(m, component);
}
// bsdf::diffuse_reflectance: the albedo of a diffuse BSDF, passed through by the coatings
LRT_HD f3 bsdf_diffuse_reflectance(const MatRec* mats, int32_t mid) {
    const MatRec& m = mats[mid];
    if(m.type == LRT_COATING || m.type == LRT_ROUGH_COATING) {
        const MatRec& n = mats[m.nested];
        return n.type == LRT_DIFFUSE ? load3(n.diffuse) : mk(0.0f);
    }
    return m.type == LRT_DIFFUSE ? load3(m.diffuse) : mk(0.0f);
}

// ================= top-level dispatch =================
LRT_HD f3 bsdf_sample(const MatRec* mats, const float* tables, int32_t mid, const BsdfCtx& c, BRec& r, float ux,
                      float uy) {
    const MatRec& m = mats[mid];
    if(m.type == LRT_COATING) return coating_sample(m, mats[m.nested], tables, c, r, ux, uy);
    if(m.type == LRT_ROUGH_COATING) return rcoat_sample(m, mats[m.nested], tables, c, r, ux, uy);
    return base_sample(m, tables, c, r, ux, uy);
}
LRT_HD f3 bsdf_eval(const MatRec* mats, const float* tables, int32_t mid, const BsdfCtx& c, const BRec& r, int meas) {
    const MatRec& m = mats[mid];
    if(m.type == LRT_COATING) return coating_eval(m, mats[m.nested], tables, c, r, meas);
    if(m.type == LRT_ROUGH_COATING) return rcoat_eval(m, mats[m.nested], tables, c, r, meas);
    return base_eval(m, tables, c, r, meas);
}
LRT_HD float bsdf_pdf(const MatRec* mats, const float* tables, int32_t mid, const BsdfCtx& c, const BRec& r, int meas) {
    const MatRec& m = mats[mid];
    if(m.type == LRT_COATING) return coating_pdf(m, mats[m.nested], tables, c, r, meas);
    if(m.type == LRT_ROUGH_COATING) return rcoat_pdf(m, mats[m.nested], tables, c, r, meas);
    return base_pdf(m, tables, c, r, meas);
}

// The same three calls for a material whose type is known at compile time (kType >= 0; -1: the type is
// read from the record): only that type's code is compiled in, so a kernel specialised per material
// type holds fewer registers than one that can shade every type.
template <int kType>
LRT_HD f3 bsdf_sample_t(const MatRec* mats, const float* tables, int32_t mid, const BsdfCtx& c, BRec& r, float ux,
                        float uy) {
    const MatRec& m = mats[mid];
    if constexpr(kType == LRT_DIFFUSE) {
        return diffuse_sample(m, c, r, ux, uy);
    } else if constexpr(kType == LRT_ROUGH_CONDUCTOR) {
        return conductor_sample(m, c, r, ux, uy);
    } else if constexpr(kType == LRT_DIELECTRIC) {
        return dielectric_sample(m, c, r, ux, uy);
    } else if constexpr(kType == LRT_ROUGH_DIELECTRIC) {
        return rdiel_sample(m, c, r, ux, uy);
    } else if constexpr(kType == LRT_PLASTIC) {
        return plastic_sample(m, c, r, ux, uy);
    } else if constexpr(kType == LRT_ROUGH_PLASTIC) {
        return rplastic_sample(m, mat_table(tables, m), c, r, ux, uy);
    } else if constexpr(kType == LRT_COATING) {
        return coating_sample(m, mats[m.nested], tables, c, r, ux, uy);
    } else if constexpr(kType == LRT_ROUGH_COATING) {
        return rcoat_sample(m, mats[m.nested], tables, c, r, ux, uy);
    } else {
        return bsdf_sample(mats, tables, mid, c, r, ux, uy);
    }
}
template <int kType>
LRT_HD f3 bsdf_eval_t(const MatRec* mats, const float* tables, int32_t mid, const BsdfCtx& c, const BRec& r, int meas) {
    const MatRec& m = mats[mid];
    if constexpr(kType == LRT_DIFFUSE) {
        return diffuse_eval(m, c, r, meas);
    } else if constexpr(kType == LRT_ROUGH_CONDUCTOR) {
        return conductor_eval(m, c, r, meas);
    } else if constexpr(kType == LRT_DIELECTRIC) {
        return dielectric_eval(m, c, r, meas);
    } else if constexpr(kType == LRT_ROUGH_DIELECTRIC) {
        return rdiel_eval(m, c, r, meas);
    } else if constexpr(kType == LRT_PLASTIC) {
        return plastic_eval(m, c, r, meas);
    } else if constexpr(kType == LRT_ROUGH_PLASTIC) {
        return rplastic_eval(m, mat_table(tables, m), c, r, meas);
    } else if constexpr(kType == LRT_COATING) {
        return coating_eval(m, mats[m.nested], tables, c, r, meas);
    } else if constexpr(kType == LRT_ROUGH_COATING) {
        return rcoat_eval(m, mats[m.nested], tables, c, r, meas);
    } else {
        return bsdf_eval(mats, tables, mid, c, r, meas);
    }
}
template <int kType>
LRT_HD float bsdf_pdf_t(const MatRec* mats, const float* tables, int32_t mid, const BsdfCtx& c, const BRec& r, int meas) {
    const MatRec& m = mats[mid];
    if constexpr(kType == LRT_DIFFUSE) {
        return diffuse_pdf(m, c, r, meas);
    } else if constexpr(kType == LRT_ROUGH_CONDUCTOR) {
        return conductor_pdf(m, c, r, meas);
    } else if constexpr(kType == LRT_DIELECTRIC) {
        return dielectric_pdf(m, c, r, meas);
    } else if constexpr(kType == LRT_ROUGH_DIELECTRIC) {
        return rdiel_pdf(m, c, r, meas);
    } else if constexpr(kType == LRT_PLASTIC) {
        return plastic_pdf(m, c, r, meas);
    } else if constexpr(kType == LRT_ROUGH_PLASTIC) {
        return rplastic_pdf(m, mat_table(tables, m), c, r, meas);
    } else if constexpr(kType == LRT_COATING) {
        return coating_pdf(m, mats[m.nested], tables, c, r, meas);
    } else if constexpr(kType == LRT_ROUGH_COATING) {
        return rcoat_pdf(m, mats[m.nested], tables, c, r, meas);
    } else {
        return bsdf_pdf(mats, tables, mid, c, r, meas);
    }
}

}  // namespace lrt
