// lrt_math.cuh — FP32 vector math, orthonormal basis and the scrambled Sobol sampler.
//
// Every operation keeps the reference's operand order (src/core/vec3.h:71-109): a dot product is
// (x*x' + y*y') + z*z', a vec3/scalar divides each component, a scalar*vec3 multiplies componentwise.
// The library is compiled with -fmad=false (device) and -ffp-contract=off (host), so each product and
// sum is rounded separately as in the reference's x86-64 build; this is what makes traversal and
// triangle tests bit-identical to the reference.
#pragma once

#include <math.h>
#include <stdint.h>

#ifdef __CUDACC__
#define LRT_HD __host__ __device__ __forceinline__
#else
#define LRT_HD inline
#endif

namespace lrt {

constexpr float kPi = 3.14159265358979323846f;  // M_PI<float> (src/core/core.h:7)

struct f3 {
    float x, y, z;
};

LRT_HD f3 mk(float x, float y, float z) { return f3{x, y, z}; }
LRT_HD f3 mk(float v) { return f3{v, v, v}; }
LRT_HD f3 load3(const float* p) { return f3{p[0], p[1], p[2]}; }
LRT_HD void store3(float* p, f3 v) { p[0] = v.x; p[1] = v.y; p[2] = v.z; }
LRT_HD float comp(f3 v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : v.z); }

LRT_HD f3 operator-(f3 a) { return f3{-a.x, -a.y, -a.z}; }
LRT_HD f3 operator+(f3 a, f3 b) { return f3{a.x + b.x, a.y + b.y, a.z + b.z}; }
LRT_HD f3 operator-(f3 a, f3 b) { return f3{a.x - b.x, a.y - b.y, a.z - b.z}; }
LRT_HD f3 operator*(f3 a, float s) { return f3{a.x * s, a.y * s, a.z * s}; }
LRT_HD f3 operator*(float s, f3 a) { return a * s; }
LRT_HD f3 operator*(f3 a, f3 b) { return f3{a.x * b.x, a.y * b.y, a.z * b.z}; }
LRT_HD f3 operator/(f3 a, float s) { return f3{a.x / s, a.y / s, a.z / s}; }
LRT_HD f3& operator+=(f3& a, f3 b) { a.x += b.x; a.y += b.y; a.z += b.z; return a; }
LRT_HD f3& operator*=(f3& a, f3 b) { a.x *= b.x; a.y *= b.y; a.z *= b.z; return a; }
LRT_HD f3& operator*=(f3& a, float s) { a.x *= s; a.y *= s; a.z *= s; return a; }
LRT_HD f3& operator/=(f3& a, float s) { a.x /= s; a.y /= s; a.z /= s; return a; }

LRT_HD float dot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
LRT_HD f3 cross(f3 a, f3 b) {
    return f3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
LRT_HD float length_squared(f3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
LRT_HD float length(f3 a) { return sqrtf(a.x * a.x + a.y * a.y + a.z * a.z); }
LRT_HD f3 normalize(f3 a) { return a / length(a); }
LRT_HD bool is_zero(f3 a) { return a.x == 0.0f && a.y == 0.0f && a.z == 0.0f; }

// std::min / std::max / std::clamp semantics (NaN handling included): min(a,b) = b<a ? b : a.
LRT_HD float smin(float a, float b) { return (b < a) ? b : a; }
LRT_HD float smax(float a, float b) { return (a < b) ? b : a; }
LRT_HD float sclamp(float v, float lo, float hi) { return (v < lo) ? lo : ((hi < v) ? hi : v); }
LRT_HD float max3(f3 v) {  // std::max({r, g, b})
    float m = v.x;
    if(m < v.y) m = v.y;
    if(m < v.z) m = v.z;
    return m;
}
LRT_HD float signum(float v) { return static_cast<float>((v > 0.0f) - (v < 0.0f)); }

// Single-precision sin/cos, x^(1/4) (the reference's powf(x, 0.25f)), exp and acos as the reference's
// libm returns them. glibc's float versions (sinf/cosf/powf/expf, under 0.6-0.9 ulp) give the correctly
// rounded result for nearly every argument; CUDA's float versions are within 1-2 ulp and left about 1%
// of arguments an ulp away, which grazing reflections and the Catmull-Rom table lookups amplify past
// 1e-5. On the device these evaluate in double precision and round once to float, which is the
// correctly rounded value except where the double result lies within a double ulp or so of a float
// rounding boundary.
#ifdef __CUDA_ARCH__
__device__ __forceinline__ void sincos_rn(float x, float& s, float& c) {
    double sd, cd;
    sincos(static_cast<double>(x), &sd, &cd);
    s = static_cast<float>(sd);
    c = static_cast<float>(cd);
}
// x^(1/4) for x >= 0 as two double-precision square roots (each correctly rounded)
__device__ __forceinline__ float quartic_root_rn(float x) {
    return static_cast<float>(sqrt(sqrt(static_cast<double>(x))));
}
__device__ __forceinline__ float exp_rn(float x) { return static_cast<float>(exp(static_cast<double>(x))); }
__device__ __forceinline__ float acos_rn(float x) { return static_cast<float>(acos(static_cast<double>(x))); }
#else
inline void sincos_rn(float x, float& s, float& c) {
    s = sinf(x);
    c = cosf(x);
}
inline float quartic_root_rn(float x) { return powf(x, 0.25f); }
inline float exp_rn(float x) { return expf(x); }
inline float acos_rn(float x) { return acosf(x); }
#endif

// onb::build_from_normal / local_to_world / world_to_local (src/core/onb.h:8-23)
struct Onb {
    f3 a0, a1, a2;
};
LRT_HD Onb onb_from_normal(f3 n) {
    Onb b;
    b.a2 = normalize(n);
    const f3 a = (fabsf(b.a2.x) > 0.9f) ? f3{0.0f, 1.0f, 0.0f} : f3{1.0f, 0.0f, 0.0f};
    b.a1 = normalize(cross(b.a2, a));
    b.a0 = cross(b.a2, b.a1);
    return b;
}
LRT_HD f3 to_world(const Onb& b, f3 a) { return b.a0 * a.x + b.a1 * a.y + b.a2 * a.z; }
LRT_HD f3 to_local(const Onb& b, f3 a) { return f3{dot(a, b.a0), dot(a, b.a1), dot(a, b.a2)}; }

// ---- scrambled Sobol sampler (src/core/sampler.h:12-33, src/core/sobol.h:12-41) ----

LRT_HD uint32_t mix_bits(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

constexpr uint32_t kSobolDims = 16;

// dims >= 16 fall back to a hash (sobol.h:16-19)
LRT_HD uint32_t sobol_bits(const uint32_t (*table)[32], uint32_t index, uint32_t dimension) {
    if(dimension >= kSobolDims) {
        return mix_bits(index + dimension * 0x9e3779b9u);
    }
    uint32_t gray = index ^ (index >> 1);
    uint32_t value = 0;
    const uint32_t* row = table[dimension];
    while(gray != 0u) {
#ifdef __CUDA_ARCH__
        const int bit = __ffs(gray) - 1;
        value ^= __ldg(row + bit);
#else
        const int bit = __builtin_ctz(gray);
        value ^= row[bit];
#endif
        gray &= gray - 1u;
    }
    return value;
}

struct Sampler {
    uint32_t index;
    uint32_t dimension;
    uint32_t seed;
};

LRT_HD Sampler sampler_start(uint32_t pixel_index, uint32_t sample_index) {
    return Sampler{sample_index, 0u, mix_bits(pixel_index)};
}

LRT_HD float sampler_next_1d(const uint32_t (*table)[32], Sampler& s) {
    const uint32_t d = s.dimension++;
    const uint32_t scrambled = sobol_bits(table, s.index, d) ^ mix_bits(s.seed + d * 0x9e3779b9u);
    return static_cast<float>(scrambled) * (1.0f / 4294967296.0f);
}

// sampler::next_2d is `vec2(next_1d(), next_1d())` (sampler.h:25-27). C++ leaves the evaluation order
// of those two arguments unspecified; the compiled reference (g++, and MSVC on x64) evaluates them
// right to left, so y takes dimension d and x takes dimension d + 1. The same holds one level up for
// f(next_2d(), next_2d()): the right argument draws first.
struct F2 {
    float x, y;
};
LRT_HD F2 sampler_next_2d(const uint32_t (*table)[32], Sampler& s) {
    const float y = sampler_next_1d(table, s);
    const float x = sampler_next_1d(table, s);
    return F2{x, y};
}

}  // namespace lrt
