// lrt_image.cu — the float-to-byte step of the reference's image output (io/image_write.cpp:10-20 and
// the optional vertical flip of image_write.cpp:60-69), on the device, so that a rendered image leaves
// the GPU as 3 bytes per pixel instead of 12.
//
// The reference's to_byte is NaN -> 0, v = powf(v, 1.0f / 2.2f), clamp to [0, 0.999], truncate v * 256.
// For every finite v >= 0 that is a non-decreasing step function of v with 255 steps, so it is fully
// described by its 255 thresholds: t[k] = the smallest float whose byte is >= k. The thresholds are
// found once per process on the host with the host C library's powf -- the function the reference's
// to_byte calls -- by bisection over the float bit patterns (8k powf calls), and the kernel counts the
// thresholds at or below each value (8 steps of a binary search over a table in shared memory). This
// reproduces the host powf's own last-bit rounding at the byte boundaries, which a device-side power
// does not: glibc's powf is not correctly rounded everywhere, and at 0.36048645f its result lands on
// 161/256 where the correctly rounded power is the float below it.
//
// Outside the table: NaN -> 0; a negative value (powf gives NaN, which the reference's conversion of
// NaN * 256 turns into 0 on x86-64) -> 0; -inf (powf(-inf, y) = +inf) -> 255.
//
// The kernel is a pure stream (12 bytes read and 3 written per pixel): one component per thread in a
// grid-stride loop, reads and writes both coalesced along a row.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>

#include "lrt_context.cuh"
#include "lrt_math.cuh"

using namespace lrt;

namespace {

struct ByteThresholds {
    float t[256];  // t[k] (k = 1..255): the smallest float whose byte is >= k; t[0] = 0
};

// to_byte of image_write.cpp:10-20 on the host, with this process's C library
unsigned char host_to_byte(float value) {
    if(std::isnan(value)) value = 0.0f;
    value = std::pow(value, 1.0f / 2.2f);
    value = std::clamp(value, 0.0f, 0.999f);
    if(std::isnan(value)) return 0;
    return static_cast<unsigned char>(static_cast<int>(value * 256.0f));
}

float float_of(uint32_t bits) {
    float f;
    std::memcpy(&f, &bits, 4);
    return f;
}

// Bisection over the non-negative float bit patterns (their order is the values' order): the first
// pattern in [0, +inf] whose byte is >= k. Returns false when the step function is not monotonic
// around a threshold (checked over 256 patterns on each side).
bool compute_thresholds(ByteThresholds& out) {
    out.t[0] = 0.0f;
    const uint32_t inf_bits = 0x7f800000u;
    for(int k = 1; k < 256; ++k) {
        uint32_t lo = 0, hi = inf_bits;  // byte(lo) < k <= byte(hi)
        while(hi - lo > 1) {
            const uint32_t mid = lo + (hi - lo) / 2;
            if(host_to_byte(float_of(mid)) >= k) {
                hi = mid;
            } else {
                lo = mid;
            }
        }
        out.t[k] = float_of(hi);
        const uint32_t a = hi > 256 ? hi - 256 : 0, b = std::min(hi + 256, inf_bits);
        for(uint32_t bits = a; bits <= b; ++bits) {
            if((host_to_byte(float_of(bits)) >= k) != (bits >= hi)) return false;
        }
    }
    for(int k = 2; k < 256; ++k) {
        if(!(out.t[k - 1] <= out.t[k])) return false;
    }
    return true;
}

std::once_flag g_thresholds_once;
ByteThresholds g_thresholds;
bool g_thresholds_ok = false;

const ByteThresholds* thresholds() {
    std::call_once(g_thresholds_once, [] { g_thresholds_ok = compute_thresholds(g_thresholds); });
    return g_thresholds_ok ? &g_thresholds : nullptr;
}

__device__ __forceinline__ uint8_t to_byte(float v, const float* t) {
    if(isnan(v)) return 0;
    if(v == -INFINITY) return 255;
    if(v < 0.0f) return 0;
    int lo = 0;  // t[lo] <= v
#pragma unroll
    for(int step = 128; step > 0; step >>= 1) {
        if(lo + step <= 255 && t[lo + step] <= v) lo += step;
    }
    return static_cast<uint8_t>(lo);
}

__global__ void __launch_bounds__(256) k_tonemap(const float* __restrict__ rgb, uint32_t width, uint32_t height,
                                                 int flip, uint8_t* __restrict__ out, ByteThresholds table) {
    __shared__ float t[256];
    t[threadIdx.x] = table.t[threadIdx.x];
    __syncthreads();
    const uint64_t row_len = 3ull * width;
    const uint64_t total = row_len * height;
    for(uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < total;
        i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint64_t row = i / row_len;
        const uint64_t col = i - row * row_len;
        const uint64_t dst_row = flip ? (height - 1 - row) : row;
        out[dst_row * row_len + col] = to_byte(__ldg(rgb + i), t);
    }
}

int tonemap_launch(lrt_context* ctx, const float* rgb_dev, uint32_t width, uint32_t height, int flip,
                   uint8_t* bytes_dev) {
    const ByteThresholds* table = thresholds();
    if(!table) return fail(ctx, LRT_ERR_RANGE, "tonemap: the host powf's byte steps are not monotonic");
    const uint64_t total = 3ull * width * height;
    if(total == 0) return LRT_OK;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
    const uint64_t blocks = std::min<uint64_t>((total + 255) / 256, 8ull * sms);
    k_tonemap<<<static_cast<unsigned>(blocks), 256, 0, ctx->stream>>>(rgb_dev, width, height, flip, bytes_dev,
                                                                      *table);
    LRT_CUDA(ctx, cudaGetLastError());
    ctx->stats.kernel_launches += 1;
    return LRT_OK;
}

}  // namespace

int lrt_tonemap_table(float* out) {
    if(!out) return LRT_ERR_INVALID_ARGUMENT;
    const ByteThresholds* table = thresholds();
    if(!table) return LRT_ERR_RANGE;
    std::memcpy(out, table->t, sizeof(table->t));
    return LRT_OK;
}

int lrt_tonemap_dev(lrt_context* ctx, const float* rgb_dev, uint32_t width, uint32_t height, int flip,
                    uint8_t* bytes_dev) {
    if(!ctx) return LRT_ERR_INVALID_ARGUMENT;
    if(width == 0 || height == 0) return LRT_OK;
    if(!rgb_dev || !bytes_dev) return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "null argument");
    LRT_CUDA(ctx, cudaSetDevice(ctx->device));
    return tonemap_launch(ctx, rgb_dev, width, height, flip, bytes_dev);
}

int lrt_tonemap(lrt_context* ctx, const float* rgb, uint32_t width, uint32_t height, int flip, uint8_t* bytes) {
    if(!ctx) return LRT_ERR_INVALID_ARGUMENT;
    if(width == 0 || height == 0) return LRT_OK;
    if(!rgb || !bytes) return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "null argument");
    LRT_CUDA(ctx, cudaSetDevice(ctx->device));
    const size_t n = 3ull * width * height;
    const size_t in_bytes = (4 * n + 255) / 256 * 256;
    LRT_CUDA(ctx, ctx->scratch_a.ensure(in_bytes + n));
    float* d_rgb = ctx->scratch_a.as<float>();
    uint8_t* d_bytes = ctx->scratch_a.as<uint8_t>() + in_bytes;
    LRT_CUDA(ctx, cudaMemcpyAsync(d_rgb, rgb, 4 * n, cudaMemcpyHostToDevice, ctx->stream));
    const int st = tonemap_launch(ctx, d_rgb, width, height, flip, d_bytes);
    if(st != LRT_OK) return st;
    LRT_CUDA(ctx, cudaMemcpyAsync(bytes, d_bytes, n, cudaMemcpyDeviceToHost, ctx->stream));
    LRT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return LRT_OK;
}
