// lrt_autotune.cu — launch-shape autotuner of lrt_render_batch (C ABI lrt_autotune).
//
// Three knobs change only the speed of a batch, never its images: paths per wave, resident blocks per
// SM of every grid, and the path order inside a job (bands of pixel_tile rows walked column by
// column). The tuner times the caller's jobs, with spp scaled so that one trial holds about 150M
// paths, over the candidates of one knob at a time (coordinate descent from the library defaults),
// keeps the fastest configuration on the context, and caches it in a text file keyed by the scene's
// and the batch's size class: triangles and paths rounded up to powers of two, material and emitter
// counts.
#include "lrt_context.cuh"

#include <cmath>
#include <cstdio>
#include <fstream>
#include <sstream>

namespace lrt {

namespace {

constexpr uint64_t kPathsPerTrial = 150000000ull;
constexpr int kRepeats = 2;
const uint32_t kWaveCandidates[] = {1u << 19, 1u << 20, 1u << 21, 1u << 22, 1u << 23, 1u << 24};
const uint32_t kTileCandidates[] = {1u, 4u, 8u, 16u};
const uint32_t kBlockCandidates[] = {0u, 2u, 3u};

struct Config {
    uint32_t knob[3];  // wave_capacity, pixel_tile, blocks_per_sm
};

uint32_t ceil_log2(uint64_t x) { return x <= 1 ? 0u : 64u - static_cast<uint32_t>(__builtin_clzll(x - 1)); }

void apply(lrt_context* ctx, const Config& c) {
    ctx->wave_capacity = c.knob[0];
    ctx->pixel_tile = c.knob[1];
    ctx->blocks_per_sm_cap = c.knob[2];
}

// seconds of the fastest of kRepeats renders after one warm render (CUDA events on the context's stream)
int time_batch(lrt_context* ctx, const std::vector<lrt_job_desc>& jobs, int32_t max_depth, int32_t rr_depth,
               float* rgb_dev, float& seconds) {
    int st = lrt_render_batch_dev(ctx, jobs.data(), static_cast<uint32_t>(jobs.size()), max_depth, rr_depth, rgb_dev);
    if(st != LRT_OK) return st;
    cudaEvent_t e0, e1;
    LRT_CUDA(ctx, cudaEventCreate(&e0));
    LRT_CUDA(ctx, cudaEventCreate(&e1));
    float best = INFINITY;
    for(int r = 0; r < kRepeats && st == LRT_OK; ++r) {
        cudaEventRecord(e0, ctx->stream);
        st = lrt_render_batch_dev(ctx, jobs.data(), static_cast<uint32_t>(jobs.size()), max_depth, rr_depth, rgb_dev);
        cudaEventRecord(e1, ctx->stream);
        float ms = 0.0f;
        if(st == LRT_OK && cudaEventSynchronize(e1) == cudaSuccess && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess) {
            best = std::min(best, ms * 1e-3f);
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    seconds = best;
    return st;
}

bool read_cache(const char* path, const std::string& key, Config& c, float& seconds) {
    std::ifstream in(path);
    std::string line;
    bool found = false;
    while(std::getline(in, line)) {  // the last line of a key wins
        std::istringstream ls(line);
        std::string k;
        Config t{};
        float s = 0.0f;
        if(ls >> k >> t.knob[0] >> t.knob[1] >> t.knob[2] >> s && k == key) {
            c = t;
            seconds = s;
            found = true;
        }
    }
    return found;
}

}  // namespace

}  // namespace lrt

using namespace lrt;

extern "C" {

int lrt_autotune(lrt_context* ctx, const lrt_job_desc* jobs, uint32_t n_jobs, int32_t max_depth, int32_t rr_depth,
                 float* rgb_dev, const char* cache_path, lrt_launch_config* out) {
    if(!ctx) return LRT_ERR_INVALID_ARGUMENT;
    if(!ctx->has_scene) return fail(ctx, LRT_ERR_NO_SCENE, "no scene uploaded");
    if(!jobs || n_jobs == 0 || !rgb_dev || !out) return fail(ctx, LRT_ERR_INVALID_ARGUMENT, "null argument or no jobs");
    LRT_CUDA(ctx, cudaSetDevice(ctx->device));
    uint64_t tris = 0, paths = 0;
    for(const ObjRec& o : ctx->host.objects) {
        if(o.kind == LRT_OBJECT_MESH) tris += o.n_tris;
    }
    for(uint32_t j = 0; j < n_jobs; ++j) paths += static_cast<uint64_t>(jobs[j].width) * jobs[j].height * jobs[j].spp;
    char key[128];
    snprintf(key, sizeof(key), "tris2^%u_mats%zu_emitters%zu_paths2^%u", ceil_log2(std::max<uint64_t>(1, tris)),
             ctx->host.materials.size(), ctx->host.emitters.size(), ceil_log2(std::max<uint64_t>(1, paths)));

    Config best{{1u << 24, 1u, 0u}};
    float best_s = 0.0f;
    if(cache_path && read_cache(cache_path, key, best, best_s)) {
        apply(ctx, best);
        *out = lrt_launch_config{best.knob[0], best.knob[1], best.knob[2], 1u, best_s, 0u};
        return LRT_OK;
    }

    // the jobs with spp scaled so that a trial holds about kPathsPerTrial paths
    std::vector<lrt_job_desc> trial(jobs, jobs + n_jobs);
    const double f = std::min(1.0, static_cast<double>(kPathsPerTrial) / static_cast<double>(std::max<uint64_t>(1, paths)));
    for(lrt_job_desc& j : trial) j.spp = std::max<uint32_t>(1, static_cast<uint32_t>(std::lround(j.spp * f)));

    const Config saved{{ctx->wave_capacity, ctx->pixel_tile, ctx->blocks_per_sm_cap}};
    apply(ctx, best);
    int st = time_batch(ctx, trial, max_depth, rr_depth, rgb_dev, best_s);
    uint32_t trials = 1;
    const uint32_t* candidates[3] = {kWaveCandidates, kTileCandidates, kBlockCandidates};
    const size_t n_candidates[3] = {sizeof(kWaveCandidates) / 4, sizeof(kTileCandidates) / 4, sizeof(kBlockCandidates) / 4};
    for(int knob = 0; knob < 3 && st == LRT_OK; ++knob) {
        const uint32_t start = best.knob[knob];  // timed already, with the other knobs as they are now
        for(size_t c = 0; c < n_candidates[knob] && st == LRT_OK; ++c) {
            if(candidates[knob][c] == start) continue;
            Config cfg = best;
            cfg.knob[knob] = candidates[knob][c];
            apply(ctx, cfg);
            float s = INFINITY;
            st = time_batch(ctx, trial, max_depth, rr_depth, rgb_dev, s);
            ++trials;
            if(st == LRT_OK && s < best_s) {
                best = cfg;
                best_s = s;
            }
        }
    }
    if(st != LRT_OK) {
        apply(ctx, saved);
        return st;
    }
    apply(ctx, best);
    if(cache_path) {
        FILE* fcache = fopen(cache_path, "a");
        if(!fcache) return fail(ctx, LRT_ERR_IO, "autotune cache %s: cannot append", cache_path);
        fprintf(fcache, "%s %u %u %u %.6g\n", key, best.knob[0], best.knob[1], best.knob[2], best_s);
        fclose(fcache);
    }
    *out = lrt_launch_config{best.knob[0], best.knob[1], best.knob[2], 0u, best_s, trials};
    return LRT_OK;
}

}  // extern "C"
