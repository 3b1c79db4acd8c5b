/* lrt_oracle.c — TEST INFRASTRUCTURE (see lrt_oracle.h). Compiled with -ffp-contract=off: every float
 * product and sum is rounded separately, as in the reference's own x86-64 build. */
#include "lrt_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ---- Sobol: src/core/sobol.h:12-41 (sample_bits, mix_bits) and 44-106 (direction numbers) ---- */

static uint32_t mix_bits(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

void oro_sobol_table(uint32_t table[16][32]) {
    /* degree, polynomial coefficient bits a, initial m_1..m_degree (Joe & Kuo, dimensions 2..16) */
    static const uint32_t poly[15][8] = {
        {1, 0, 1},           {2, 1, 1, 3},          {3, 1, 1, 3, 1},       {3, 2, 1, 1, 1},
        {4, 1, 1, 1, 3, 3},  {4, 4, 1, 3, 5, 13},   {5, 2, 1, 1, 5, 5, 17}, {5, 4, 1, 1, 5, 5, 5},
        {5, 7, 1, 1, 7, 11, 19}, {5, 11, 1, 1, 5, 1, 1}, {5, 13, 1, 1, 1, 3, 11}, {5, 14, 1, 3, 5, 5, 13},
        {6, 1, 1, 3, 3, 9, 7, 49}, {6, 13, 1, 1, 1, 15, 21, 21}, {6, 16, 1, 3, 1, 13, 27, 49},
    };
    for(int b = 0; b < 32; ++b) table[0][b] = 1u << (31 - b);
    for(int d = 0; d < 15; ++d) {
        const uint32_t s = poly[d][0], a = poly[d][1];
        uint32_t m[33] = {0};
        for(uint32_t i = 1; i <= s; ++i) m[i] = poly[d][1 + i];
        for(uint32_t i = s + 1; i <= 32; ++i) {
            uint32_t v = (m[i - s] << s) ^ m[i - s];
            for(uint32_t k = 1; k < s; ++k) {
                if((a >> (s - 1 - k)) & 1u) v ^= m[i - k] << k;
            }
            if(i < 32) v &= (1u << i) - 1u;
            m[i] = v;
        }
        for(int i = 1; i <= 32; ++i) table[d + 1][i - 1] = m[i] << (32 - i);
    }
}

float oro_sampler_value(uint32_t pixel, uint32_t sample, uint32_t dim) {
    static uint32_t table[16][32];
    static int ready = 0;
    if(!ready) {
        oro_sobol_table(table);
        ready = 1;
    }
    uint32_t bits;
    if(dim >= 16) {
        bits = mix_bits(sample + dim * 0x9e3779b9u);
    } else {
        const uint32_t gray = sample ^ (sample >> 1);
        bits = 0;
        for(int b = 0; b < 32; ++b) {
            if((gray >> b) & 1u) bits ^= table[dim][b];
        }
    }
    const uint32_t scramble = mix_bits(mix_bits(pixel) + dim * 0x9e3779b9u);
    return (float)(bits ^ scramble) * (1.0f / 4294967296.0f);
}

/* ---- kd-tree traversal + Moller-Trumbore ---- */

static float fmin_ref(float a, float b) { return (b < a) ? b : a; } /* std::min */

static float dot3(const float* a, const float* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
static void cross3(const float* a, const float* b, float* o) {
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}

static int hit_triangle(const float* positions, const uint32_t* indices, uint32_t t_index, const float* o,
                        const float* d, float t0, float t1, float* closest, float* uo, float* vo) {
    const float* p0 = positions + 3 * indices[3 * t_index];
    const float* p1 = positions + 3 * indices[3 * t_index + 1];
    const float* p2 = positions + 3 * indices[3 * t_index + 2];
    float e1[3], e2[3], g[3], pvec[3], tvec[3], qvec[3];
    for(int i = 0; i < 3; ++i) {
        e1[i] = p1[i] - p0[i];
        e2[i] = p2[i] - p0[i];
    }
    cross3(e1, e2, g);
    if(g[0] * g[0] + g[1] * g[1] + g[2] * g[2] <= 0.0f) return 0;
    cross3(d, e2, pvec);
    const float det = dot3(e1, pvec);
    if(fabsf(det) < 1e-8f) return 0;
    const float inv_det = 1.0f / det;
    for(int i = 0; i < 3; ++i) tvec[i] = o[i] - p0[i];
    const float u = dot3(tvec, pvec) * inv_det;
    if(u < 0.0f || u > 1.0f) return 0;
    cross3(tvec, e1, qvec);
    const float v = dot3(d, qvec) * inv_det;
    if(v < 0.0f || u + v > 1.0f) return 0;
    const float t = dot3(e2, qvec) * inv_det;
    if(t < t0 || t > t1) return 0;
    *closest = t;
    *uo = u;
    *vo = v;
    return 1;
}

int oro_mesh_hit(const uint32_t* nodes, const uint32_t* refs, const float* positions, const uint32_t* indices,
                 const float origin[3], const float direction[3], float t_min, float* closest, uint32_t* tri,
                 float* u, float* v) {
    struct item {
        uint32_t node;
        float mint, maxt;
    } stack[48];
    int top = 0, hit_any = 0;
    float mint = t_min, maxt = *closest;
    uint32_t node = 0;
    for(;;) {
        if(*closest < mint) break;
        const uint32_t w0 = nodes[2 * node], w1 = nodes[2 * node + 1];
        if((w1 & 3u) == 3u) {
            const uint32_t count = w1 >> 2;
            float limit = fmin_ref(maxt, *closest);
            for(uint32_t i = 0; i < count; ++i) {
                if(hit_triangle(positions, indices, refs[w0 + i], origin, direction, mint, limit, closest, u, v)) {
                    hit_any = 1;
                    *tri = refs[w0 + i];
                }
                limit = fmin_ref(maxt, *closest);
            }
            if(top == 0) break;
            --top;
            node = stack[top].node;
            mint = stack[top].mint;
            maxt = stack[top].maxt;
            continue;
        }
        const uint32_t axis = w1 & 3u, right = w1 >> 2;
        float split;
        memcpy(&split, &w0, 4);
        const float t_plane = (split - origin[axis]) * (1.0f / direction[axis]);
        const int left_of_split = origin[axis] < split || (origin[axis] == split && direction[axis] <= 0.0f);
        const uint32_t first = left_of_split ? node + 1 : right;
        const uint32_t second = left_of_split ? right : node + 1;
        if(t_plane > maxt || t_plane <= 0.0f) {
            node = first;
        } else if(t_plane < mint) {
            node = second;
        } else {
            if(top >= 48) return -1;
            stack[top].node = second;
            stack[top].mint = t_plane;
            stack[top].maxt = maxt;
            ++top;
            node = first;
            maxt = t_plane;
        }
    }
    return hit_any;
}

/* ---- k-NN by brute force ---- */

typedef struct {
    float d2;
    uint32_t idx;
} pair_t;

static int pair_desc(const void* a, const void* b) {
    const pair_t* x = (const pair_t*)a;
    const pair_t* y = (const pair_t*)b;
    if(x->d2 != y->d2) return x->d2 < y->d2 ? 1 : -1;
    return x->idx < y->idx ? 1 : (x->idx > y->idx ? -1 : 0);
}

uint32_t oro_knn(const float* positions, uint32_t n, const float point[3], float r2, uint32_t k, uint32_t* idx,
                 float* d2) {
    pair_t* all = (pair_t*)malloc(sizeof(pair_t) * (n ? n : 1));
    uint32_t m = 0;
    for(uint32_t i = 0; i < n; ++i) {
        const float dx = positions[3 * i] - point[0];
        const float dy = positions[3 * i + 1] - point[1];
        const float dz = positions[3 * i + 2] - point[2];
        const float d = dx * dx + dy * dy + dz * dz;
        if(d <= r2) {
            all[m].d2 = d;
            all[m].idx = i;
            ++m;
        }
    }
    qsort(all, m, sizeof(pair_t), pair_desc);
    const uint32_t keep = m < k ? m : k;
    for(uint32_t j = 0; j < keep; ++j) { /* the k smallest, still in descending order */
        idx[j] = all[m - keep + j].idx;
        d2[j] = all[m - keep + j].d2;
    }
    free(all);
    return keep;
}
