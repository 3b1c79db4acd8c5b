/* lrt_oracle.h — TEST INFRASTRUCTURE: a plain-C restatement of the integer and bit-exact parts of the
 * LinRT hot path, used only by tests as an independent checker (never by the library or its bench).
 *
 *   sampler      src/core/sampler.h:12-33, src/core/sobol.h:12-106
 *   traversal    src/accelerator/sah_kdtree.h:62-121 over a packed tree, with the Moller-Trumbore
 *                test of src/geometry/triangle_mesh.h:43-99
 *   k-NN         the set photon_map::nearest returns (src/integrator/photonmapper/photon_map.h:117-165):
 *                the k smallest squared distances not above r2, found here by brute force
 */
#ifndef LRT_ORACLE_H
#define LRT_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

void oro_sobol_table(uint32_t table[16][32]);
/* the value of dimension `dim` of sampler.start(pixel, sample) */
float oro_sampler_value(uint32_t pixel, uint32_t sample, uint32_t dim);

/* closest hit of one ray against one mesh's packed kd-tree (two uint32 words per node: interior =
 * split bits, right << 2 | axis; leaf = first, count << 2 | 3). Returns 1 on a hit. */
int oro_mesh_hit(const uint32_t* nodes, const uint32_t* refs, const float* positions, const uint32_t* indices,
                 const float origin[3], const float direction[3], float t_min, float* closest, uint32_t* tri,
                 float* u, float* v);

/* up to k (index, d2) pairs with the smallest d2 <= r2, sorted by (d2, index) descending; returns count */
uint32_t oro_knn(const float* positions, uint32_t n, const float point[3], float r2, uint32_t k, uint32_t* idx,
                 float* d2);

#ifdef __cplusplus
}
#endif

#endif
