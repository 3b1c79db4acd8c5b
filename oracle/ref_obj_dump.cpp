/* oracle/ref_obj_dump.cpp — test infrastructure: runs the UNMODIFIED reference loader load_obj
 * (src/io/obj_loader.h:44-141) on one file and writes the loaded triangle_mesh's arrays:
 *   uint32 n_vertices, uint32 n_indices, float positions[3 n_vertices], uint32 indices[n_indices],
 *   float corner_normals[3 n_indices]   (little endian)
 * Exit code 1 when load_obj returns no mesh, 2 on a usage or output error. Built into oracle/_ref by
 * oracle/Makefile; the tests compare liblrt's lrt_load_obj with it. */
#include <cstdint>
#include <cstdio>

#define private public
#include "io/obj_loader.h"
#undef private

int main(int argc, char** argv) {
    if(argc != 3) return 2;
    const auto mesh = LinRT::load_obj(argv[1]);
    if(!mesh) return 1;
    std::FILE* f = std::fopen(argv[2], "wb");
    if(!f) return 2;
    const uint32_t counts[2] = {static_cast<uint32_t>(mesh->positions.size()), static_cast<uint32_t>(mesh->indices.size())};
    std::fwrite(counts, 4, 2, f);
    for(const auto& p : mesh->positions) {
        const float v[3] = {p.x, p.y, p.z};
        std::fwrite(v, 4, 3, f);
    }
    std::fwrite(mesh->indices.data(), 4, mesh->indices.size(), f);
    for(const auto& n : mesh->corner_normals) {
        const float v[3] = {n.x, n.y, n.z};
        std::fwrite(v, 4, 3, f);
    }
    return std::fclose(f) == 0 ? 0 : 2;
}
