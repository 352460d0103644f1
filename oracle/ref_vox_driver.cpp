// Test infrastructure: drives the reference's CPU solid voxeliser
// (voxelizer/cpu_voxelizer.cpp:262-322, cpu_voxelize_mesh_solid), compiled unchanged against the
// GLM and trimesh2 stand-ins in ref_stubs/, on a mesh and a voxel box given by the caller, so the
// oracle's voxeliser can be checked against it.  Only tests load the library.
#include <cstdint>
#include <cstring>

#include "cpu_voxelizer.h"

extern "C" __attribute__((visibility("default"))) void ref_voxelize_solid(const float* coords, long nvert,
                                                                         const int* tris, long ntri,
                                                                         const float bmin[3], const float bmax[3],
                                                                         int reso, uint32_t* bits) {
    trimesh::TriMesh mesh;
    mesh.vertices.resize(nvert);
    for (long i = 0; i < nvert; i++) mesh.vertices[i] = trimesh::point(coords[3 * i], coords[3 * i + 1], coords[3 * i + 2]);
    mesh.faces.resize(ntri);
    for (long t = 0; t < ntri; t++)
        for (int k = 0; k < 3; k++) mesh.faces[t][k] = tris[3 * t + k];
    AABox<glm::vec3> box(glm::vec3(bmin[0], bmin[1], bmin[2]), glm::vec3(bmax[0], bmax[1], bmax[2]));
    voxinfo info(box, glm::uvec3(reso, reso, reso), (size_t)ntri);
    const size_t words = ((size_t)reso * reso * reso + 31) / 32;
    memset(bits, 0, words * 4);
    cpu_voxelizer::cpu_voxelize_mesh_solid(info, &mesh, bits, false);
}
