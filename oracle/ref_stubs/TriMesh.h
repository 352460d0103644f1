// Test infrastructure: the part of the trimesh2 library's TriMesh that the reference's CPU
// voxeliser (voxelizer/cpu_voxelizer.cpp) touches, written here so that file compiles unchanged
// (trimesh2 is not in this image): vertex positions and triangle index triples.
#pragma once
#include <vector>

namespace trimesh {

struct vec3 {
    float v[3] = {0, 0, 0};
    vec3() = default;
    vec3(float a, float b, float c) : v{a, b, c} {}
    float& operator[](int i) { return v[i]; }
    float operator[](int i) const { return v[i]; }
};
inline vec3 operator-(const vec3& a, const vec3& b) { return vec3(a[0] - b[0], a[1] - b[1], a[2] - b[2]); }
typedef vec3 point;

struct TriMesh {
    struct Face {
        int v[3] = {0, 0, 0};
        int& operator[](int i) { return v[i]; }
        int operator[](int i) const { return v[i]; }
    };
    std::vector<point> vertices;
    std::vector<Face> faces;
};

}  // namespace trimesh
