// Pieces of the uniform mesh generator shared by the host builder
// (host_setup.cpp) and the GPU builder (lbfs_mesh_gpu.cu).
#pragma once

#include <cstdint>
#include <vector>

#ifdef __CUDACC__
#define LBFS_HD __host__ __device__
#else
#define LBFS_HD
#endif

namespace lbfs {

struct UniformDims {
    int nx, ny, nz;
    double dx, dy, dz;
    int n_cells, n_faces, n_interior, n_bc, n_fx, n_fy, n_fz;
};

// unstructured_mesh::create_uniform_openfoam_mesh, unstructured_mesh.cpp:252-401
UniformDims uniform_dims(double X, double Y, double Z, double dt);

// Vertex coordinates along one axis of n cells (unstructured_mesh.cpp:290-378):
// uniform, cosine-clustered, or the plateau function normalised to the length.
std::vector<double> axis_vertices(int mesh_type, bool clustered, int n, double origin, double length, double step,
                                  double ap, double bp);

// Seeded uniform variate in [-1, 1) for (seed, vertex, axis): splitmix64 of
// the combined key, top 53 bits.  The product and the difference are rounded
// separately on the host and the device alike.
LBFS_HD inline double jitter_unit(uint64_t seed, uint64_t vertex, int axis) {
    uint64_t z = seed * 0x9E3779B97F4A7C15ull + vertex * 3 + (uint64_t)axis + 0x632BE59BD9B4E019ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z = z ^ (z >> 31);
#ifdef __CUDA_ARCH__
    return __dadd_rn(__dmul_rn((double)(z >> 11), 2.0 / 9007199254740992.0), -1.0);
#else
    return (double)(z >> 11) * (2.0 / 9007199254740992.0) - 1.0;
#endif
}

}  // namespace lbfs
