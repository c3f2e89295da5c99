// Internal declarations shared by the host runtime and the kernels.
#pragma once

#include <cstdint>
#include <string>

#include "lbfs_b200.h"

namespace lbfs {

// Thread-local last-error text behind lbfs_last_error; returns `code`.
int set_error(int code, const std::string &msg);

// Returns the error status of a failed CUDA runtime call from the enclosing
// entry point (allocation failures as LBFS_ERR_NOMEM).
#define LBFS_CUDA(call)                                                                                  \
    do {                                                                                                 \
        cudaError_t e_ = (call);                                                                         \
        if (e_ != cudaSuccess)                                                                           \
            return lbfs::set_error(e_ == cudaErrorMemoryAllocation ? LBFS_ERR_NOMEM : LBFS_ERR_CUDA,     \
                                   std::string(#call) + ": " + cudaGetErrorString(e_));                  \
    } while (0)

// Geometry and least-squares matrices of a hex mesh given as lists (float
// vertices, four vertex ids per face, owner per face, neighbour per interior
// face; boundary neighbours are written as their ghosts) built on GPU
// `device` (lbfs_mesh_gpu.cu): the host routine's arrays bit for bit.
int mesh_geometry_gpu(int device, int np, int nc, int nf, int ni, const float *vx, const float *vy, const float *vz,
                      const int *fv, const int32_t *owner, int32_t *neighbour, double visc, double fneq_min,
                      int32_t gradient_hybrid, bool closed_faces, double *face_area, double *face_normal,
                      double *face_centroid, double *streaming_dt, double *cell_volume, double *cell_centroid,
                      int32_t *gradient_stencil, double *lhs_inverse, double *rhs);

// Largest membrane patch (cells of the IBM stencil's bounding box) a membrane
// may cover; 48^3 cells covers a red cell of radius 8 cells deformed to twice
// its diameter with the 4-point stencil margin.
constexpr int kMaxPatchCells = 48 * 48 * 48;
// Threads of the one-CTA-per-membrane kernel (512 leaves 128 registers per
// thread for the spring-force derivatives).
constexpr int kMembraneThreads = 1024;
// Largest membrane handled by one CTA (nodes; springs = 3 (nodes - 2)).
constexpr int kMaxMembraneNodes = 16384;

// D3Q15 weights and velocities, ordering of gpu_solver::populate_e_alpha
// (Solver_gpu.cu:1407-1445).
constexpr int kQ = 15;

// Per-membrane device-side scalars (one record per membrane).
struct MembraneScalars {
    double V, V0, A, A0, MAD, MAD0;
    double Vc, Ac;                   // current totals from the totals kernel (when it runs)
    double bbox_lo[3], bbox_hi[3];   // node coordinate bounds (interior viscosity test)
    int patch_lo[3], patch_dim[3];   // IBM patch: first cell and extent per axis
    int patch_cells;                 // product of patch_dim (0 when the patch overflowed)
    int patch_off;                   // first cell of this membrane's slice of the patch arrays (set at create)
};

// Per-membrane constants (moduli) and ranges into the concatenated arrays.
struct MembraneConst {
    int node0, n_nodes, tri0, n_tris, spring0, n_springs;
    int inc0;  // start of this membrane's node->(spring,slot) incidence list
    int periodic;  // lagrangian_object::periodic (check_periodic_object)
    double volume_modulus, local_area_modulus, global_area_modulus, shear_modulus;
    double global_bending_modulus, local_bending_modulus, membrane_thickness, viscosity;
    double wlc_ratio, curvature_ratio, volume_ratio, internal_viscosity_ratio, reference_length;
    int pivkin_length, sphere_reference;
    // IBM grid of the membrane's instance
    int cell0, gnx, gny, gnz;
    double gorigin[3], gdx, gdh;
    int instance, patch_bound;  // patch cells the spread launch covers
    double domain_z0, domain_Z;  // origin_z and Z of the instance's domain (check_periodic_object)
};

// One ensemble instance as the kernels see it.
struct InstanceGrid {
    int cell0, nx, ny, nz;
    int mem0, mem1;  // membranes [mem0, mem1) live in this instance
    int pad0, pad1;
};

}  // namespace lbfs
