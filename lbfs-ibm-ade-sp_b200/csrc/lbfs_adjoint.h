// Buffers and launchers of the discrete adjoint (lbfs_adjoint.cu).
#pragma once

#include <cuda_runtime.h>

#include "lbfs_fluid.cuh"
#include "lbfs_kernels.h"

namespace lbfs {

struct AdjointArgs {
    double dt;                   // time-marching step
    double4 *lam_t1;             // [nc] adjoint of soln_t1 (mom x, y, z, mass)
    double *lam_face;            // [2][nf][16] per side (owner, then neighbour) and face: state (4), grad (12)
    int nf;                      // faces (the stride between the two sides)
    double *lam_bcv;             // [4 nb] Dirichlet boundary values seen by the boundary-face reconstruction
    double *lam_rs;              // [12 nc] lambda_R = LHS^-T lambda_grad per cell
    double *lam_state;           // [4 nc] state adjoint from the cell's faces, ghosts and stencil self terms
    const int *tst_start;        // [nc + 1] transposed gradient stencil (interior entries only)
    const int *tst;              // codes 8 i + q: cell i uses this cell as its stencil entry q
    double *sigma_acc;           // [nc] d J / d sigma per cell, summed over the steps
    const double *lam_u_ibm;     // [3 nc] adjoint of the cell velocities through the IBM interpolation (or null)
};

// Membrane part of the adjoint (lbfs_adjoint_mem.cu).
struct MemAdjArgs {
    double dt;
    const double4 *lam_t1;       // fluid adjoint of t1_{n+1}: the IBM force adjoint is dt * its momentum part
    double *lam_x;               // [3 N] node-position adjoint, carried between steps (in: x_{n+1}, out: x_n)
    double *lam_xp;              // [3 N] adjoint of x' = x_{n+1} within the step
    double *lam_F;               // [3 N] node-force adjoint
    double *adjm;                // [17 S] spring adjoint per input direction
    double *lam_mad;             // [M] MAD adjoint, carried (in: MAD_{n+1}, out: MAD_n)
    double *red;                 // [5 M] per-membrane sums of the step
    double *gs_acc, *kb_acc;     // [M] d J / d G_s, d J / d k_b, summed over the steps
    const double *mad_n;         // [M] MAD at the start of the step
    const int *tri_start;        // [N + 1] node -> triangle incidence
    const int *tri_inc;          // codes 4 t + vertex
    const double *xn, *yn, *zn;  // node positions at the start of the step
    double *lam_u_ibm;           // [3 nc] cell velocity adjoint through the IBM interpolation
    MembraneArgs mb;             // sort / spread buffers of the interpolation transpose (positions xn)
};

void launch_adjm_get_mad(const MembraneArgs &A, double *out, cudaStream_t s);
void launch_adjm_set_mad(const MembraneArgs &A, const double *in, cudaStream_t s);
void launch_adj_membrane_sort(const MemAdjArgs &J, cudaStream_t s);
int launch_adj_membrane(const MembraneArgs &A, const MemAdjArgs &J, int nc, const int *cell_instance,
                        const InstanceGrid *instances, cudaStream_t s);

void launch_adj_prim(const FluidArgs<double> &a, cudaStream_t s);

// Up to kMaxCopyJobs device-to-device copies of doubles in one launch (the
// per-step stores of the segment re-run): job q copies n[q] values,
// dst[q][i] = src[q][i * src_stride[q]].
constexpr int kMaxCopyJobs = 12;
struct CopyList {
    const double *src[kMaxCopyJobs];
    double *dst[kMaxCopyJobs];
    long long n[kMaxCopyJobs];
    int src_stride[kMaxCopyJobs];
    int count;
    void add(const void *from, void *to, long long doubles, int stride = 1) {
        if (doubles <= 0) return;
        src[count] = static_cast<const double *>(from);
        dst[count] = static_cast<double *>(to);
        n[count] = doubles;
        src_stride[count] = stride;
        count++;
    }
};
void launch_copy_list(const CopyList &l, cudaStream_t s);
void launch_adj_velocity_seed(const FluidArgs<double> &a, const AdjointArgs &j, const double *weights, cudaStream_t s);
int launch_adj_fluid(const FluidArgs<double> &a, const AdjointArgs &j, cudaStream_t s);
// the phases of launch_adj_fluid: A1 on axis and on general faces (independent,
// disjoint face records), A2 after both, A3 after A2 and the membrane part
void launch_adj_flux_axis(const FluidArgs<double> &a, const AdjointArgs &j, cudaStream_t s);
void launch_adj_flux_general(const FluidArgs<double> &a, const AdjointArgs &j, cudaStream_t s);
// pdl: launched as a programmatic dependent launch behind the kernel before it on the stream
void launch_adj_cells(const FluidArgs<double> &a, const AdjointArgs &j, cudaStream_t s, bool pdl = false);
void launch_adj_gather(const FluidArgs<double> &a, const AdjointArgs &j, cudaStream_t s, bool pdl = false);

}  // namespace lbfs
