// Buffers and launchers of the discrete adjoint (lbfs_adjoint.cu).
#pragma once

#include <cuda_runtime.h>

#include "lbfs_fluid.cuh"
#include "lbfs_kernels.h"

namespace lbfs {

struct AdjointArgs {
    double dt;                   // time-marching step
    double4 *lam_t1;             // [nc] adjoint of soln_t1 (mom x, y, z, mass)
    double *lam_face;            // [32 nf] per face: owner state, neighbour state, owner grad, neighbour grad
    double *lam_bcv;             // [4 nb] Dirichlet boundary values seen by the boundary-face reconstruction
    double *lam_rs;              // [12 nc] lambda_R = LHS^-T lambda_grad per cell
    double *lam_state;           // [4 nc] state adjoint from the cell's faces, ghosts and stencil self terms
    const int *tst_start;        // [nc + 1] transposed gradient stencil (interior entries only)
    const int *tst;              // codes 8 i + q: cell i uses this cell as its stencil entry q
    double *sigma_acc;           // [nc] d J / d sigma per cell, summed over the steps
    const double *lam_u_ibm;     // [3 nc] adjoint of the cell velocities through the IBM interpolation (or null)
};

void launch_adj_prim(const FluidArgs<double> &a, cudaStream_t s);
void launch_adj_velocity_seed(const FluidArgs<double> &a, const AdjointArgs &j, const double *weights, cudaStream_t s);
int launch_adj_fluid(const FluidArgs<double> &a, const AdjointArgs &j, cudaStream_t s);

}  // namespace lbfs
