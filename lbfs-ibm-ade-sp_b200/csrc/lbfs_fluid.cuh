// Fluid-side kernels of one LBFS time step (sm_100a).
//
//   K1 cell_gradients : least-squares cell gradients, one thread per interior
//                       cell, the ghost states of its stencil formed in
//                       registers.  Replaces get_interior_gradients
//                       (LBFS.cu:2177-2240) and, for its own use,
//                       update_unstructured_bcs (LBFS.cu:1843-1928).
//   K2 face_flux      : D3Q15 reconstruction at the face lattice nodes,
//                       equilibria, interface BGK relaxation and the face flux,
//                       one thread per face, all in registers.  Replaces
//                       calc_face_flux_x/_y/_z (LBFS.cu:2283-2569),
//                       calc_face_flux (LBFS.cu:2574-2687) and calc_face_flux_bc
//                       (LBFS.cu:2691-2810); the boundary-face thread also
//                       forms and stores its ghost's state and gradients
//                       (update_unstructured_bcs, get_bc_gradients,
//                       LBFS.cu:1933-2048), which keeps that tail and its
//                       registers out of K1.
//   K3 cell_update    : deterministic gather of the face fluxes of each cell,
//                       body + IBM force, forward-Euler update of soln_t1 and
//                       of the primitive state, residual partial sums, status
//                       flags.  Replaces add_face_flux_to_cell (LBFS.cu:2242-2281,
//                       8 CAS atomics per face), add (common_kernels.cu:220-233),
//                       time_integration (LBFS.cu:2089-2172), square + total<128>
//                       (Solver_gpu.cu:1033-1046).
//
// Storage type R is double (the drop-in) or float (the FP32-bulk form).  In
// the float form the density is carried as rho' = rho - rho0 and every
// equilibrium as f' = f - w_k rho0; the two forms are the same algebra (the
// reconstruction and the BGK relaxation are linear in f), except that the
// constant normal-momentum flux rho0/3 * n * area is left out, which cancels
// exactly in the sum over the closed faces of each cell.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

namespace lbfs {

// D3Q15 velocity set (gpu_solver::populate_e_alpha, Solver_gpu.cu:1407-1445):
//   ex = {0, 1,-1, 0, 0, 0, 0, 1,-1, 1,-1, 1,-1,-1, 1}
//   ey = {0, 0, 0, 1,-1, 0, 0, 1,-1, 1,-1,-1, 1, 1,-1}
//   ez = {0, 0, 0, 0, 0, 1,-1, 1,-1,-1, 1, 1,-1, 1,-1}
// as constexpr functions so that fully unrolled loops fold every branch.
__host__ __device__ constexpr int c_ex(int k) {
    return (k == 1 || k == 7 || k == 9 || k == 11 || k == 14) ? 1 : ((k == 2 || k == 8 || k == 10 || k == 12 || k == 13) ? -1 : 0);
}
__host__ __device__ constexpr int c_ey(int k) {
    return (k == 3 || k == 7 || k == 9 || k == 12 || k == 13) ? 1 : ((k == 4 || k == 8 || k == 10 || k == 11 || k == 14) ? -1 : 0);
}
__host__ __device__ constexpr int c_ez(int k) {
    return (k == 5 || k == 7 || k == 10 || k == 11 || k == 13) ? 1 : ((k == 6 || k == 8 || k == 9 || k == 12 || k == 14) ? -1 : 0);
}

// 4-value record with natural vector alignment (32 B in FP64, 16 B in FP32) so
// loads and stores are emitted as vector instructions.
template <typename R> struct alignas(4 * sizeof(R)) Vec4 { R u, v, w, rho; };

template <typename R> __host__ __device__ constexpr R lattice_w(int k) {
    return k == 0 ? R(2.0 / 9.0) : (k < 7 ? R(1.0 / 9.0) : R(1.0 / 72.0));
}

// Equilibrium deviation  f'_k = w_k (rho' (1 + X) + rho0 X),
// X = 3 e.u + q (4.5 (e.u)^2 - 1.5 |u|^2)  (q the preconditioning factor),
// formed as w_k (rho' + (rho' + rho0) X).  With rho0 = 0 it is the reference's
// equilibrium w_k rho (1 + X) (populate_feq_lattice_explicit, LBFS.cu:1041-1354,
// which expands (e.u)^2 into its component products; the same polynomial with
// fewer operations).
template <typename R>
__device__ __forceinline__ R feq_dev(int k, R rho, R u, R v, R w, R rho0, R qscale) {
    const int ex = c_ex(k), ey = c_ey(k), ez = c_ez(k);
    R eu = R(0);
    if (ex) eu = ex > 0 ? eu + u : eu - u;
    if (ey) eu = ey > 0 ? eu + v : eu - v;
    if (ez) eu = ez > 0 ? eu + w : eu - w;
    const R usq = u * u + v * v + w * w;
    const R X = R(3.0) * eu + qscale * (R(4.5) * eu * eu - R(1.5) * usq);
    return lattice_w<R>(k) * (rho + (rho + rho0) * X);
}

// Programmatic dependent launch: a kernel lets the next one on its stream be
// scheduled as soon as all its CTAs have started (pdl_trigger), and the next
// one, launched with the programmatic-serialization attribute, waits in
// pdl_wait until this grid has completed and its writes are visible; before the
// wait it touches nothing a kernel of the step writes.  Without the attribute
// the wait returns at once.
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

}  // namespace lbfs

namespace lbfs {

// Per-boundary-face record used by K1 (ghost state and ghost gradient).
// d = ghost centroid - owner centroid, dmag = |d|, dn = d / dmag
// (get_bc_gradients, LBFS.cu:1968-1979); m = 1 - |face normal| (Neumann);
// gy, gz = ghost centroid y, z (bc types 9 and 10, LBFS.cu:1885-1913).
template <typename R> struct BcRec {
    R dmag, dnx, dny, dnz, mx, my, mz, gy, gz;
};

// Face geometry of an axis-aligned interior face: area, streaming dt,
// t1 = owner centroid - face centroid and t2 = neighbour centroid - face
// centroid along the face axis (LBFS.cu:2313-2315, 2950-2951).
template <typename R> struct alignas(4 * sizeof(R)) AxisFace {
    R area, dt, t1, t2;
};

// Face geometry of a general face (boundary faces always; interior faces of
// meshes that are not axis aligned): area, dt, unit normal, and the full
// vectors t1 = c_owner - x_face, t2 = c_neighbour - x_face (LBFS.cu:335-337).
// bc_branch is 1 on boundary faces that take the boundary reconstruction: the
// reference tests neighbour > n_cells, so the face of the first ghost cell
// (index n_cells) takes the interior branch; in an ensemble, the face of each
// instance's first ghost does.
template <typename R> struct alignas(16) GenFace {
    R area, dt, nx, ny, nz, t1x, t1y, t1z, t2x, t2y, t2z, bc_branch;
};

// Least-squares geometry of one cell: RHS weights of the 6 stencil entries
// (x, y, z each) then LHS^-1 row major, padded to 28 values (16-B multiple).
template <typename R> struct alignas(16) LsRec {
    R rhs[18];
    R lhs[9];
    R pad;
};

// The same geometry folded for K1: per stencil entry q the gradient weights
// W_q = LHS^-1 RHS_q (x, y, z), so that grad = sum_q W_q (s_q - s_i).  The
// reference forms LHS^-1 (sum_q RHS_q (s_q - s_i)) (get_interior_gradients,
// LBFS.cu:2177-2240): the same linear map with its products regrouped
// (rounding differences of a few ulps), and 18 values per cell to load
// instead of 27.
template <typename R> struct alignas(16) LsW {
    R w[18];
};

// Gradients of one cell: grad rho, grad u, grad v, grad w (x, y, z each).
template <typename R> struct alignas(16) GradRec {
    R g[12];
};

// The six faces of cell c of the generator's structured mesh of nx x ny x nz
// cells (x, y, z interior faces in the generator's loop order, then the
// patches left, right, bottom, top, back, front; unstructured_mesh.cpp:415-664)
// in increasing face index, signed as the cell update's face table: +(f + 1)
// where the cell owns face f, -(f + 1) where it is the face's neighbour.
__host__ __device__ inline void grid_cell_faces(int c, int nx, int ny, int nz, int (&cf)[6]) {
    const int i = c % nx, j = (c / nx) % ny, k = c / (nx * ny);
    const int nfx = (nx - 1) * ny * nz, nfy = nx * (ny - 1) * nz, nfz = nx * ny * (nz - 1);
    const int nyz = ny * nz, nxz = nx * nz;
    const int bl = nfx + nfy + nfz, br = bl + nyz, bb = br + nyz, bt = bb + nxz, bk = bt + nxz, bf = bk + nx * ny;
    int f[6], sg[6];
    f[0] = i > 0 ? (i - 1) + (nx - 1) * (j + ny * k) : bl + j + ny * k;
    sg[0] = i > 0 ? -1 : 1;
    f[1] = i < nx - 1 ? i + (nx - 1) * (j + ny * k) : br + j + ny * k;
    sg[1] = 1;
    f[2] = j > 0 ? nfx + i + nx * ((j - 1) + (ny - 1) * k) : bb + i + nx * k;
    sg[2] = j > 0 ? -1 : 1;
    f[3] = j < ny - 1 ? nfx + i + nx * (j + (ny - 1) * k) : bt + i + nx * k;
    sg[3] = 1;
    f[4] = k > 0 ? nfx + nfy + i + nx * (j + ny * (k - 1)) : bk + i + nx * j;
    sg[4] = k > 0 ? -1 : 1;
    f[5] = k < nz - 1 ? nfx + nfy + i + nx * (j + ny * k) : bf + i + nx * j;
    sg[5] = 1;
    for (int a = 1; a < 6; a++)  // insertion sort by face index
        for (int b = a; b > 0 && f[b] < f[b - 1]; b--) {
            const int tf = f[b], ts = sg[b];
            f[b] = f[b - 1]; sg[b] = sg[b - 1];
            f[b - 1] = tf; sg[b - 1] = ts;
        }
#pragma unroll
    for (int q = 0; q < 6; q++) cf[q] = sg[q] * (f[q] + 1);
}

template <typename R> struct FluidArgs {
    int nc, nf, ni, nb, nfx, nfy, nfz, axis_aligned;
    int testcase;
    R rho0;          // density offset of the stored state (0 in FP64)
    R gamma_inv, visc;
    R recon_q;       // quadratic factor of the general-face lattice equilibria: gamma_inv when preconditioning, else 1
    double delta_t, H2, H4;
    double force[3];
    // state and gradients
    Vec4<R> *state;              // [nc+nb]
    R *grad;                     // [12*(nc+nb)] rho(x,y,z) u(x,y,z) v(x,y,z) w(x,y,z)
    // K1 geometry
    const int2 *stencil;         // [3*nc] (6 stencil entries per cell)
    const LsRec<R> *ls;          // [nc] RHS and LHS^-1 (the adjoint's; null for FP32-bulk handles)
    const LsW<R> *lsw;           // [nc] K1's folded weights
    // Meshes whose per-slot weight vectors W_q take at most 8 distinct values
    // (the generator's uniform meshes: +-1/(4 dx) along one axis, in a
    // per-cell order): each cell's six vectors as 3-bit indices into lsw_tab,
    // checked bit for bit at create (null: read lsw)
    const unsigned *lsw_code;    // [nc]
    R lsw_tab[8][3];
    // ls_coded (FP64 handles, with lsw_code): every cell has the same LHS^-1 (ls_lhs) and its RHS
    // vectors are ls_rhs_tab[k] for the same codes; the adjoint reads these instead of ls
    int ls_coded;
    R ls_lhs[9];
    R ls_rhs_tab[8][3];
    const int *bc_rho_type, *bc_vel_type;
    const int *bc_periodic;      // [nb] partner cell of a type-3 ghost (Boundary_Conditions::periodic_node)
    const Vec4<R> *bc_val;       // [nb] (u, v, w, rho - rho0)
    const BcRec<R> *bc_rec;      // [nb]
    // K2 geometry
    const int2 *face_cells;      // [nf] owner, neighbour
    const AxisFace<R> *axis_face;  // [ni] when axis_aligned
    // axis_uniform: every interior face of an axis has the same geometry (the
    // generator's uniform meshes, also across ensemble instances of one
    // spacing), checked bit for bit at create; the interior-face kernels then
    // take it from here instead of reading axis_face, with the owner/neighbour
    // interpolation weights |t2 / (t2 - t1)|, |t1 / (t2 - t1)| formed once
    int axis_uniform;
    R axis_geo[3][4];            // per axis: area, dt, t1, t2
    R axis_wa[3], axis_wb[3];
    const GenFace<R> *gen_face;  // [nb] bc faces, or [nf] when not axis aligned (indexed by face)
    const R *visc_factor;        // [nc]
    Vec4<R> *flux;               // [nf]
    // tiles of tb_flux cells for the face kernel: [3 (n_tiles + 1)], first face of each axis owned by
    // a tile (null: faces not ordered by owner, the per-axis face ranges are used)
    const int *flux_tiles;
    int n_tiles;
    // K3
    const int *cell_faces;       // [6*nc] +(f+1) owner, -(f+1) neighbour
    // grid_faces: the mesh is the generator's structured mesh of grid_n cells (one instance) and its
    // face table is grid_cell_faces's, checked entry for entry at create: K3 forms each cell's faces
    // instead of loading them.  inv_volume_uniform: every cell has the same 1 / volume (bitwise).
    int grid_faces, grid_n[3];
    int inv_volume_uniform;
    double inv_volume_all;
    const double *cell_volume;   // [nc]
    const double *cell_inv_volume;  // [nc] 1 / cell_volume
    // FP32 bulk on meshes whose cell faces do not close: per cell the momentum
    // residual of the constant flux rho0/3 n area that the deviation form
    // leaves out, sum over the faces of -+ rho0/3 n area / volume (null when
    // every cell closes, where it vanishes)
    const double *closure;       // [3 nc]
    double4 *t1;                 // [nc] (u, v, w, rho) conservative accumulator, FP64
    double *res_out;             // [4*nc] residuals kept for parity checks (null = not stored)
    // IBM patches (one per membrane), grouped by ensemble instance
    int n_membranes;
    const void *membrane_scalars;  // MembraneScalars[n_membranes]
    const void *instances;       // InstanceGrid[n_instances]
    const int *cell_instance;    // [nc] instance of each cell; null with one instance
    const double *patch_force;   // [n_membranes * kMaxPatchCells * 3]
    // reductions and flags
    double *partials;            // [4 * gridDim of K3]
    unsigned int *ticket;
    double *residual_sums;       // [4] sum of squares of the last step
    unsigned int *flags;
    // launch shape (read by the host launchers only; lbfs_autotune picks it)
    int tb_grad, tb_flux, tb_gen, tb_update, update_blocks;
    // time stepping other than constant (get_cfl_device, LBFS.cu:2868-2932)
    int time_stepping;           // LBFS_DT_*; 0 or LBFS_DT_CONSTANT: delta_t
    const double4 *cfl;          // [nc] (cfl area x, y, z, cell volume)
    double *dt_local;            // [nc] per-cell step of the current step
    double *dt_min;              // [1] minimum over the cells (the step's delta_t)
    double *dt_partials;         // [kCflBlocks] block minima
    unsigned int *dt_ticket;
    double cfl_factor, cfl_esos, cfl_gamma, cfl_visc, cfl_max_velocity;
};

constexpr int kCflBlocks = 148 * 4;  // grid of the CFL kernel (grid-stride over the cells)

// Up to three ranges of axis-aligned interior faces (x, y, z) for one launch
// of the face flux: a chunk of the pipelined K1 -> K2.
struct FaceRanges {
    int start[3], count[3];
};
constexpr int kMaxFluxChunks = 8;

}  // namespace lbfs
