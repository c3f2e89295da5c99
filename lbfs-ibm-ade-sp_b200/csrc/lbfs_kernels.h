// Launch wrappers shared by the runtime and the kernel files.
#pragma once

#include <cuda_runtime.h>

#include "lbfs_fluid.cuh"
#include "lbfs_internal.h"

namespace lbfs {

constexpr int kK3MaxBlocks = 148 * 8;      // default grid cap of the cell update (grid-stride)
constexpr int kSpreadMaxBlocks = 148 * 8;  // default spread grid cap (grid-stride over the tiles)
constexpr int kK3PatchCache = 32;          // membranes whose patches the cell update caches per block
constexpr int kK3BlocksLimit = LBFS_MAX_UPDATE_BLOCKS;  // partial-sum slots allocated for the update

template <typename R> void launch_fluid_gradients(const FluidArgs<R> &a, cudaStream_t s);
// K1 over cells [begin, end) and K2 over up to three axis face ranges (the pipelined form)
template <typename R> void launch_fluid_gradients_range(const FluidArgs<R> &a, int begin, int end, cudaStream_t s);
template <typename R> void launch_fluid_flux_axis_ranges(const FluidArgs<R> &a, const FaceRanges &r, cudaStream_t s);
// K2 over the faces owned by tiles [tile0, tile1) of a.flux_tiles (axis-aligned meshes whose faces are
// ordered by owner within each axis)
template <typename R>
void launch_fluid_flux_tiles(const FluidArgs<R> &a, int tile0, int tile1, cudaStream_t s, bool pdl = false);
template <typename R> void launch_fluid_flux(const FluidArgs<R> &a, cudaStream_t s);
// pdl: launched with the programmatic-serialization attribute, directly behind
// the gradient kernel on the same stream
template <typename R> void launch_fluid_flux_axis(const FluidArgs<R> &a, cudaStream_t s, bool pdl = false);
template <typename R> void launch_fluid_flux_general(const FluidArgs<R> &a, cudaStream_t s);
// pdl: launched with the programmatic-serialization attribute behind the face kernels
template <typename R> void launch_fluid_update(const FluidArgs<R> &a, cudaStream_t s, bool pdl = false);
// per-cell step and its minimum (time stepping other than constant)
template <typename R> void launch_fluid_cfl(const FluidArgs<R> &a, cudaStream_t s);
// stage = 4 planes of n_cells doubles (rho, u, v, w); pack also resets soln_t1
// to the primitive state (Solver_gpu.cu:746)
template <typename R> void launch_pack_state(const FluidArgs<R> &a, const double *stage, cudaStream_t s);
template <typename R> void launch_unpack_state(const FluidArgs<R> &a, double *stage, cudaStream_t s);

// Membrane work modes.
enum MembraneMode : int {
    kModeReference = 0,  // stress-free mesh: contour lengths, spring constants, reference curvature
    kModeInitial = 1,    // initial mesh: V0, A0, MAD0, spring_area_0, spring_angle_0
    kModeStep = 2,       // one time step: interpolate, advect, forces, spread
};




// Spring blocks of 128 per membrane the MAD partials can hold.
constexpr int kMaxSpringBlocks = (3 * kMaxMembraneNodes + 127) / 128;

struct MembraneArgs {
    int n_membranes;
    int mode;
    int ibm_stencil;             // 2 or 4
    double delta_t;
    const double *dt_dev;        // [1] the step's delta_t on the device (time stepping not constant), else null
    // fluid state (read) and IBM grid
    const void *state;           // Vec4<R>[nc]
    int state_is_float;
    int nc;
    // membranes
    const MembraneConst *mc;     // [n_membranes]
    MembraneScalars *ms;         // [n_membranes]
    const int *tri;              // [3*total_tris]   global node ids
    const int *spring;           // [4*total_springs] global node ids
    const int *inc;              // node -> 4*spring + slot, CSR by node (in spring order)
    const int *inc_start;        // [total_nodes + 1]
    double *x, *y, *z;           // node positions [total_nodes]
    double *vx, *vy, *vz;        // node velocities
    double *fx, *fy, *fz;        // node forces
    double *contour, *kspring, *curv, *curv0, *angle0, *area0, *area; // per spring (area, area0: 2 per spring)
    double *contrib;             // [12*total_springs] per-spring node forces (scratch)
    unsigned long long *keys;    // [total_nodes] bin keys (scratch)
    double *patch_force;         // [sum of patch_bound * 3], membrane m from cell ms[m].patch_off
    unsigned int *flags;
    int sort_capacity;           // power of two >= nodes of the largest membrane
    int max_nodes;               // nodes of the largest membrane
    int total_nodes, total_springs;
    const int *spring_mem;       // [total_springs] membrane of each spring
    int *bin_start;              // [sum of (patch_bound + 1)] first sorted node of each bin, from patch_off + m
    int *bin_cursor;             // [sum of (patch_bound + 1)] placement cursors of the node sort (scratch)
    int *cell_start;             // [n_membranes + 1] first spread cell of each membrane (prefix over patches)
    unsigned int *sort_ticket;   // membranes whose patch is known in this launch; zero between launches
    int spread_blocks;           // grid of the spread kernel (grid-stride over the tiles)
    int force_cluster;           // 8 or 16: totals, node sort, spring and node forces as one cluster of
                                 // that many CTAs per membrane (k_mem_step); 0: four kernels
    int *node_base;              // [3 total_nodes] first IBM stencil cell per axis at the current positions
    double *node_w;              // [12 total_nodes] 1D stencil weights per axis (4 slots) at the current positions
    int *sorted_node;            // [total_nodes] each membrane's nodes in (bin, node) order, from node0
    // LBFS_IBM_VANDERMONDE4 (rectilinear meshes, one instance): per axis the
    // vertex coordinates [n + 1] and the centroid coordinate of each cell row [n]
    // (centroid[i].x, centroid[j nx].y, centroid[k nx ny].z), and the cell volumes
    const double *grid_v[3];
    const double *grid_c[3];
    const double *cell_volume;
    int max_springs;             // springs of the largest membrane
    int max_patch_bound;         // largest patch_bound over the membranes (spread grid)
    const int *node_mem;         // [total_nodes] membrane of each node
    double *mad_partials;        // [n_membranes * kMaxSpringBlocks] (scratch)
    unsigned int *mad_ticket;    // [n_membranes], zero between launches
    // IBM window along z (lbfs_set_ibm_window): a patch whose z cells leave
    // [ibm_z_lo, ibm_z_hi) of its grid is an IBM range error (whole grid by default)
    int ibm_z_lo, ibm_z_hi;
};

// points per axis of an IBM stencil
__host__ __device__ constexpr int stencil_width(int ibm_stencil) { return ibm_stencil == 2 ? 2 : 4; }

// Shared-memory limits of the kernels for the largest membrane.
void membrane_prepare(int sort_capacity, int max_nodes);
// Whether membranes of max_nodes nodes fit the one-cluster-per-membrane step.
bool membrane_cluster_fits(int max_nodes);
// Enqueues the membrane kernels of the current mode on `s` (the node sort on
// `s_side`, joined back before the spread, when the side stream and its two
// events are given); returns the launch count.  without_spread: everything
// but the spread, which the caller launches (launch_membrane_spread).
int launch_membrane(const MembraneArgs &a, cudaStream_t s, cudaStream_t s_side = nullptr,
                    cudaEvent_t ev_advected = nullptr, cudaEvent_t ev_sorted = nullptr, bool without_spread = false);

// Per membrane, the y-z binning of its triangles for the interior test: bins
// of size >= every triangle's y-z extent and >= 4 delta_h over the membrane's
// box (+- 2 delta_h), at most kViscBins of them.
constexpr int kViscBins = 64 * 64;
struct ViscBins {
    double y0, z0, inv_b;
    int ny, nz;
};

struct ViscArgs {
    int nc, n_membranes;
    ViscBins *bins;              // [n_membranes]
    int *bin_start;              // [n_membranes * (kViscBins + 1)] first list entry of each bin
    int *bin_list;               // [4 total_tris] triangles (global ids) per bin, membrane m from 4 tri0
    int total_tris;
    const double *centroid;      // [3*nc]
    const MembraneConst *mc;
    const MembraneScalars *ms;
    const InstanceGrid *instances;
    const int *cell_instance;    // null with one instance
    const int *tri;
    const double *x, *y, *z;
    void *visc_factor;           // R[nc]
    int visc_is_float;
};

void launch_interior_viscosity(const ViscArgs &a, cudaStream_t s);
// stencil tables at the current positions (k_mem_advect writes them at x')
void launch_membrane_tables(const MembraneArgs &a, cudaStream_t s);
// advection, totals, spring and node forces only (adjoint recomputation)
void launch_membrane_forces(const MembraneArgs &a, cudaStream_t s);
// single phases of the membrane chain (autotuner): node sort + patches, spread
void launch_membrane_sort(const MembraneArgs &a, cudaStream_t s);
// programmatic: launched behind the membrane kernel before it on the same stream (its CTAs placed
// behind that kernel's last wave)
void launch_membrane_spread(const MembraneArgs &a, cudaStream_t s, bool programmatic = false);
// per membrane the local area, local bending and spring energy sums, out[3 n_membranes]
void launch_membrane_energies(const MembraneArgs &a, double *out, cudaStream_t s);
// check_periodic_object for the membranes flagged periodic (after a step's fluid update)
void launch_membrane_wrap(const MembraneArgs &a, cudaStream_t s);

}  // namespace lbfs
