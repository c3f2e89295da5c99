/*
 * lbfs_b200.h -- C ABI of the B200 (sm_100a) implementation of the LBFS-IBM
 * time step: D3Q15 lattice-Boltzmann flux solver on an unstructured
 * finite-volume hex mesh, immersed-boundary coupling, spring-network red blood
 * cell membranes.
 *
 * The reference (CHRG-Developer/LBFS-IBM-ADE-SP) has no plugin layer: its
 * solver entry point is the C++ method
 *     void gpu_solver::General_Purpose_Solver_mk_i(unstructured_mesh&, Solution&,
 *         Boundary_Conditions&, external_forces&, global_variables&, domain_geometry&,
 *         initial_conditions&, unstructured_bcs&, int mg, Solution& residual, int fmg,
 *         post_processing&, std::vector<lagrangian_object>&)      (Solver_gpu.h:28-31)
 * which copies the host objects into ~80 managed arrays (Solver_gpu.cu:473-655),
 * runs the time loop (Solver_gpu.cu:749-1246) and writes the solution back.
 * This header is what a drop-in replacement of that method binds to: the
 * descriptors below carry exactly the arrays the reference copies (same
 * ordering, same meaning), lbfs_create replaces the set-up block, lbfs_step
 * replaces one iteration of the time loop, and lbfs_get_state replaces the
 * write-back into Solution.  lbfs-ibm-ade-sp_b200/integration/Solver_gpu_lbfs.cpp
 * is that method written over this ABI.
 *
 * Conventions: every entry point returns an int status (LBFS_OK = 0); no C++
 * exception crosses the boundary; all pointers in descriptors are HOST
 * pointers owned by the caller and only read during lbfs_create; device
 * buffers are owned by the library; a handle is not thread-safe.
 */
#ifndef LBFS_B200_H
#define LBFS_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define LBFS_OK 0
#define LBFS_ERR_ARG 1          /* invalid argument or descriptor            */
#define LBFS_ERR_CUDA 2         /* CUDA runtime error (message via lbfs_last_error) */
#define LBFS_ERR_NOMEM 3        /* device allocation failed                  */
#define LBFS_ERR_STATE 4        /* solution flagged non-finite / invalid      */
#define LBFS_ERR_UNSUPPORTED 5  /* option not implemented                    */
#define LBFS_ERR_LIMIT 6        /* size beyond a documented maximum          */

/* ---- status flags (lbfs_status) ---------------------------------------- */
#define LBFS_FLAG_NONFINITE 1u  /* NaN/Inf in the fluid state (reference: LBFS.cu:2833-2865 traps; here a flag) */
#define LBFS_FLAG_RHO_RANGE 2u  /* rho <= 0 or rho > 1000 (same limit as LBFS.cu:2852)                       */
#define LBFS_FLAG_IBM_RANGE 4u  /* a membrane node's IBM patch exceeded its bounding allocation            */

/* ---- precision ----------------------------------------------------------- */
#define LBFS_FP64 0             /* plain FP64: the drop-in                                   */
#define LBFS_FP32_BULK 1        /* FP32 flux/gradient/IBM arithmetic, rho stored as rho-rho0,
                                   FP64 reductions, FP64 node integration                     */

/* ---- IBM kernels ---------------------------------------------------------- */
#define LBFS_IBM_HAT2 2         /* 2-point hat stencil (immersed_boundary_method.cu:14-97, 947-1024) */
#define LBFS_IBM_PESKIN4 4      /* 4-point Peskin cosine-free delta (new; no reference counterpart)  */
#define LBFS_IBM_VANDERMONDE4 5 /* 4x4x4 Lagrange (Vandermonde first column) weights on a rectilinear
                                   mesh, the mesh_type 4 kernels (immersed_boundary_method.cu:588-872,
                                   919-941); needs lbfs_mesh_desc.grid_x/y/z                       */

/* One instance of a batched ensemble: a contiguous range of interior cells
 * that forms its own uniform IBM grid (cell index = cell0 + i + nx (j + ny k)). */
typedef struct lbfs_grid_desc {
    int32_t cell0, n_cells;
    double origin[3], length[3];
    double delta_x, delta_h;
} lbfs_grid_desc;

/* Mesh arrays, in the reference's layout and order.  Sizes: nc = n_cells,
 * nb = n_bc (boundary faces = ghost cells, ghost of bc face i is cell nc+i),
 * nf = n_faces = n_interior + n_bc (boundary faces last).
 * Source of every array: unstructured_mesh / gradients (Solver_gpu.cu:625-655). */
typedef struct lbfs_mesh_desc {
    int32_t n_cells, n_faces, n_interior, n_bc;
    /* Axis-sorted prefix of the interior faces (x faces, then y, then z) for
     * meshes whose interior faces are axis aligned (mesh_type 4..7, flux kernels
     * calc_face_flux_x/_y/_z).  axis_aligned = 0 selects the general-normal
     * reconstruction of calc_face_flux (mesh_type 3). */
    int32_t n_face_x, n_face_y, n_face_z;
    int32_t axis_aligned;
    const int32_t *owner;          /* [nf]              mesh_owner              */
    const int32_t *neighbour;      /* [nf]              mesh_neighbour (ghost index for bc faces) */
    const double *face_area;       /* [nf]              surface_area            */
    const double *face_normal;     /* [3*nf]            face_normal (unit)      */
    const double *face_centroid;   /* [3*nf]            face_centroid           */
    const double *streaming_dt;    /* [nf]              delta_t_face            */
    const double *cell_volume;     /* [nc+nb]           cell_volume             */
    const double *cell_centroid;   /* [3*(nc+nb)]       cell_centroid           */
    const int32_t *gradient_stencil; /* [6*nc]          gradient_cells          */
    const double *lhs_inverse;     /* [9*nc]  row major LHS_xx,LHS_xy,...,LHS_zz */
    const double *rhs;             /* [18*nc] RHS_arr (6 neighbours x 3)        */
    const int32_t *bc_rho_type;    /* [nb]    1 Dirichlet, 2 Neumann, 3 periodic */
    const int32_t *bc_vel_type;    /* [nb]    1 Dirichlet, 2 Neumann, 3 periodic, 9 duct, 10 shear */
    const double *bc_values;       /* [4*nb]  (u, v, w, rho) = bcs_arr          */
    /* Uniform Eulerian grid seen by the IBM stencils (Solver_gpu.cu:448, 538-544). */
    double origin[3];              /* domain.origin_x/y/z                        */
    double length[3];              /* domain.X/Y/Z                               */
    double delta_x;                /* 2 * domain.dt                              */
    double delta_h;                /* unstructured_mesh::get_delta_h()           */
    /* Batched ensemble (no reference counterpart): n_instances independent
     * meshes concatenated into this one (interior cells, then ghosts; x, y, z
     * interior faces, then boundary faces, each category instance by
     * instance).  0 = one instance described by origin/length/delta_x/delta_h. */
    int32_t n_instances;
    const lbfs_grid_desc *instances;
    /* Vertex coordinates per axis of a rectilinear mesh, [nx+1], [ny+1], [nz+1]
     * (plateau_x, plateau_y, plateau_z, Solver_gpu.cu:637-639): read only by
     * LBFS_IBM_VANDERMONDE4; null otherwise. */
    const double *grid_x, *grid_y, *grid_z;
    /* Periodic boundaries (type 3; Boundary_Conditions::periodic_node,
     * Boundary_Conditions.cpp:417-432): per ghost the interior cell whose
     * state (Solution::update_unstructured_bcs, Solution.cpp:777-803) and
     * gradients (gradients::Get_LS_Gradients, gradients.cpp:428-440) a type-3
     * ghost takes, e.g. from lbfs_mesh_find_periodic_nodes.  Required when a
     * boundary has type 3, ignored for other ghosts; null otherwise.  The
     * reference's GPU kernels implement no periodic type (LBFS.cu:1872-1918):
     * this is its CPU solver's definition on the GPU path. */
    const int32_t *periodic_node;
} lbfs_mesh_desc;

/* Scalars of global_variables / initial_conditions used by the step. */
typedef struct lbfs_params {
    double visc;                /* globals.visc                                           */
    double delta_t;             /* globals.time_marching_step (time_stepping = constant)   */
    double gamma_inv;           /* 1 / globals.pre_conditioned_gamma                       */
    double channel_diameter;    /* domain.Y (bc type 9)                                    */
    double body_force[3];       /* init_conds.force_x/y/z                                  */
    double ref_rho;             /* globals.ref_rho (residual normalisation)                */
    double max_velocity;        /* globals.max_velocity (residual normalisation)           */
    double rho0;                /* density offset carried by LBFS_FP32_BULK                */
    double visc_factor_initial; /* visc_factor before the first interior-viscosity update */
    int32_t testcase;           /* globals.testcase (8 = inviscid)                          */
    int32_t precision;          /* LBFS_FP64 or LBFS_FP32_BULK                               */
    int32_t ibm_stencil;        /* LBFS_IBM_HAT2 or LBFS_IBM_PESKIN4                         */
    int32_t viscosity_period;   /* interior viscosity update when t % period == 1 (10000); 0 = never */
    /* Time stepping (globals.gpu_time_stepping, global_variables.h:59).  0 or
     * LBFS_DT_CONSTANT: delta_t is the step.  Otherwise every step starts with
     * get_cfl_device (LBFS.cu:2868-2932): a per-cell step
     * delta_t * volume / (CFL eigenvalue) and its minimum over the cells
     * (min<128> + min_block, Solver_gpu.cu:767-787); LBFS_DT_LOCAL advances each
     * cell with its own step, LBFS_DT_MIN and LBFS_DT_TALTS with the minimum
     * (time_integration, LBFS.cu:2089-2172); node advection always uses the
     * minimum. */
    int32_t time_stepping;
    double pre_conditioned_gamma; /* globals.pre_conditioned_gamma (get_cfl_device); 0 = 1 / gamma_inv */
    /* globals.preconditioning_active: the lattice equilibria of the general-normal
     * and boundary faces take the 1/gamma factor (populate_feq, LBFS.cu:940-1036,
     * chosen at LBFS.cu:2637-2647); the interface equilibria and relaxation take
     * gamma_inv in any case. */
    int32_t preconditioning;
} lbfs_params;

#define LBFS_DT_LOCAL 1
#define LBFS_DT_CONSTANT 2
#define LBFS_DT_MIN 3
#define LBFS_DT_TALTS 4         /* as LBFS_DT_MIN: the GPU path advances talts with the minimum step */

/* One spring-network membrane (lagrangian_object with type == 2). */
typedef struct lbfs_rbc_desc {
    int32_t n_nodes, n_tris, n_springs;
    const int32_t *tri;             /* [3*n_tris]   sorted_triIdx                         */
    const int32_t *spring;          /* [4*n_springs] sprIdx (a, b, c, d): edge a-c, wings b, d */
    const double *xyz_stress_free;  /* [3*n_nodes]  stress-free mesh (contour lengths, c0) */
    const double *xyz_initial;      /* [3*n_nodes]  initial mesh (V0, A0, MAD0, angles)   */
    double volume_modulus, local_area_modulus, global_area_modulus, shear_modulus;
    double global_bending_modulus, local_bending_modulus, membrane_thickness, viscosity;
    double wlc_ratio, curvature_ratio, volume_ratio, internal_viscosity_ratio, reference_length;
    int32_t pivkin_length, sphere_reference;
    int32_t instance;               /* ensemble instance the membrane lives in (0 without an ensemble) */
    /* lagrangian_object::periodic (its XML key): at t % 5000 == 1, after the
     * step's fluid update, nodes whose mean z exceeds origin_z + 0.75 Z move by
     * -0.5 Z in z (gpu_solver::check_periodic_object, Solver_gpu.cu:1027-1029,
     * 1277-1304).  0: never; LBFS_WRAP_OWN: this membrane by the mean of its own
     * nodes; LBFS_WRAP_ALL (membrane 0 only, as the reference gates on
     * object_vec[0].periodic): the mean over the nodes of every membrane of the
     * handle together, and every membrane moves when it exceeds the bound -- the
     * reference's behaviour with several objects. */
    int32_t periodic;
} lbfs_rbc_desc;

#define LBFS_WRAP_OWN 1
#define LBFS_WRAP_ALL 2

typedef struct lbfs_solver lbfs_solver;

/* Create a solver on CUDA device `device`, upload the mesh and membranes and
 * run the membrane set-up (Solver_gpu.cu:659-735).  n_rbc may be 0.
 * Replaces the set-up half of gpu_solver::General_Purpose_Solver_mk_i
 * (Solver_gpu.cu:178-746). */
int lbfs_create(const lbfs_mesh_desc *mesh, const lbfs_params *params, const lbfs_rbc_desc *rbc, int32_t n_rbc,
                int32_t device, lbfs_solver **out);
int lbfs_destroy(lbfs_solver *s);

/* Fluid state (primitive rho, u, v, w per interior cell), host arrays of n_cells.
 * set_state also resets soln_t1 to the primitive state, as Solver_gpu.cu:746 does. */
int lbfs_set_state(lbfs_solver *s, const double *rho, const double *u, const double *v, const double *w);
int lbfs_get_state(lbfs_solver *s, double *rho, double *u, double *v, double *w);

/* set_state / get_state copy four planes (rho, u, v, w) with one cudaMemcpyAsync
 * each, so page-locked host arrays transfer at full DMA bandwidth. */

/* Advance n_steps time steps (one iteration of Solver_gpu.cu:749-1046 each).
 * Enqueued on the solver's stream; returns without waiting. */
int lbfs_step(lbfs_solver *s, int32_t n_steps);
/* Same, with the per-step work replayed from a CUDA graph captured on first use. */
int lbfs_step_graph(lbfs_solver *s, int32_t n_steps);
int lbfs_synchronize(lbfs_solver *s);
/* The reference's time loop with its convergence test (Solver_gpu.cu:1206-1208:
 * stop after the first step whose residual norms, as lbfs_get_residuals gives
 * them, have their maximum below `tolerance`) and the drop-in's divergence test
 * (stop once LBFS_FLAG_NONFINITE or LBFS_FLAG_RHO_RANGE is set), for at most
 * max_steps steps.  The tests run on the device: the steps between
 * interior-viscosity updates and object wraps are one launch of a CUDA graph
 * whose while node repeats the step and a one-thread check kernel, so no host
 * round trip separates two steps (those special steps, and every step while
 * profiling, go one at a time with the tests on the host).  *steps_done gets
 * the number of steps taken, residuals[4] (may be null) the last step's norms.
 * Results equal lbfs_step_graph + lbfs_get_residuals step by step. */
int lbfs_step_until(lbfs_solver *s, int32_t max_steps, double tolerance, int32_t *steps_done, double *residuals);

/* Use a caller stream (a cudaStream_t) instead of the solver's own. */
int lbfs_set_stream(lbfs_solver *s, void *cuda_stream);

/* Membrane node positions / velocities / forces of all membranes, host [3*total_nodes] (x,y,z per node). */
int lbfs_get_nodes(lbfs_solver *s, int32_t which, double *out);
int lbfs_set_nodes(lbfs_solver *s, const double *xyz);
#define LBFS_NODES_POSITION 0
#define LBFS_NODES_VELOCITY 1
#define LBFS_NODES_FORCE 2

/* Membrane totals, host [6*n_rbc]: V, V0, A, A0, MAD, MAD0 per membrane
 * (lagrangian_object::total_volume ... total_MAD_0). */
int lbfs_get_totals(lbfs_solver *s, double *out);
/* Membrane energies, host [7*n_rbc]: volume, global area, local area, local
 * bending, ADE, spring (WLC) and total energy per membrane, the columns of the
 * reference's energy_log.txt (Solver_gpu.cu:1073-1136; the per-spring sums
 * of get_area_energy, get_bending_energy and get_spring_energy,
 * spring_network.cu:1687-1768, formed on the device in FP64). */
int lbfs_get_energies(lbfs_solver *s, double *out);
/* RMS residuals of the last step, host [4]: rho, u, v, w (residuals::l2_norm_rms_moukallad). */
int lbfs_get_residuals(lbfs_solver *s, double *out);
/* The time step of the last step (the solver loop's delta_t): params.delta_t
 * with constant time stepping, else the minimum of the per-cell steps
 * (Solver_gpu.cu:776). */
int lbfs_get_time_step(lbfs_solver *s, double *delta_t);

/* Internal arrays for parity checking, copied to host.  Layouts:
 *  LBFS_FIELD_GRADIENTS  [12*(nc+nb)]  per cell: grad rho, grad u, grad v, grad w (x,y,z each)
 *  LBFS_FIELD_FACE_FLUX  [4*nf]        per face: (u, v, w, rho) components of res_face
 *  LBFS_FIELD_RESIDUAL   [4*nc]        per cell: res_rho, res_u, res_v, res_w (forces included)
 *  LBFS_FIELD_FORCE      [3*nc]        per cell: force density (body force + IBM spread)
 *  LBFS_FIELD_T1         [4*nc]        per cell: soln_t1 (u, v, w, rho)
 *  LBFS_FIELD_VISC       [nc]          per cell: visc_factor
 *  LBFS_FIELD_GHOST      [4*nb]        per ghost: (u, v, w, rho)
 *  LBFS_FIELD_SPRING     [9*total_springs] contour length, spring constant, curvature,
 *                        curvature_0, angle_0, area_0[2], area[2]
 *  LBFS_FIELD_DT_LOCAL   [nc]          per cell: delta_t_local of the last step (the constant step, the
 *                        cell's own CFL step with local or talts, the minimum with min)     */
int lbfs_get_field(lbfs_solver *s, int32_t which, double *out);
#define LBFS_FIELD_GRADIENTS 0
#define LBFS_FIELD_FACE_FLUX 1
#define LBFS_FIELD_RESIDUAL 2
#define LBFS_FIELD_FORCE 3
#define LBFS_FIELD_T1 4
#define LBFS_FIELD_VISC 5
#define LBFS_FIELD_GHOST 6
#define LBFS_FIELD_SPRING 7
#define LBFS_FIELD_DT_LOCAL 8

/* Keep the per-cell residuals of every step for lbfs_get_field(LBFS_FIELD_RESIDUAL).
 * Off by default: it adds 32 bytes of writes per cell per step. */
int lbfs_keep_residuals(lbfs_solver *s, int32_t on);

/* Accumulated status flags (LBFS_FLAG_*) since creation; reading does not clear. */
int lbfs_status(lbfs_solver *s, uint32_t *flags);
/* Timing with CUDA events, also inside the captured graph.  level 1: events
 * around each whole step; level 2: also around every kernel (or kernel group);
 * 0: off.  lbfs_get_phase_times writes the durations in ms of the last step:
 * [0] membrane kernels, [1] ghost+gradients, [2] face flux, [3] cell update,
 * [4] interior viscosity (0 when not launched or not level 2), and [5] the
 * whole step (first launch to last, on the solver's stream). */
int lbfs_set_profiling(lbfs_solver *s, int32_t on);
int lbfs_get_phase_times(lbfs_solver *s, double *ms);

/* Kernel launches issued per time step by this handle (graph or stream). */
int lbfs_launches_per_step(lbfs_solver *s, int32_t *launches);
/* Copy of the last error message (NUL terminated, truncated to len). */
int lbfs_last_error(char *buf, int32_t len);

/* ---- launch shapes and the autotuner (no reference counterpart) ----------- *
 * Block sizes and grid caps of the per-phase kernels.  Results do not depend on
 * the shape, except the last bits of the residual norms, whose block partials
 * follow the cell-update grid.  lbfs_autotune searches the shape coordinate by
 * coordinate, timing each candidate as `reps` whole steps (CUDA-graph replays,
 * CUDA events) from the handle's current state, which it saves and puts back;
 * it keeps a candidate only for a gain above 1 %.  The next lbfs_step_graph
 * captures a new graph.  `shape` (may be null) receives the choice;
 * time_us[0] is its mean step time in microseconds. */
#define LBFS_MAX_UPDATE_BLOCKS (148 * 16)
#define LBFS_MAX_SPREAD_BLOCKS (148 * 16)
typedef struct lbfs_launch_shape {
    int32_t gradient_threads;       /* 128, 256 or 512 */
    int32_t flux_threads;           /* interior faces of an axis-aligned mesh: 64, 128 or 256 */
    int32_t general_flux_threads;   /* boundary / general-normal faces: 64, 128 or 256 */
    int32_t update_threads;         /* 128, 256 or 512 */
    int32_t update_blocks;          /* grid cap of the cell update, 1 .. LBFS_MAX_UPDATE_BLOCKS */
    int32_t spread_blocks;          /* grid of the IBM spread, 1 .. LBFS_MAX_SPREAD_BLOCKS */
    int32_t flux_chunks;            /* 1, 2, 4 or 8: gradients and interior-face fluxes of an axis-aligned
                                       mesh pipelined in that many chunks of cells on two streams
                                       (0 = 1; meshes that do not allow it use 1) */
    int32_t membrane_cluster;       /* 8 or 16: a membrane's totals, spring and node forces as one
                                       thread-block cluster of that many CTAs; 0: three kernels.  It
                                       changes the summation order of V, A and MAD (rounding only) */
    int32_t membrane_after_k1;      /* 1: in a captured step the membrane kernels start once every block
                                       of the gradient kernel has begun (a programmatic edge from its
                                       launch-completion port) instead of beside it from the step's
                                       start; 0: from the step's start.  Order only: results unchanged */
    double time_us[5];              /* autotune: [0] mean step time of the chosen shape (us) */
} lbfs_launch_shape;
int lbfs_get_launch_shape(lbfs_solver *s, lbfs_launch_shape *shape);
int lbfs_set_launch_shape(lbfs_solver *s, const lbfs_launch_shape *shape);
int lbfs_autotune(lbfs_solver *s, int32_t reps, lbfs_launch_shape *shape);

/* ---- lossless checkpoint / restart ------------------------------------------ *
 * Replaces the reference's restart from its 6-digit text output
 * (Solution::output, Solution.cpp:221-251; Solver_gpu.cu:1953-1980): a
 * caller-owned binary blob with soln_t1, the state with its ghosts, the
 * viscosity field, the step counter and every membrane array, so a run resumed
 * from it continues bit for bit.  Load checks sizes and precision against the
 * handle (LBFS_ERR_ARG otherwise). */
int lbfs_checkpoint_size(lbfs_solver *s, uint64_t *bytes);
int lbfs_checkpoint_save(lbfs_solver *s, void *buf, uint64_t bytes);
int lbfs_checkpoint_load(lbfs_solver *s, const void *buf, uint64_t bytes);

/* ---- discrete adjoint (no reference counterpart) --------------------------- *
 * lbfs_adjoint runs n_steps forward from the handle's state, keeping soln_t1
 * (and, with membranes, node positions and MAD) every `checkpoint_every`
 * steps, evaluates the objective on the final state, then sweeps backwards
 * segment by segment: each segment is recomputed from its checkpoint and the
 * discrete adjoint of every step is applied in reverse.  When every segment's
 * per-step intermediates fit in half the free device memory (at most
 * LBFS_ADJOINT_MEMORY_MB MiB if that environment variable is set; 0 forces the
 * recomputation), the forward sweep keeps them and the reverse sweep
 * recomputes nothing; the results are the same bit for bit.  FP64 handles without
 * preconditioning.  On return the handle holds the final forward state and
 * the step counter has advanced by n_steps.
 *   J        objective value
 *   grad[0]  dJ / d(shear modulus of every membrane)
 *   grad[1]  dJ / d(global bending modulus of every membrane)
 *   grad[2]  dJ / d sigma, every boundary velocity value scaled by sigma at 1
 *   times_ms (may be null): forward sweep and reverse sweep, device time. */
#define LBFS_OBJ_VELOCITY 0   /* J = sum over cells of w_c . (u, v, w)_c at the final step */
#define LBFS_OBJ_TAYLOR 1     /* J = Taylor deformation (L - B) / (L + B) of one membrane in the x-y plane */
typedef struct lbfs_objective {
    int32_t kind;
    int32_t membrane;             /* LBFS_OBJ_TAYLOR */
    const double *cell_weights;   /* LBFS_OBJ_VELOCITY: 3 per interior cell */
} lbfs_objective;
int lbfs_adjoint(lbfs_solver *s, int32_t n_steps, int32_t checkpoint_every, const lbfs_objective *obj, double *J,
                 double *grad, double *times_ms);

/* ---- residual norms without device allocation ---------------------------- */

/* No counterpart in the reference.  For callers that cannot call cudaMalloc --
 * host code that drives the step from inside a CUDA-graph capture or a stream
 * callback (cudaMalloc is illegal during capture and synchronises the device),
 * or integrations whose device memory is all reserved by their own pool:
 * the RMS norms of a residual field, as lbfs_get_residuals reports them, with
 * the reduction's scratch in a fixed __device__ array of the library instead
 * of allocated memory.  d_res: device [4*n_cells] (res_rho, res_u, res_v,
 * res_w per cell); d_rms: device [4] (rho, u, v, w norms); stream: a
 * cudaStream_t (0 = default stream).  Enqueued, not waited for.
 * Limits: n_cells <= LBFS_NOALLOC_MAX_CELLS (LBFS_ERR_LIMIT beyond); the
 * scratch array (2 MiB per GPU that loads the library, held until exit) is
 * shared by every call, so calls that overlap on the GPU race -- serialise
 * them.  The first call on a device resolves the array's device address
 * (cudaGetSymbolAddress) and must come before any stream capture on that
 * device.  The scratch is the CURRENT device's: `stream` must belong to the
 * current device (LBFS_ERR_ARG otherwise).  The resolved address is kept for
 * the life of the process; after cudaDeviceReset on a device, do not call
 * this entry point on that device again in the same process. */
#define LBFS_NOALLOC_MAX_BLOCKS 65536
#define LBFS_NOALLOC_MAX_CELLS (LBFS_NOALLOC_MAX_BLOCKS * 256)
int lbfs_residual_rms_noalloc(const double *d_res, int32_t n_cells, double ref_rho, double max_velocity,
                              double *d_rms, void *stream);

/* ---- host-side set-up helpers ------------------------------------------- */

/* Sizes of the uniform mesh generated for a domain X x Y x Z with streaming
 * step dt (unstructured_mesh::create_uniform_openfoam_mesh, mesh_type 6):
 * out[0..7] = n_cells, n_faces, n_interior, n_bc, n_face_x, n_face_y, n_face_z,
 * n_cells + n_bc. */
int lbfs_mesh_uniform_counts(double X, double Y, double Z, double dt, int32_t *out);

/* Fill the mesh arrays of that uniform mesh (same ordering and geometry as
 * unstructured_mesh.cpp:239-666, 1592-1692, 1963-1996 and
 * gradients.cpp:214-315).  Output buffers must be sized from
 * lbfs_mesh_uniform_counts; bc faces are tagged with patch ids
 * 0 left, 1 right, 2 bottom, 3 top, 4 back, 5 front in bc_patch[nb].
 * gradient_hybrid: 0 "LS", 1 "hybrid". */
int lbfs_mesh_build_uniform(double X, double Y, double Z, double dt, const double *origin, double visc,
                            double fneq_min, int32_t gradient_hybrid, int32_t *owner, int32_t *neighbour,
                            double *face_area, double *face_normal, double *face_centroid, double *streaming_dt,
                            double *cell_volume, double *cell_centroid, int32_t *gradient_stencil,
                            double *lhs_inverse, double *rhs, int32_t *bc_patch, double *delta_h);

/* Rectilinear meshes of the reference generator (create_uniform_openfoam_mesh,
 * unstructured_mesh.cpp:238-380): mesh_type 6 uniform, 7 cosine-clustered in
 * x and y, 5 in x, y and z, 4 the plateau mesh (domain.plateau_width,
 * plateau_slope).  Outputs as lbfs_mesh_build_uniform, plus grid_xyz
 * [(nx+1) + (ny+1) + (nz+1)]: the vertex coordinates per axis (for mesh_type 4
 * the plateau arrays the 4x4x4 IBM stencil searches).  Faces stay axis
 * aligned (axis_aligned = 1). */
int lbfs_mesh_build_rectilinear(double X, double Y, double Z, double dt, const double *origin, double visc,
                                double fneq_min, int32_t gradient_hybrid, int32_t mesh_type, double plateau_width,
                                double plateau_slope, int32_t *owner, int32_t *neighbour, double *face_area,
                                double *face_normal, double *face_centroid, double *streaming_dt,
                                double *cell_volume, double *cell_centroid, int32_t *gradient_stencil,
                                double *lhs_inverse, double *rhs, int32_t *bc_patch, double *delta_h,
                                double *grid_xyz);

/* The same mesh with every interior vertex moved by a seeded uniform
 * perturbation of up to `jitter` (< 0.25) times the cell spacing per axis
 * (boundary vertices stay, so the box and its patches stay).  Faces are then
 * non-planar quadrilaterals and normals general, as in the imported
 * (mesh_type 3) meshes; step it with axis_aligned = 0.  closed_faces = 0
 * gives exactly the geometry the reference's importer forms from this mesh
 * written as a polyMesh (lbfs_mesh_write_openfoam): a face's area is the sum
 * of its two triangles' areas, which on a warped face makes the vector areas
 * of a cell's faces fail to close, so a fluid at rest starts to move.
 * closed_faces = 1 uses the length of the face's vector area instead (the
 * faces of every cell close; the one deviation from the reference's
 * formulas). */
int lbfs_mesh_build_jittered(double X, double Y, double Z, double dt, const double *origin, double visc,
                             double fneq_min, int32_t gradient_hybrid, double jitter, uint64_t seed,
                             int32_t closed_faces, int32_t *owner, int32_t *neighbour, double *face_area,
                             double *face_normal, double *face_centroid, double *streaming_dt, double *cell_volume,
                             double *cell_centroid, int32_t *gradient_stencil, double *lhs_inverse, double *rhs,
                             int32_t *bc_patch, double *delta_h);

/* OpenFOAM polyMesh.  lbfs_mesh_write_openfoam writes the generator's mesh
 * (mesh_type 4-7, or 6 with jitter) as <dir>/points, faces, owner, neighbour
 * and boundary (ASCII; patches left, right, bottom, top, back, front; the
 * owner file's 13th line carries the note the reference's importer reads).
 * lbfs_mesh_openfoam_counts reads the sizes: counts[6] = n_points, n_cells,
 * n_faces, n_internal_faces, n_boundary_faces, n_patches.
 * lbfs_mesh_import_openfoam reads a polyMesh as unstructured_mesh::
 * import_openfoam_mesh and import_openfoam_BC_tags do (unstructured_mesh.cpp:
 * 670-941, 2533-2608: the header note, lists between a line starting with "("
 * and one starting with ")", points read as float, faces "4(a b c d)") and
 * forms the geometry and least-squares matrices with the same code as the
 * generated meshes (generate_internal_mesh); hexahedral cells only.  bc_patch
 * is each boundary face's patch index in the boundary file, names the patch
 * names separated by newlines.  The imported mesh steps with axis_aligned = 0
 * (mesh_type 3). */
/* The generator's meshes built on GPU `device` (mesh_type 4-7 as
 * lbfs_mesh_build_rectilinear, jitter > 0 as lbfs_mesh_build_jittered; grid_xyz
 * may be null): the same arrays bit for bit (unstructured_mesh::
 * generate_internal_mesh, unstructured_mesh.cpp:1592-1692, and gradients::
 * pre_fill_LHS_and_RHS_matrix, gradients.cpp:214-315, otherwise serial host
 * loops), one thread per vertex, face or cell, in a fraction of the host
 * builder's time at 128^3.  Device memory is allocated for the build and
 * released before it returns. */
int lbfs_mesh_build_gpu(double X, double Y, double Z, double dt, const double *origin, double visc, double fneq_min,
                        int32_t gradient_hybrid, int32_t mesh_type, double plateau_width, double plateau_slope,
                        double jitter, uint64_t seed, int32_t closed_faces, int32_t device, int32_t *owner,
                        int32_t *neighbour, double *face_area, double *face_normal, double *face_centroid,
                        double *streaming_dt, double *cell_volume, double *cell_centroid, int32_t *gradient_stencil,
                        double *lhs_inverse, double *rhs, int32_t *bc_patch, double *delta_h, double *grid_xyz);

/* Slab decomposition of one mesh over several handles (one per GPU): each
 * handle holds a slab of z planes plus halo planes of its neighbours' cells,
 * and between steps the halo planes are refreshed from the neighbours (the
 * reference has no multi-GPU path; its step is Solver_gpu.cu:749-1021 on one
 * device).  lbfs_halo_bytes: bytes of the buffer for n_cells cells.
 * lbfs_halo_pack / lbfs_halo_unpack copy the state records and the FP64
 * accumulators (soln_t1) of interior cells [first_cell, first_cell + n_cells)
 * to / from the DEVICE buffer `d_buf` on the handle's stream, device to
 * device, without synchronising (order NCCL or peer copies on the same
 * stream, lbfs_set_stream).  lbfs_set_ibm_window confines the IBM patches of
 * the handle's membranes to z cells [z_lo, z_hi) of its grid: a patch that
 * leaves the window spreads nothing and raises LBFS_FLAG_IBM_RANGE, so a
 * membrane cannot reach a halo plane unnoticed. */
int lbfs_halo_bytes(lbfs_solver *s, int32_t n_cells, uint64_t *bytes);
int lbfs_halo_pack(lbfs_solver *s, int32_t first_cell, int32_t n_cells, void *d_buf);
int lbfs_halo_unpack(lbfs_solver *s, int32_t first_cell, int32_t n_cells, const void *d_buf);
int lbfs_set_ibm_window(lbfs_solver *s, int32_t z_lo, int32_t z_hi);

/* Periodic partners (Boundary_Conditions::assign_boundary_conditions,
 * Boundary_Conditions.cpp:417-432): for every ghost b whose rho or velocity
 * type is 3, out[b] = the interior cell whose centroid is nearest to the
 * ghost's centroid moved by +translation or by -translation (the smaller
 * distance; ties to the lower cell index); 0 for other ghosts, as the
 * reference leaves them.  The reference searches all cells per ghost from an
 * uninitialised cell index (`nb`, line 420); here the point is the ghost's
 * own centroid, and the search bins the cells (O(cells + ghosts) instead of
 * O(cells x ghosts)) with the same result as the all-cell search.  Needs the
 * descriptor's sizes, owner/neighbour, cell_centroid and bc types. */
int lbfs_mesh_find_periodic_nodes(const lbfs_mesh_desc *mesh, const double *translation, int32_t *out);

int lbfs_mesh_write_openfoam(const char *dir, double X, double Y, double Z, double dt, const double *origin,
                             int32_t mesh_type, double plateau_width, double plateau_slope, double jitter,
                             uint64_t seed);
int lbfs_mesh_openfoam_counts(const char *dir, int32_t *counts);
int lbfs_mesh_import_openfoam(const char *dir, double visc, double fneq_min, int32_t gradient_hybrid,
                              int32_t closed_faces, int32_t *owner, int32_t *neighbour, double *face_area,
                              double *face_normal, double *face_centroid, double *streaming_dt, double *cell_volume,
                              double *cell_centroid, int32_t *gradient_stencil, double *lhs_inverse, double *rhs,
                              int32_t *bc_patch, char *names, int32_t names_len);
/* lbfs_mesh_import_openfoam with the geometry and least-squares matrices
 * formed on GPU `device`: the file is read on the host as above, then one
 * thread per face forms the face geometry and one per cell gathers its six
 * faces in increasing face index (the order of the host routine's face loop)
 * for the volume, centroid and LS sums, so every array equals
 * lbfs_mesh_import_openfoam's bit for bit.  Rejects (LBFS_ERR_ARG) a face
 * whose neighbour is its owner and a cell without six faces.  Device memory
 * is allocated for the build and released before it returns. */
int lbfs_mesh_import_openfoam_gpu(const char *dir, double visc, double fneq_min, int32_t gradient_hybrid,
                                  int32_t closed_faces, int32_t device, int32_t *owner, int32_t *neighbour,
                                  double *face_area, double *face_normal, double *face_centroid,
                                  double *streaming_dt, double *cell_volume, double *cell_centroid,
                                  int32_t *gradient_stencil, double *lhs_inverse, double *rhs, int32_t *bc_patch,
                                  char *names, int32_t names_len);

/* Spring connectivity of a closed triangulated membrane, in the order the
 * reference's Osay reader produces it (lagrangian_object.cpp:238-481).
 * spring_out must hold 4 * capacity ints; *n_springs receives the count. */
int lbfs_rbc_build_springs(int32_t n_nodes, int32_t n_tris, const int32_t *tri, int32_t capacity,
                           int32_t *spring_out, int32_t *n_springs);

#ifdef __cplusplus
}
#endif

#endif /* LBFS_B200_H */
