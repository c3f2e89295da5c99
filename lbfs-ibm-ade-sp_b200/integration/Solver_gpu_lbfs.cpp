// Drop-in replacement of the reference's GPU solver entry point,
//     gpu_solver::General_Purpose_Solver_mk_i   (Solver_gpu.h:28-31, Solver_gpu.cu:178-1275),
// over the C ABI of include/lbfs_b200.h.  A reference build links this file
// (and liblbfs_b200.so) in place of Solver_gpu.cu; program::run
// (program.cpp:113-115) calls it unchanged with the objects it built from the
// XML deck, the mesh and the membrane files.
//
// What it forwards: the arrays the reference copies into managed memory
// (Solver_gpu.cu:625-655, 1821-2151), the scalars of global_variables /
// initial_conditions the loop uses, and the type-2 lagrangian_objects with
// their stress-free and initial meshes (Solver_gpu.cu:659-735).  What it keeps
// from the reference loop: the step count ceil(simulation_length), the
// write-back into `soln`, and the convergence test on the RMS residuals
// (Solver_gpu.cu:1033-1046, 1206-1210).  File output (TecIO, text dumps) stays
// with the caller.  Errors end the process with a message, as the reference's
// post_kernel_checks does (Solver_gpu.cu:1806-1818).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "Solver_gpu.h"
#include "gradients.h"
#include "lagrangian_object.h"
#include "lbfs_b200.h"

namespace {

void lbfs_check(int rc, const char *what) {
    if (rc == LBFS_OK) return;
    char msg[512];
    lbfs_last_error(msg, sizeof(msg));
    std::fprintf(stderr, "lbfs_b200: %s failed (%d): %s\n", what, rc, msg);
    std::exit(-1);
}

}  // namespace

// The rest of the class as Solver_gpu.cu defines it (this file takes that
// translation unit's place in a build): construction and destruction hold no state.
gpu_solver::gpu_solver() {}
gpu_solver::~gpu_solver() {}

void gpu_solver::General_Purpose_Solver_mk_i(unstructured_mesh &Mesh, Solution &soln, Boundary_Conditions &bcs,
                                             external_forces &source, global_variables &globals,
                                             domain_geometry &domain, initial_conditions &init_conds,
                                             unstructured_bcs &quad_bcs_orig, int mg, Solution &residual, int fmg,
                                             post_processing &pp, std::vector<lagrangian_object> &object_vec) {
    const int nc = Mesh.get_n_cells(), nf = Mesh.get_n_faces(), ni = Mesh.get_n_neighbours();
    const int nb = Mesh.get_num_bc(), nt = Mesh.get_total_cells();

    // least-squares geometry, as Solver_gpu.cu:394 prepares it
    gradients grads(nt);
    grads.pre_fill_LHS_and_RHS_matrix(bcs, Mesh, domain, soln, globals);

    std::vector<int32_t> owner(nf), neighbour(nf), stencil(6 * (size_t)nc), rho_type(nb), vel_type(nb);
    std::vector<double> area(nf), normal(3 * (size_t)nf), fcen(3 * (size_t)nf), sdt(nf), vol(nt),
        cen(3 * (size_t)nt), lhs(9 * (size_t)nc), rhs(18 * (size_t)nc), bcv(4 * (size_t)nb);
    for (int f = 0; f < nf; f++) {
        owner[f] = Mesh.get_mesh_owner(f);
        neighbour[f] = Mesh.get_mesh_neighbour(f);
        area[f] = Mesh.get_face_area(f);
        sdt[f] = Mesh.get_delta_t_face(f);
        normal[3 * f] = Mesh.get_face_i(f); normal[3 * f + 1] = Mesh.get_face_j(f); normal[3 * f + 2] = Mesh.get_face_k(f);
        fcen[3 * f] = Mesh.get_face_x(f); fcen[3 * f + 1] = Mesh.get_face_y(f); fcen[3 * f + 2] = Mesh.get_face_z(f);
    }
    for (int i = 0; i < nt; i++) {
        vol[i] = Mesh.get_cell_volume(i);
        cen[3 * i] = Mesh.get_centroid_x(i); cen[3 * i + 1] = Mesh.get_centroid_y(i); cen[3 * i + 2] = Mesh.get_centroid_z(i);
    }
    for (int i = 0; i < nc; i++) {
        for (int j = 0; j < 6; j++) {
            stencil[6 * i + j] = Mesh.gradient_cells[i][j];
            rhs[18 * i + 3 * j] = grads.RHS_x[6 * i + j];
            rhs[18 * i + 3 * j + 1] = grads.RHS_y[6 * i + j];
            rhs[18 * i + 3 * j + 2] = grads.RHS_z[6 * i + j];
        }
        const double L[9] = {grads.LHS_xx[i], grads.LHS_xy[i], grads.LHS_xz[i], grads.LHS_yx[i], grads.LHS_yy[i],
                             grads.LHS_yz[i], grads.LHS_zx[i], grads.LHS_zy[i], grads.LHS_zz[i]};
        for (int k = 0; k < 9; k++) lhs[9 * i + k] = L[k];
    }
    for (int i = 0; i < nb; i++) {  // bcs_to_array / bcs_to_array_double, Solver_gpu.cu:1821-1855
        rho_type[i] = bcs.get_rho_type(i);
        vel_type[i] = bcs.get_vel_type(i);
        bcv[4 * i] = bcs.get_u(i); bcv[4 * i + 1] = bcs.get_v(i); bcv[4 * i + 2] = bcs.get_w(i); bcv[4 * i + 3] = bcs.get_rho(i);
    }
    lbfs_mesh_desc md = {};
    md.n_cells = nc; md.n_faces = nf; md.n_interior = ni; md.n_bc = nb;
    md.n_face_x = Mesh.get_n_face_x(); md.n_face_y = Mesh.get_n_face_y(); md.n_face_z = Mesh.get_n_face_z();
    md.axis_aligned = globals.mesh_type != 3;  // calc_face_flux_x/_y/_z vs calc_face_flux (Solver_gpu.cu:953-981)
    md.owner = owner.data(); md.neighbour = neighbour.data(); md.face_area = area.data();
    md.face_normal = normal.data(); md.face_centroid = fcen.data(); md.streaming_dt = sdt.data();
    md.cell_volume = vol.data(); md.cell_centroid = cen.data(); md.gradient_stencil = stencil.data();
    md.lhs_inverse = lhs.data(); md.rhs = rhs.data();
    md.bc_rho_type = rho_type.data(); md.bc_vel_type = vel_type.data(); md.bc_values = bcv.data();
    md.origin[0] = domain.origin_x; md.origin[1] = domain.origin_y; md.origin[2] = domain.origin_z;
    md.length[0] = domain.X; md.length[1] = domain.Y; md.length[2] = domain.Z;
    md.delta_x = domain.dt * 2;
    md.delta_h = Mesh.get_delta_h();
    // periodic boundaries (type 3; the CPU solver's, Solution.cpp:777-803): each ghost's partner cell by
    // the deck's periodic_translation (preprocessor.cpp:532-534, Boundary_Conditions.cpp:417-432)
    std::vector<int32_t> partner(nb, 0);
    bool any_periodic = false;
    for (int i = 0; i < nb; i++) any_periodic = any_periodic || rho_type[i] == 3 || vel_type[i] == 3;
    if (any_periodic) {
        const double T[3] = {quad_bcs_orig.per_translate_x, quad_bcs_orig.per_translate_y,
                             quad_bcs_orig.per_translate_z};
        lbfs_check(lbfs_mesh_find_periodic_nodes(&md, T, partner.data()), "lbfs_mesh_find_periodic_nodes");
        md.periodic_node = partner.data();
    }
    // plateau meshes: the vertex coordinates the 4x4x4 IBM searches (Solver_gpu.cu:497-499, 637-639)
    std::vector<double> plateau[3];
    if (globals.mesh_type == 4) {
        const double len[3] = {domain.X, domain.Y, domain.Z};
        for (int a = 0; a < 3; a++) {
            const int n = (int)std::ceil(len[a] / domain.dt * 0.5) + 1;
            plateau[a].resize(n);
            for (int i = 0; i < n; i++)
                plateau[a][i] = a == 0 ? Mesh.get_plateau_x(i) : (a == 1 ? Mesh.get_plateau_y(i) : Mesh.get_plateau_z(i));
        }
        md.grid_x = plateau[0].data(); md.grid_y = plateau[1].data(); md.grid_z = plateau[2].data();
    }

    lbfs_params p = {};
    p.visc = globals.visc;
    p.delta_t = globals.time_marching_step;
    p.gamma_inv = 1 / globals.pre_conditioned_gamma;
    p.channel_diameter = domain.Y;
    p.body_force[0] = init_conds.force_x; p.body_force[1] = init_conds.force_y; p.body_force[2] = init_conds.force_z;
    p.ref_rho = globals.ref_rho;
    p.max_velocity = globals.max_velocity;
    p.rho0 = init_conds.average_rho;
    // visc_factor: 1 for testcase 2 (Solver_gpu.cu:738); otherwise the
    // reference reads it before its first update at t = 1 (zero-filled pages)
    p.visc_factor_initial = globals.testcase == 2 ? 1.0 : 0.0;
    p.testcase = globals.testcase;
    p.precision = LBFS_FP64;
    // interpolate_velocities_on_nodes(_non_uniform_grid), Solver_gpu.cu:810-820
    p.ibm_stencil = globals.mesh_type == 4 ? LBFS_IBM_VANDERMONDE4 : LBFS_IBM_HAT2;
    p.viscosity_period = 10000;
    // local = 1, constant = 2, min = 3, talts = 4 (global_variables.h:59)
    p.time_stepping = globals.gpu_time_stepping;
    p.pre_conditioned_gamma = globals.pre_conditioned_gamma;
    p.preconditioning = globals.preconditioning_active ? 1 : 0;

    // membranes (Solver_gpu.cu:659-735): sprIdx / sorted_triIdx / stress-free
    // coordinates, then the initial mesh read over the node arrays
    std::vector<lbfs_rbc_desc> rbc;
    std::vector<std::vector<double>> sf, init;
    if (globals.testcase != 2) {
        for (lagrangian_object &o : object_vec) {
            if (o.type != 2) continue;
            sf.emplace_back(o.sorted_coordinate, o.sorted_coordinate + 3 * (size_t)o.num_nodes);
            if (o.mz_importer) o.read_initial_mesh_MZ(o.mesh_file);
            else o.read_initial_mesh(o.mesh_file);
            std::vector<double> xyz(3 * (size_t)o.num_nodes);
            for (int n = 0; n < o.num_nodes; n++) {
                xyz[3 * n] = o.node_x[n]; xyz[3 * n + 1] = o.node_y[n]; xyz[3 * n + 2] = o.node_z[n];
            }
            init.push_back(xyz);
            lbfs_rbc_desc d = {};
            d.n_nodes = o.num_nodes; d.n_tris = o.num_tets; d.n_springs = o.num_springs;
            d.tri = o.sorted_triIdx; d.spring = o.sprIdx;
            d.volume_modulus = o.volume_modulus; d.local_area_modulus = o.local_area_modulus;
            d.global_area_modulus = o.global_area_modulus; d.shear_modulus = o.shear_modulus;
            d.global_bending_modulus = o.global_bending_modulus; d.local_bending_modulus = o.local_bending_modulus;
            d.membrane_thickness = o.membrane_thickness; d.viscosity = o.viscosity; d.wlc_ratio = o.wlc_ratio;
            d.curvature_ratio = o.curvature_ratio; d.volume_ratio = o.volume_ratio;
            d.internal_viscosity_ratio = o.internal_viscosity_ratio; d.reference_length = o.reference_length;
            d.pivkin_length = o.pivkin_length; d.sphere_reference = o.sphere_reference;
            // the reference's gate of check_periodic_object (Solver_gpu.cu:1027): object 0's flag, one mean
            // over every object's nodes, all objects moved together
            d.periodic = object_vec[0].periodic ? LBFS_WRAP_ALL : 0;
            rbc.push_back(d);
        }
        for (size_t k = 0; k < rbc.size(); k++) {
            rbc[k].xyz_stress_free = sf[k].data();
            rbc[k].xyz_initial = init[k].data();
        }
    }

    lbfs_solver *s = nullptr;
    lbfs_check(lbfs_create(&md, &p, rbc.data(), (int32_t)rbc.size(), globals.gpu_device, &s), "lbfs_create");
    std::vector<double> rho(nc), u(nc), v(nc), w(nc);
    for (int i = 0; i < nc; i++) { rho[i] = soln.get_rho(i); u[i] = soln.get_u(i); v[i] = soln.get_v(i); w[i] = soln.get_w(i); }
    lbfs_check(lbfs_set_state(s, rho.data(), u.data(), v.data(), w.data()), "lbfs_set_state");

    const int timesteps = (int)std::ceil(globals.simulation_length);
    // the reference tests convergence on the residuals after every step (Solver_gpu.cu:1206); with a
    // tolerance the library runs that test on the device after every step (lbfs_step_until), without
    // one the steps go in chunks of output_step
    if (globals.tolerance > 0) {
        int32_t done = 0;
        double rms[4];
        lbfs_check(lbfs_step_until(s, timesteps, globals.tolerance, &done, rms), "lbfs_step_until");
        uint32_t flags = 0;
        lbfs_check(lbfs_status(s, &flags), "lbfs_status");
        if (flags & (LBFS_FLAG_NONFINITE | LBFS_FLAG_RHO_RANGE)) {
            std::fprintf(stderr, "lbfs_b200: solution diverged (flags %u) at step %d\n", flags, done);
            std::exit(-1);
        }
    }
    const int chunk = globals.output_step > 0 ? globals.output_step : 1;
    for (int t = 0; globals.tolerance <= 0 && t < timesteps; t += chunk) {
        const int n = std::min(chunk, timesteps - t);
        lbfs_check(lbfs_step_graph(s, n), "lbfs_step_graph");
        double rms[4];
        lbfs_check(lbfs_get_residuals(s, rms), "lbfs_get_residuals");
        uint32_t flags = 0;
        lbfs_check(lbfs_status(s, &flags), "lbfs_status");
        if (flags & (LBFS_FLAG_NONFINITE | LBFS_FLAG_RHO_RANGE)) {
            std::fprintf(stderr, "lbfs_b200: solution diverged (flags %u) at step %d\n", flags, t + n);
            std::exit(-1);
        }
    }
    lbfs_check(lbfs_get_state(s, rho.data(), u.data(), v.data(), w.data()), "lbfs_get_state");
    for (int i = 0; i < nc; i++) soln.update(rho[i], u[i], v[i], w[i], i);
    lbfs_destroy(s);
}
