// Driver of the reference's own program set-up (test and bench infrastructure).
//
// It performs what program::run does (program.cpp:40-113): the XML deck through
// the reference's preprocessor (preprocessor::initialise_program_variables), the
// lagrangian object's initialise, the generated unstructured mesh, the boundary
// conditions, the external force and the initial solution -- and then calls
// gpu_solver::General_Purpose_Solver_mk_i with those objects.  oracle/build_ref.sh
// links it with the drop-in replacement of that method
// (lbfs-ibm-ade-sp_b200/integration/Solver_gpu_lbfs.cpp over liblbfs_b200.so):
// the reference's host code calling this repository's library through the
// reference's own entry point.  oracle/build_ref_gpu.sh links it with the
// reference's own Solver_gpu.cu built for sm_100a (the reference GPU
// baseline), and built with REF_CPU_SOLVER it calls the reference's CPU
// Solver::General_Purpose_Solver_mk_i instead (program.cpp:120-123).
//
//   dropin_program DECK.xml OUT_PREFIX [STATE0.bin] [--dump-only]
//
// STATE0.bin (optional): n_cells doubles each of rho, u, v, w replacing the
// deck's initial solution (a seeded perturbation, Solution::update).
// Writes OUT_PREFIX_params.txt (the scalars and sizes as the solver receives
// them), OUT_PREFIX_inputs.bin (initial rho, u, v, w; bc rho/vel types and
// values; membrane triangles, springs, stress-free and initial coordinates),
// and, unless --dump-only, OUT_PREFIX_state.bin (rho, u, v, w after the solver
// call) and OUT_PREFIX_run.txt (host wall-clock seconds of the call).
#include <chrono>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "Boundary_Conditions.h"
#include "Solution.h"
#ifdef REF_CPU_SOLVER
#include "Solver.h"
#else
#include "Solver_gpu.h"
#endif
#ifdef REF_GPU_PROGRAM
#include <cuda_runtime.h>
#endif
#include "domain_geometry.h"
#include "external_forces.h"
#include "global_variables.h"
#include "initial_conditions.h"
#include "lagrangian_object.h"
#include "post_processing.h"
#include "preprocessor.h"
#include "quad_bcs_plus.h"
#include "unstructured_bcs.h"
#include "unstructured_mesh.h"

namespace {

template <typename T> void put(std::ofstream &f, const T *p, size_t n) { f.write((const char *)p, sizeof(T) * n); }

}  // namespace

int main(int argc, char **argv) {
    if (argc < 3) {
        std::fprintf(stderr, "usage: %s DECK.xml OUT_PREFIX [STATE0.bin] [--dump-only]\n", argv[0]);
        return 2;
    }
    const std::string deck = argv[1], out = argv[2];
    std::string state_file;
    bool dump_only = false;
    for (int a = 3; a < argc; a++) {
        if (std::strcmp(argv[a], "--dump-only") == 0) dump_only = true;
        else state_file = argv[a];
    }
    std::streambuf *cout_buf = std::cout.rdbuf();
    std::ofstream log(out + "_log.txt");
    std::cout.rdbuf(log.rdbuf());  // the reference's progress printing goes to the log

    quad_bcs_plus bcs;
    unstructured_bcs u_bcs;
    global_variables globals;
    domain_geometry domain;
    initial_conditions initial_conds;
    std::vector<lagrangian_object> objects;
    preprocessor pre;
    std::vector<char> deck_path(deck.begin(), deck.end());
    deck_path.push_back('\0');
    pre.initialise_program_variables(deck_path.data(), globals, domain, initial_conds, bcs, u_bcs, objects);
    std::filesystem::create_directories(globals.output_file);  // program.cpp copies the deck there first
    objects[0].initialise(globals.PI);

    Solution soln, residual;
    unstructured_mesh mesh(domain, globals);
    Boundary_Conditions bc(mesh.get_num_bc());
    external_forces source_term(mesh.get_total_cells());
    source_term.set_uniform_force(initial_conds.pressure_gradient);
    soln.assign_memory(mesh.get_total_cells());
    residual.assign_memory(mesh.get_total_cells());
    post_processing post_processor(mesh.get_total_cells());
    soln.assign_pressure_gradient(initial_conds.rho_gradient, initial_conds.origin_loc, initial_conds.rho_origin_mag,
                                  mesh, globals);
    soln.assign_velocity_gradient(initial_conds.vel_gradient, initial_conds.origin_loc, initial_conds.vel_origin_mag,
                                  mesh, globals);
    soln.set_average_rho(initial_conds.average_rho);
    const int nc = mesh.get_n_cells(), nb = mesh.get_num_bc();
    if (!state_file.empty()) {
        std::vector<double> s0(4 * (size_t)nc);
        std::ifstream f(state_file, std::ios::binary);
        f.read((char *)s0.data(), sizeof(double) * s0.size());
        if (!f) {
            std::cout.rdbuf(cout_buf);
            std::fprintf(stderr, "cannot read %zu doubles from %s\n", s0.size(), state_file.c_str());
            return 1;
        }
        for (int i = 0; i < nc; i++) soln.update(s0[i], s0[nc + i], s0[2 * (size_t)nc + i], s0[3 * (size_t)nc + i], i);
    }
    bc.assign_boundary_conditions(mesh, u_bcs);

    // the inputs as the solver receives them
    {
        lagrangian_object &o = objects[0];
        std::ofstream p(out + "_params.txt");
        p.precision(17);
        p << "n_cells " << nc << "\nn_bc " << nb << "\nn_faces " << mesh.get_n_faces() << "\n";
        p << "X " << domain.X << "\nY " << domain.Y << "\nZ " << domain.Z << "\ndt " << domain.dt << "\n";
        p << "origin_x " << domain.origin_x << "\norigin_y " << domain.origin_y << "\norigin_z " << domain.origin_z << "\n";
        p << "visc " << globals.visc << "\ndelta_t " << globals.time_marching_step << "\n";
        p << "pre_conditioned_gamma " << globals.pre_conditioned_gamma << "\n";
        p << "preconditioning " << (globals.preconditioning_active ? 1 : 0) << "\n";
        p << "time_stepping " << globals.gpu_time_stepping << "\n";
        p << "force_x " << initial_conds.force_x << "\nforce_y " << initial_conds.force_y << "\nforce_z "
          << initial_conds.force_z << "\n";
        p << "ref_rho " << globals.ref_rho << "\nmax_velocity " << globals.max_velocity << "\n";
        p << "testcase " << globals.testcase << "\nmesh_type " << globals.mesh_type << "\n";
        p << "simulation_length " << globals.simulation_length << "\ntolerance " << globals.tolerance << "\n";
        p << "average_rho " << initial_conds.average_rho << "\n";
        p << "n_nodes " << o.num_nodes << "\nn_tris " << o.num_tets << "\nn_springs " << o.num_springs << "\n";
        p << "volume_modulus " << o.volume_modulus << "\nlocal_area_modulus " << o.local_area_modulus << "\n";
        p << "global_area_modulus " << o.global_area_modulus << "\nshear_modulus " << o.shear_modulus << "\n";
        p << "global_bending_modulus " << o.global_bending_modulus << "\nlocal_bending_modulus "
          << o.local_bending_modulus << "\n";
        p << "membrane_thickness " << o.membrane_thickness << "\nviscosity " << o.viscosity << "\n";
        p << "wlc_ratio " << o.wlc_ratio << "\ncurvature_ratio " << o.curvature_ratio << "\n";
        p << "volume_ratio " << o.volume_ratio << "\ninternal_viscosity_ratio " << o.internal_viscosity_ratio << "\n";
        p << "reference_length " << o.reference_length << "\npivkin_length " << (o.pivkin_length ? 1 : 0) << "\n";
        p << "sphere_reference " << (o.sphere_reference ? 1 : 0) << "\nperiodic " << (o.periodic ? 1 : 0) << "\n";
        std::ofstream b(out + "_inputs.bin", std::ios::binary);
        std::vector<double> s(nc);
        for (int i = 0; i < nc; i++) s[i] = soln.get_rho(i);
        put(b, s.data(), nc);
        for (int i = 0; i < nc; i++) s[i] = soln.get_u(i);
        put(b, s.data(), nc);
        for (int i = 0; i < nc; i++) s[i] = soln.get_v(i);
        put(b, s.data(), nc);
        for (int i = 0; i < nc; i++) s[i] = soln.get_w(i);
        put(b, s.data(), nc);
        std::vector<int> rt(nb), vt(nb);
        std::vector<double> bv(4 * (size_t)nb);
        for (int i = 0; i < nb; i++) {
            rt[i] = bc.get_rho_type(i);
            vt[i] = bc.get_vel_type(i);
            bv[4 * i] = bc.get_u(i); bv[4 * i + 1] = bc.get_v(i); bv[4 * i + 2] = bc.get_w(i); bv[4 * i + 3] = bc.get_rho(i);
        }
        put(b, rt.data(), nb);
        put(b, vt.data(), nb);
        put(b, bv.data(), bv.size());
        put(b, o.sorted_triIdx, 3 * (size_t)o.num_tets);
        put(b, o.sprIdx, 4 * (size_t)o.num_springs);
        put(b, o.sorted_coordinate, 3 * (size_t)o.num_nodes);
        // the initial mesh the solver reads over the nodes (Solver_gpu.cu:717); the drop-in reads it again
        lagrangian_object probe = o;
        probe.read_initial_mesh(o.mesh_file);
        std::vector<double> xyz(3 * (size_t)o.num_nodes);
        for (int n = 0; n < o.num_nodes; n++) {
            xyz[3 * n] = probe.node_x[n]; xyz[3 * n + 1] = probe.node_y[n]; xyz[3 * n + 2] = probe.node_z[n];
        }
        put(b, xyz.data(), xyz.size());
    }
    if (dump_only) {
        std::cout.rdbuf(cout_buf);
        return 0;
    }

#ifdef REF_CPU_SOLVER
    // the reference's CPU path (program.cpp:120-123): fluid only, serial
    Solver solve;
    const auto t0 = std::chrono::steady_clock::now();
    solve.General_Purpose_Solver_mk_i(mesh, soln, bc, source_term, globals, domain, initial_conds, u_bcs, 0, residual,
                                      0, post_processor);
#else
#ifdef REF_GPU_PROGRAM
    // the CUDA context is created before the timed call: it is not part of the solver's work
    cudaSetDevice(globals.gpu_device);
    cudaFree(nullptr);
#endif
    gpu_solver gpu;
    const auto t0 = std::chrono::steady_clock::now();
    gpu.General_Purpose_Solver_mk_i(mesh, soln, bc, source_term, globals, domain, initial_conds, u_bcs, 0, residual, 0,
                                    post_processor, objects);
#endif
    const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::cout.rdbuf(cout_buf);
    {
        std::ofstream b(out + "_state.bin", std::ios::binary);
        std::vector<double> s(nc);
        for (int i = 0; i < nc; i++) s[i] = soln.get_rho(i);
        put(b, s.data(), nc);
        for (int i = 0; i < nc; i++) s[i] = soln.get_u(i);
        put(b, s.data(), nc);
        for (int i = 0; i < nc; i++) s[i] = soln.get_v(i);
        put(b, s.data(), nc);
        for (int i = 0; i < nc; i++) s[i] = soln.get_w(i);
        put(b, s.data(), nc);
        std::ofstream r(out + "_run.txt");
        r.precision(17);
        r << "seconds " << sec << "\nn_cells " << nc << "\nsteps " << globals.simulation_length << "\n";
    }
    return 0;
}
