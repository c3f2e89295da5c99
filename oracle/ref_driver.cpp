// Reference driver: runs the UNMODIFIED reference sources, compiled for the
// host with the stubs in oracle/ref_stub/, to produce golden vectors.
//
// Test infrastructure only.  It is built by oracle/build_ref.sh into
// oracle/_ref/libref_lbfs.so and is called from tests/golden/make_golden.py
// (fixture generation) and from bench.py's reference arm.  Nothing in the
// product links or loads it.
//
// What it drives:
//   * unstructured_mesh (uniform OpenFOAM-layout generator, mesh_type 6) and
//     gradients::pre_fill_LHS_and_RHS_matrix  -> mesh arrays exactly as
//     gpu_solver::General_Purpose_Solver_mk_i copies them (Solver_gpu.cu:625-655);
//   * lagrangian_object::initialise (Osay reader, spring hashing)
//     -> sprIdx / triangle arrays as lagrangian_spring_network_to_array copies
//     them (Solver_gpu.cu:1891-1945);
//   * the GPU time loop Solver_gpu.cu:749-1021 restated as a sequence of calls
//     to the reference's own __global__ kernel bodies (run serially on the host,
//     one "launch" = one direct call with a 1x1 grid), including the host-side
//     block-partial sums of total<128> / sum_product_curvature<128>.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "unstructured_mesh.h"
#include "gradients.h"
#include "Boundary_Conditions.h"
#include "Solution.h"
#include "lagrangian_object.h"
#include "LBFS.hpp"
#include "immersed_boundary_method.hpp"
#include "spring_network.hpp"
#include "common_kernels.hpp"

uint3 threadIdx = {0, 0, 0};
uint3 blockIdx = {0, 0, 0};
dim3 blockDim = {1, 1, 1};
dim3 gridDim = {1, 1, 1};

namespace {

struct NullBuf : std::streambuf {
    int overflow(int c) override { return c; }
};

struct Quiet {  // silence the reference's progress printing on std::cout
    NullBuf nb;
    std::streambuf *old;
    Quiet() { old = std::cout.rdbuf(&nb); }
    ~Quiet() { std::cout.rdbuf(old); }
};

struct RefMesh {
    domain_geometry domain;
    global_variables globals;
    unstructured_mesh *mesh = nullptr;
    gradients *grads = nullptr;
};

// Host emulation of total<128> launched on ceil(n/128) blocks
// (common_kernels.hpp:71-94): each block tree-sums 256 consecutive entries,
// then the host adds the block partials in order (lagrangian_object::add_*,
// residuals::l2_norm_rms_moukallad).
double block_tree_total(const double *v, int n, int n_blocks, const double *v2 = nullptr, bool curvature = false) {
    double total = 0.0;
    for (int b = 0; b < n_blocks; b++) {
        double part[256];
        unsigned start = 2u * b * 128u;
        for (int t = 0; t < 256; t++) {
            unsigned idx = start + t;
            if ((int)idx < n) {
                if (curvature) part[t] = v[idx] * (v2[idx * 2] + v2[idx * 2 + 1]) * 1 / 3;
                else part[t] = v[idx];
            } else {
                part[t] = 0;
            }
        }
        for (unsigned stride = 128; stride >= 1; stride >>= 1)
            for (unsigned t = 0; t < stride; t++) part[t] += part[t + stride];
        total = total + part[0];
    }
    return total;
}

double block_min_max(const double *v, int n, int n_blocks, bool is_min) {
    // min<128>/max<128> (common_kernels.hpp:147-196) then min_block/max_block on the host.
    double r = is_min ? 100000000.0 : -100000000.0;
    for (int b = 0; b < n_blocks; b++) {
        double part[256];
        unsigned start = 2u * b * 128u;
        for (int t = 0; t < 256; t++) {
            unsigned idx = start + t;
            part[t] = ((int)idx < n) ? v[idx] : (is_min ? 100000000 : -100000000);
        }
        for (unsigned stride = 128; stride >= 1; stride >>= 1)
            for (unsigned t = 0; t < stride; t++)
                part[t] = is_min ? std::fmin(part[t + stride], part[t]) : std::fmax(part[t + stride], part[t]);
        r = is_min ? std::fmin(r, part[0]) : std::fmax(r, part[0]);
    }
    return r;
}

}  // namespace

// ---------------------------------------------------------------- mesh ----
extern "C" void *ref_mesh_create(double X, double Y, double Z, double dt, double ox, double oy, double oz,
                                 double visc, int gradient_hybrid, const char *outdir, int mesh_type,
                                 double plateau_width, double plateau_slope, const char *import_dir) {
    Quiet q;
    RefMesh *m = new RefMesh();
    m->domain.X = X; m->domain.Y = Y; m->domain.Z = Z; m->domain.dt = dt;
    m->domain.dx = 2 * dt; m->domain.dy = 2 * dt; m->domain.dz = 2 * dt;
    m->domain.origin_x = ox; m->domain.origin_y = oy; m->domain.origin_z = oz;
    m->domain.ref_length = Y; m->domain.plateau_width = plateau_width; m->domain.plateau_slope = plateau_slope;
    m->domain.IBM_face = "none";
    m->globals.mesh_type = mesh_type;
    m->globals.import_format = "openfoam";
    // mesh_type 3 reads the polyMesh in import_dir (import_openfoam_mesh); the
    // generated types find no boundary file here
    m->globals.import_file = import_dir ? std::string(import_dir) + "/" : std::string(outdir) + "/no_such_case/";
    m->globals.output_file = outdir;
    m->globals.testcase = 1;
    m->globals.visc = visc;
    m->globals.pre_conditioned_gamma = 1;
    m->globals.fneq_min = 0.0;
    m->globals.gradient_calc_type = gradient_hybrid ? "hybrid" : "LS";
    m->mesh = new unstructured_mesh(m->domain, m->globals);
    m->grads = new gradients(m->mesh->get_total_cells());
    Boundary_Conditions bcs(m->mesh->get_num_bc());
    Solution soln(m->mesh->get_total_cells());
    m->grads->pre_fill_LHS_and_RHS_matrix(bcs, *m->mesh, m->domain, soln, m->globals);
    return m;
}

extern "C" void ref_mesh_counts(void *h, int *out) {
    RefMesh *m = (RefMesh *)h;
    out[0] = m->mesh->get_n_cells();
    out[1] = m->mesh->get_n_faces();
    out[2] = m->mesh->get_n_neighbours();
    out[3] = m->mesh->get_num_bc();
    out[4] = m->mesh->get_n_face_x();
    out[5] = m->mesh->get_n_face_y();
    out[6] = m->mesh->get_n_face_z();
    out[7] = m->mesh->get_total_cells();
}

extern "C" void ref_mesh_dump(void *h, int *owner, int *neighbour, double *area, double *normal, double *fcen,
                              double *sdt, double *vol, double *ccen, int *stencil, double *lhs, double *rhs,
                              double *delta_h) {
    RefMesh *m = (RefMesh *)h;
    unstructured_mesh &M = *m->mesh;
    int nf = M.get_n_faces(), nt = M.get_total_cells(), nc = M.get_n_cells();
    for (int f = 0; f < nf; f++) {
        owner[f] = M.get_mesh_owner(f);
        neighbour[f] = M.get_mesh_neighbour(f);
        area[f] = M.get_face_area(f);
        normal[3 * f] = M.get_face_i(f); normal[3 * f + 1] = M.get_face_j(f); normal[3 * f + 2] = M.get_face_k(f);
        fcen[3 * f] = M.get_face_x(f); fcen[3 * f + 1] = M.get_face_y(f); fcen[3 * f + 2] = M.get_face_z(f);
        sdt[f] = M.get_delta_t_face(f);
    }
    for (int c = 0; c < nt; c++) {
        vol[c] = M.get_cell_volume(c);
        ccen[3 * c] = M.get_centroid_x(c); ccen[3 * c + 1] = M.get_centroid_y(c); ccen[3 * c + 2] = M.get_centroid_z(c);
    }
    gradients &G = *m->grads;
    for (int c = 0; c < nc; c++) {
        for (int j = 0; j < 6; j++) {
            stencil[6 * c + j] = M.gradient_cells[c][j];
            rhs[18 * c + 3 * j] = G.RHS_x[c * 6 + j];
            rhs[18 * c + 3 * j + 1] = G.RHS_y[c * 6 + j];
            rhs[18 * c + 3 * j + 2] = G.RHS_z[c * 6 + j];
        }
        double *L = lhs + 9 * c;
        L[0] = G.LHS_xx[c]; L[1] = G.LHS_xy[c]; L[2] = G.LHS_xz[c];
        L[3] = G.LHS_yx[c]; L[4] = G.LHS_yy[c]; L[5] = G.LHS_yz[c];
        L[6] = G.LHS_zx[c]; L[7] = G.LHS_zy[c]; L[8] = G.LHS_zz[c];
    }
    *delta_h = M.get_delta_h();
}

// The generator's plateau arrays (Solver_gpu.cu:637-639, mesh_to_array): [nx+1], [ny+1], [nz+1].
extern "C" void ref_mesh_plateau(void *h, int nx, int ny, int nz, double *out) {
    unstructured_mesh &M = *((RefMesh *)h)->mesh;
    for (int i = 0; i < nx + 1; i++) out[i] = M.get_plateau_x(i);
    for (int i = 0; i < ny + 1; i++) out[nx + 1 + i] = M.get_plateau_y(i);
    for (int i = 0; i < nz + 1; i++) out[nx + ny + 2 + i] = M.get_plateau_z(i);
}

extern "C" void ref_mesh_free(void *h) { delete (RefMesh *)h; }

// ----------------------------------------------------------------- RBC ----
extern "C" void *ref_rbc_create(const char *stress_free_file, double cx, double cy, double cz) {
    Quiet q;
    lagrangian_object *o = new lagrangian_object();
    o->type = 2;
    o->mz_importer = false;
    o->stress_free_mesh = stress_free_file;
    o->centre_x = cx; o->centre_y = cy; o->centre_z = cz;
    o->initialise(acos(-1.0));
    return o;
}

extern "C" void ref_rbc_counts(void *h, int *out) {
    lagrangian_object *o = (lagrangian_object *)h;
    out[0] = o->num_nodes; out[1] = o->num_tets; out[2] = o->num_springs; out[3] = o->maxFreedom;
}

extern "C" void ref_rbc_dump(void *h, int *spr, int *tri, double *xyz) {
    lagrangian_object *o = (lagrangian_object *)h;
    for (int i = 0; i < o->num_springs * 4; i++) spr[i] = o->sprIdx[i];
    for (int i = 0; i < o->num_tets * 3; i++) tri[i] = o->sorted_triIdx[i];
    for (int i = 0; i < o->num_nodes * 3; i++) xyz[i] = o->sorted_coordinate[i];
}

extern "C" void ref_rbc_free(void *h) { delete (lagrangian_object *)h; }

// ------------------------------------------------------------ time loop ----
// Parameters of one case.  Field meanings follow global_variables /
// lagrangian_object; values arrive already scaled (as after
// preprocessor::mach_number_factor).
struct ref_params {
    double visc, delta_t, gamma_inv, channel_diameter;
    double force[3];
    double ref_rho, max_velocity;
    int testcase;
    double visc_factor_initial;
    int has_rbc;
    // RBC (object_vec[0])
    double volume_modulus, local_area_modulus, global_area_modulus, shear_modulus;
    double global_bending_modulus, local_bending_modulus, membrane_thickness, viscosity;
    double wlc_ratio, curvature_ratio, volume_ratio, internal_viscosity_ratio, reference_length;
    int pivkin_length, sphere_reference;
    int viscosity_period;  // update_viscosities when t % period == 1
    int time_stepping;     // globals.gpu_time_stepping: 1 local, 2 constant, 3 min, 4 talts (0 = 2)
    double pre_conditioned_gamma;  // get_cfl_device's gamma (0 = 1 / gamma_inv)
    int preconditioning;           // globals.preconditioning_active
    int object_periodic;           // object_vec[0].periodic (check_periodic_object)
};

namespace {
struct RefCase {
    RefMesh *m;
    ref_params p;
    int nc, nf, nn, nb, nt, nfx, nfy, nfz;
    std::vector<double4> soln, t0, t1, bcs_arr, res_face;
    std::vector<int> owner, neighbour, stencil, rho_type, vel_type;
    std::vector<double3> ccen, fnorm, fcen, rhs, g_rho, g_u, g_v, g_w;
    std::vector<double> vol, area, sdt, L[9], res_rho, res_u, res_v, res_w, fx, fy, fz, visc_factor, local_fneq, dtl;
    std::vector<double3> cfl_areas;
    double delta_t = 0;  // the step's delta_t (the loop's variable)
    std::vector<double> plateau[3];  // mesh_type 4: vertex coordinates per axis (Solver_gpu.cu:637-639)
    double residual_rms[4];
    // RBC
    int n_nodes = 0, n_tets = 0, n_springs = 0;
    std::vector<int> spr, tri;
    std::vector<double> x, y, z, vx, vy, vz, nfx_, nfy_, nfz_, tet_area, tet_vol, tnx, tny, tnz;
    std::vector<double> contour, kspring, curv, curv0, sangle, sangle0, sarea, sarea0, dummy;
    double V = 0, V0 = 0, A = 0, A0 = 0, MAD = 0, MAD0 = 0;
    int t = 0;
};

void spring_network_pass(RefCase &c, bool initials) {
    // gpu_solver::run_spring_network_functions_atomics, Solver_gpu.cu:2311-2361
    update_spring_network_tet_parameters(c.n_tets, c.x.data(), c.y.data(), c.z.data(), c.tri.data(), c.dummy.data(),
                                         c.tet_vol.data(), c.tet_area.data(), c.tnx.data(), c.tny.data(), c.tnz.data());
    int n_tet_blocks = (c.n_tets + 127) / 128;
    c.V = block_tree_total(c.tet_vol.data(), c.n_tets, n_tet_blocks);
    if (initials) c.V0 = c.V * c.p.volume_ratio;
    c.A = block_tree_total(c.tet_area.data(), c.n_tets, n_tet_blocks);
    if (initials) c.A0 = c.A;
    get_spring_forces_atomics(c.n_springs, c.nfx_.data(), c.nfy_.data(), c.nfz_.data(), c.x.data(), c.y.data(), c.z.data(),
                              c.p.volume_modulus, c.V, c.V0, c.spr.data(), nullptr, 0,
                              c.p.local_area_modulus, c.p.global_area_modulus, c.A, c.A0, c.sarea.data(), c.sarea0.data(),
                              c.tnx.data(), c.tny.data(), c.tnz.data(), nullptr, c.contour.data(), c.kspring.data(),
                              c.p.global_bending_modulus, c.MAD, c.MAD0, c.p.membrane_thickness, c.p.local_bending_modulus,
                              c.curv.data(), c.curv0.data(), c.sangle.data(), c.p.viscosity, c.vx.data(), c.vy.data(), c.vz.data(),
                              c.p.wlc_ratio, nullptr, nullptr, nullptr, c.sangle0.data(), c.p.shear_modulus, initials, 0.0);
    int n_node_blocks = (c.n_nodes + 127) / 128;
    c.MAD = block_tree_total(c.curv.data(), c.n_nodes, n_node_blocks, c.sarea.data(), true);
    c.MAD = c.MAD / c.A;
    if (initials) c.MAD0 = c.MAD;
}
}  // namespace

extern "C" void *ref_case_create(void *mesh, const ref_params *p, const int *rho_type, const int *vel_type,
                                 const double *bc_values /* 4*n_bc: u,v,w,rho */) {
    RefCase *c = new RefCase();
    c->m = (RefMesh *)mesh;
    c->p = *p;
    unstructured_mesh &M = *c->m->mesh;
    c->nc = M.get_n_cells(); c->nf = M.get_n_faces(); c->nn = M.get_n_neighbours(); c->nb = M.get_num_bc();
    c->nt = M.get_total_cells(); c->nfx = M.get_n_face_x(); c->nfy = M.get_n_face_y(); c->nfz = M.get_n_face_z();
    int nt = c->nt, nf = c->nf, nc = c->nc, nb = c->nb;
    c->soln.assign(nt, make_double4(0, 0, 0, 0)); c->t0 = c->soln; c->t1 = c->soln;
    c->res_face.assign(nf, make_double4(0, 0, 0, 0));
    c->owner.resize(nf); c->neighbour.resize(nf); c->area.resize(nf); c->sdt.resize(nf); c->fnorm.resize(nf); c->fcen.resize(nf);
    for (int f = 0; f < nf; f++) {
        c->owner[f] = M.get_mesh_owner(f); c->neighbour[f] = M.get_mesh_neighbour(f);
        c->area[f] = M.get_face_area(f); c->sdt[f] = M.get_delta_t_face(f);
        c->fnorm[f] = make_double3(M.get_face_i(f), M.get_face_j(f), M.get_face_k(f));
        c->fcen[f] = make_double3(M.get_face_x(f), M.get_face_y(f), M.get_face_z(f));
    }
    c->vol.resize(nt); c->ccen.resize(nt);
    for (int i = 0; i < nt; i++) {
        c->vol[i] = M.get_cell_volume(i);
        c->ccen[i] = make_double3(M.get_centroid_x(i), M.get_centroid_y(i), M.get_centroid_z(i));
    }
    c->stencil.resize(6 * nc); c->rhs.resize(6 * nc);
    gradients &G = *c->m->grads;
    for (int k = 0; k < 9; k++) c->L[k].resize(nc);
    for (int i = 0; i < nc; i++) {
        for (int j = 0; j < 6; j++) {
            c->stencil[6 * i + j] = M.gradient_cells[i][j];
            c->rhs[6 * i + j] = make_double3(G.RHS_x[6 * i + j], G.RHS_y[6 * i + j], G.RHS_z[6 * i + j]);
        }
        c->L[0][i] = G.LHS_xx[i]; c->L[1][i] = G.LHS_xy[i]; c->L[2][i] = G.LHS_xz[i];
        c->L[3][i] = G.LHS_yx[i]; c->L[4][i] = G.LHS_yy[i]; c->L[5][i] = G.LHS_yz[i];
        c->L[6][i] = G.LHS_zx[i]; c->L[7][i] = G.LHS_zy[i]; c->L[8][i] = G.LHS_zz[i];
    }
    c->rho_type.assign(rho_type, rho_type + nb);
    c->vel_type.assign(vel_type, vel_type + nb);
    c->bcs_arr.resize(nb);
    for (int i = 0; i < nb; i++)
        c->bcs_arr[i] = make_double4(bc_values[4 * i], bc_values[4 * i + 1], bc_values[4 * i + 2], bc_values[4 * i + 3]);
    c->g_rho.assign(nt, make_double3(0, 0, 0)); c->g_u = c->g_rho; c->g_v = c->g_rho; c->g_w = c->g_rho;
    c->res_rho.assign(nt, 0.0); c->res_u = c->res_rho; c->res_v = c->res_rho; c->res_w = c->res_rho;
    c->fx.assign(nt, 0.0); c->fy = c->fx; c->fz = c->fx;
    c->visc_factor.assign(nc, p->visc_factor_initial);
    c->local_fneq.assign(nt, 0.0);
    c->dtl.assign(nc, p->delta_t);
    c->delta_t = p->delta_t;
    if (c->m->globals.mesh_type != 3) {  // generated meshes only: the importer allocates no plateau arrays
        domain_geometry &D = c->m->domain;
        const int n[3] = {(int)ceil(D.X / D.dt * 0.5), (int)ceil(D.Y / D.dt * 0.5), (int)ceil(D.Z / D.dt * 0.5)};
        for (int a = 0; a < 3; a++) {
            c->plateau[a].resize(n[a] + 1);
            for (int i = 0; i < n[a] + 1; i++)
                c->plateau[a][i] = a == 0 ? M.get_plateau_x(i) : (a == 1 ? M.get_plateau_y(i) : M.get_plateau_z(i));
        }
    }
    // gpu_solver::populate_cfl_areas (Solver_gpu.cu:1657-1687), restated: the
    // method is a member of the GPU solver class, which is not built here
    c->cfl_areas.assign(nc, make_double3(0, 0, 0));
    for (int i = 0; i < nc; i++) {
        double ax = 0, ay = 0, az = 0;
        for (int f = 0; f < (int)M.gradient_faces[i].size(); f++) {
            const int face = M.gradient_faces[i][f];
            ax = ax + fabs(M.get_face_i(face) * M.get_face_area(face));
            ay = ay + fabs(M.get_face_j(face) * M.get_face_area(face));
            az = az + fabs(M.get_face_k(face) * M.get_face_area(face));
        }
        c->cfl_areas[i] = make_double3(ax / 2, ay / 2, az / 2);
    }
    // D3Q15 weights, gpu_solver::populate_e_alpha (Solver_gpu.cu:1407-1445)
    for (int k = 0; k < 15; k++) lattice_weight[k] = (k > 0 && k < 7) ? 1.0 / 9.0 : (k > 6 ? 1.0 / 72.0 : 2.0 / 9.0);
    return c;
}

extern "C" void ref_case_set_state(void *h, const double *rho, const double *u, const double *v, const double *w) {
    RefCase *c = (RefCase *)h;
    for (int i = 0; i < c->nc; i++) c->soln[i] = make_double4(u[i], v[i], w[i], rho[i]);
    // Solver_gpu.cu:746: soln_t1 starts as a copy of the primitive state
    for (int i = 0; i < c->nc; i++) c->t1[i] = c->soln[i];
}

// Set-up of the membrane (Solver_gpu.cu:659-735): contour lengths and reference
// curvatures on the stress-free coordinates, then the initial coordinates and
// the initial pass that fixes V0, A0, MAD0, spring_area_0 and spring_angle_0.
extern "C" void ref_case_set_rbc(void *h, int n_nodes, int n_tets, int n_springs, const int *tri, const int *spr,
                                 const double *xyz_stress_free, const double *xyz_initial) {
    RefCase *c = (RefCase *)h;
    c->n_nodes = n_nodes; c->n_tets = n_tets; c->n_springs = n_springs;
    c->tri.assign(tri, tri + 3 * n_tets);
    c->spr.assign(spr, spr + 4 * n_springs);
    auto fill = [](std::vector<double> &v, int n) { v.assign(n, 0.0); };
    fill(c->x, n_nodes); fill(c->y, n_nodes); fill(c->z, n_nodes);
    fill(c->vx, n_nodes); fill(c->vy, n_nodes); fill(c->vz, n_nodes);
    fill(c->nfx_, n_nodes); fill(c->nfy_, n_nodes); fill(c->nfz_, n_nodes);
    fill(c->tet_area, n_tets); fill(c->tet_vol, n_tets); fill(c->tnx, n_tets); fill(c->tny, n_tets); fill(c->tnz, n_tets);
    fill(c->dummy, n_nodes);
    fill(c->contour, n_springs); fill(c->kspring, n_springs); fill(c->curv, n_springs); fill(c->curv0, n_springs);
    fill(c->sangle, n_springs); fill(c->sangle0, n_springs); fill(c->sarea, 2 * n_springs); fill(c->sarea0, 2 * n_springs);
    for (int i = 0; i < n_nodes; i++) {
        c->x[i] = xyz_stress_free[3 * i]; c->y[i] = xyz_stress_free[3 * i + 1]; c->z[i] = xyz_stress_free[3 * i + 2];
    }
    get_contour_lengths(n_springs, c->x.data(), c->y.data(), c->z.data(), c->spr.data(), c->contour.data(),
                        c->kspring.data(), c->p.wlc_ratio, c->p.shear_modulus, c->p.pivkin_length != 0, c->p.reference_length);
    get_reference_curvatures(n_springs, c->x.data(), c->y.data(), c->z.data(), c->spr.data(), c->sarea.data(),
                             c->sarea0.data(), c->curv.data(), c->curv0.data(), c->sangle.data(), c->sangle0.data(),
                             c->p.sphere_reference != 0, c->p.curvature_ratio);
    for (int i = 0; i < n_nodes; i++) {
        c->x[i] = xyz_initial[3 * i]; c->y[i] = xyz_initial[3 * i + 1]; c->z[i] = xyz_initial[3 * i + 2];
    }
    // MAD and MAD0 are read by the initial force pass before they are set; the
    // forces of that pass are discarded (node forces are refilled every step).
    c->MAD = 0.0; c->MAD0 = 0.0;
    spring_network_pass(*c, true);
}

extern "C" void ref_case_step(void *h, int n_steps) {
    RefCase *c = (RefCase *)h;
    ref_params &p = c->p;
    unstructured_mesh &M = *c->m->mesh;
    domain_geometry &D = c->m->domain;
    double3 origin = make_double3(D.origin_x, D.origin_y, D.origin_z);
    double3 lengths = make_double3(D.X, D.Y, D.Z);
    double delta_x = D.dt * 2;
    int nc = c->nc;
    for (int s = 0; s < n_steps; s++, c->t++) {
        int t = c->t;
        clone_a_to_b(nc, c->t1.data(), c->t0.data());
        // local time stepping calculation (Solver_gpu.cu:767-787)
        const int mode = p.time_stepping == 0 ? 2 : p.time_stepping;
        double delta_t = p.delta_t;
        if (mode != 2) {
            const double gamma = p.pre_conditioned_gamma > 0 ? p.pre_conditioned_gamma : 1 / p.gamma_inv;
            get_cfl_device(nc, c->soln.data(), c->vol.data(), c->dtl.data(), c->cfl_areas.data(), p.delta_t,
                           p.max_velocity, gamma, p.visc, mode);
            delta_t = block_min_max(c->dtl.data(), nc, (nc + 127) / 128, true);
        }
        if (mode == 3) fill_double(nc, c->dtl.data(), delta_t);
        else if (mode == 2) fill_double(nc, c->dtl.data(), p.delta_t);
        c->delta_t = delta_t;
        const bool plateau_ibm = c->m->globals.mesh_type == 4;  // Solver_gpu.cu:810-820, 899-912
        if (p.has_rbc) {
            if (plateau_ibm)
                interpolate_velocities_on_nodes_non_uniform_grid(
                    c->n_nodes, c->vx.data(), c->vy.data(), c->vz.data(), c->x.data(), c->y.data(), c->z.data(), origin,
                    lengths, delta_x, c->soln.data(), nc, acos(-1.0), c->ccen.data(), c->vol.data(),
                    c->plateau[0].data(), c->plateau[1].data(), c->plateau[2].data());
            else
            interpolate_velocities_on_nodes(c->n_nodes, c->vx.data(), c->vy.data(), c->vz.data(), c->x.data(), c->y.data(),
                                            c->z.data(), origin, lengths, delta_x, c->soln.data(), nc);
            update_node_positions(c->n_nodes, c->vx.data(), c->vy.data(), c->vz.data(), c->x.data(), c->y.data(), c->z.data(),
                                  delta_t, c->n_nodes, 1);
        }
        fill_double(nc, c->fx.data(), p.force[0]);
        fill_double(nc, c->fy.data(), p.force[1]);
        fill_double(nc, c->fz.data(), p.force[2]);
        if (p.has_rbc) {
            fill_double(c->n_nodes, c->nfx_.data(), 0.0);
            fill_double(c->n_nodes, c->nfy_.data(), 0.0);
            fill_double(c->n_nodes, c->nfz_.data(), 0.0);
            spring_network_pass(*c, false);
            if (p.viscosity_period > 0 && t % p.viscosity_period == 1) {
                // gpu_solver::update_viscosities, Solver_gpu.cu:2153-2208
                int nb_n = (c->n_nodes + 127) / 128;
                double mnx = block_min_max(c->x.data(), c->n_nodes, nb_n, true);
                double mny = block_min_max(c->y.data(), c->n_nodes, nb_n, true);
                double mnz = block_min_max(c->z.data(), c->n_nodes, nb_n, true);
                double mxx = block_min_max(c->x.data(), c->n_nodes, nb_n, false);
                double mxy = block_min_max(c->y.data(), c->n_nodes, nb_n, false);
                double mxz = block_min_max(c->z.data(), c->n_nodes, nb_n, false);
                fill_double(nc, c->visc_factor.data(), 1.0);
                update_interior_viscosities_plucker(nc, c->ccen.data(), c->x.data(), c->y.data(), c->z.data(), mnx, mxx, mny,
                                                    mxy, mnz, mxz, c->n_nodes, c->visc_factor.data(), M.get_delta_h(),
                                                    acos(-1.0), p.internal_viscosity_ratio, c->n_tets, c->tri.data());
            }
            if (plateau_ibm)
                spread_forces_on_non_uniform_grid(c->n_nodes, c->nfx_.data(), c->nfy_.data(), c->nfz_.data(),
                                                  c->x.data(), c->y.data(), c->z.data(), origin, lengths, delta_x,
                                                  c->fx.data(), c->fy.data(), c->fz.data(), nc, acos(-1.0),
                                                  c->ccen.data(), c->vol.data(), c->plateau[0].data(),
                                                  c->plateau[1].data(), c->plateau[2].data());
            else
            spread_forces_on_structured_grid(c->n_nodes, c->nfx_.data(), c->nfy_.data(), c->nfz_.data(), c->x.data(),
                                             c->y.data(), c->z.data(), origin, lengths, delta_x, c->fx.data(),
                                             c->fy.data(), c->fz.data(), nc);
        }
        // one RK stage (RungeKutta.timesteps = 1)
        update_unstructured_bcs(c->nb, c->nn, nc, c->owner.data(), c->rho_type.data(), c->vel_type.data(), c->soln.data(),
                                c->bcs_arr.data(), c->ccen.data(), p.channel_diameter);
        fill_zero(nc, c->res_rho.data()); fill_zero(nc, c->res_u.data()); fill_zero(nc, c->res_v.data());
        fill_zero(nc, c->res_w.data());
        for (auto &r : c->res_face) r = make_double4(0, 0, 0, 0);
        get_interior_gradients(nc, c->stencil.data(), c->soln.data(), c->rhs.data(), c->L[0].data(), c->L[1].data(),
                               c->L[2].data(), c->L[3].data(), c->L[4].data(), c->L[5].data(), c->L[6].data(),
                               c->L[7].data(), c->L[8].data(), c->g_rho.data(), c->g_u.data(), c->g_v.data(), c->g_w.data());
        get_bc_gradients(c->nb, c->nn, nc, c->owner.data(), c->rho_type.data(), c->vel_type.data(), c->soln.data(),
                         c->fnorm.data(), c->ccen.data(), c->bcs_arr.data(), c->g_rho.data(), c->g_u.data(), c->g_v.data(),
                         c->g_w.data());
        if (c->m->globals.mesh_type == 3) {  // imported meshes: general-normal interior faces (Solver_gpu.cu:970-976)
            calc_face_flux(c->nn, c->soln.data(), c->vol.data(), c->area.data(), c->owner.data(), c->neighbour.data(),
                           c->ccen.data(), c->fcen.data(), c->fnorm.data(), c->sdt.data(), c->g_rho.data(),
                           c->g_u.data(), c->g_v.data(), c->g_w.data(), nc, p.gamma_inv, c->local_fneq.data(), p.visc,
                           c->res_rho.data(), c->res_u.data(), c->res_v.data(), c->res_w.data(), c->res_face.data(),
                           c->rho_type.data(), c->vel_type.data(), c->bcs_arr.data(), acos(-1.0), p.testcase,
                           c->visc_factor.data(), p.preconditioning != 0);
        } else {
        calc_face_flux_x(c->nfx, c->soln.data(), c->vol.data(), c->area.data(), c->owner.data(), c->neighbour.data(),
                         c->ccen.data(), c->fcen.data(), c->fnorm.data(), c->sdt.data(), c->g_rho.data(), c->g_u.data(),
                         c->g_v.data(), c->g_w.data(), nc, p.gamma_inv, c->local_fneq.data(), p.visc, c->res_rho.data(),
                         c->res_u.data(), c->res_v.data(), c->res_w.data(), c->res_face.data(), c->rho_type.data(),
                         c->vel_type.data(), c->bcs_arr.data(), acos(-1.0), c->visc_factor.data(), p.testcase);
        calc_face_flux_y(c->nfy, c->soln.data(), c->vol.data(), c->area.data(), c->owner.data(), c->neighbour.data(),
                         c->ccen.data(), c->fcen.data(), c->fnorm.data(), c->sdt.data(), c->g_rho.data(), c->g_u.data(),
                         c->g_v.data(), c->g_w.data(), nc, p.gamma_inv, c->local_fneq.data(), p.visc, c->res_rho.data(),
                         c->res_u.data(), c->res_v.data(), c->res_w.data(), c->res_face.data(), c->rho_type.data(),
                         c->vel_type.data(), c->bcs_arr.data(), acos(-1.0), c->nfx, c->visc_factor.data(), p.testcase);
        calc_face_flux_z(c->nfz, c->soln.data(), c->vol.data(), c->area.data(), c->owner.data(), c->neighbour.data(),
                         c->ccen.data(), c->fcen.data(), c->fnorm.data(), c->sdt.data(), c->g_rho.data(), c->g_u.data(),
                         c->g_v.data(), c->g_w.data(), nc, p.gamma_inv, c->local_fneq.data(), p.visc, c->res_rho.data(),
                         c->res_u.data(), c->res_v.data(), c->res_w.data(), c->res_face.data(), c->rho_type.data(),
                         c->vel_type.data(), c->bcs_arr.data(), acos(-1.0), c->nfx + c->nfy, c->visc_factor.data(),
                         p.testcase);
        }
        calc_face_flux_bc(c->nb, c->soln.data(), c->vol.data(), c->area.data(), c->owner.data(), c->neighbour.data(),
                          c->ccen.data(), c->fcen.data(), c->fnorm.data(), c->sdt.data(), c->g_rho.data(), c->g_u.data(),
                          c->g_v.data(), c->g_w.data(), nc, p.gamma_inv, c->local_fneq.data(), p.visc, c->res_rho.data(),
                          c->res_u.data(), c->res_v.data(), c->res_w.data(), c->res_face.data(), c->rho_type.data(),
                          c->vel_type.data(), c->bcs_arr.data(), acos(-1.0), c->nn, p.testcase, p.preconditioning != 0);
        add_face_flux_to_cell(c->nf, c->res_face.data(), c->vol.data(), c->owner.data(), c->neighbour.data(),
                              c->res_rho.data(), c->res_u.data(), c->res_v.data(), c->res_w.data());
        add(nc, c->res_u.data(), c->fx.data());
        add(nc, c->res_v.data(), c->fy.data());
        add(nc, c->res_w.data(), c->fz.data());
        time_integration(nc, 0, 1, c->dtl.data(), c->t0.data(), c->t1.data(), c->soln.data(), c->res_rho.data(),
                         c->res_u.data(), c->res_v.data(), c->res_w.data(), delta_t, mode);
        // gpu_solver::check_periodic_object (Solver_gpu.cu:1027-1029, 1277-1304): total<128> over
        // n_node_Blocks = ceil(n / 128) blocks, host sum, add_double
        if (p.has_rbc && t % 5000 == 1 && p.object_periodic) {
            const double sum_add = block_tree_total(c->z.data(), c->n_nodes, (c->n_nodes + 127) / 128);
            const double object_centre_z = sum_add / c->n_nodes;
            if (object_centre_z > (D.origin_z + 0.75 * D.Z)) add_double(c->n_nodes, c->z.data(), (-0.5 * D.Z));
        }
        // residual RMS (Solver_gpu.cu:1033-1046, residuals.cpp:114-133)
        int nblk = (nc + 127) / 128;
        std::vector<double> sq(nc);
        double *rs[4] = {c->res_rho.data(), c->res_u.data(), c->res_v.data(), c->res_w.data()};
        double ref_mom = p.ref_rho * p.max_velocity;
        for (int k = 0; k < 4; k++) {
            for (int i = 0; i < nc; i++) sq[i] = rs[k][i] * rs[k][i];
            double s2 = block_tree_total(sq.data(), nc, nblk);
            c->residual_rms[k] = sqrt(s2 / nc) / (k == 0 ? p.ref_rho : ref_mom);
        }
    }
}

// Output selectors for ref_case_get.
enum {
    REF_RHO = 0, REF_U, REF_V, REF_W,             // n_cells (primitive state soln)
    REF_T1 = 4,                                   // 4*n_cells (u,v,w,rho of soln_t1)
    REF_GRAD = 5,                                 // 12*(n_cells+n_bc): rho,u,v,w gradients (x,y,z)
    REF_RES_FACE = 6,                             // 4*n_faces: (u,v,w,rho) fluxes
    REF_RES = 7,                                  // 4*n_cells: res_rho,res_u,res_v,res_w (after force add)
    REF_FORCE = 8,                                // 3*n_cells: cell force densities
    REF_NODE_X = 9,                               // 3*n_nodes
    REF_NODE_V = 10,                              // 3*n_nodes
    REF_NODE_F = 11,                              // 3*n_nodes
    REF_TOTALS = 12,                              // V, V0, A, A0, MAD, MAD0
    REF_VISC = 13,                                // n_cells visc_factor
    REF_SPRING = 14,                              // per spring: contour, k, curvature, curvature0, angle0, area0[2], area[2]
    REF_RESID = 15,                               // 4 residual rms
    REF_GHOST = 16,                               // 4*n_bc ghost (u,v,w,rho)
    REF_DT_LOCAL = 17,                            // n_cells delta_t_local
    REF_DELTA_T = 18,                             // 1: the last step's delta_t
    REF_ENERGY = 19,                              // 7: volume, global area, local area, local bending, ADE, spring, total
};

extern "C" void ref_case_get(void *h, int which, double *out) {
    RefCase *c = (RefCase *)h;
    int nc = c->nc, nt = c->nt;
    switch (which) {
    case REF_RHO: for (int i = 0; i < nc; i++) out[i] = c->soln[i].w; break;
    case REF_U: for (int i = 0; i < nc; i++) out[i] = c->soln[i].x; break;
    case REF_V: for (int i = 0; i < nc; i++) out[i] = c->soln[i].y; break;
    case REF_W: for (int i = 0; i < nc; i++) out[i] = c->soln[i].z; break;
    case REF_T1:
        for (int i = 0; i < nc; i++) {
            out[4 * i] = c->t1[i].x; out[4 * i + 1] = c->t1[i].y; out[4 * i + 2] = c->t1[i].z; out[4 * i + 3] = c->t1[i].w;
        }
        break;
    case REF_GRAD: {
        const std::vector<double3> *g[4] = {&c->g_rho, &c->g_u, &c->g_v, &c->g_w};
        for (int i = 0; i < nt; i++)
            for (int k = 0; k < 4; k++) {
                out[12 * i + 3 * k] = (*g[k])[i].x; out[12 * i + 3 * k + 1] = (*g[k])[i].y; out[12 * i + 3 * k + 2] = (*g[k])[i].z;
            }
        break;
    }
    case REF_RES_FACE:
        for (int f = 0; f < c->nf; f++) {
            out[4 * f] = c->res_face[f].x; out[4 * f + 1] = c->res_face[f].y; out[4 * f + 2] = c->res_face[f].z;
            out[4 * f + 3] = c->res_face[f].w;
        }
        break;
    case REF_RES:
        for (int i = 0; i < nc; i++) {
            out[4 * i] = c->res_rho[i]; out[4 * i + 1] = c->res_u[i]; out[4 * i + 2] = c->res_v[i]; out[4 * i + 3] = c->res_w[i];
        }
        break;
    case REF_FORCE:
        for (int i = 0; i < nc; i++) { out[3 * i] = c->fx[i]; out[3 * i + 1] = c->fy[i]; out[3 * i + 2] = c->fz[i]; }
        break;
    case REF_NODE_X:
        for (int i = 0; i < c->n_nodes; i++) { out[3 * i] = c->x[i]; out[3 * i + 1] = c->y[i]; out[3 * i + 2] = c->z[i]; }
        break;
    case REF_NODE_V:
        for (int i = 0; i < c->n_nodes; i++) { out[3 * i] = c->vx[i]; out[3 * i + 1] = c->vy[i]; out[3 * i + 2] = c->vz[i]; }
        break;
    case REF_NODE_F:
        for (int i = 0; i < c->n_nodes; i++) {
            out[3 * i] = c->nfx_[i]; out[3 * i + 1] = c->nfy_[i]; out[3 * i + 2] = c->nfz_[i];
        }
        break;
    case REF_TOTALS:
        out[0] = c->V; out[1] = c->V0; out[2] = c->A; out[3] = c->A0; out[4] = c->MAD; out[5] = c->MAD0;
        break;
    case REF_VISC: for (int i = 0; i < nc; i++) out[i] = c->visc_factor[i]; break;
    case REF_SPRING:
        for (int s = 0; s < c->n_springs; s++) {
            double *o = out + 9 * s;
            o[0] = c->contour[s]; o[1] = c->kspring[s]; o[2] = c->curv[s]; o[3] = c->curv0[s]; o[4] = c->sangle0[s];
            o[5] = c->sarea0[2 * s]; o[6] = c->sarea0[2 * s + 1]; o[7] = c->sarea[2 * s]; o[8] = c->sarea[2 * s + 1];
        }
        break;
    case REF_RESID: for (int k = 0; k < 4; k++) out[k] = c->residual_rms[k]; break;
    case REF_GHOST:
        for (int i = 0; i < c->nb; i++) {
            double4 g = c->soln[nc + i];
            out[4 * i] = g.x; out[4 * i + 1] = g.y; out[4 * i + 2] = g.z; out[4 * i + 3] = g.w;
        }
        break;
    case REF_DT_LOCAL:
        for (int i = 0; i < nc; i++) out[i] = c->dtl[i];
        break;
    case REF_DELTA_T:
        out[0] = c->delta_t;
        break;
    case REF_ENERGY: {
        // the energy log of Solver_gpu.cu:1060-1136: host formulas for the
        // global terms, the reference's kernels summed as total<128> block
        // partials, of which the host adds the first n_tet_Blocks
        const ref_params &p = c->p;
        const int S = c->n_springs, nblk = (c->n_tets + 127) / 128;
        std::vector<double> ea(S), eb(S), es(S);
        get_area_energy(S, c->sarea.data(), c->sarea0.data(), ea.data(), p.global_area_modulus);
        get_bending_energy(S, c->curv.data(), c->curv0.data(), eb.data(), c->sarea.data(), p.local_bending_modulus);
        get_spring_energy(S, c->spr.data(), c->spr.data(), c->x.data(), c->y.data(), c->z.data(), 0,
                          c->contour.data(), 1 / p.wlc_ratio, es.data(), c->kspring.data());
        const double ade = 0.5 * p.global_bending_modulus * (c->MAD - c->MAD0) * (c->MAD - c->MAD0) / c->A0;
        const double vol = 0.5 * p.volume_modulus * (c->V - c->V0) * (c->V - c->V0) / c->V0;
        const double gar = 0.5 * p.global_area_modulus * (c->A - c->A0) * (c->A - c->A0) / c->A0;
        const double la = block_tree_total(ea.data(), S, nblk), lb = block_tree_total(eb.data(), S, nblk),
                     sp = block_tree_total(es.data(), S, nblk);
        out[0] = vol; out[1] = gar; out[2] = la; out[3] = lb; out[4] = ade; out[5] = sp;
        out[6] = vol + gar + la + lb + ade + sp;
        break;
    }
    }
}

extern "C" void ref_case_free(void *h) { delete (RefCase *)h; }
