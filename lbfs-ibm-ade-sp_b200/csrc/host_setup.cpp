// Host-side set-up of the inputs the time step consumes: the uniform
// OpenFOAM-layout hex mesh with its least-squares gradient geometry, and the
// spring connectivity of a triangulated membrane.  These reproduce the
// reference's orderings exactly (face order, gradient stencil order, sprIdx
// order), because the step's results depend on them.
//
// Compiled with -ffp-contract=off so every multiply and add rounds on its own,
// as the reference's host code does; the geometry is then bit-identical.
#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <limits>
#include <unordered_set>
#include <vector>

#include "lbfs_b200.h"
#include "lbfs_internal.h"
#include "lbfs_mesh_common.h"

using lbfs::UniformDims;
using lbfs::axis_vertices;
using lbfs::jitter_unit;
using lbfs::uniform_dims;

namespace {

struct V3 {
    double x, y, z;
};
inline V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 add(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline double mag(V3 a) { return std::sqrt(std::pow(a.x, 2) + std::pow(a.y, 2) + std::pow(a.z, 2)); }

}  // namespace

// unstructured_mesh::create_uniform_openfoam_mesh, unstructured_mesh.cpp:252-401
lbfs::UniformDims lbfs::uniform_dims(double X, double Y, double Z, double dt) {
    UniformDims d;
    d.nx = (int)std::ceil(X / dt * 0.5);
    d.ny = (int)std::ceil(Y / dt * 0.5);
    d.nz = (int)std::ceil(Z / dt * 0.5);
    d.dx = X / d.nx;
    d.dy = Y / d.ny;
    d.dz = Z / d.nz;
    d.n_cells = d.nx * d.ny * d.nz;
    d.n_faces = (d.nx + 1) * d.ny * d.nz + d.nx * (d.ny + 1) * d.nz + d.nx * d.ny * (d.nz + 1);
    d.n_interior = d.n_faces - 2 * d.ny * d.nx - 2 * d.nx * d.nz - 2 * d.ny * d.nz;
    d.n_bc = d.n_faces - d.n_interior;
    d.n_fx = (d.nx - 1) * d.ny * d.nz;
    d.n_fy = d.nx * (d.ny - 1) * d.nz;
    d.n_fz = d.nx * d.ny * (d.nz - 1);
    return d;
}

extern "C" int lbfs_mesh_uniform_counts(double X, double Y, double Z, double dt, int32_t *out) {
    if (!out || !(dt > 0) || !(X > 0) || !(Y > 0) || !(Z > 0)) return lbfs::set_error(LBFS_ERR_ARG, "bad domain");
    UniformDims d = uniform_dims(X, Y, Z, dt);
    if (d.nx < 2 || d.ny < 2 || d.nz < 2) return lbfs::set_error(LBFS_ERR_ARG, "mesh needs >= 2 cells per axis");
    out[0] = d.n_cells; out[1] = d.n_faces; out[2] = d.n_interior; out[3] = d.n_bc;
    out[4] = d.n_fx; out[5] = d.n_fy; out[6] = d.n_fz; out[7] = d.n_cells + d.n_bc;
    return LBFS_OK;
}

namespace {

// How the generator places the vertices: the reference's mesh types
// (unstructured_mesh.cpp:354-378) and the seeded jitter of interior vertices.
struct VertexSpec {
    int mesh_type = 6;           // 6 uniform, 7 cosine in x and y, 5 cosine in x, y, z, 4 plateau
    double plateau_width = 0.0;  // domain.plateau_width (mesh_type 4)
    double plateau_slope = 0.0;  // domain.plateau_slope (mesh_type 4)
    double jitter = 0.0;
    uint64_t seed = 0;
    bool closed_faces = true;    // jittered faces: vector areas (true) or the reference's triangle sums
};

int build_mesh(double X, double Y, double Z, double dt, const double *origin, double visc, double fneq_min,
               int32_t gradient_hybrid, const VertexSpec &vs, int32_t *owner, int32_t *neighbour,
               double *face_area, double *face_normal, double *face_centroid, double *streaming_dt,
               double *cell_volume, double *cell_centroid, int32_t *gradient_stencil, double *lhs_inverse,
               double *rhs, int32_t *bc_patch, double *delta_h, double *grid_xyz,
               std::vector<float> *verts_out = nullptr, std::vector<int> *faces_out = nullptr);

}  // namespace

extern "C" int lbfs_mesh_build_uniform(double X, double Y, double Z, double dt, const double *origin, double visc,
                                       double fneq_min, int32_t gradient_hybrid, int32_t *owner, int32_t *neighbour,
                                       double *face_area, double *face_normal, double *face_centroid,
                                       double *streaming_dt, double *cell_volume, double *cell_centroid,
                                       int32_t *gradient_stencil, double *lhs_inverse, double *rhs, int32_t *bc_patch,
                                       double *delta_h) {
    return build_mesh(X, Y, Z, dt, origin, visc, fneq_min, gradient_hybrid, VertexSpec(), owner, neighbour, face_area,
                      face_normal, face_centroid, streaming_dt, cell_volume, cell_centroid, gradient_stencil,
                      lhs_inverse, rhs, bc_patch, delta_h, nullptr);
}

extern "C" int lbfs_mesh_build_rectilinear(double X, double Y, double Z, double dt, const double *origin, double visc,
                                           double fneq_min, int32_t gradient_hybrid, int32_t mesh_type,
                                           double plateau_width, double plateau_slope, int32_t *owner,
                                           int32_t *neighbour, double *face_area, double *face_normal,
                                           double *face_centroid, double *streaming_dt, double *cell_volume,
                                           double *cell_centroid, int32_t *gradient_stencil, double *lhs_inverse,
                                           double *rhs, int32_t *bc_patch, double *delta_h, double *grid_xyz) {
    if (mesh_type != 4 && mesh_type != 5 && mesh_type != 6 && mesh_type != 7)
        return lbfs::set_error(LBFS_ERR_ARG, "mesh_type must be 4 (plateau), 5, 6 (uniform) or 7 (cosine)");
    if (!grid_xyz) return lbfs::set_error(LBFS_ERR_ARG, "null output buffer");
    VertexSpec vs;
    vs.mesh_type = mesh_type;
    vs.plateau_width = plateau_width;
    vs.plateau_slope = plateau_slope;
    return build_mesh(X, Y, Z, dt, origin, visc, fneq_min, gradient_hybrid, vs, owner, neighbour, face_area,
                      face_normal, face_centroid, streaming_dt, cell_volume, cell_centroid, gradient_stencil,
                      lhs_inverse, rhs, bc_patch, delta_h, grid_xyz);
}

extern "C" int lbfs_mesh_build_jittered(double X, double Y, double Z, double dt, const double *origin, double visc,
                                        double fneq_min, int32_t gradient_hybrid, double jitter, uint64_t seed,
                                        int32_t closed_faces, int32_t *owner, int32_t *neighbour, double *face_area,
                                        double *face_normal, double *face_centroid, double *streaming_dt,
                                        double *cell_volume, double *cell_centroid, int32_t *gradient_stencil,
                                        double *lhs_inverse, double *rhs, int32_t *bc_patch, double *delta_h) {
    if (!(jitter >= 0.0 && jitter < 0.25))
        return lbfs::set_error(LBFS_ERR_ARG, "jitter must be in [0, 0.25) of the cell spacing");
    VertexSpec vs;
    vs.jitter = jitter;
    vs.seed = seed;
    vs.closed_faces = closed_faces != 0;
    return build_mesh(X, Y, Z, dt, origin, visc, fneq_min, gradient_hybrid, vs, owner, neighbour,
                      face_area, face_normal, face_centroid, streaming_dt, cell_volume, cell_centroid,
                      gradient_stencil, lhs_inverse, rhs, bc_patch, delta_h, nullptr);
}

// Vertex coordinates along one axis of n cells (unstructured_mesh.cpp:290-378):
// uniform, cosine-clustered, or the plateau function normalised to the length.
std::vector<double> lbfs::axis_vertices(int mesh_type, bool clustered, int n, double origin, double length,
                                        double step, double ap, double bp) {
    std::vector<double> v(n + 1);
    const double PI = std::acos(-1.0);  // globals.PI
    if (mesh_type == 4) {
        double sum = 0.0;
        for (int i = 1; i < n + 1; i++) {
            const double fx = i - n / 2.0 - 0.5;
            v[i] = (std::exp(bp * (fx - ap)) + 1) * (std::exp(bp * (-fx - ap)) + 1);
            sum = sum + v[i];
        }
        for (int i = 0; i < n + 1; i++) v[i] = i == 0 ? origin : v[i - 1] + v[i] * length / sum;
    } else if (clustered) {
        for (int i = 0; i < n + 1; i++) v[i] = origin + 0.5 * (1 - std::cos(i / (double)(n)*PI)) * length;
    } else {
        for (int i = 0; i < n + 1; i++) v[i] = origin + i * step;
    }
    return v;
}

namespace {

// Geometry and least-squares matrices of a hex mesh given as float vertices,
// quadrilateral faces (4 vertex ids each, winding giving the owner -> neighbour
// normal), owner and neighbour (boundary faces: any neighbour, replaced by
// the ghost cell n_cells + f - n_interior): unstructured_mesh::
// generate_internal_mesh (unstructured_mesh.cpp:1592-1692), tet_volume
// (:1015-1040), cell_tet_area (:1170-1204), calc_face_delta_t (:1349-1446),
// populate_ghost_cell_from_foam_face (:1963-1996) and gradients::
// pre_fill_LHS_and_RHS_matrix (gradients.cpp:214-315).  closed_faces: a
// face's area is the length of its vector area (see lbfs_mesh_build_jittered)
// instead of the reference's sum of its triangles' areas.
int mesh_geometry(int nc, int nf, int ni, const float *vx, const float *vy, const float *vz, const int *fv,
                  int32_t *owner, int32_t *neighbour, double visc, double fneq_min, int32_t gradient_hybrid,
                  bool closed_faces, double *face_area, double *face_normal, double *face_centroid,
                  double *streaming_dt, double *cell_volume, double *cell_centroid, int32_t *gradient_stencil,
                  double *lhs_inverse, double *rhs) {
    const int nt = nc + (nf - ni);
    // Geometry: unstructured_mesh::generate_internal_mesh (unstructured_mesh.cpp:1592-1692),
    // tet_volume (:1015-1040), cell_tet_area (:1170-1204), calc_face_delta_t (:1349-1446).
    std::vector<double> cvol(nt, 0.0), csum_area(nt, 0.0), cx(nt, 0.0), cy(nt, 0.0), cz(nt, 0.0);
    std::vector<std::vector<int>> gcells(nt), gfaces(nt);
    const double reference_dt = visc * 3 / 1.0 / fneq_min;  // pre_conditioned_gamma = 1
    for (int f = 0; f < nf; f++) {
        V3 nd[4];
        for (int q = 0; q < 4; q++) {
            int t = fv[4 * f + q];
            nd[q] = {(double)vx[t], (double)vy[t], (double)vz[t]};
        }
        for (int t = 0; t < 2; t++) {
            V3 a = nd[0], b = sub(nd[t + 1], a), c = sub(nd[t + 2], a);
            double vol = dot(a, cross(b, c)) / 6;
            cvol[owner[f]] = cvol[owner[f]] + vol;
            if (f < ni) cvol[neighbour[f]] = cvol[neighbour[f]] - vol;
        }
        double area_f = 0.0;
        V3 fcen = {0, 0, 0}, fnorm = {0, 0, 0};
        for (int t = 0; t < 2; t++) {
            V3 a = nd[0], b = nd[t + 1], c = nd[t + 2];
            V3 cen = {(a.x + b.x + c.x) / 3, (a.y + b.y + c.y) / 3, (a.z + b.z + c.z) / 3};
            V3 n = cross(sub(b, a), sub(c, a));
            double ar = 0.5 * mag(n);
            area_f = area_f + ar;
            double inv = 1 / ar;  // vector_var::factor divides by its argument
            cen = {cen.x / inv, cen.y / inv, cen.z / inv};
            fcen = add(fcen, cen);
            fnorm = add(fnorm, n);
        }
        // Warped faces: the face's vector area is the sum of its triangles'
        // vector areas, |N1 + N2| / 2 along (N1 + N2).  The reference's scalar
        // sum |N1| / 2 + |N2| / 2 (kept for the area-weighted centroids) is
        // longer whenever N1 and N2 are not parallel, so the vector areas of a
        // cell's faces would not close and a fluid at rest would be pushed by
        // its own pressure.
        face_area[f] = closed_faces ? 0.5 * mag(fnorm) : area_f;
        csum_area[owner[f]] = csum_area[owner[f]] + area_f;
        cx[owner[f]] = cx[owner[f]] + fcen.x;
        cy[owner[f]] = cy[owner[f]] + fcen.y;
        cz[owner[f]] = cz[owner[f]] + fcen.z;
        face_centroid[3 * f] = fcen.x / area_f;
        face_centroid[3 * f + 1] = fcen.y / area_f;
        face_centroid[3 * f + 2] = fcen.z / area_f;
        double nm = mag(fnorm);
        face_normal[3 * f] = fnorm.x / nm;
        face_normal[3 * f + 1] = fnorm.y / nm;
        face_normal[3 * f + 2] = fnorm.z / nm;
        double face_dt = 0.5 * std::sqrt(area_f);
        streaming_dt[f] = std::min(face_dt, reference_dt);
        if (f > ni - 1) {
            int g = f - ni + nc;
            gcells[owner[f]].push_back(g);
            gfaces[owner[f]].push_back(f);
        } else {
            int nb = neighbour[f];
            csum_area[nb] = csum_area[nb] + area_f;
            cx[nb] = cx[nb] + fcen.x;
            cy[nb] = cy[nb] + fcen.y;
            cz[nb] = cz[nb] + fcen.z;
            gcells[owner[f]].push_back(nb);
            gcells[nb].push_back(owner[f]);
            gfaces[owner[f]].push_back(f);
            gfaces[nb].push_back(f);
        }
    }
    for (int i = 0; i < nc; i++) {
        cx[i] = cx[i] / csum_area[i];
        cy[i] = cy[i] / csum_area[i];
        cz[i] = cz[i] / csum_area[i];
    }
    // ghost centroids: populate_ghost_cell_from_foam_face, unstructured_mesh.cpp:1963-1996
    for (int f = ni; f < nf; f++) {
        int g = nc + f - ni, o = owner[f];
        double ex = (face_centroid[3 * f] - cx[o]) / 0.5;
        double ey = (face_centroid[3 * f + 1] - cy[o]) / 0.5;
        double ez = (face_centroid[3 * f + 2] - cz[o]) / 0.5;
        cx[g] = cx[o] + ex;
        cy[g] = cy[o] + ey;
        cz[g] = cz[o] + ez;
        neighbour[f] = g;
    }
    for (int i = 0; i < nt; i++) {
        cell_volume[i] = cvol[i];
        cell_centroid[3 * i] = cx[i];
        cell_centroid[3 * i + 1] = cy[i];
        cell_centroid[3 * i + 2] = cz[i];
    }
    // Least-squares / hybrid gradient geometry: gradients::pre_fill_LHS_and_RHS_matrix
    // (gradients.cpp:214-315) and add_non_macrovariable_contributions (:149-211).
    for (int i = 0; i < nc; i++) {
        if (gcells[i].size() != 6) return lbfs::set_error(LBFS_ERR_ARG, "hex cell without 6 stencil entries");
        double L[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        double max_area = 0.0, max_disp = 0.0;
        for (int q = 0; q < 6; q++) {
            int i1 = gcells[i][q], f = gfaces[i][q];
            max_area = std::max(max_area, face_area[f]);
            double ddx = cx[i1] - cx[i], ddy = cy[i1] - cy[i], ddz = cz[i1] - cz[i];
            max_disp = std::max(std::sqrt(ddx * ddx + ddy * ddy + ddz * ddz), max_disp);
        }
        double aspect = 2 * std::fabs(max_disp) * max_area / cvol[i];
        double beta = gradient_hybrid ? std::min(1.0, (2 / aspect)) : 1.0;
        L[0] = L[0] + 2 * (1 - beta) * cvol[i];
        L[4] = L[4] + 2 * (1 - beta) * cvol[i];
        L[8] = L[8] + 2 * (1 - beta) * cvol[i];
        for (int q = 0; q < 6; q++) {
            int i1 = gcells[i][q], f = gfaces[i][q];
            double fi = face_normal[3 * f], fj = face_normal[3 * f + 1], fk = face_normal[3 * f + 2];
            double ddx = face_centroid[3 * f] - cx[i], ddy = face_centroid[3 * f + 1] - cy[i],
                   ddz = face_centroid[3 * f + 2] - cz[i];
            double l_norm = ddx * fi + ddy * fj + ddz * fk;
            ddx = cx[i1] - cx[i]; ddy = cy[i1] - cy[i]; ddz = cz[i1] - cz[i];
            double Ld = std::sqrt(std::pow(ddx, 2.0) + std::pow(ddy, 2.0) + std::pow(ddz, 2.0));
            double s = face_area[f];
            double L_norm = ddx * fi + ddy * fj + ddz * fk;
            double alpha_w = std::pow(2 * l_norm / L_norm, 2.0);
            double w = alpha_w * s / Ld;
            L[0] = L[0] + w * ddx * ddx * beta; L[1] = L[1] + w * ddx * ddy * beta; L[2] = L[2] + w * ddx * ddz * beta;
            L[3] = L[3] + w * ddy * ddx * beta; L[4] = L[4] + w * ddy * ddy * beta; L[5] = L[5] + w * ddy * ddz * beta;
            L[6] = L[6] + w * ddz * ddx * beta; L[7] = L[7] + w * ddz * ddy * beta; L[8] = L[8] + w * ddz * ddz * beta;
            double sgn = (owner[f] == i) ? 1.0 : -1.0;
            double *R = rhs + 18 * i + 3 * q;
            if (sgn > 0) {
                R[0] = (beta * w * ddx + 2 * (1 - beta) * 0.5 * fi * s);
                R[1] = (beta * w * ddy + 2 * (1 - beta) * 0.5 * fj * s);
                R[2] = (beta * w * ddz + 2 * (1 - beta) * 0.5 * fk * s);
            } else {
                R[0] = (beta * w * ddx + 2 * (1 - beta) * 0.5 * fi * -1 * s);
                R[1] = (beta * w * ddy + 2 * (1 - beta) * 0.5 * fj * -1 * s);
                R[2] = (beta * w * ddz + 2 * (1 - beta) * 0.5 * fk * -1 * s);
            }
            gradient_stencil[6 * i + q] = i1;
        }
        // Determinant exactly as the reference forms it (gradients.cpp:282-284;
        // its second cofactor is not the true one, which only matters on
        // non-orthogonal meshes), then the adjugate / det.
        double det = L[0] * (L[4] * L[8] - L[5] * L[7]) + L[1] * (L[3] * L[8] - L[5] - L[6]) +
                     L[2] * (L[3] * L[7] - L[4] * L[6]);
        double a = L[0], b = L[1], c = L[2], dd = L[3], e = L[4], f = L[5], g = L[6], h = L[7], k = L[8];
        double *I = lhs_inverse + 9 * i;
        I[0] = 1 / det * (e * k - f * h);
        I[1] = 1 / det * (c * h - b * k);
        I[2] = 1 / det * (b * f - c * e);
        I[3] = 1 / det * (f * g - dd * k);
        I[4] = 1 / det * (a * k - c * g);
        I[5] = 1 / det * (c * dd - a * f);
        I[6] = 1 / det * (dd * h - e * g);
        I[7] = 1 / det * (b * g - a * h);
        I[8] = 1 / det * (a * e - b * dd);
    }
    return LBFS_OK;
}

int build_mesh(double X, double Y, double Z, double dt, const double *origin, double visc, double fneq_min,
               int32_t gradient_hybrid, const VertexSpec &vs, int32_t *owner, int32_t *neighbour,
               double *face_area, double *face_normal, double *face_centroid, double *streaming_dt,
               double *cell_volume, double *cell_centroid, int32_t *gradient_stencil, double *lhs_inverse,
               double *rhs, int32_t *bc_patch, double *delta_h, double *grid_xyz, std::vector<float> *verts_out,
               std::vector<int> *faces_out) {
    const double jitter = vs.jitter;
    const uint64_t seed = vs.seed;
    int32_t cnt[8];
    int rc = lbfs_mesh_uniform_counts(X, Y, Z, dt, cnt);
    if (rc) return rc;
    if (!origin || !owner || !neighbour || !face_area || !face_normal || !face_centroid || !streaming_dt ||
        !cell_volume || !cell_centroid || !gradient_stencil || !lhs_inverse || !rhs || !bc_patch || !delta_h)
        return lbfs::set_error(LBFS_ERR_ARG, "null output buffer");
    UniformDims d = uniform_dims(X, Y, Z, dt);
    const int nvx = d.nx + 1, nvy = d.ny + 1, nvz = d.nz + 1;
    const int nc = d.n_cells, nf = d.n_faces, ni = d.n_interior, nt = nc + d.n_bc;

    // Vertices are stored as float in the reference (unstructured_mesh.h:59).
    const int mt = vs.mesh_type;
    const std::vector<double> ax = axis_vertices(mt, mt == 5 || mt == 7, d.nx, origin[0], X, d.dx, vs.plateau_width,
                                                 vs.plateau_slope),
                              ay = axis_vertices(mt, mt == 5 || mt == 7, d.ny, origin[1], Y, d.dy, vs.plateau_width,
                                                 vs.plateau_slope),
                              az = axis_vertices(mt, mt == 5, d.nz, origin[2], Z, d.dz, vs.plateau_width,
                                                 vs.plateau_slope);
    if (grid_xyz) {
        std::copy(ax.begin(), ax.end(), grid_xyz);
        std::copy(ay.begin(), ay.end(), grid_xyz + nvx);
        std::copy(az.begin(), az.end(), grid_xyz + nvx + nvy);
    }
    std::vector<float> vx((size_t)nvx * nvy * nvz), vy(vx.size()), vz(vx.size());
    {
        size_t t = 0;
        for (int k = 0; k < nvz; k++)
            for (int j = 0; j < nvy; j++)
                for (int i = 0; i < nvx; i++, t++) {
                    double px = ax[i], py = ay[j], pz = az[k];
                    // interior vertices move by up to jitter * spacing per axis (the box stays a box)
                    if (jitter > 0 && i > 0 && j > 0 && k > 0 && i < nvx - 1 && j < nvy - 1 && k < nvz - 1) {
                        px += jitter * d.dx * jitter_unit(seed, t, 0);
                        py += jitter * d.dy * jitter_unit(seed, t, 1);
                        pz += jitter * d.dz * jitter_unit(seed, t, 2);
                    }
                    vx[t] = (float)px;
                    vy[t] = (float)py;
                    vz[t] = (float)pz;
                }
    }
    // Face loop order and vertex winding: unstructured_mesh.cpp:415-664.
    std::vector<int> fv((size_t)4 * nf);
    int face = 0;
    const int sxy = nvx * nvy;
    auto put = [&](int a, int b, int c, int dd, int own, int nb) {
        fv[4 * face] = a; fv[4 * face + 1] = b; fv[4 * face + 2] = c; fv[4 * face + 3] = dd;
        owner[face] = own;
        neighbour[face] = nb;
        face++;
    };
    for (int k = 0; k < nvz - 1; k++)
        for (int j = 0; j < nvy - 1; j++)
            for (int i = 1; i < nvx - 1; i++) {
                int a = k * sxy + j * nvx + i, b = a + nvx, c = b + sxy, dd = a + sxy;
                int own = (i - 1) + j * d.nx + k * d.nx * d.ny;
                put(a, b, c, dd, own, own + 1);
            }
    for (int k = 0; k < nvz - 1; k++)
        for (int j = 1; j < nvy - 1; j++)
            for (int i = 0; i < nvx - 1; i++) {
                int a = k * sxy + j * nvx + i, b = a + sxy, c = b + 1, dd = a + 1;
                int own = i + (j - 1) * d.nx + k * d.nx * d.ny;
                put(a, b, c, dd, own, own + d.nx);
            }
    for (int k = 1; k < nvz - 1; k++)
        for (int j = 0; j < nvy - 1; j++)
            for (int i = 0; i < nvx - 1; i++) {
                int a = k * sxy + j * nvx + i, b = a + 1, c = b + nvx, dd = c - 1;
                int own = i + j * d.nx + (k - 1) * d.nx * d.ny;
                put(a, b, c, dd, own, own + d.nx * d.ny);
            }
    int bci = 0;
    for (int k = 0; k < nvz - 1; k++)
        for (int j = 0; j < nvy - 1; j++) {  // left
            int i = 0, a = k * sxy + j * nvx + i;
            bc_patch[bci++] = 0;
            put(a, a + sxy, a + nvx + sxy, a + nvx, i + j * d.nx + k * d.nx * d.ny, 0);
        }
    for (int k = 0; k < nvz - 1; k++)
        for (int j = 0; j < nvy - 1; j++) {  // right
            int i = nvx - 1, a = k * sxy + j * nvx + i, b = a + nvx;
            bc_patch[bci++] = 1;
            put(a, b, b + sxy, a + sxy, (i - 1) + j * d.nx + k * d.nx * d.ny, 0);
        }
    for (int k = 0; k < nvz - 1; k++)
        for (int i = 0; i < nvx - 1; i++) {  // bottom
            int j = 0, a = k * sxy + j * nvx + i;
            bc_patch[bci++] = 2;
            put(a, a + 1, a + sxy + 1, a + sxy, i + j * d.nx + k * d.nx * d.ny, 0);
        }
    for (int k = 0; k < nvz - 1; k++)
        for (int i = 0; i < nvx - 1; i++) {  // top
            int j = nvy - 1, a = k * sxy + j * nvx + i, b = a + sxy;
            bc_patch[bci++] = 3;
            put(a, b, b + 1, a + 1, i + (j - 1) * d.nx + k * d.nx * d.ny, 0);
        }
    for (int j = 0; j < nvy - 1; j++)
        for (int i = 0; i < nvx - 1; i++) {  // back
            int k = 0, a = k * sxy + j * nvx + i, b = a + nvx;
            bc_patch[bci++] = 4;
            put(a, b, b + 1, a + 1, i + j * d.nx + k * d.nx * d.ny, 0);
        }
    for (int j = 0; j < nvy - 1; j++)
        for (int i = 0; i < nvx - 1; i++) {  // front
            int k = nvz - 1, a = k * sxy + j * nvx + i, b = a + 1, c = b + nvx;
            bc_patch[bci++] = 5;
            put(a, b, c, c - 1, i + j * d.nx + (k - 1) * d.nx * d.ny, 0);
        }

    double dh = std::min(d.dx, std::min(d.dy, d.dz)) * 0.5;
    *delta_h = std::min(dh, 0.1);
    if (verts_out) {
        verts_out->resize(3 * vx.size());
        for (size_t t = 0; t < vx.size(); t++) {
            (*verts_out)[3 * t] = vx[t];
            (*verts_out)[3 * t + 1] = vy[t];
            (*verts_out)[3 * t + 2] = vz[t];
        }
    }
    if (faces_out) *faces_out = fv;

    return mesh_geometry(nc, nf, ni, vx.data(), vy.data(), vz.data(), fv.data(), owner, neighbour, visc, fneq_min,
                         gradient_hybrid, jitter > 0 && vs.closed_faces, face_area, face_normal, face_centroid,
                         streaming_dt, cell_volume, cell_centroid, gradient_stencil, lhs_inverse, rhs);
}

}  // namespace

// ---- OpenFOAM polyMesh ------------------------------------------------------

namespace {

const char *const kPatchNames[6] = {"left", "right", "bottom", "top", "back", "front"};

void foam_header(std::FILE *f, const char *cls, const char *object, const std::string &note) {
    std::fprintf(f,
                 "/*--------------------------------*- C++ -*----------------------------------*\\\n"
                 "  =========                 |\n"
                 "  \\\\      /  F ield         | polyMesh written by lbfs_mesh_write_openfoam\n"
                 "   \\\\    /   O peration     |\n"
                 "    \\\\  /    A nd           |\n"
                 "     \\\\/     M anipulation  |\n"
                 "\\*---------------------------------------------------------------------------*/\n"
                 "FoamFile\n{\n    version     2.0;\n    format      ascii;\n    class       %s;\n", cls);
    if (!note.empty()) std::fprintf(f, "    note        \"%s\";\n", note.c_str());
    std::fprintf(f, "    location    \"constant/polyMesh\";\n    object      %s;\n}\n"
                    "// * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * //\n\n\n", object);
}

// Lines of a file; false if it cannot be opened.
bool read_lines(const std::string &path, std::vector<std::string> &lines) {
    std::ifstream in(path);
    if (!in) return false;
    std::string line;
    while (std::getline(in, line)) lines.push_back(line);
    return true;
}

// The entries of the list of a polyMesh file: the lines after the first line
// that starts with '(' up to the next line that starts with ')', as the
// reference's reader delimits them (unstructured_mesh.cpp:749-770).
std::vector<std::string> list_entries(const std::vector<std::string> &lines) {
    std::vector<std::string> out;
    bool start = false;
    for (const std::string &l : lines) {
        const char c = l.empty() ? 0 : l[0];
        if (c == ')') start = false;
        if (start && !l.empty()) out.push_back(l);
        if (c == '(') start = true;
    }
    return out;
}

// A polyMesh file read whole, with the [begin, end) offsets of its list's
// entries (delimited as list_entries does).  The large lists (points, faces,
// owner, neighbour) are parsed from it with strtof / strtol, which read a
// well-formed entry as the stream extractions of the reference's reader do.
struct FoamText {
    std::string text;
    std::vector<std::pair<size_t, size_t>> entries;
    std::string buf;  // the entry being parsed, NUL-terminated
    const char *entry(size_t k) {
        buf.assign(text, entries[k].first, entries[k].second - entries[k].first);
        return buf.c_str();
    }
    // Line `k` (0-based) of the file, without its newline; empty past the end.
    std::string line(int k) const {
        size_t b = 0;
        for (int i = 0; i < k && b < text.size(); i++) {
            const size_t e = text.find('\n', b);
            b = e == std::string::npos ? text.size() : e + 1;
        }
        const size_t e = std::min(text.find('\n', b), text.size());
        return b < text.size() ? text.substr(b, e - b) : std::string();
    }
};

bool read_foam_text(const std::string &path, FoamText &t) {
    std::FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) return false;
    char chunk[1 << 16];
    size_t n;
    while ((n = std::fread(chunk, 1, sizeof chunk, f)) > 0) t.text.append(chunk, n);
    std::fclose(f);
    bool start = false;
    for (size_t b = 0; b < t.text.size();) {
        size_t e = t.text.find('\n', b);
        if (e == std::string::npos) e = t.text.size();
        const char c = e > b ? t.text[b] : 0;
        if (c == ')') start = false;
        if (start && e > b) t.entries.push_back({b, e});
        if (c == '(') start = true;
        b = e + 1;
    }
    return true;
}

// One int from p (leading blanks skipped, as the stream extraction does);
// false when nothing was read or it does not fit an int.
bool parse_int(const char *&p, int &v) {
    char *end = nullptr;
    errno = 0;
    const long r = std::strtol(p, &end, 10);
    if (end == p || errno == ERANGE || r < std::numeric_limits<int>::min() || r > std::numeric_limits<int>::max())
        return false;
    v = (int)r;
    p = end;
    return true;
}

// One float from p, read as float (unstructured_mesh.h:59): false when
// nothing was read or the value overflows a float.
bool parse_float(const char *&p, float &v) {
    char *end = nullptr;
    errno = 0;
    const float r = std::strtof(p, &end);
    if (end == p || !std::isfinite(r)) return false;
    v = r;
    p = end;
    return true;
}

struct FoamMesh {
    int n_points = 0, n_cells = 0, n_faces = 0, n_internal = 0;
    std::vector<float> x, y, z;
    std::vector<int> fv, owner, neighbour;
    std::vector<std::string> patch_names;
    std::vector<int> patch_faces;
};

// The owner file's note on its 13th line (nPoints, nCells, nFaces,
// nInternalFaces), the lists of points, faces, owner and neighbour, and the
// patch names and face counts of the boundary file (import_openfoam_mesh,
// unstructured_mesh.cpp:670-941; import_openfoam_BC_tags, :2533-2608).
int read_foam(const std::string &dir0, FoamMesh &m, bool header_only) {
    const std::string dir = dir0.empty() || dir0.back() == '/' ? dir0 : dir0 + "/";
    FoamText own;
    if (!read_foam_text(dir + "owner", own)) return lbfs::set_error(LBFS_ERR_ARG, "cannot open " + dir + "owner");
    const std::string note = own.line(12);
    if (note.empty()) return lbfs::set_error(LBFS_ERR_ARG, "owner: no header note on line 13");
    auto field = [&](const char *key, int &v) {
        const size_t p = note.find(key);
        if (p == std::string::npos) return false;
        std::istringstream is(note.substr(p + std::strlen(key)));
        return (bool)(is >> v);
    };
    if (!field("nPoints:", m.n_points) || !field("nCells:", m.n_cells) || !field("nFaces:", m.n_faces) ||
        !field("nInternalFaces:", m.n_internal))
        return lbfs::set_error(LBFS_ERR_ARG, "owner: line 13 must carry nPoints:, nCells:, nFaces:, nInternalFaces:");
    if (m.n_points <= 0 || m.n_cells <= 0 || m.n_internal < 0 || m.n_faces <= m.n_internal)
        return lbfs::set_error(LBFS_ERR_ARG, "owner: inconsistent sizes in the header note");
    std::vector<std::string> bnd;
    if (!read_lines(dir + "boundary", bnd)) return lbfs::set_error(LBFS_ERR_ARG, "cannot open " + dir + "boundary");
    {
        std::string last_name;
        for (const std::string &l : list_entries(bnd)) {
            std::istringstream is(l);
            std::string t1, t2;
            is >> t1 >> t2;
            if (t1 == "{" || t1 == "}" || t1.empty()) continue;
            if (t2.empty()) { last_name = t1; continue; }
            if (t1 == "nFaces") {
                if (!t2.empty() && t2.back() == ';') t2.pop_back();
                m.patch_names.push_back(last_name);
                m.patch_faces.push_back(std::stoi(t2));
            }
        }
    }
    int nbf = 0;
    for (int n : m.patch_faces) nbf += n;
    if (nbf != m.n_faces - m.n_internal)
        return lbfs::set_error(LBFS_ERR_ARG, "boundary: patch face counts do not add up to the boundary faces");
    if (header_only) return LBFS_OK;
    FoamText P, F, N;
    if (!read_foam_text(dir + "points", P) || !read_foam_text(dir + "faces", F) ||
        !read_foam_text(dir + "neighbour", N))
        return lbfs::set_error(LBFS_ERR_ARG, "cannot open points, faces or neighbour in " + dir);
    FoamText &O = own;
    if ((int)P.entries.size() != m.n_points || (int)F.entries.size() != m.n_faces ||
        (int)O.entries.size() != m.n_faces || (int)N.entries.size() != m.n_internal)
        return lbfs::set_error(LBFS_ERR_ARG, "polyMesh lists do not match the owner file's header note");
    m.x.resize(m.n_points); m.y.resize(m.n_points); m.z.resize(m.n_points);
    for (int i = 0; i < m.n_points; i++) {
        const char *p = P.entry(i) + 1;  // past '('; the coordinates are read as float (unstructured_mesh.h:59)
        if (!parse_float(p, m.x[i]) || !parse_float(p, m.y[i]) || !parse_float(p, m.z[i]))
            return lbfs::set_error(LBFS_ERR_ARG, "points: bad entry");
    }
    m.fv.resize(4 * (size_t)m.n_faces);
    for (int f = 0; f < m.n_faces; f++) {
        const char *p = F.entry(f);
        int n = 0;
        if (!parse_int(p, n) || n != 4)
            return lbfs::set_error(LBFS_ERR_UNSUPPORTED, "faces: quadrilaterals only (hexahedral cells)");
        if (*p) p++;  // '('
        for (int q = 0; q < 4; q++) {
            if (!parse_int(p, m.fv[4 * f + q]) || m.fv[4 * f + q] < 0 || m.fv[4 * f + q] >= m.n_points)
                return lbfs::set_error(LBFS_ERR_ARG, "faces: bad vertex index");
        }
    }
    m.owner.resize(m.n_faces);
    m.neighbour.assign(m.n_faces, 0);
    for (int f = 0; f < m.n_faces; f++) {
        const char *p = O.entry(f);
        if (!parse_int(p, m.owner[f]) || m.owner[f] < 0 || m.owner[f] >= m.n_cells)
            return lbfs::set_error(LBFS_ERR_ARG, "owner: bad cell index");
    }
    for (int f = 0; f < m.n_internal; f++) {
        const char *p = N.entry(f);
        if (!parse_int(p, m.neighbour[f]) || m.neighbour[f] < 0 || m.neighbour[f] >= m.n_cells)
            return lbfs::set_error(LBFS_ERR_ARG, "neighbour: bad cell index");
    }
    return LBFS_OK;
}

}  // namespace

extern "C" int lbfs_mesh_write_openfoam(const char *dir, double X, double Y, double Z, double dt, const double *origin,
                                        int32_t mesh_type, double plateau_width, double plateau_slope, double jitter,
                                        uint64_t seed) {
    if (!dir || !origin) return lbfs::set_error(LBFS_ERR_ARG, "null argument");
    if (mesh_type != 4 && mesh_type != 5 && mesh_type != 6 && mesh_type != 7)
        return lbfs::set_error(LBFS_ERR_ARG, "mesh_type must be 4, 5, 6 or 7");
    if (!(jitter >= 0.0 && jitter < 0.25) || (jitter > 0 && mesh_type != 6))
        return lbfs::set_error(LBFS_ERR_ARG, "jitter must be in [0, 0.25), on the uniform mesh only");
    int32_t cnt[8];
    int rc = lbfs_mesh_uniform_counts(X, Y, Z, dt, cnt);
    if (rc) return rc;
    const int nc = cnt[0], nf = cnt[1], ni = cnt[2], nb = cnt[3], nt = cnt[7];
    VertexSpec vs;
    vs.mesh_type = mesh_type; vs.plateau_width = plateau_width; vs.plateau_slope = plateau_slope;
    vs.jitter = jitter; vs.seed = seed;
    std::vector<int32_t> owner(nf), neighbour(nf), stencil(6 * (size_t)nc), patch(nb);
    std::vector<double> area(nf), normal(3 * (size_t)nf), fcen(3 * (size_t)nf), sdt(nf), vol(nt),
        cen(3 * (size_t)nt), lhs(9 * (size_t)nc), rhs(18 * (size_t)nc);
    double dh = 0;
    std::vector<float> verts;
    std::vector<int> fv;
    if ((rc = build_mesh(X, Y, Z, dt, origin, 0.1, 0.0, 0, vs, owner.data(), neighbour.data(), area.data(),
                         normal.data(), fcen.data(), sdt.data(), vol.data(), cen.data(), stencil.data(), lhs.data(),
                         rhs.data(), patch.data(), &dh, nullptr, &verts, &fv)))
        return rc;
    const std::string d = std::string(dir) + (std::string(dir).back() == '/' ? "" : "/");
    const int np = (int)(verts.size() / 3);
    char note[256];
    std::snprintf(note, sizeof note, "nPoints:%d  nCells:%d  nFaces:%d  nInternalFaces:%d", np, nc, nf, ni);
    auto open = [&](const char *name) { return std::fopen((d + name).c_str(), "w"); };
    std::FILE *f = open("points");
    if (!f) return lbfs::set_error(LBFS_ERR_ARG, "cannot write " + d + "points");
    foam_header(f, "vectorField", "points", "");
    std::fprintf(f, "%d\n(\n", np);
    for (int t = 0; t < np; t++)  // %.9g reproduces a float exactly
        std::fprintf(f, "(%.9g %.9g %.9g)\n", verts[3 * t], verts[3 * t + 1], verts[3 * t + 2]);
    std::fprintf(f, ")\n");
    std::fclose(f);
    if (!(f = open("faces"))) return lbfs::set_error(LBFS_ERR_ARG, "cannot write " + d + "faces");
    foam_header(f, "faceList", "faces", "");
    std::fprintf(f, "%d\n(\n", nf);
    for (int q = 0; q < nf; q++) std::fprintf(f, "4(%d %d %d %d)\n", fv[4 * q], fv[4 * q + 1], fv[4 * q + 2], fv[4 * q + 3]);
    std::fprintf(f, ")\n");
    std::fclose(f);
    if (!(f = open("owner"))) return lbfs::set_error(LBFS_ERR_ARG, "cannot write " + d + "owner");
    foam_header(f, "labelList", "owner", note);
    std::fprintf(f, "%d\n(\n", nf);
    for (int q = 0; q < nf; q++) std::fprintf(f, "%d\n", owner[q]);
    std::fprintf(f, ")\n");
    std::fclose(f);
    if (!(f = open("neighbour"))) return lbfs::set_error(LBFS_ERR_ARG, "cannot write " + d + "neighbour");
    foam_header(f, "labelList", "neighbour", note);
    std::fprintf(f, "%d\n(\n", ni);
    for (int q = 0; q < ni; q++) std::fprintf(f, "%d\n", neighbour[q]);
    std::fprintf(f, ")\n");
    std::fclose(f);
    if (!(f = open("boundary"))) return lbfs::set_error(LBFS_ERR_ARG, "cannot write " + d + "boundary");
    foam_header(f, "polyBoundaryMesh", "boundary", "");
    std::fprintf(f, "6\n(\n");
    int start = ni;
    for (int p = 0; p < 6; p++) {
        int n = 0;
        for (int b = 0; b < nb; b++) n += patch[b] == p ? 1 : 0;
        std::fprintf(f, "    %s\n    {\n        type            patch;\n        nFaces          %d;\n"
                        "        startFace       %d;\n    }\n", kPatchNames[p], n, start);
        start += n;
    }
    std::fprintf(f, ")\n");
    std::fclose(f);
    return LBFS_OK;
}

extern "C" int lbfs_mesh_openfoam_counts(const char *dir, int32_t *counts) {
    if (!dir || !counts) return lbfs::set_error(LBFS_ERR_ARG, "null argument");
    FoamMesh m;
    int rc = read_foam(dir, m, true);
    if (rc) return rc;
    counts[0] = m.n_points; counts[1] = m.n_cells; counts[2] = m.n_faces; counts[3] = m.n_internal;
    counts[4] = m.n_faces - m.n_internal; counts[5] = (int32_t)m.patch_names.size();
    return LBFS_OK;
}

extern "C" int lbfs_mesh_import_openfoam(const char *dir, double visc, double fneq_min, int32_t gradient_hybrid,
                                         int32_t closed_faces, int32_t *owner, int32_t *neighbour, double *face_area,
                                         double *face_normal, double *face_centroid, double *streaming_dt,
                                         double *cell_volume, double *cell_centroid, int32_t *gradient_stencil,
                                         double *lhs_inverse, double *rhs, int32_t *bc_patch, char *names,
                                         int32_t names_len) {
    if (!dir || !owner || !neighbour || !face_area || !face_normal || !face_centroid || !streaming_dt ||
        !cell_volume || !cell_centroid || !gradient_stencil || !lhs_inverse || !rhs || !bc_patch)
        return lbfs::set_error(LBFS_ERR_ARG, "null argument");
    FoamMesh m;
    int rc = read_foam(dir, m, false);
    if (rc) return rc;
    std::copy(m.owner.begin(), m.owner.end(), owner);
    std::copy(m.neighbour.begin(), m.neighbour.end(), neighbour);
    int b = 0;
    for (size_t p = 0; p < m.patch_faces.size(); p++)
        for (int q = 0; q < m.patch_faces[p]; q++) bc_patch[b++] = (int32_t)p;
    if (names && names_len > 0) {
        std::string all;
        for (const std::string &n : m.patch_names) all += n + "\n";
        std::snprintf(names, (size_t)names_len, "%s", all.c_str());
    }
    return mesh_geometry(m.n_cells, m.n_faces, m.n_internal, m.x.data(), m.y.data(), m.z.data(), m.fv.data(), owner,
                         neighbour, visc, fneq_min, gradient_hybrid, closed_faces != 0, face_area, face_normal,
                         face_centroid, streaming_dt, cell_volume, cell_centroid, gradient_stencil, lhs_inverse, rhs);
}

extern "C" int lbfs_mesh_import_openfoam_gpu(const char *dir, double visc, double fneq_min, int32_t gradient_hybrid,
                                             int32_t closed_faces, int32_t device, int32_t *owner, int32_t *neighbour,
                                             double *face_area, double *face_normal, double *face_centroid,
                                             double *streaming_dt, double *cell_volume, double *cell_centroid,
                                             int32_t *gradient_stencil, double *lhs_inverse, double *rhs,
                                             int32_t *bc_patch, char *names, int32_t names_len) {
    if (!dir || !owner || !neighbour || !face_area || !face_normal || !face_centroid || !streaming_dt ||
        !cell_volume || !cell_centroid || !gradient_stencil || !lhs_inverse || !rhs || !bc_patch)
        return lbfs::set_error(LBFS_ERR_ARG, "null argument");
    FoamMesh m;
    int rc = read_foam(dir, m, false);
    if (rc) return rc;
    std::copy(m.owner.begin(), m.owner.end(), owner);
    std::copy(m.neighbour.begin(), m.neighbour.end(), neighbour);
    int b = 0;
    for (size_t p = 0; p < m.patch_faces.size(); p++)
        for (int q = 0; q < m.patch_faces[p]; q++) bc_patch[b++] = (int32_t)p;
    if (names && names_len > 0) {
        std::string all;
        for (const std::string &n : m.patch_names) all += n + "\n";
        std::snprintf(names, (size_t)names_len, "%s", all.c_str());
    }
    return lbfs::mesh_geometry_gpu(device, m.n_points, m.n_cells, m.n_faces, m.n_internal, m.x.data(), m.y.data(),
                                   m.z.data(), m.fv.data(), owner, neighbour, visc, fneq_min, gradient_hybrid,
                                   closed_faces != 0, face_area, face_normal, face_centroid, streaming_dt,
                                   cell_volume, cell_centroid, gradient_stencil, lhs_inverse, rhs);
}

// Periodic partners (Boundary_Conditions::assign_boundary_conditions,
// Boundary_Conditions.cpp:417-432): the interior cell nearest to a point,
// distance |c_i - p| formed as vector_var::Magnitude does, the lowest index
// among equal distances (the reference's strict < over ascending i).  The
// cells are binned on a uniform grid over their centroids' box and the search
// walks shells of bins outwards: a cell in a bin r shells away from the
// point's (clamped) bin is at least (r - 1) times the smallest bin width away,
// so the walk stops once the best distance is below r times that width; the
// result is the all-cell search's.
namespace {
struct CellBins {
    int n[3];
    double lo[3], w[3], wmin;
    std::vector<int> start, list;
};

CellBins bin_cells(const double *cen, int nc) {
    CellBins b;
    double hi[3];
    for (int a = 0; a < 3; a++) b.lo[a] = hi[a] = cen[a];
    for (int i = 1; i < nc; i++)
        for (int a = 0; a < 3; a++) {
            b.lo[a] = std::min(b.lo[a], cen[3 * (size_t)i + a]);
            hi[a] = std::max(hi[a], cen[3 * (size_t)i + a]);
        }
    const double ext_max = std::max(hi[0] - b.lo[0], std::max(hi[1] - b.lo[1], hi[2] - b.lo[2]));
    const double h = ext_max > 0 ? ext_max / std::cbrt((double)nc) : 1.0;
    b.wmin = std::numeric_limits<double>::infinity();
    for (int a = 0; a < 3; a++) {
        const double ext = hi[a] - b.lo[a];
        b.n[a] = ext > 0 ? std::max(1, std::min(1 << 10, (int)std::ceil(ext / h))) : 1;
        b.w[a] = ext > 0 ? ext / b.n[a] : h;
        b.wmin = std::min(b.wmin, b.w[a]);
    }
    const size_t nbins = (size_t)b.n[0] * b.n[1] * b.n[2];
    b.start.assign(nbins + 1, 0);
    std::vector<int> key(nc);
    for (int i = 0; i < nc; i++) {
        int k[3];
        for (int a = 0; a < 3; a++) {
            const int q = (int)std::floor((cen[3 * (size_t)i + a] - b.lo[a]) / b.w[a]);
            k[a] = std::max(0, std::min(b.n[a] - 1, q));
        }
        key[i] = k[0] + b.n[0] * (k[1] + b.n[1] * k[2]);
        b.start[key[i] + 1]++;
    }
    for (size_t q = 0; q < nbins; q++) b.start[q + 1] += b.start[q];
    b.list.resize(nc);
    std::vector<int> fill(b.start.begin(), b.start.end() - 1);
    for (int i = 0; i < nc; i++) b.list[fill[key[i]]++] = i;  // ascending cell index within a bin
    return b;
}

void nearest_cell(const CellBins &b, const double *cen, V3 p, double &best, int &best_i) {
    int c[3];
    const double pp[3] = {p.x, p.y, p.z};
    for (int a = 0; a < 3; a++) {
        const double q = std::floor((pp[a] - b.lo[a]) / b.w[a]);
        c[a] = (int)std::max(0.0, std::min((double)(b.n[a] - 1), q));
    }
    const int rmax = std::max(b.n[0], std::max(b.n[1], b.n[2]));
    for (int r = 0; r <= rmax; r++) {
        for (int k = c[2] - r; k <= c[2] + r; k++) {
            if (k < 0 || k >= b.n[2]) continue;
            for (int j = c[1] - r; j <= c[1] + r; j++) {
                if (j < 0 || j >= b.n[1]) continue;
                for (int i = c[0] - r; i <= c[0] + r; i++) {
                    if (i < 0 || i >= b.n[0]) continue;
                    const int cheb = std::max(std::abs(i - c[0]), std::max(std::abs(j - c[1]), std::abs(k - c[2])));
                    if (cheb != r) continue;
                    const int bin = i + b.n[0] * (j + b.n[1] * k);
                    for (int q = b.start[bin]; q < b.start[bin + 1]; q++) {
                        const int cell = b.list[q];
                        const V3 ci = {cen[3 * (size_t)cell], cen[3 * (size_t)cell + 1], cen[3 * (size_t)cell + 2]};
                        const double d = mag(sub(ci, p));
                        if (d < best || (d == best && cell < best_i)) {
                            best = d;
                            best_i = cell;
                        }
                    }
                }
            }
        }
        if (best < r * b.wmin) break;
    }
}
}  // namespace

extern "C" int lbfs_mesh_find_periodic_nodes(const lbfs_mesh_desc *m, const double *translation, int32_t *out) {
    if (!m || !translation || !out || !m->cell_centroid || m->n_cells <= 0 || m->n_bc < 0 ||
        (m->n_bc > 0 && (!m->bc_rho_type || !m->bc_vel_type)))
        return lbfs::set_error(LBFS_ERR_ARG, "lbfs_mesh_find_periodic_nodes: bad arguments");
    const int nc = m->n_cells;
    const double *cen = m->cell_centroid;
    const CellBins bins = bin_cells(cen, nc);
    const V3 T = {translation[0], translation[1], translation[2]};
    for (int b = 0; b < m->n_bc; b++) {
        out[b] = 0;
        if (m->bc_rho_type[b] != 3 && m->bc_vel_type[b] != 3) continue;
        const size_t g = (size_t)nc + b;
        const V3 c = {cen[3 * g], cen[3 * g + 1], cen[3 * g + 2]};
        double best = std::numeric_limits<double>::infinity();
        int best_i = -1;
        nearest_cell(bins, cen, add(c, T), best, best_i);
        nearest_cell(bins, cen, sub(c, T), best, best_i);
        out[b] = best_i;
    }
    return LBFS_OK;
}

// Spring connectivity: the neighbour-ring construction, duplicate removal and
// spring hashing of lagrangian_object::osay_mesh_read (lagrangian_object.cpp:
// 299-481).  The ring is assembled by the same sequence of pair swaps, so the
// (a, b, c, d) quadruples come out in the reference's order.
extern "C" int lbfs_rbc_build_springs(int32_t n_nodes, int32_t n_tris, const int32_t *tri, int32_t capacity,
                                      int32_t *spring_out, int32_t *n_springs) {
    if (n_nodes <= 0 || n_tris <= 0 || !tri || !spring_out || !n_springs)
        return lbfs::set_error(LBFS_ERR_ARG, "bad membrane arguments");
    std::vector<std::vector<int>> ring(n_nodes);
    std::vector<int> degree(n_nodes, 0);
    for (int i = 0; i < 3 * n_tris; i++) {
        if (tri[i] < 0 || tri[i] >= n_nodes) return lbfs::set_error(LBFS_ERR_ARG, "triangle index out of range");
        degree[tri[i]]++;
    }
    for (int t = 0; t < n_tris; t++) {
        int v0 = tri[3 * t], v1 = tri[3 * t + 1], v2 = tri[3 * t + 2];
        ring[v0].push_back(v1); ring[v0].push_back(v2);
        ring[v1].push_back(v2); ring[v1].push_back(v0);
        ring[v2].push_back(v0); ring[v2].push_back(v1);
    }
    for (int i = 0; i < n_nodes; i++) {
        std::vector<int> &r = ring[i];
        if (r.size() < 4) return lbfs::set_error(LBFS_ERR_ARG, "node with fewer than two triangles");
        size_t it = 1;
        for (size_t t = 3; t < r.size(); t += 2) {
            size_t j = it + 1;
            while (j < r.size() && r[j] != r[it]) j++;
            if (j == r.size()) return lbfs::set_error(LBFS_ERR_ARG, "membrane is not a closed manifold");
            size_t num = j - it;
            if (num % 2 == 0) {
                if (it + num - 1 >= r.size()) return lbfs::set_error(LBFS_ERR_ARG, "membrane ring walk failed");
                std::swap(r[it + 1], r[it + num]);
                std::swap(r[it + 2], r[it + num - 1]);
            } else {
                if (it + num + 1 >= r.size()) return lbfs::set_error(LBFS_ERR_ARG, "membrane ring walk failed");
                std::swap(r[it + 1], r[it + num]);
                std::swap(r[it + 2], r[it + num + 1]);
            }
            it += 2;
        }
        // Remove repeated ids keeping the survivor the reference's uniquify
        // keeps: positions sorted by value with std::sort, first of each run
        // of equal values retained, survivors in original order.
        std::vector<size_t> pos(r.size());
        for (size_t q = 0; q < r.size(); q++) pos[q] = q;
        std::sort(pos.begin(), pos.end(), [&](size_t a, size_t b) { return r[a] < r[b]; });
        pos.erase(std::unique(pos.begin(), pos.end(), [&](size_t a, size_t b) { return r[a] == r[b]; }), pos.end());
        std::sort(pos.begin(), pos.end());
        std::vector<int> kept;
        kept.reserve(pos.size());
        for (size_t q : pos) kept.push_back(r[q]);
        r.swap(kept);
    }
    long long total = 0;
    for (int i = 0; i < n_nodes; i++) total += degree[i];
    const int expected = (int)(total / 2);
    if (expected > capacity) return lbfs::set_error(LBFS_ERR_LIMIT, "spring capacity too small");
    const int factor = (int)std::ceil(std::log10((double)n_nodes));
    std::unordered_set<long long> seen;
    int count = 0;
    for (int i = 0; i < n_nodes; i++) {
        const std::vector<int> &r = ring[i];
        const size_t m = r.size();
        for (size_t j = 0; j < m; j++) {
            int a = r[j], b = r[(j + 1) % m], c = r[(j + 2) % m];
            int q[4] = {i, a, b, c};
            std::sort(q, q + 4);
            long long h = 0;
            for (int t = 0; t < 4; t++) h = (long long)(h + q[t] * std::pow(10, factor * t));
            if (seen.insert(h).second) {
                if (count >= expected) return lbfs::set_error(LBFS_ERR_ARG, "more springs than edges");
                spring_out[4 * count] = i;
                spring_out[4 * count + 1] = a;
                spring_out[4 * count + 2] = b;
                spring_out[4 * count + 3] = c;
                count++;
            }
        }
    }
    *n_springs = count;
    return LBFS_OK;
}
