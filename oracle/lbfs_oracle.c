/*
 * lbfs_oracle.c -- TEST INFRASTRUCTURE ONLY.  CPU restatement, in plain serial
 * C, of the reference GPU time step of CHRG-Developer/LBFS-IBM-ADE-SP
 * (gpu_solver::General_Purpose_Solver_mk_i, Solver_gpu.cu:749-1046, and the
 * kernels it launches).  It is the checker the parity tests compare the CUDA
 * path against; the product never links it.
 *
 * Parity of this restatement is pinned against the reference itself: the
 * golden fixtures in tests/golden/ are produced by the reference's own kernel
 * sources compiled for the host (oracle/build_ref.sh, oracle/ref_driver.cpp),
 * and tests/test_oracle_golden.py checks this file against them.
 *
 * Same inputs as the product (include/lbfs_b200.h descriptors), FP64 only.
 * Evaluation order follows the reference kernels; sums that the reference
 * forms with atomics are formed here in face / node order.
 * Extensions without a reference counterpart (parity unpinned): the 4-point
 * Peskin delta (ibm_stencil = 4) and several membranes (each handled on its
 * own index range).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "lbfs_b200.h"

/* D3Q15 velocities and weights (gpu_solver::populate_e_alpha, Solver_gpu.cu:1407-1445) */
static const int EX[15] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1};
static const int EY[15] = {0, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, -1, 1, 1, -1};
static const int EZ[15] = {0, 0, 0, 0, 0, 1, -1, 1, -1, -1, 1, 1, -1, 1, -1};
static double W(int k) { return k == 0 ? 2.0 / 9.0 : (k < 7 ? 1.0 / 9.0 : 1.0 / 72.0); }

typedef struct {
    int n_nodes, n_tris, n_springs, node0, tri0, spring0;
    lbfs_rbc_desc d;
    double V, V0, A, A0, MAD, MAD0;
} omem;

typedef struct oracle_case {
    lbfs_mesh_desc m;
    lbfs_params p;
    int nc, nf, ni, nb, nt;
    /* copies of the mesh arrays (the descriptor's pointers are the caller's) */
    int *owner, *neighbour, *stencil, *rt, *vt, *per;
    double *area, *normal, *fcen, *sdt, *vol, *cen, *lhs, *rhs, *bcv;
    /* state: (u, v, w, rho) per cell incl. ghosts, soln_t1 per cell */
    double *soln, *t1, *grad, *flux, *res, *force, *visc;
    double *cfl, *dtl; /* cfl areas (x, y, z per cell), per-cell step */
    /* LBFS_IBM_VANDERMONDE4: vertex coordinates and cell-row centroids per axis */
    double *gv[3], *gc[3];
    int gn[3];
    double dt;         /* the step's delta_t */
    double resid[4];
    long long t;
    /* membranes */
    int n_mem, N, T, S;
    omem *mem;
    int *tri, *spr;
    double *x, *y, *z, *vx, *vy, *vz, *fx, *fy, *fz;
    double *contour, *kspr, *curv, *curv0, *ang0, *area0, *sarea;
} oracle_case;

static void *dup(const void *src, size_t bytes) {
    void *p = malloc(bytes ? bytes : 1);
    if (src && bytes) memcpy(p, src, bytes);
    else memset(p, 0, bytes ? bytes : 1);
    return p;
}

/* ------------------------------------------------------------ fluid ---- */

/* update_unstructured_bcs, LBFS.cu:1843-1928; type 3 (periodic) as the CPU
 * solver's Solution::update_unstructured_bcs (Solution.cpp:777-803): the
 * partner cell's values. */
static void ghost_update(oracle_case *o) {
    const double H2 = o->p.channel_diameter * 0.5;
    const double H4 = o->p.channel_diameter * o->p.channel_diameter * o->p.channel_diameter * o->p.channel_diameter;
    for (int i = 0; i < o->nb; i++) {
        const int j = i + o->nc, nb = o->owner[i + o->ni];
        const double *s = o->soln + 4 * nb, *bc = o->bcv + 4 * i;
        double *g = o->soln + 4 * j;
        /* soln layout: 0 u, 1 v, 2 w, 3 rho; bcv layout: u, v, w, rho */
        const double *ps = o->soln + 4 * o->per[i];
        if (o->rt[i] == 1) g[3] = bc[3] - (s[3] - bc[3]);
        else if (o->rt[i] == 3) g[3] = ps[3];
        else g[3] = s[3];
        if (o->vt[i] == 3) {
            for (int c = 0; c < 3; c++) g[c] = ps[c];
        } else if (o->vt[i] == 1) {
            for (int c = 0; c < 3; c++) g[c] = bc[c] - (s[c] - bc[c]);
        } else if (o->vt[i] == 2) {
            for (int c = 0; c < 3; c++) g[c] = s[c];
        } else {
            const double *cell = o->cen + 3 * j;
            double ut;
            if (o->vt[i] == 9) ut = 16 * bc[0] * (H2 + cell[1]) * (H2 - cell[1]) * (H2 + cell[2]) * (H2 - cell[2]) / H4;
            else ut = (cell[1]) * bc[0];
            g[0] = ut - (s[0] - ut);
            g[1] = bc[1] - (s[1] - bc[1]);
            g[2] = bc[2] - (s[2] - bc[2]);
        }
    }
}

/* get_interior_gradients + add_LS_contributions, LBFS.cu:2177-2240, 2051-2083.
 * grad layout per cell: rho(x,y,z), u(x,y,z), v(x,y,z), w(x,y,z). */
static void interior_gradients(oracle_case *o) {
    static const int var[4] = {3, 0, 1, 2}; /* rho, u, v, w in soln order */
    for (int i = 0; i < o->nc; i++) {
        double R[4][3] = {{0}};
        for (int q = 0; q < 6; q++) {
            const int i1 = o->stencil[6 * i + q];
            const double *r3 = o->rhs + 18 * i + 3 * q;
            for (int m = 0; m < 4; m++) {
                const double d = o->soln[4 * i1 + var[m]] - o->soln[4 * i + var[m]];
                for (int c = 0; c < 3; c++) R[m][c] = R[m][c] + r3[c] * d;
            }
        }
        const double *L = o->lhs + 9 * i;
        double *g = o->grad + 12 * i;
        for (int m = 0; m < 4; m++)
            for (int r = 0; r < 3; r++) g[3 * m + r] = L[3 * r] * R[m][0] + L[3 * r + 1] * R[m][1] + L[3 * r + 2] * R[m][2];
    }
}

/* get_bc_gradients, LBFS.cu:1933-2048; a periodic (type 3) component takes
 * the partner cell's gradient (gradients::Get_LS_Gradients,
 * gradients.cpp:428-440), formed before the ghosts' as there. */
static void bc_gradients(oracle_case *o) {
    static const int var[4] = {3, 0, 1, 2};
    for (int i = 0; i < o->nb; i++) {
        const int face = o->ni + i, nbi = o->owner[face], j = i + o->nc;
        const double *n = o->normal + 3 * face;
        const double dx = o->cen[3 * j] - o->cen[3 * nbi], dy = o->cen[3 * j + 1] - o->cen[3 * nbi + 1],
                     dz = o->cen[3 * j + 2] - o->cen[3 * nbi + 2];
        const double dmag = sqrt(pow(dx, 2.0) + pow(dy, 2.0) + pow(dz, 2.0));
        const double un[3] = {dx / dmag, dy / dmag, dz / dmag};
        double *g = o->grad + 12 * j;
        const double *go = o->grad + 12 * nbi;
        for (int m = 0; m < 4; m++) {
            const int dirichlet = (m == 0) ? (o->rt[i] == 1) : (o->vt[i] == 1 || o->vt[i] == 9 || o->vt[i] == 10);
            const int periodic = (m == 0) ? (o->rt[i] == 3) : (o->vt[i] == 3);
            const double d = o->soln[4 * j + var[m]] - o->soln[4 * nbi + var[m]];
            const double *gp = o->grad + 12 * o->per[i];
            for (int c = 0; c < 3; c++)
                g[3 * m + c] = periodic ? gp[3 * m + c]
                                        : (dirichlet ? d / dmag * un[c] : go[3 * m + c] * (1 - fabs(n[c])));
        }
    }
}

/* feq of populate_feq_lattice_explicit (LBFS.cu:1041-1354) and of
 * calculate_flux_at_interface (q scales the quadratic terms: 1/gamma there). */
static double feq(int k, double rho, double u, double v, double w, double q) {
    const double uu2 = u * u * q, vv2 = v * v * q, ww2 = w * w * q, u2v2w2 = (uu2 + vv2 + ww2) * 1.5;
    if (k == 0) return W(k) * rho * (1.0 - u2v2w2);
    if (k < 7) {
        const double c = EX[k] ? u : (EY[k] ? v : w), c2 = EX[k] ? uu2 : (EY[k] ? vv2 : ww2);
        const double s = EX[k] + EY[k] + EZ[k];
        return W(k) * rho * (1.0 + s * 3.0 * c + 4.5 * c2 - u2v2w2);
    }
    const double uv = u * v * 9.0 * q, uw = u * w * 9.0 * q, vw = v * w * 9.0 * q;
    return W(k) * rho *
           (1.0 + EX[k] * 3.0 * u + EY[k] * 3.0 * v + EZ[k] * 3.0 * w + EX[k] * EY[k] * uv + EX[k] * EZ[k] * uw +
            EY[k] * EZ[k] * vw + 4.5 * uu2 + 4.5 * vv2 + 4.5 * ww2 - u2v2w2);
}

/* Interface moments, BGK relaxation and flux (calculate_flux_at_interface,
 * LBFS.cu:1462-1648; axis forms LBFS.cu:3648-4092).  out = (u, v, w, rho). */
static void flux_from_lattice(const double fl[15], double tau, double q, double area, int axis, const double *n,
                              double out[4]) {
    double rho = 0, mx = 0, my = 0, mz = 0;
    for (int k = 0; k < 15; k++) rho += fl[k];
    for (int k = 1; k < 15; k++) { mx += EX[k] * fl[k]; my += EY[k] * fl[k]; mz += EZ[k] * fl[k]; }
    const double ux = 1 / rho * mx, uy = 1 / rho * my, uz = 1 / rho * mz;
    double F[3][4] = {{0}};
    for (int k = 1; k < 15; k++) {
        const int e[3] = {EX[k], EY[k], EZ[k]};
        if (axis >= 0 && !e[axis]) continue;
        double f = feq(k, rho, ux, uy, uz, q);
        f = f - tau * (f - fl[k]);
        for (int c = 0; c < 3; c++) {
            if (!e[c]) continue;
            F[c][3] += e[c] * f;
            for (int mm = 0; mm < 3; mm++) F[c][mm] += e[c] * e[mm] * f;
        }
    }
    for (int m = 0; m < 4; m++)
        out[m] = (axis >= 0) ? F[axis][m] * area : (F[0][m] * n[0] + F[1][m] * n[1] + F[2][m] * n[2]) * area;
}

/* Value at the lattice node x_f - e_k dt extrapolated from base value b with gradient g:
 * the reference subtracts/adds g_x dt, g_y dt, g_z dt in that order. */
static double extrap(double b, const double *g, const int e[3], double dt) {
    for (int d = 0; d < 3; d++) {
        if (e[d] > 0) b = b - g[d] * dt;
        else if (e[d] < 0) b = b + g[d] * dt;
    }
    return b;
}

/* calc_face_flux_x/_y/_z with populate_lattice_macros_uniform_{x,y,z}
 * (LBFS.cu:2283-2569, 2939-3644). */
static void axis_face(oracle_case *o, int f, int axis) {
    static const int var[4] = {3, 0, 1, 2};
    const int i = o->owner[f], nb = o->neighbour[f];
    const double dt = o->sdt[f];
    const double t1 = o->cen[3 * i + axis] - o->fcen[3 * f + axis], t2 = o->cen[3 * nb + axis] - o->fcen[3 * f + axis];
    const double c = o->cen[3 * nb + axis] - o->cen[3 * i + axis];
    const double a = fabs(t2 / c), b = fabs(t1 / c);
    double L[15][4];
    for (int m = 0; m < 4; m++) {
        const double *g1 = o->grad + 12 * i + 3 * m, *g2 = o->grad + 12 * nb + 3 * m;
        const double pi = o->soln[4 * i + var[m]] - t1 * g1[axis];
        const double pn = o->soln[4 * nb + var[m]] - (t2 * g2[axis]);
        const double p0 = (pi + pn) * 0.5;
        double g3[3];
        for (int d = 0; d < 3; d++) g3[d] = (g1[d] * a + g2[d] * b);
        for (int k = 0; k < 15; k++) {
            const int e[3] = {EX[k], EY[k], EZ[k]};
            if (e[axis] > 0) L[k][m] = extrap(pi, g1, e, dt);      /* owner (west) side */
            else if (e[axis] < 0) L[k][m] = extrap(pn, g2, e, dt); /* neighbour (east) side */
            else L[k][m] = extrap(p0, g3, e, dt);                  /* on the face plane */
        }
    }
    double fl[15];
    for (int k = 0; k < 15; k++) fl[k] = feq(k, L[k][0], L[k][1], L[k][2], L[k][3], 1.0);
    const double tau = (o->p.testcase == 8) ? 0.0 : (o->p.visc * o->visc[i] * 3 / dt * o->p.gamma_inv);
    flux_from_lattice(fl, tau, 1.0, o->area[f], axis, NULL, o->flux + 4 * f);
}

/* calc_face_flux / calc_face_flux_bc with populate_lattice_macros
 * (LBFS.cu:2574-2810, 323-936). */
static void general_face(oracle_case *o, int f, int is_bc) {
    static const int var[4] = {3, 0, 1, 2};
    const int i = o->owner[f], nb = o->neighbour[f];
    const double dt = o->sdt[f];
    const double *n = o->normal + 3 * f;
    double t1[3], t2[3];
    for (int d = 0; d < 3; d++) {
        t1[d] = o->cen[3 * i + d] - o->fcen[3 * f + d];
        t2[d] = o->cen[3 * nb + d] - o->fcen[3 * f + d];
    }
    const double d1 = 0.001 * dt; /* LBFS.cu:351-352 */
    double L[15][4];
    for (int m = 0; m < 4; m++) {
        const double *g1 = o->grad + 12 * i + 3 * m, *g2 = o->grad + 12 * nb + 3 * m;
        double pi, pn, p0, g3[3];
        const double *G1 = g1;
        if (nb > o->nc) {
            const int bi = nb - o->nc;
            const int dir = (m == 0) ? (o->rt[bi] == 1) : (o->vt[bi] == 1);
            const double bcval = o->bcv[4 * bi + var[m]];
            p0 = dir ? bcval : o->soln[4 * i + var[m]] - (t1[0] * g2[0] + t1[1] * g2[1] + t1[2] * g2[2]);
            pi = p0;
            pn = p0;
            for (int d = 0; d < 3; d++) g3[d] = g2[d];
            G1 = g2;
        } else {
            pi = o->soln[4 * i + var[m]] - (t1[0] * g1[0] + t1[1] * g1[1] + t1[2] * g1[2]);
            pn = o->soln[4 * nb + var[m]] - (t2[0] * g2[0] + t2[1] * g2[1] + t2[2] * g2[2]);
            p0 = (pi + pn) * 0.5;
            for (int d = 0; d < 3; d++) g3[d] = (g1[d] + g2[d]) * 0.5;
        }
        L[0][m] = p0;
        for (int k = 1; k < 15; k += 2) {
            const int e[3] = {EX[k], EY[k], EZ[k]}, eo[3] = {-EX[k], -EY[k], -EZ[k]};
            const double s = (k < 7) ? (e[0] ? n[0] : (e[1] ? n[1] : n[2])) : (e[0] * n[0] + e[1] * n[1] + e[2] * n[2]);
            if (s > d1) {
                L[k][m] = extrap(pi, G1, e, dt);
                L[k + 1][m] = extrap(pn, g2, eo, dt);
            } else if (s < -d1) {
                L[k][m] = extrap(pn, g2, e, dt);
                L[k + 1][m] = extrap(pi, G1, eo, dt);
            } else {
                L[k][m] = extrap(p0, g3, e, dt);
                L[k + 1][m] = extrap(p0, g3, eo, dt);
            }
        }
    }
    double fl[15];
    /* populate_feq with 1/gamma when preconditioning, else the explicit form (LBFS.cu:2637-2647) */
    const double q = o->p.preconditioning ? o->p.gamma_inv : 1.0;
    for (int k = 0; k < 15; k++) fl[k] = feq(k, L[k][0], L[k][1], L[k][2], L[k][3], q);
    const double vf = is_bc ? 1.0 : o->visc[i];
    const double tau = (o->p.testcase == 8) ? 0.0 : (o->p.visc * vf * 3 / dt * o->p.gamma_inv);
    flux_from_lattice(fl, tau, o->p.gamma_inv, o->area[f], -1, n, o->flux + 4 * f);
}

/* ---------------------------------------------------------- membranes ---- */

static double peskin4(double r) {
    r = fabs(r);
    if (r < 1.0) return (3.0 - 2.0 * r + sqrt(1.0 + 4.0 * r - 4.0 * r * r)) * 0.125;
    if (r < 2.0) return (5.0 - 2.0 * r - sqrt(-7.0 + 12.0 * r - 4.0 * r * r)) * 0.125;
    return 0.0;
}

/* IBM stencil of a node: reference coordinates (y, z mirrored with fabs as in
 * immersed_boundary_method.cu:45-58), first cell, width and weights. */
static void node_stencil(const oracle_case *o, double x, double y, double z, double r[3], int i0[3], int *S) {
    r[0] = (x - o->m.origin[0]) / o->m.delta_x;
    r[1] = fabs((y - o->m.origin[1]) / o->m.delta_x);
    r[2] = fabs((z - o->m.origin[2]) / o->m.delta_x);
    if (o->p.ibm_stencil == LBFS_IBM_PESKIN4) {
        *S = 4;
        for (int c = 0; c < 3; c++) i0[c] = (int)floor(r[c] - 0.5) - 1;
    } else {
        *S = 2;
        for (int c = 0; c < 3; c++) i0[c] = (int)round(r[c]) - 1;
    }
}
static double ibm_weight(const oracle_case *o, double d) {
    return o->p.ibm_stencil == LBFS_IBM_PESKIN4 ? peskin4(d) : 1 - fabs(d);
}

/* find_index_closest (immersed_boundary_method.cu:588-630), as written there. */
static int find_index_closest(const double *arr, int n, double target) {
    if (target <= arr[0]) return 0;
    if (target >= arr[n - 1]) return n - 1;
    int i = 0, j = n, mid = 0;
    while (i < j) {
        mid = (i + j) / 2;
        if (arr[mid] == target) return mid;
        if (target < arr[mid]) {
            if (mid > 0 && target > arr[mid - 1]) return (target - arr[mid - 1] >= arr[mid] - target) ? mid : mid - 1;
            j = mid;
        } else {
            if (mid < n - 1 && target < arr[mid + 1]) return (target - arr[mid] >= arr[mid + 1] - target) ? mid + 1 : mid;
            i = mid + 1;
        }
    }
    return mid;
}

/* vandemonde_inverse, 4 points (immersed_boundary_method.cu:919-941). */
static void vandermonde_inverse4(double x, double y, double z, double w, double out[4]) {
    const double sub_xy = 1 / (x - y), sub_xz = 1 / (x - z), sub_xw = 1 / (x - w);
    const double sub_yz = 1 / (y - z), sub_yw = 1 / (y - w), sub_zw = 1 / (z - w);
    out[0] = -1 * y * z * w * sub_xy * sub_xz * sub_xw;
    out[1] = x * z * w * sub_xy * sub_yz * sub_yw;
    out[2] = -1 * x * y * w * sub_xz * sub_yz * sub_zw;
    out[3] = x * y * z * sub_xw * sub_yw * sub_zw;
}

/* The 4x4x4 stencil of the mesh_type 4 kernels (immersed_boundary_method.cu:
 * 685-740, 790-840): first cell per axis (closest vertex - 2) and the 1D
 * weights from the cell-row centroid offsets.  A stencil leaving the mesh
 * (the reference reads outside its arrays) gets zero weights. */
static void vandermonde_stencil(const oracle_case *o, const double p[3], int i0[3], double w[3][4]) {
    for (int a = 0; a < 3; a++) {
        i0[a] = find_index_closest(o->gv[a], o->gn[a] + 1, p[a]) - 2;
        if (i0[a] < 0 || i0[a] + 3 >= o->gn[a]) {
            for (int q = 0; q < 4; q++) w[a][q] = 0.0;
            continue;
        }
        const double *c = o->gc[a] + i0[a];
        vandermonde_inverse4(c[0] - p[a], c[1] - p[a], c[2] - p[a], c[3] - p[a], w[a]);
    }
}

/* interpolate_velocities_on_nodes_non_uniform_grid (immersed_boundary_method.cu:633-758), one node */
static void interpolate_vandermonde(const oracle_case *o, int n, double v[3]) {
    const int nx = o->gn[0], ny = o->gn[1];
    const double p[3] = {o->x[n], o->y[n], o->z[n]};
    int i0[3];
    double w[3][4];
    vandermonde_stencil(o, p, i0, w);
    for (int i = i0[0]; i <= i0[0] + 3; i++)
        for (int j = i0[1]; j <= i0[1] + 3; j++)
            for (int k = i0[2]; k <= i0[2] + 3; k++) {
                const int idx = i + j * nx + k * ny * nx;
                if (idx < o->nc && idx >= 0) {
                    const double weight = w[0][i - i0[0]] * w[1][j - i0[1]] * w[2][k - i0[2]];
                    for (int c = 0; c < 3; c++) v[c] += o->soln[4 * idx + c] * weight;
                }
            }
}

/* interpolate_velocities_on_nodes + update_node_positions (immersed_boundary_method.cu:14-97, 234-264) */
static void interpolate_and_move(oracle_case *o) {
    const int nx = (int)(o->m.length[0] / o->m.delta_x), ny = (int)(o->m.length[1] / o->m.delta_x);
    for (int n = 0; n < o->N; n++) {
        if (o->p.ibm_stencil == LBFS_IBM_VANDERMONDE4) {
            double v[3] = {0.0, 0.0, 0.0};
            interpolate_vandermonde(o, n, v);
            o->vx[n] = v[0]; o->vy[n] = v[1]; o->vz[n] = v[2];
            o->x[n] += v[0] * o->dt;
            o->y[n] += v[1] * o->dt;
            o->z[n] += v[2] * o->dt;
            continue;
        }
        double r[3];
        int i0[3], S;
        node_stencil(o, o->x[n], o->y[n], o->z[n], r, i0, &S);
        double v[3] = {0.0, 0.0, 0.0};
        for (int i = i0[0]; i < i0[0] + S; i++)
            for (int j = i0[1]; j < i0[1] + S; j++)
                for (int k = i0[2]; k < i0[2] + S; k++) {
                    const int idx = i + j * nx + k * ny * nx;
                    if (idx < o->nc && idx >= 0) {
                        const double wx = ibm_weight(o, i + 0.5 - r[0]), wy = ibm_weight(o, j + 0.5 - r[1]),
                                     wz = ibm_weight(o, k + 0.5 - r[2]);
                        for (int c = 0; c < 3; c++) v[c] += o->soln[4 * idx + c] * wx * wy * wz;
                    }
                }
        o->vx[n] = v[0]; o->vy[n] = v[1]; o->vz[n] = v[2];
        o->x[n] += v[0] * o->dt;
        o->y[n] += v[1] * o->dt;
        o->z[n] += v[2] * o->dt;
    }
}

/* spread_forces_on_structured_grid (immersed_boundary_method.cu:947-1024), node order */
static void spread(oracle_case *o) {
    const int nx = (int)(o->m.length[0] / o->m.delta_x), ny = (int)(o->m.length[1] / o->m.delta_x);
    const double inv3 = 1 / o->m.delta_x / o->m.delta_x / o->m.delta_x;
    for (int n = 0; n < o->N; n++) {
        if (o->p.ibm_stencil == LBFS_IBM_VANDERMONDE4) {
            /* spread_forces_on_non_uniform_grid (immersed_boundary_method.cu:761-872) */
            const double p[3] = {o->x[n], o->y[n], o->z[n]};
            int i0[3];
            double w[3][4];
            vandermonde_stencil(o, p, i0, w);
            for (int i = i0[0]; i <= i0[0] + 3; i++)
                for (int j = i0[1]; j <= i0[1] + 3; j++)
                    for (int k = i0[2]; k <= i0[2] + 3; k++) {
                        const int idx = i + j * o->gn[0] + k * o->gn[1] * o->gn[0];
                        if (idx < o->nc && idx >= 0) {
                            const double weight = w[0][i - i0[0]] * w[1][j - i0[1]] * w[2][k - i0[2]] / o->vol[idx];
                            o->force[3 * idx] += o->fx[n] * weight;
                            o->force[3 * idx + 1] += o->fy[n] * weight;
                            o->force[3 * idx + 2] += o->fz[n] * weight;
                        }
                    }
            continue;
        }
        double r[3];
        int i0[3], S;
        node_stencil(o, o->x[n], o->y[n], o->z[n], r, i0, &S);
        for (int i = i0[0]; i < i0[0] + S; i++)
            for (int j = i0[1]; j < i0[1] + S; j++)
                for (int k = i0[2]; k < i0[2] + S; k++) {
                    const int idx = i + j * nx + k * ny * nx;
                    if (idx < o->nc && idx >= 0) {
                        const double wx = ibm_weight(o, i + 0.5 - r[0]), wy = ibm_weight(o, j + 0.5 - r[1]),
                                     wz = ibm_weight(o, k + 0.5 - r[2]);
                        o->force[3 * idx] += o->fx[n] * wx * wy * wz * inv3;
                        o->force[3 * idx + 1] += o->fy[n] * wx * wy * wz * inv3;
                        o->force[3 * idx + 2] += o->fz[n] * wx * wy * wz * inv3;
                    }
                }
    }
}

typedef struct { double x, y, z; } v3;
static v3 V3(double x, double y, double z) { v3 r = {x, y, z}; return r; }
static v3 vsub(v3 a, v3 b) { return V3(a.x - b.x, a.y - b.y, a.z - b.z); }
static v3 vadd(v3 a, v3 b) { return V3(a.x + b.x, a.y + b.y, a.z + b.z); }
static v3 vmul(v3 a, double s) { return V3(a.x * s, a.y * s, a.z * s); }
static v3 vdiv(v3 a, double s) { return V3(a.x / s, a.y / s, a.z / s); }
static double vdot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static v3 vcross(v3 a, v3 b) { return V3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
static v3 vcen(v3 a, v3 b, v3 c) { return V3((a.x + b.x + c.x) / 3, (a.y + b.y + c.y) / 3, (a.z + b.z + c.z) / 3); }
static v3 node(const oracle_case *o, int n) { return V3(o->x[n], o->y[n], o->z[n]); }

/* update_spring_network_tet_parameters + total<128> + add_volume/add_area
 * (spring_network.cu:1186-1238, lagrangian_object.cpp:601-630); sums in triangle order. */
static void triangle_totals(oracle_case *o, omem *M, int initials) {
    double V = 0, A = 0;
    for (int t = M->tri0; t < M->tri0 + M->n_tris; t++) {
        const v3 a = node(o, o->tri[3 * t]), b = node(o, o->tri[3 * t + 1]), c = node(o, o->tri[3 * t + 2]);
        const v3 nrm = vcross(vsub(b, a), vsub(c, a));
        A += sqrt(vdot(nrm, nrm)) * 0.5;
        V += vdot(nrm, vcen(a, b, c)) / 6;
    }
    M->V = V;
    M->A = A;
    if (initials) {
        M->V0 = V * M->d.volume_ratio;
        M->A0 = A;
    }
}

/* d(normal)/d(node) of the triangle (p, q, r) (get_d_normals, spring_network.cu:1348-1414):
 * dn[9 s + 3 c + k] = d normal_k / d(node s)_c, and dv[3 s + c] the volume derivative. */
static void dnormals(v3 p, v3 q, v3 r, v3 nrm, double dn[27], double dv[9]) {
    const v3 P[3] = {p, q, r};
    for (int s = 0; s < 3; s++) {
        const v3 A = P[(s + 1) % 3], B = P[(s + 2) % 3];
        /* d((q-p)x(r-p))/d(node s) is the cross-product matrix of (B - A) */
        const double dd[3] = {B.x - A.x, B.y - A.y, B.z - A.z};
        double *D = dn + 9 * s;
        D[0] = 0.0;    D[1] = dd[2];  D[2] = -dd[1];
        D[3] = -dd[2]; D[4] = 0.0;    D[5] = dd[0];
        D[6] = dd[1];  D[7] = -dd[0]; D[8] = 0.0;
    }
    const v3 cen = vcen(p, q, r), n3 = vdiv(nrm, 3.0);
    for (int s = 0; s < 3; s++) {
        const double *D = dn + 9 * s;
        dv[3 * s] = n3.x + D[1] * cen.y + D[2] * cen.z;
        dv[3 * s + 1] = n3.y + D[3] * cen.x + D[5] * cen.z;
        dv[3 * s + 2] = n3.z + D[6] * cen.x + D[7] * cen.y;
    }
}

/* get_spring_forces_atomics (spring_network.cu:613-971); forces accumulated per node in spring order */
static void spring_forces(oracle_case *o, omem *M, int initials) {
    const lbfs_rbc_desc *d = &M->d;
    const double wr = d->wlc_ratio;
    const double sfc = (0.25 * wr * wr / ((wr - 1.0) * (wr - 1.0)) - 0.25 + 1.0 / wr);
    const double vc = -1 * d->volume_modulus * (M->V / M->V0 - 1.0) / 6.0;
    const double ac = -1 * d->global_area_modulus * (M->A / M->A0 - 1.0);
    const double madc = -1 * 2.0 * d->global_bending_modulus * (M->MAD - M->MAD0) / M->A0;
    for (int s = M->spring0; s < M->spring0 + M->n_springs; s++) {
        const int id[4] = {o->spr[4 * s], o->spr[4 * s + 1], o->spr[4 * s + 2], o->spr[4 * s + 3]};
        const v3 a = node(o, id[0]), b = node(o, id[1]), c = node(o, id[2]), dd = node(o, id[3]);
        const v3 l = vsub(c, a);
        const double len = sqrt(vdot(l, l));
        const v3 na = vcross(vsub(b, a), vsub(c, a)), nb = vcross(vsub(c, a), vsub(dd, a));
        const double n1 = sqrt(vdot(na, na)), n2 = sqrt(vdot(nb, nb));
        double dN1[27], dN2[27], dV1[9], dV2[9], dn1[9], dn2[9];
        dnormals(a, b, c, na, dN1, dV1);
        dnormals(c, dd, a, nb, dN2, dV2);
        const v3 u1 = vdiv(na, n1), u2 = vdiv(nb, n2);
        for (int j = 0; j < 9; j++) {
            dn1[j] = dN1[3 * j] * u1.x + dN1[3 * j + 1] * u1.y + dN1[3 * j + 2] * u1.z;
            dn2[j] = dN2[3 * j] * u2.x + dN2[3 * j + 1] * u2.y + dN2[3 * j + 2] * u2.z;
        }
        /* 12-vectors over (a, b, c, d): triangle 1 is (a, b, c), triangle 2 is (c, d, a) */
        double dA[12], dVol[12], dAng[12];
        double da1[9], da2[9];
        const v3 h1 = vcross(u1, vdiv(l, len)), h2 = vcross(vdiv(l, len), u2);
        for (int j = 0; j < 9; j++) {
            da1[j] = -1 / n1 * (h1.x * dN1[3 * j] + h1.y * dN1[3 * j + 1] + h1.z * dN1[3 * j + 2]);
            da2[j] = -1 / n2 * (h2.x * dN2[3 * j] + h2.y * dN2[3 * j + 1] + h2.z * dN2[3 * j + 2]);
        }
        const double *t1s[3] = {dn1, dV1, da1}, *t2s[3] = {dn2, dV2, da2};
        double *outs[3] = {dA, dVol, dAng};
        for (int q = 0; q < 3; q++) {
            double *O = outs[q];
            for (int j = 0; j < 9; j++) O[j] = t1s[q][j];
            for (int j = 0; j < 3; j++) O[j + 6] += t2s[q][j];
            for (int j = 3; j < 6; j++) O[j + 6] = t2s[q][j];
            for (int j = 6; j < 9; j++) O[j - 6] += t2s[q][j];
        }
        for (int j = 0; j < 12; j++) dA[j] *= 0.166666666666666666666666666666666666666666;
        for (int j = 0; j < 12; j++) dVol[j] *= (1.0 / 18.0);
        double ca = vdot(na, nb) / (n1 * n2);
        ca = fmin(ca, 1.0);
        ca = fmax(ca, -1.0);
        const v3 c2 = vsub(vcen(a, c, dd), vcen(a, b, c));
        const double adir = vdot(na, c2);
        const double ang = ((adir < 0) - (adir > 0)) * acos(ca);
        if (initials) {
            o->ang0[s] = ang;
            o->area0[2 * s] = n1;
            o->area0[2 * s + 1] = n2;
        }
        const v3 dL = vdiv(l, len);
        double dC[12];
        for (int j = 0; j < 12; j++) dC[j] = dAng[j] * len;
        dC[0] -= dL.x * ang; dC[1] -= dL.y * ang; dC[2] -= dL.z * ang;
        dC[6] += dL.x * ang; dC[7] += dL.y * ang; dC[8] += dL.z * ang;
        double F[12] = {0};
        double lac = -1 * d->local_area_modulus * (n1 / o->area0[2 * s] - 1) + ac;
        for (int c = 0; c < 3; c++) F[3 + c] += lac * dn1[3 + c];
        lac = -1 * d->local_area_modulus * (n2 / o->area0[2 * s + 1] - 1) + ac;
        for (int c = 0; c < 3; c++) F[9 + c] += lac * dn2[3 + c];
        for (int j = 0; j < 12; j++) F[j] += vc * dVol[j];
        {
            const v3 dv = vsub(V3(o->vx[id[2]], o->vy[id[2]], o->vz[id[2]]), V3(o->vx[id[0]], o->vy[id[0]], o->vz[id[0]]));
            const v3 visc = vmul(vdiv(vmul(vmul(vmul(dL, -1), vdot(dL, dv)), 4), sqrt(3.0)), d->viscosity);
            F[6] += visc.x; F[7] += visc.y; F[8] += visc.z;
            F[0] -= visc.x; F[1] -= visc.y; F[2] -= visc.z;
        }
        const double curvature = ang * len / ((n1 + n2) / 6.0);
        o->curv[s] = curvature;
        o->sarea[2 * s] = n1;
        o->sarea[2 * s + 1] = n2;
        const double c0 = o->curv0[s];
        const double lbc = -0.5 * d->local_bending_modulus * (c0 - curvature) * (c0 - curvature);
        const double cc = -1 * d->global_bending_modulus * (curvature - c0) + madc;
        for (int j = 0; j < 12; j++) F[j] += lbc * dA[j];
        for (int j = 0; j < 12; j++) F[j] += cc * dC[j];
        const double sr = len / o->contour[s];
        const double fcoef = -1 * o->kspr[s] * ((0.25 / ((1.0 - sr) * (1.0 - sr))) - 0.25 + sr - sfc);
        F[6] += dL.x * fcoef; F[7] += dL.y * fcoef; F[8] += dL.z * fcoef;
        F[0] -= dL.x * fcoef; F[1] -= dL.y * fcoef; F[2] -= dL.z * fcoef;
        for (int q = 0; q < 4; q++) {
            o->fx[id[q]] += F[3 * q];
            o->fy[id[q]] += F[3 * q + 1];
            o->fz[id[q]] += F[3 * q + 2];
        }
    }
}

/* sum_product_curvature<128> over the first n_nodes springs + add_MAD (common_kernels.hpp:97-119, lagrangian_object.cpp:633-650) */
static void mad(oracle_case *o, omem *M, int initials) {
    double s = 0;
    const int n = M->n_nodes < M->n_springs ? M->n_nodes : M->n_springs;
    for (int i = M->spring0; i < M->spring0 + n; i++) s += o->curv[i] * (o->sarea[2 * i] + o->sarea[2 * i + 1]) * 1 / 3;
    M->MAD = s / M->A;
    if (initials) M->MAD0 = M->MAD;
}

/* get_contour_lengths + get_reference_curvatures on the stress-free mesh (spring_network.cu:389-604) */
static void reference_pass(oracle_case *o, omem *M) {
    const lbfs_rbc_desc *d = &M->d;
    for (int s = M->spring0; s < M->spring0 + M->n_springs; s++) {
        const v3 a = node(o, o->spr[4 * s]), b = node(o, o->spr[4 * s + 1]), c = node(o, o->spr[4 * s + 2]),
                 dd = node(o, o->spr[4 * s + 3]);
        const v3 l = vsub(c, a);
        const double len = sqrt(vdot(l, l));
        const double cons = (0.5 * pow(1.0 - 1 / d->wlc_ratio, -3.0) + 1.0);
        const double L0 = d->pivkin_length ? d->reference_length : len;
        o->kspr[s] = ((4.0 * d->wlc_ratio * L0 * d->shear_modulus) / (sqrt(3.0) * cons));
        o->contour[s] = L0 * d->wlc_ratio;
        const v3 na = vcross(vsub(b, a), vsub(c, a)), nb = vcross(vsub(c, a), vsub(dd, a));
        const double n1 = sqrt(vdot(na, na)), n2 = sqrt(vdot(nb, nb));
        double ca = vdot(na, nb) / (n1 * n2);
        ca = fmin(ca, 1.0);
        ca = fmax(ca, -1.0);
        const double adir = vdot(vsub(nb, na), vsub(vcen(a, c, dd), vcen(a, b, c)));
        const double ang = ((adir > 0) - (adir < 0)) * acos(ca);
        o->curv[s] = ang * len / ((n1 + n2) / 6.0);
        o->sarea[2 * s] = n1;
        o->sarea[2 * s + 1] = n2;
        o->curv0[s] = d->sphere_reference ? d->curvature_ratio / 3.265483301 : 0.0;
        o->ang0[s] = ang;
        o->area0[2 * s] = n1;
        o->area0[2 * s + 1] = n2;
    }
}

/* update_viscosities + update_interior_viscosities_plucker (Solver_gpu.cu:2153-2208,
 * immersed_boundary_method.cu:389-527), per membrane bounding box */
static void interior_viscosity(oracle_case *o) {
    const double pi = acos(-1.0), dh = o->m.delta_h;
    for (int i = 0; i < o->nc; i++) o->visc[i] = 1.0;
    for (int mi = 0; mi < o->n_mem; mi++) {
        omem *M = o->mem + mi;
        double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
        for (int n = M->node0; n < M->node0 + M->n_nodes; n++) {
            const double p[3] = {o->x[n], o->y[n], o->z[n]};
            for (int c = 0; c < 3; c++) { lo[c] = fmin(lo[c], p[c]); hi[c] = fmax(hi[c], p[c]); }
        }
        for (int c = 0; c < 3; c++) { lo[c] -= 2 * dh; hi[c] += 2 * dh; }
        for (int i = 1; i < o->nc; i++) {
            const v3 cc = V3(o->cen[3 * i], o->cen[3 * i + 1], o->cen[3 * i + 2]);
            if (!(cc.x >= lo[0] && cc.x <= hi[0] && cc.y >= lo[1] && cc.y <= hi[1] && cc.z >= lo[2] && cc.z <= hi[2]))
                continue;
            const double xb = hi[0];
            const double pc[3] = {cc.x * cc.y - xb * cc.y, cc.x * cc.z - xb * cc.z, cc.x - xb};
            int crossings = 0;
            double md = 1000000000;
            for (int t = M->tri0; t < M->tri0 + M->n_tris; t++) {
                const v3 P[3] = {node(o, o->tri[3 * t]), node(o, o->tri[3 * t + 1]), node(o, o->tri[3 * t + 2])};
                if (!(P[0].x > cc.x && P[1].x > cc.x && P[2].x > cc.x)) continue;
                double side[3];
                for (int e = 0; e < 3; e++) {
                    const v3 a = P[e], b = P[(e + 1) % 3];
                    const double pe[3] = {a.y * b.z - b.y * a.z, a.z - b.z, b.y - a.y};
                    side[e] = pc[0] * pe[1] + pc[1] * pe[2] + pc[2] * pe[0];
                }
                if ((side[0] < 0 && side[1] < 0 && side[2] < 0) || (side[0] > 0 && side[1] > 0 && side[2] > 0)) crossings++;
                for (int e = 0; e < 3; e++) md = fmin(sqrt(vdot(vsub(cc, P[e]), vsub(cc, P[e]))), md);
            }
            const double r = M->d.internal_viscosity_ratio;
            const double fac = 2.0 * fmin(0.5, (md * 0.5 / dh + 1.0 / pi * sin(pi * md / dh) * 0.5));
            const double v = (crossings % 2) ? (r + 1.0) + (r - 1.0) * fac : (r + 1.0) + (1.0 - r) * fac;
            o->visc[i] = v * 0.5;
        }
    }
}

/* -------------------------------------------------------- time step ---- */

static int dynamic_dt(const oracle_case *o) { return o->p.time_stepping != 0 && o->p.time_stepping != LBFS_DT_CONSTANT; }

/* populate_cfl_areas (Solver_gpu.cu:1657-1687): per cell, half the sums of
 * |n_c * area| over its faces in gradient_faces order (the face loop,
 * unstructured_mesh.cpp:1645-1665). */
static void cfl_areas(oracle_case *o) {
    for (int f = 0; f < o->nf; f++) {
        const int cells[2] = {o->owner[f], f < o->ni ? o->neighbour[f] : -1};
        for (int k = 0; k < 2; k++) {
            const int c = cells[k];
            if (c < 0 || c >= o->nc) continue;
            for (int d = 0; d < 3; d++) o->cfl[3 * c + d] = o->cfl[3 * c + d] + fabs(o->normal[3 * f + d] * o->area[f]);
        }
    }
    for (int i = 0; i < 3 * o->nc; i++) o->cfl[i] = o->cfl[i] / 2;
}

/* get_cfl_device (LBFS.cu:2868-2932) per cell, then min<128> + min_block
 * (common_kernels.hpp:147-170, Solver_gpu.cu:57-66, 767-787): the minimum of
 * the per-cell steps and of min<128>'s padding value 1e8. */
static void time_step(oracle_case *o) {
    if (!dynamic_dt(o)) { o->dt = o->p.delta_t; return; }
    const double g = o->p.pre_conditioned_gamma > 0 ? o->p.pre_conditioned_gamma : 1.0 / o->p.gamma_inv;
    const double mv = o->p.max_velocity, factor = o->p.delta_t;
    const double esos = mv * sqrt(1 - g + pow(g / sqrt(3.0) / mv, 2));
    double mn = 100000000.0;
    for (int i = 0; i < o->nc; i++) {
        const double *a = o->cfl + 3 * i;
        double eig = (mv + esos) * a[0] + (mv + esos) * a[1] + (mv + esos) * a[2];
        eig = eig / g;
        double ve = 2 * o->p.visc / g / o->soln[4 * i + 3] / o->vol[i];
        ve = ve * (a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
        eig = eig + 4 * ve;
        o->dtl[i] = factor * o->vol[i] / eig;
        mn = fmin(o->dtl[i], mn);
    }
    o->dt = mn;
    if (o->p.time_stepping == LBFS_DT_MIN)
        for (int i = 0; i < o->nc; i++) o->dtl[i] = mn; /* fill_double (Solver_gpu.cu:781-783) */
}

/* ------------------------------------------------------------- API ---- */

oracle_case *oracle_create(const lbfs_mesh_desc *m, const lbfs_params *p, const lbfs_rbc_desc *rbc, int n_rbc) {
    if (m->n_instances > 1) return NULL; /* one case per oracle object: check ensembles instance by instance */
    oracle_case *o = (oracle_case *)calloc(1, sizeof(oracle_case));
    o->m = *m;
    o->p = *p;
    o->nc = m->n_cells; o->nf = m->n_faces; o->ni = m->n_interior; o->nb = m->n_bc; o->nt = o->nc + o->nb;
    const size_t nf = o->nf, nt = o->nt, nc = o->nc, nb = o->nb;
    o->owner = dup(m->owner, nf * sizeof(int));
    o->neighbour = dup(m->neighbour, nf * sizeof(int));
    o->stencil = dup(m->gradient_stencil, 6 * nc * sizeof(int));
    o->rt = dup(m->bc_rho_type, nb * sizeof(int));
    o->vt = dup(m->bc_vel_type, nb * sizeof(int));
    o->per = dup(m->periodic_node, nb * sizeof(int)); /* zeros when absent */
    o->area = dup(m->face_area, nf * sizeof(double));
    o->normal = dup(m->face_normal, 3 * nf * sizeof(double));
    o->fcen = dup(m->face_centroid, 3 * nf * sizeof(double));
    o->sdt = dup(m->streaming_dt, nf * sizeof(double));
    o->vol = dup(m->cell_volume, nt * sizeof(double));
    o->cen = dup(m->cell_centroid, 3 * nt * sizeof(double));
    o->lhs = dup(m->lhs_inverse, 9 * nc * sizeof(double));
    o->rhs = dup(m->rhs, 18 * nc * sizeof(double));
    o->bcv = dup(m->bc_values, 4 * nb * sizeof(double));
    o->soln = dup(NULL, 4 * nt * sizeof(double));
    o->t1 = dup(NULL, 4 * nc * sizeof(double));
    o->grad = dup(NULL, 12 * nt * sizeof(double));
    o->flux = dup(NULL, 4 * nf * sizeof(double));
    o->res = dup(NULL, 4 * nt * sizeof(double));
    o->force = dup(NULL, 3 * nc * sizeof(double));
    o->visc = (double *)malloc(nc * sizeof(double));
    for (size_t i = 0; i < nc; i++) o->visc[i] = p->visc_factor_initial;
    o->cfl = dup(NULL, 3 * nc * sizeof(double));
    o->dtl = (double *)malloc(nc * sizeof(double));
    for (size_t i = 0; i < nc; i++) o->dtl[i] = p->delta_t;
    o->dt = p->delta_t;
    cfl_areas(o);
    {
        const double *g[3] = {m->grid_x, m->grid_y, m->grid_z};
        for (int a = 0; a < 3; a++) {
            o->gn[a] = (int)(m->length[a] / m->delta_x);
            const long long stride = a == 0 ? 1 : (a == 1 ? o->gn[0] : (long long)o->gn[0] * o->gn[1]);
            o->gv[a] = dup(g[a], g[a] ? (o->gn[a] + 1) * sizeof(double) : 0);
            o->gc[a] = (double *)malloc((o->gn[a] + 1) * sizeof(double));
            for (int i = 0; i < o->gn[a] && i * stride < o->nc; i++) o->gc[a][i] = m->cell_centroid[3 * (i * stride) + a];
        }
    }
    o->n_mem = n_rbc;
    o->mem = (omem *)calloc(n_rbc > 0 ? n_rbc : 1, sizeof(omem));
    for (int r = 0; r < n_rbc; r++) {
        omem *M = o->mem + r;
        M->d = rbc[r];
        M->n_nodes = rbc[r].n_nodes; M->n_tris = rbc[r].n_tris; M->n_springs = rbc[r].n_springs;
        M->node0 = o->N; M->tri0 = o->T; M->spring0 = o->S;
        o->N += M->n_nodes; o->T += M->n_tris; o->S += M->n_springs;
    }
    const size_t N = o->N, T = o->T, S = o->S;
    o->tri = (int *)malloc((3 * T + 1) * sizeof(int));
    o->spr = (int *)malloc((4 * S + 1) * sizeof(int));
    double *d[18];
    for (int k = 0; k < 9; k++) d[k] = dup(NULL, N * sizeof(double));
    o->x = d[0]; o->y = d[1]; o->z = d[2]; o->vx = d[3]; o->vy = d[4]; o->vz = d[5]; o->fx = d[6]; o->fy = d[7]; o->fz = d[8];
    o->contour = dup(NULL, S * sizeof(double)); o->kspr = dup(NULL, S * sizeof(double));
    o->curv = dup(NULL, S * sizeof(double)); o->curv0 = dup(NULL, S * sizeof(double));
    o->ang0 = dup(NULL, S * sizeof(double)); o->area0 = dup(NULL, 2 * S * sizeof(double));
    o->sarea = dup(NULL, 2 * S * sizeof(double));
    for (int r = 0; r < n_rbc; r++) {
        omem *M = o->mem + r;
        for (int i = 0; i < 3 * M->n_tris; i++) o->tri[3 * M->tri0 + i] = rbc[r].tri[i] + M->node0;
        for (int i = 0; i < 4 * M->n_springs; i++) o->spr[4 * M->spring0 + i] = rbc[r].spring[i] + M->node0;
        for (int n = 0; n < M->n_nodes; n++) {
            o->x[M->node0 + n] = rbc[r].xyz_stress_free[3 * n];
            o->y[M->node0 + n] = rbc[r].xyz_stress_free[3 * n + 1];
            o->z[M->node0 + n] = rbc[r].xyz_stress_free[3 * n + 2];
        }
        reference_pass(o, M);
        for (int n = 0; n < M->n_nodes; n++) {
            o->x[M->node0 + n] = rbc[r].xyz_initial[3 * n];
            o->y[M->node0 + n] = rbc[r].xyz_initial[3 * n + 1];
            o->z[M->node0 + n] = rbc[r].xyz_initial[3 * n + 2];
        }
        /* initial pass (Solver_gpu.cu:726-732): V0, A0, angles, areas, MAD0 */
        M->MAD = 0.0;
        M->MAD0 = 0.0;
        triangle_totals(o, M, 1);
        spring_forces(o, M, 1);
        mad(o, M, 1);
    }
    return o;
}

void oracle_free(oracle_case *o) {
    if (!o) return;
    void *ptrs[] = {o->owner, o->neighbour, o->stencil, o->rt, o->vt, o->per, o->area, o->normal, o->fcen, o->sdt, o->vol,
                    o->cen, o->lhs, o->rhs, o->bcv, o->soln, o->t1, o->grad, o->flux, o->res, o->force, o->visc, o->mem,
                    o->tri, o->spr, o->x, o->y, o->z, o->vx, o->vy, o->vz, o->fx, o->fy, o->fz, o->contour, o->kspr,
                    o->curv, o->curv0, o->ang0, o->area0, o->sarea, o->cfl, o->dtl, o->gv[0], o->gv[1],
                    o->gv[2], o->gc[0], o->gc[1], o->gc[2]};
    for (size_t i = 0; i < sizeof(ptrs) / sizeof(ptrs[0]); i++) free(ptrs[i]);
    free(o);
}

void oracle_set_state(oracle_case *o, const double *rho, const double *u, const double *v, const double *w) {
    for (int i = 0; i < o->nc; i++) {
        double *s = o->soln + 4 * i;
        s[0] = u[i]; s[1] = v[i]; s[2] = w[i]; s[3] = rho[i];
        memcpy(o->t1 + 4 * i, s, 4 * sizeof(double)); /* Solver_gpu.cu:746 */
    }
}

void oracle_get_state(const oracle_case *o, double *rho, double *u, double *v, double *w) {
    for (int i = 0; i < o->nc; i++) {
        const double *s = o->soln + 4 * i;
        u[i] = s[0]; v[i] = s[1]; w[i] = s[2]; rho[i] = s[3];
    }
}

/* gpu_solver::check_periodic_object (Solver_gpu.cu:1027-1029, 1277-1304), per
 * periodic membrane: the mean node z as total<128> sums it (256 nodes per
 * block tree-summed, stride 128 down to 1; the block sums added in order
 * from 0), and a move by -0.5 Z when it exceeds origin_z + 0.75 Z. */
static void wrap_nodes(double *z, int n_nodes, double z0, double Z) {
    double sum = 0.0;
    for (int s0 = 0; s0 < n_nodes; s0 += 256) {
        double part[256];
        for (int t = 0; t < 256; t++) part[t] = s0 + t < n_nodes ? z[s0 + t] : 0.0;
        for (int stride = 128; stride >= 1; stride >>= 1)
            for (int t = 0; t < stride; t++) part[t] += part[t + stride];
        sum = sum + part[0];
    }
    if (sum / n_nodes > z0 + 0.75 * Z)
        for (int n = 0; n < n_nodes; n++) z[n] = z[n] + -0.5 * Z;
}

/* LBFS_WRAP_ALL on membrane 0: as the reference (object_z holds every
 * object's nodes), one mean over all membranes' nodes and one move of all. */
static void periodic_wrap(oracle_case *o) {
    const double z0 = o->m.origin[2], Z = o->m.length[2];
    if (o->n_mem > 0 && o->mem[0].d.periodic == LBFS_WRAP_ALL) {
        wrap_nodes(o->z, o->N, z0, Z);
        return;
    }
    for (int r = 0; r < o->n_mem; r++) {
        const omem *M = o->mem + r;
        if (M->d.periodic) wrap_nodes(o->z + M->node0, M->n_nodes, z0, Z);
    }
}

/* One iteration of the time loop, Solver_gpu.cu:749-1046 (one RK stage). */
void oracle_step(oracle_case *o, int n_steps) {
    for (int st = 0; st < n_steps; st++, o->t++) {
        time_step(o);
        const int local = o->p.time_stepping == LBFS_DT_LOCAL;
        if (o->n_mem > 0) interpolate_and_move(o);
        for (int i = 0; i < o->nc; i++)
            for (int c = 0; c < 3; c++) o->force[3 * i + c] = o->p.body_force[c];
        if (o->n_mem > 0) {
            memset(o->fx, 0, o->N * sizeof(double));
            memset(o->fy, 0, o->N * sizeof(double));
            memset(o->fz, 0, o->N * sizeof(double));
            for (int r = 0; r < o->n_mem; r++) {
                triangle_totals(o, o->mem + r, 0);
                spring_forces(o, o->mem + r, 0);
                mad(o, o->mem + r, 0);
            }
            if (o->p.viscosity_period > 0 && o->t % o->p.viscosity_period == 1) interior_viscosity(o);
            spread(o);
        }
        ghost_update(o);
        memset(o->res, 0, 4 * (size_t)o->nt * sizeof(double));
        interior_gradients(o);
        bc_gradients(o);
        if (o->m.axis_aligned) {
            const int nfx = o->m.n_face_x, nfy = o->m.n_face_y;
            for (int f = 0; f < o->ni; f++) axis_face(o, f, f < nfx ? 0 : (f < nfx + nfy ? 1 : 2));
        } else {
            for (int f = 0; f < o->ni; f++) general_face(o, f, 0);
        }
        for (int f = o->ni; f < o->nf; f++) general_face(o, f, 1);
        /* add_face_flux_to_cell (LBFS.cu:2242-2281), face order; res layout rho, u, v, w */
        for (int f = 0; f < o->nf; f++) {
            const int i = o->owner[f], nb = o->neighbour[f];
            const double *F = o->flux + 4 * f;
            const double fl[4] = {F[3], F[0], F[1], F[2]};
            for (int m = 0; m < 4; m++) {
                o->res[4 * i + m] += -fl[m] / o->vol[i];
                if (nb < o->nc) o->res[4 * nb + m] += fl[m] / o->vol[nb];
            }
        }
        double sq[4] = {0, 0, 0, 0};
        for (int i = 0; i < o->nc; i++) {
            double *r = o->res + 4 * i, *t1 = o->t1 + 4 * i, *s = o->soln + 4 * i;
            for (int c = 0; c < 3; c++) r[1 + c] = r[1 + c] + o->force[3 * i + c];
            /* time_integration, last (only) stage (LBFS.cu:2089-2172) */
            const double dtm = local ? o->dtl[i] : o->dt;
            t1[3] = t1[3] + dtm * 1.0 * r[0];
            t1[0] = t1[0] + dtm * 1.0 * r[1];
            t1[1] = t1[1] + dtm * 1.0 * r[2];
            t1[2] = t1[2] + dtm * 1.0 * r[3];
            s[3] = t1[3];
            s[0] = t1[0] / t1[3];
            s[1] = t1[1] / t1[3];
            s[2] = t1[2] / t1[3];
            for (int m = 0; m < 4; m++) sq[m] += r[m] * r[m];
        }
        if (o->n_mem > 0 && o->t % 5000 == 1) periodic_wrap(o);
        const double ref_mom = o->p.ref_rho * o->p.max_velocity;
        for (int m = 0; m < 4; m++) o->resid[m] = sqrt(sq[m] / o->nc) / (m == 0 ? o->p.ref_rho : ref_mom);
    }
}

/* Same layouts as lbfs_get_field / lbfs_get_nodes / lbfs_get_totals / lbfs_get_residuals. */
int oracle_get_field(const oracle_case *o, int which, double *out) {
    switch (which) {
    case LBFS_FIELD_GRADIENTS: memcpy(out, o->grad, 12 * (size_t)o->nt * sizeof(double)); return 0;
    case LBFS_FIELD_FACE_FLUX: memcpy(out, o->flux, 4 * (size_t)o->nf * sizeof(double)); return 0;
    case LBFS_FIELD_RESIDUAL: memcpy(out, o->res, 4 * (size_t)o->nc * sizeof(double)); return 0;
    case LBFS_FIELD_FORCE: memcpy(out, o->force, 3 * (size_t)o->nc * sizeof(double)); return 0;
    case LBFS_FIELD_T1: memcpy(out, o->t1, 4 * (size_t)o->nc * sizeof(double)); return 0;
    case LBFS_FIELD_VISC: memcpy(out, o->visc, (size_t)o->nc * sizeof(double)); return 0;
    case LBFS_FIELD_DT_LOCAL: memcpy(out, o->dtl, (size_t)o->nc * sizeof(double)); return 0;
    case LBFS_FIELD_GHOST: memcpy(out, o->soln + 4 * (size_t)o->nc, 4 * (size_t)o->nb * sizeof(double)); return 0;
    case LBFS_FIELD_SPRING:
        for (int s = 0; s < o->S; s++) {
            double *q = out + 9 * (size_t)s;
            q[0] = o->contour[s]; q[1] = o->kspr[s]; q[2] = o->curv[s]; q[3] = o->curv0[s]; q[4] = o->ang0[s];
            q[5] = o->area0[2 * s]; q[6] = o->area0[2 * s + 1]; q[7] = o->sarea[2 * s]; q[8] = o->sarea[2 * s + 1];
        }
        return 0;
    }
    return 1;
}

void oracle_get_nodes(const oracle_case *o, int which, double *out) {
    const double *src[3];
    if (which == LBFS_NODES_POSITION) { src[0] = o->x; src[1] = o->y; src[2] = o->z; }
    else if (which == LBFS_NODES_VELOCITY) { src[0] = o->vx; src[1] = o->vy; src[2] = o->vz; }
    else { src[0] = o->fx; src[1] = o->fy; src[2] = o->fz; }
    for (int n = 0; n < o->N; n++)
        for (int c = 0; c < 3; c++) out[3 * n + c] = src[c][n];
}

void oracle_get_totals(const oracle_case *o, double *out) {
    for (int r = 0; r < o->n_mem; r++) {
        const omem *M = o->mem + r;
        out[6 * r] = M->V; out[6 * r + 1] = M->V0; out[6 * r + 2] = M->A;
        out[6 * r + 3] = M->A0; out[6 * r + 4] = M->MAD; out[6 * r + 5] = M->MAD0;
    }
}

void oracle_get_residuals(const oracle_case *o, double *out) { memcpy(out, o->resid, 4 * sizeof(double)); }

double oracle_time_step(const oracle_case *o) { return o->dt; }

/* The energy log of Solver_gpu.cu:1060-1136 per membrane: volume, global area,
 * local area, local bending, ADE, spring (WLC) and total energy; the per-spring
 * terms of get_area_energy, get_bending_energy and get_spring_energy
 * (spring_network.cu:1687-1768) summed in spring order. */
void oracle_get_energies(const oracle_case *o, double *out) {
    for (int r = 0; r < o->n_mem; r++) {
        const omem *M = o->mem + r;
        const lbfs_rbc_desc *d = &M->d;
        const double w = 1 / d->wlc_ratio;
        const double c1 = (0.25 / (1 - w) / (1 - w) - 0.25 + w);
        const double c2 = w * w * (3.0 - 2.0 * w) / (1.0 - w) - 4 * c1 * w;
        double la = 0, lb = 0, sp = 0;
        for (int q = 0; q < M->n_springs; q++) {
            const int i = M->spring0 + q;
            const double *a = o->sarea + 2 * (size_t)i, *a0 = o->area0 + 2 * (size_t)i;
            la += d->global_area_modulus * 0.5 *
                  ((a[0] - a0[0]) * (a[0] - a0[0]) / a0[0] + (a[1] - a0[1]) * (a[1] - a0[1]) / a0[1]);
            lb += 0.5 * d->local_bending_modulus * (o->curv[i] - o->curv0[i]) * (o->curv[i] - o->curv0[i]) /
                  o->sarea[i]; /* the reference passes spring_area as the nodal area, indexed by spring */
            const int na = o->spr[4 * i], nc = o->spr[4 * i + 2];
            const double dx = o->x[nc] - o->x[na], dy = o->y[nc] - o->y[na], dz = o->z[nc] - o->z[na];
            const double len = sqrt(dx * dx + dy * dy + dz * dz), sr = len / o->contour[i];
            sp += 0.5 * o->kspr[i] * fabs(0.25 * o->contour[i] * (sr * sr * (3.0 - 2.0 * sr) / (1.0 - sr) - 4 * sr * c1 - c2));
        }
        const double ade = 0.5 * d->global_bending_modulus * (M->MAD - M->MAD0) * (M->MAD - M->MAD0) / M->A0;
        const double vol = 0.5 * d->volume_modulus * (M->V - M->V0) * (M->V - M->V0) / M->V0;
        const double gar = 0.5 * d->global_area_modulus * (M->A - M->A0) * (M->A - M->A0) / M->A0;
        double *e = out + 7 * (size_t)r;
        e[0] = vol; e[1] = gar; e[2] = la; e[3] = lb; e[4] = ade; e[5] = sp;
        e[6] = vol + gar + la + lb + ade + sp;
    }
}
