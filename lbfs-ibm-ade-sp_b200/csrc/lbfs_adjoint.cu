// Discrete adjoint of the FP64 time step (no reference counterpart).
//
// The forward step maps (soln_t1, node positions, MAD) at step n to step n+1:
//   state_n = primitive(t1_n)                       (K3 of the previous step)
//   grad_n  = G(state_n, bc)                        (K1, ghosts included)
//   flux    = Phi(state_n, grad_n, bc)              (K2, per face)
//   t1_{n+1} = t1_n + dt (sum_f +-flux_f / vol + f_ibm + f_body)   (K3)
// plus the membrane chain for the IBM force.  These kernels run the step
// backwards: given the adjoint of t1_{n+1} they form the adjoint of t1_n and
// accumulate the sensitivity to the boundary-velocity scale.  Every sum that
// the forward step forms by gathering is formed here by gathering too (per
// face, then per cell through the cell's face list and through the transposed
// gradient stencil), so the adjoint is deterministic.
//
//   A1 k_adj_flux    one thread per face: recomputes the face's lattice
//                    reconstruction, equilibria and interface flux, then
//                    back-propagates the flux adjoint to the two cells'
//                    states and gradients (and to Dirichlet boundary values).
//   A2 k_adj_cell    one thread per cell: gathers its faces' adjoints, takes
//                    its ghost cells back through the ghost gradients and
//                    states, and forms lambda_R = LHS^-T lambda_grad.
//   A3 k_adj_gather  one thread per cell: the transposed-stencil gather of
//                    lambda_R, the IBM interpolation term, and the primitive
//                    -> conservative transpose into lambda_t1.
#include <cuda_runtime.h>

#include "lbfs_adjoint.h"
#include "lbfs_fluid.cuh"

namespace lbfs {
namespace {

struct Dir3 {
    int ex, ey, ez;
};
__device__ __forceinline__ Dir3 dir3(int k) { return {c_ex(k), c_ey(k), c_ez(k)}; }

// d feq_k / d(rho, u, v, w) of w_k rho (1 + X), X = 3 e.u + 4.5 (e.u)^2 - 1.5 |u|^2
// (FP64 form: rho0 = 0, no preconditioning).
__device__ __forceinline__ void feq_grad(int k, double rho, double u, double v, double w, double (&d)[4]) {
    const int ex = c_ex(k), ey = c_ey(k), ez = c_ez(k);
    const double eu = ex * u + ey * v + ez * w;
    const double X = 3.0 * eu + 4.5 * eu * eu - 1.5 * (u * u + v * v + w * w);
    const double wk = lattice_w<double>(k);
    d[0] = wk * (1.0 + X);
    d[1] = wk * rho * (3.0 * ex + 9.0 * eu * ex - 3.0 * u);
    d[2] = wk * rho * (3.0 * ey + 9.0 * eu * ey - 3.0 * v);
    d[3] = wk * rho * (3.0 * ez + 9.0 * eu * ez - 3.0 * w);
}

// Adjoint of interface_flux (FP64, rho0 = 0, qscale = 1): lo = adjoint of the
// face flux (mass, momentum x, y, z); lfl += adjoint of the 15 reconstructed
// equilibria.  The forward flux is (1 - tau) F_eq(rho, u) + tau F_fl with the
// interface moments rho = sum fl, rho u = sum e fl.
__device__ __forceinline__ void interface_flux_bwd(const double (&fl)[15], double tau, double area, int axis,
                                                   double nx, double ny, double nz, const double (&lo)[4],
                                                   double (&lfl)[15]) {
    double rho = fl[0];
#pragma unroll
    for (int k = 1; k < 15; k++) rho = rho + fl[k];
    double m[3] = {0, 0, 0};
#pragma unroll
    for (int k = 1; k < 15; k++) {
        const Dir3 e = dir3(k);
        m[0] += e.ex * fl[k];
        m[1] += e.ey * fl[k];
        m[2] += e.ez * fl[k];
    }
    const double inv = 1.0 / rho;
    const double u[3] = {inv * m[0], inv * m[1], inv * m[2]};
    const double n[3] = {nx, ny, nz};
    double lF[3][4];
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
        for (int j = 0; j < 4; j++) lF[c][j] = axis >= 0 ? (c == axis ? area * lo[j] : 0.0) : area * n[c] * lo[j];
    // fr = (1 - tau) f + tau fl: the reconstructed populations' share
#pragma unroll
    for (int k = 1; k < 15; k++) {
        const Dir3 e = dir3(k);
        const int ee[3] = {e.ex, e.ey, e.ez};
        if (axis >= 0 && !ee[axis]) continue;
        double lfr = 0.0;
#pragma unroll
        for (int c = 0; c < 3; c++) {
            if (axis >= 0 && c != axis) continue;
            if (!ee[c]) continue;
            double t = lF[c][0];
#pragma unroll
            for (int q = 0; q < 3; q++)
                if (ee[q]) t += ee[q] * lF[c][1 + q];
            lfr += ee[c] * t;
        }
        lfl[k] += tau * lfr;
    }
    // the equilibrium's share, through the closed-form moments the forward
    // kernel forms (rho u_c and rho (u_c u_m + d_cm / 3)), not 14 equilibria
    const double keep = 1.0 - tau;
    double lrho = 0.0, lu[3] = {0, 0, 0};
#pragma unroll
    for (int c = 0; c < 3; c++) {
        if (axis >= 0 && c != axis) continue;
        lrho += lF[c][0] * u[c];
        lu[c] += rho * lF[c][0];
#pragma unroll
        for (int q = 0; q < 3; q++) {
            lrho += lF[c][1 + q] * (u[c] * u[q] + (q == c ? 1.0 / 3.0 : 0.0));
            lu[c] += rho * lF[c][1 + q] * u[q];
            lu[q] += rho * lF[c][1 + q] * u[c];
        }
    }
    lrho *= keep;
#pragma unroll
    for (int c = 0; c < 3; c++) lu[c] *= keep;
    // u = m / rho
    const double lm[3] = {lu[0] * inv, lu[1] * inv, lu[2] * inv};
    lrho -= (lu[0] * u[0] + lu[1] * u[1] + lu[2] * u[2]) * inv;
#pragma unroll
    for (int k = 0; k < 15; k++) {
        const Dir3 e = dir3(k);
        lfl[k] += lrho + e.ex * lm[0] + e.ey * lm[1] + e.ez * lm[2];
    }
}

// 12 consecutive doubles (16-B aligned) as six vector loads through the
// read-only path (the array is not written while the kernel runs).
__device__ __forceinline__ void load12(const double *p, double (&g)[12]) {
    const double2 *q = reinterpret_cast<const double2 *>(p);
#pragma unroll
    for (int t = 0; t < 6; t++) {
        const double2 v = __ldg(q + t);
        g[2 * t] = v.x;
        g[2 * t + 1] = v.y;
    }
}
__device__ __forceinline__ void load4(const double *p, double (&g)[4]) {
    const double2 *q = reinterpret_cast<const double2 *>(p);
    const double2 v0 = __ldg(q), v1 = __ldg(q + 1);
    g[0] = v0.x; g[1] = v0.y; g[2] = v1.x; g[3] = v1.y;
}

// Face adjoint record: lambda of owner state (rho, u, v, w), neighbour state,
// owner gradient (12), neighbour gradient (12).
struct FaceAdj {
    double s1[4], s2[4], g1[12], g2[12];
};

// One side of a face record: lambda of the side's state (4) and gradient (12),
// 128 contiguous bytes; the owner sides of all faces, then the neighbour
// sides, so that the per-cell gather (A2) reads whole records of neighbouring
// faces.
__device__ __forceinline__ double *face_side(const AdjointArgs &j, int f, int side) {
    return j.lam_face + 16 * ((size_t)side * j.nf + f);
}
__device__ __forceinline__ void store_face_side(const AdjointArgs &j, int f, int side, const double (&ls)[4],
                                                const double (&lg)[12]) {
    double2 *o = reinterpret_cast<double2 *>(face_side(j, f, side));
    o[0] = make_double2(ls[0], ls[1]);
    o[1] = make_double2(ls[2], ls[3]);
#pragma unroll
    for (int t = 0; t < 6; t++) o[2 + t] = make_double2(lg[2 * t], lg[2 * t + 1]);
}

// Axis-aligned interior face (axis_face_flux of the forward kernel): writes
// the face's adjoint record.
template <int axis>
__device__ __forceinline__ void axis_face_bwd(const FluidArgs<double> &a, const AdjointArgs &j, int f,
                                              const double (&lo)[4]) {
    const int2 oc = __ldg(a.face_cells + f);
    AxisFace<double> geo;
    if (a.axis_uniform) geo = {a.axis_geo[axis][0], a.axis_geo[axis][1], a.axis_geo[axis][2], a.axis_geo[axis][3]};
    else geo = a.axis_face[f];
    const Vec4<double> s1 = a.state[oc.x], s2 = a.state[oc.y];
    double g1[12], g2[12];
    load12(a.grad + 12 * (size_t)oc.x, g1);
    load12(a.grad + 12 * (size_t)oc.y, g2);
    const double dt = geo.dt, t1 = geo.t1, t2 = geo.t2;
    const double c = t2 - t1;
    const double wa = fabs(t2 / c), wb = fabs(t1 / c);
    const double S1[4] = {s1.rho, s1.u, s1.v, s1.w}, S2[4] = {s2.rho, s2.u, s2.v, s2.w};
    double pi[4], pn[4], p0[4];
#pragma unroll
    for (int m = 0; m < 4; m++) {
        pi[m] = S1[m] - t1 * g1[3 * m + axis];
        pn[m] = S2[m] - (t2 * g2[3 * m + axis]);
        p0[m] = (pi[m] + pn[m]) * 0.5;
    }
    constexpr int ob = axis == 0 ? 1 : 0;
    constexpr int oc2 = axis == 2 ? 1 : 2;
    // lattice value L[m] of direction k
    auto recon = [&](int k, double (&L)[4]) {
        const Dir3 e = dir3(k);
        const int ee[3] = {e.ex, e.ey, e.ez};
#pragma unroll
        for (int m = 0; m < 4; m++) {
            double val;
            if (ee[axis] > 0) {
                val = pi[m] - g1[3 * m + axis] * dt;
                if (ee[ob]) val = (ee[ob] > 0) ? val - g1[3 * m + ob] * dt : val + g1[3 * m + ob] * dt;
                if (ee[oc2]) val = (ee[oc2] > 0) ? val - g1[3 * m + oc2] * dt : val + g1[3 * m + oc2] * dt;
            } else if (ee[axis] < 0) {
                val = pn[m] + g2[3 * m + axis] * dt;
                if (ee[ob]) val = (ee[ob] > 0) ? val - g2[3 * m + ob] * dt : val + g2[3 * m + ob] * dt;
                if (ee[oc2]) val = (ee[oc2] > 0) ? val - g2[3 * m + oc2] * dt : val + g2[3 * m + oc2] * dt;
            } else {
                val = p0[m];
                if (ee[ob]) {
                    const double gi = g1[3 * m + ob] * wa + g2[3 * m + ob] * wb;
                    val = (ee[ob] > 0) ? val - gi * dt : val + gi * dt;
                }
                if (ee[oc2]) {
                    const double gi = g1[3 * m + oc2] * wa + g2[3 * m + oc2] * wb;
                    val = (ee[oc2] > 0) ? val - gi * dt : val + gi * dt;
                }
            }
            L[m] = val;
        }
    };
    double fl[15];
#pragma unroll
    for (int k = 0; k < 15; k++) {
        double L[4];
        recon(k, L);
        fl[k] = feq_dev<double>(k, L[0], L[1], L[2], L[3], 0.0, 1.0);
    }
    const double vf = a.visc_factor[oc.x];
    const double tau = (a.testcase == 8) ? 0.0 : (a.visc * vf * 3.0 / dt * a.gamma_inv);
    double lfl[15];
#pragma unroll
    for (int k = 0; k < 15; k++) lfl[k] = 0.0;
    interface_flux_bwd(fl, tau, geo.area, axis, 0, 0, 0, lo, lfl);
    // Reconstruction backward, one side at a time so that only one side's
    // outputs are live: the centre directions (e_axis = 0, lattice value from
    // p0 and the distance-weighted gradients) first, then the owner's
    // directions (stored), then the neighbour's (stored).  The lattice values
    // are recomputed here rather than kept from the forward pass (60 values):
    // the empty asm statements hide that the inputs are unchanged.
#pragma unroll
    for (int t = 0; t < 12; t++) {
        asm volatile("" : "+d"(g1[t]));
        asm volatile("" : "+d"(g2[t]));
    }
#pragma unroll
    for (int m = 0; m < 4; m++) {
        asm volatile("" : "+d"(pi[m]));
        asm volatile("" : "+d"(pn[m]));
        asm volatile("" : "+d"(p0[m]));
    }
    double lp0[4] = {0, 0, 0, 0}, lgc[12];  // lgc[3 m + c] = sum_k e_c lL_k[m] over the centre directions
#pragma unroll
    for (int t = 0; t < 12; t++) lgc[t] = 0.0;
#pragma unroll
    for (int k = 0; k < 15; k++) {
        const Dir3 e = dir3(k);
        const int ee[3] = {e.ex, e.ey, e.ez};
        if (ee[axis] != 0) continue;
        double L[4], d[4];
        recon(k, L);
        feq_grad(k, L[0], L[1], L[2], L[3], d);
#pragma unroll
        for (int m = 0; m < 4; m++) {
            const double lL = lfl[k] * d[m];
            lp0[m] += lL;
            if (ee[ob]) lgc[3 * m + ob] += ee[ob] * lL;
            if (ee[oc2]) lgc[3 * m + oc2] += ee[oc2] * lL;
        }
    }
#pragma unroll
    for (int side = 0; side < 2; side++) {
        const int sgn = side == 0 ? 1 : -1;  // the side's upwind directions have e_axis = sgn
        const double wside = side == 0 ? wa : wb, tside = side == 0 ? t1 : t2;
        double lp[4] = {0, 0, 0, 0}, lg[12];
#pragma unroll
        for (int t = 0; t < 12; t++) lg[t] = 0.0;
#pragma unroll
        for (int k = 1; k < 15; k++) {
            const Dir3 e = dir3(k);
            const int ee[3] = {e.ex, e.ey, e.ez};
            if (ee[axis] != sgn) continue;
            double L[4], d[4];
            recon(k, L);
            feq_grad(k, L[0], L[1], L[2], L[3], d);
#pragma unroll
            for (int m = 0; m < 4; m++) {
                const double lL = lfl[k] * d[m];
                lp[m] += lL;
                if (sgn > 0) lg[3 * m + axis] -= lL * dt;
                else lg[3 * m + axis] += lL * dt;
                if (ee[ob]) lg[3 * m + ob] -= ee[ob] * lL * dt;
                if (ee[oc2]) lg[3 * m + oc2] -= ee[oc2] * lL * dt;
            }
        }
#pragma unroll
        for (int m = 0; m < 4; m++) {
            lp[m] += 0.5 * lp0[m];
            lg[3 * m + ob] -= lgc[3 * m + ob] * wside * dt;
            lg[3 * m + oc2] -= lgc[3 * m + oc2] * wside * dt;
            lg[3 * m + axis] -= tside * lp[m];
        }
        store_face_side(j, f, side, lp, lg);
    }
}

// General-normal face (general_face_flux of the forward kernel); boundary
// faces that take the boundary branch also return the adjoint of their
// Dirichlet boundary values in lbc.
__device__ __forceinline__ void general_face_bwd(const FluidArgs<double> &a, int f, bool is_bc, const double (&lo)[4],
                                                 FaceAdj &out, double (&lbc)[4]) {
    const int2 oc = __ldg(a.face_cells + f);
    const GenFace<double> geo = a.gen_face[a.axis_aligned ? f - a.ni : f];
    const Vec4<double> s1 = a.state[oc.x], s2 = a.state[oc.y];
    double g1[12], g2[12];
    load12(a.grad + 12 * (size_t)oc.x, g1);
    load12(a.grad + 12 * (size_t)oc.y, g2);
    const double dt = geo.dt;
    const double S1[4] = {s1.rho, s1.u, s1.v, s1.w}, S2[4] = {s2.rho, s2.u, s2.v, s2.w};
    const double t1v[3] = {geo.t1x, geo.t1y, geo.t1z}, t2v[3] = {geo.t2x, geo.t2y, geo.t2z};
    const bool bcb = geo.bc_branch != 0.0;
    double pi[4], pn[4], p0[4], g3[12];
    bool dir[4] = {false, false, false, false};
    double bcv[4] = {0, 0, 0, 0};
    if (bcb) {
        const int b = oc.y - a.nc;
        const Vec4<double> bc = a.bc_val[b];
        const bool rd = a.bc_rho_type[b] == 1, vd = a.bc_vel_type[b] == 1;
        bcv[0] = bc.rho; bcv[1] = bc.u; bcv[2] = bc.v; bcv[3] = bc.w;
#pragma unroll
        for (int m = 0; m < 4; m++) {
            dir[m] = (m == 0) ? rd : vd;
            p0[m] = dir[m] ? bcv[m] : S1[m] - (t1v[0] * g2[3 * m] + t1v[1] * g2[3 * m + 1] + t1v[2] * g2[3 * m + 2]);
            pi[m] = p0[m];
            pn[m] = p0[m];
        }
#pragma unroll
        for (int t = 0; t < 12; t++) { g3[t] = g2[t]; g1[t] = g2[t]; }
    } else {
#pragma unroll
        for (int m = 0; m < 4; m++) {
            pi[m] = S1[m] - (t1v[0] * g1[3 * m] + t1v[1] * g1[3 * m + 1] + t1v[2] * g1[3 * m + 2]);
            pn[m] = S2[m] - (t2v[0] * g2[3 * m] + t2v[1] * g2[3 * m + 1] + t2v[2] * g2[3 * m + 2]);
            p0[m] = (pi[m] + pn[m]) * 0.5;
        }
#pragma unroll
        for (int t = 0; t < 12; t++) g3[t] = (g1[t] + g2[t]) * 0.5;
    }
    const double thr = 0.001 * dt;
    const double nrm[3] = {geo.nx, geo.ny, geo.nz};
    // side of direction kk: 0 owner, 1 neighbour, 2 centre
    auto side_of = [&](int kk) {
        if (kk == 0) return 2;
        const int k = (kk & 1) ? kk : kk - 1;
        const Dir3 e = dir3(k);
        const double s = (k < 7) ? (e.ex ? nrm[0] : (e.ey ? nrm[1] : nrm[2]))
                                 : (double(e.ex) * nrm[0] + double(e.ey) * nrm[1] + double(e.ez) * nrm[2]);
        const int side_k = (s > thr) ? 0 : ((s < -thr) ? 1 : 2);
        if (kk == k) return side_k;
        return side_k == 2 ? 2 : 1 - side_k;
    };
    auto recon = [&](int kk, int side, double (&L)[4]) {
        const Dir3 e = dir3(kk);
        const int ee[3] = {e.ex, e.ey, e.ez};
#pragma unroll
        for (int m = 0; m < 4; m++) {
            double val = side == 0 ? pi[m] : (side == 1 ? pn[m] : p0[m]);
#pragma unroll
            for (int d = 0; d < 3; d++) {
                if (!ee[d]) continue;
                const double gd = side == 0 ? g1[3 * m + d] : (side == 1 ? g2[3 * m + d] : g3[3 * m + d]);
                val = (ee[d] > 0) ? val - gd * dt : val + gd * dt;
            }
            L[m] = val;
        }
    };
    double fl[15];
    fl[0] = feq_dev<double>(0, p0[0], p0[1], p0[2], p0[3], 0.0, 1.0);
#pragma unroll
    for (int kk = 1; kk < 15; kk++) {
        double L[4];
        recon(kk, side_of(kk), L);
        fl[kk] = feq_dev<double>(kk, L[0], L[1], L[2], L[3], 0.0, 1.0);
    }
    const double vf = is_bc ? 1.0 : a.visc_factor[oc.x];
    const double tau = (a.testcase == 8) ? 0.0 : (a.visc * vf * 3.0 / dt * a.gamma_inv);
    double lfl[15];
#pragma unroll
    for (int k = 0; k < 15; k++) lfl[k] = 0.0;
    interface_flux_bwd(fl, tau, geo.area, -1, geo.nx, geo.ny, geo.nz, lo, lfl);
    double lpi[4] = {0, 0, 0, 0}, lpn[4] = {0, 0, 0, 0}, lp0[4] = {0, 0, 0, 0};
    double lg1[12], lg2[12], lg3[12];
#pragma unroll
    for (int t = 0; t < 12; t++) { lg1[t] = 0.0; lg2[t] = 0.0; lg3[t] = 0.0; }
    {
        double d[4];
        feq_grad(0, p0[0], p0[1], p0[2], p0[3], d);
#pragma unroll
        for (int m = 0; m < 4; m++) lp0[m] += lfl[0] * d[m];
    }
#pragma unroll
    for (int kk = 1; kk < 15; kk++) {
        const int side = side_of(kk);
        double L[4], d[4];
        recon(kk, side, L);
        feq_grad(kk, L[0], L[1], L[2], L[3], d);
        const Dir3 e = dir3(kk);
        const int ee[3] = {e.ex, e.ey, e.ez};
#pragma unroll
        for (int m = 0; m < 4; m++) {
            const double lL = lfl[kk] * d[m];
            // branches instead of a selected pointer keep the arrays in registers
            if (side == 0) {
                lpi[m] += lL;
#pragma unroll
                for (int q = 0; q < 3; q++)
                    if (ee[q]) lg1[3 * m + q] -= ee[q] * lL * dt;
            } else if (side == 1) {
                lpn[m] += lL;
#pragma unroll
                for (int q = 0; q < 3; q++)
                    if (ee[q]) lg2[3 * m + q] -= ee[q] * lL * dt;
            } else {
                lp0[m] += lL;
#pragma unroll
                for (int q = 0; q < 3; q++)
                    if (ee[q]) lg3[3 * m + q] -= ee[q] * lL * dt;
            }
        }
    }
#pragma unroll
    for (int m = 0; m < 4; m++) { out.s1[m] = 0.0; out.s2[m] = 0.0; lbc[m] = 0.0; }
    if (bcb) {
#pragma unroll
        for (int t = 0; t < 12; t++) { out.g1[t] = 0.0; out.g2[t] = lg1[t] + lg2[t] + lg3[t]; }
#pragma unroll
        for (int m = 0; m < 4; m++) {
            const double lp = lpi[m] + lpn[m] + lp0[m];
            if (dir[m]) {
                lbc[m] = lp;
            } else {
                out.s1[m] = lp;
#pragma unroll
                for (int q = 0; q < 3; q++) out.g2[3 * m + q] -= t1v[q] * lp;
            }
        }
    } else {
#pragma unroll
        for (int t = 0; t < 12; t++) {
            out.g1[t] = lg1[t] + 0.5 * lg3[t];
            out.g2[t] = lg2[t] + 0.5 * lg3[t];
        }
#pragma unroll
        for (int m = 0; m < 4; m++) {
            lpi[m] += 0.5 * lp0[m];
            lpn[m] += 0.5 * lp0[m];
            out.s1[m] = lpi[m];
            out.s2[m] = lpn[m];
#pragma unroll
            for (int q = 0; q < 3; q++) {
                out.g1[3 * m + q] -= t1v[q] * lpi[m];
                out.g2[3 * m + q] -= t2v[q] * lpn[m];
            }
        }
    }
}

// Adjoint of the face flux (mass, mom x, y, z) from the cells' t1 adjoints:
// K3 adds -flux / vol_owner and +flux / vol_neighbour, times dt.
__device__ __forceinline__ void face_flux_adjoint(const FluidArgs<double> &a, const AdjointArgs &j, int f,
                                                  double (&lo)[4]) {
    const int2 oc = __ldg(a.face_cells + f);
    const double4 lo_t = j.lam_t1[oc.x];
    const double vo = a.cell_volume[oc.x];
    lo[0] = -j.dt * lo_t.w / vo;
    lo[1] = -j.dt * lo_t.x / vo;
    lo[2] = -j.dt * lo_t.y / vo;
    lo[3] = -j.dt * lo_t.z / vo;
    if (f < a.ni) {
        const double4 ln = j.lam_t1[oc.y];
        const double vn = a.cell_volume[oc.y];
        lo[0] += j.dt * ln.w / vn;
        lo[1] += j.dt * ln.x / vn;
        lo[2] += j.dt * ln.y / vn;
        lo[3] += j.dt * ln.z / vn;
    }
}

__device__ __forceinline__ void store_face(const AdjointArgs &j, int f, const FaceAdj &r) {
    store_face_side(j, f, 0, r.s1, r.g1);
    store_face_side(j, f, 1, r.s2, r.g2);
}

__global__ void __launch_bounds__(128, 3) k_adj_flux_axis(FluidArgs<double> a, AdjointArgs j) {
    pdl_trigger();
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= a.ni) return;
    double lo[4];
    face_flux_adjoint(a, j, f, lo);
    if (f < a.nfx) axis_face_bwd<0>(a, j, f, lo);
    else if (f < a.nfx + a.nfy) axis_face_bwd<1>(a, j, f, lo);
    else axis_face_bwd<2>(a, j, f, lo);
}

// A1 over the forward step's face tiles (k_face_flux_tiles): block b takes the x, y and z faces owned
// by the cells of tile tile0 + b, so the tile's cells are read once for the three axes.  Each face's
// adjoint is written to that face's own records, so the results do not depend on the mapping.
template <int TB>
__global__ void __launch_bounds__(TB, 384 / TB) k_adj_flux_axis_tiles(FluidArgs<double> a, AdjointArgs j) {
    pdl_trigger();
    const int *tp = a.flux_tiles + 3 * (int)blockIdx.x;
    const int f0x = __ldg(tp), f0y = __ldg(tp + 1), f0z = __ldg(tp + 2);
    const int f1x = __ldg(tp + 3), f1y = __ldg(tp + 4), f1z = __ldg(tp + 5);
    double lo[4];
    for (int f = f0x + (int)threadIdx.x; f < f1x; f += TB) {
        face_flux_adjoint(a, j, f, lo);
        axis_face_bwd<0>(a, j, f, lo);
    }
    for (int f = f0y + (int)threadIdx.x; f < f1y; f += TB) {
        face_flux_adjoint(a, j, f, lo);
        axis_face_bwd<1>(a, j, f, lo);
    }
    for (int f = f0z + (int)threadIdx.x; f < f1z; f += TB) {
        face_flux_adjoint(a, j, f, lo);
        axis_face_bwd<2>(a, j, f, lo);
    }
}

__global__ void __launch_bounds__(128) k_adj_flux_general(FluidArgs<double> a, AdjointArgs j, int first) {
    const int f = first + blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= a.nf) return;
    double lo[4], lbc[4];
    face_flux_adjoint(a, j, f, lo);
    FaceAdj r;
    general_face_bwd(a, f, f >= a.ni, lo, r, lbc);
    store_face(j, f, r);
    if (f >= a.ni) {
        double *o = j.lam_bcv + 4 * (size_t)(f - a.ni);
#pragma unroll
        for (int m = 0; m < 4; m++) o[m] = lbc[m];
    }
}

// RHS vector k, component c, of a mesh with coded least-squares geometry (selects: k is not a
// compile-time index into the parameter table)
__device__ __forceinline__ double rhs_of(const FluidArgs<double> &a, unsigned k, int c) {
    double v = a.ls_rhs_tab[0][c];
#pragma unroll
    for (unsigned t = 1; t < 8; t++) v = (k == t) ? a.ls_rhs_tab[t][c] : v;
    return v;
}

// A2: per cell.  lambda of the cell's state and gradient from its faces; its
// ghost cells (boundary faces) back through the ghost gradient and the ghost
// state; lambda_R = LHS^-T lambda_grad for the stencil; the self term of the
// stencil differences and the ghost stencil entries.  The sensitivity to the
// boundary-velocity scale sigma (every boundary velocity value times sigma)
// is added to sigma_acc[cell].
__global__ void __launch_bounds__(128, 4) k_adj_cell(FluidArgs<double> a, AdjointArgs j) {
    pdl_trigger();
    pdl_wait();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.nc) return;
    double ls[4] = {0, 0, 0, 0}, lg[12];
#pragma unroll
    for (int t = 0; t < 12; t++) lg[t] = 0.0;
    int cf[6];
    if (a.grid_faces) {  // the structured mesh's faces in the table's order, formed
        grid_cell_faces(i, a.grid_n[0], a.grid_n[1], a.grid_n[2], cf);
    } else {
#pragma unroll
        for (int q = 0; q < 3; q++) {
            const int2 p = __ldg(reinterpret_cast<const int2 *>(a.cell_faces) + 3 * i + q);
            cf[2 * q] = p.x;
            cf[2 * q + 1] = p.y;
        }
    }
#pragma unroll
    for (int q = 0; q < 6; q++) {
        const int e = cf[q];
        const int f = (e > 0 ? e : -e) - 1;
        const double *r = face_side(j, f, e > 0 ? 0 : 1);
        double rs[4], rg[12];
        load4(r, rs);
        load12(r + 4, rg);
#pragma unroll
        for (int m = 0; m < 4; m++) ls[m] += rs[m];
#pragma unroll
        for (int t = 0; t < 12; t++) lg[t] += rg[t];
    }
    const Vec4<double> own = a.state[i];
    const double O[4] = {own.rho, own.u, own.v, own.w};
    int st[6];
#pragma unroll
    for (int q = 0; q < 3; q++) {
        const int2 p = a.stencil[3 * i + q];
        st[2 * q] = p.x;
        st[2 * q + 1] = p.y;
    }
    // ghosts: lambda of the ghost state collected here, then taken back to own
    double lgs[6][4];
    double sigma = 0.0;
#pragma unroll
    for (int q = 0; q < 6; q++)
#pragma unroll
        for (int m = 0; m < 4; m++) lgs[q][m] = 0.0;
#pragma unroll
    for (int q = 0; q < 6; q++) {
        const int g = st[q];
        if (g < a.nc) continue;
        const int b = g - a.nc;
        const int f = a.ni + b;
        const double *r = face_side(j, f, 1);  // the boundary face's ghost side (owner i, neighbour = ghost)
        const double *lbc = j.lam_bcv + 4 * (size_t)b;
        // Dirichlet boundary values seen by the face reconstruction
        const Vec4<double> bc = a.bc_val[b];
        sigma += lbc[1] * bc.u + lbc[2] * bc.v + lbc[3] * bc.w;
        const Vec4<double> gs = a.state[g];
        const double G[4] = {gs.rho, gs.u, gs.v, gs.w};
        const BcRec<double> br = a.bc_rec[b];
        const bool dir_rho = a.bc_rho_type[b] == 1, dir_vel = a.bc_vel_type[b] != 2;
#pragma unroll
        for (int m = 0; m < 4; m++) lgs[q][m] += r[m];
        // ghost gradient (get_bc_gradients)
#pragma unroll
        for (int m = 0; m < 4; m++) {
            const double *lgg = r + 4 + 3 * m;
            const bool dirichlet = (m == 0) ? dir_rho : dir_vel;
            if (dirichlet) {
                const double ld = (lgg[0] * br.dnx + lgg[1] * br.dny + lgg[2] * br.dnz) / br.dmag;
                lgs[q][m] += ld;
                ls[m] -= ld;
            } else {
                lg[3 * m + 0] += lgg[0] * br.mx;
                lg[3 * m + 1] += lgg[1] * br.my;
                lg[3 * m + 2] += lgg[2] * br.mz;
            }
        }
        (void)G;
    }
    // lambda_R[m][col] = sum_row LHS[row][col] lambda_grad[m][row]
    LsRec<double> L;
    if (a.ls_coded) {  // one LHS^-1, RHS vectors by the cell's codes
        const unsigned code = __ldg(a.lsw_code + i);
#pragma unroll
        for (int t = 0; t < 9; t++) L.lhs[t] = a.ls_lhs[t];
#pragma unroll
        for (int q = 0; q < 6; q++) {
            const unsigned k = (code >> (3 * q)) & 7u;
#pragma unroll
            for (int c = 0; c < 3; c++) L.rhs[3 * q + c] = rhs_of(a, k, c);
        }
    } else {
        L = a.ls[i];
    }
    double lr[12];
#pragma unroll
    for (int m = 0; m < 4; m++)
#pragma unroll
        for (int col = 0; col < 3; col++)
            lr[3 * m + col] = L.lhs[col] * lg[3 * m] + L.lhs[3 + col] * lg[3 * m + 1] + L.lhs[6 + col] * lg[3 * m + 2];
    double *o = j.lam_rs + 12 * (size_t)i;
#pragma unroll
    for (int t = 0; t < 12; t++) o[t] = lr[t];
    // stencil differences s_j - s_i: self part, and the ghost entries
#pragma unroll
    for (int q = 0; q < 6; q++) {
#pragma unroll
        for (int m = 0; m < 4; m++) {
            const double mu = L.rhs[3 * q] * lr[3 * m] + L.rhs[3 * q + 1] * lr[3 * m + 1] + L.rhs[3 * q + 2] * lr[3 * m + 2];
            ls[m] -= mu;
            if (st[q] >= a.nc) lgs[q][m] += mu;
        }
    }
    // ghost state (update_unstructured_bcs) back to the owner and the boundary values
#pragma unroll
    for (int q = 0; q < 6; q++) {
        const int g = st[q];
        if (g < a.nc) continue;
        const int b = g - a.nc;
        const Vec4<double> bc = a.bc_val[b];
        if (a.bc_rho_type[b] == 1) ls[0] -= lgs[q][0];
        else ls[0] += lgs[q][0];
        const int vt = a.bc_vel_type[b];
        if (vt == 2) {
            ls[1] += lgs[q][1]; ls[2] += lgs[q][2]; ls[3] += lgs[q][3];
        } else {
            ls[1] -= lgs[q][1]; ls[2] -= lgs[q][2]; ls[3] -= lgs[q][3];
            // g.u = 2 ut - own.u with ut linear in bc.u; g.v = 2 bc.v - own.v; g.w = 2 bc.w - own.w
            const double ut = (vt == 9) ? 16 * bc.u * (a.H2 + a.bc_rec[b].gy) * (a.H2 - a.bc_rec[b].gy) *
                                              (a.H2 + a.bc_rec[b].gz) * (a.H2 - a.bc_rec[b].gz) / a.H4
                                        : ((vt == 10) ? a.bc_rec[b].gy * bc.u : bc.u);
            sigma += 2.0 * lgs[q][1] * ut + 2.0 * lgs[q][2] * bc.v + 2.0 * lgs[q][3] * bc.w;
        }
    }
    double *so = j.lam_state + 4 * (size_t)i;
#pragma unroll
    for (int m = 0; m < 4; m++) so[m] = ls[m];
    j.sigma_acc[i] += sigma;
    (void)O;
}

// A3: per cell.  lambda_state += transposed-stencil gather of lambda_R and the
// IBM interpolation term; lambda_t1 += d primitive / d t1 ^T lambda_state.
__global__ void __launch_bounds__(128) k_adj_gather(FluidArgs<double> a, AdjointArgs j) {
    pdl_wait();
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= a.nc) return;
    double ls[4];
#pragma unroll
    for (int m = 0; m < 4; m++) ls[m] = j.lam_state[4 * (size_t)c + m];
    for (int e = j.tst_start[c]; e < j.tst_start[c + 1]; e++) {
        const int code = j.tst[e];
        const int i = code >> 3, q = code & 7;
        double r[3];
        if (a.ls_coded) {
            const unsigned k = (__ldg(a.lsw_code + i) >> (3 * q)) & 7u;
#pragma unroll
            for (int c = 0; c < 3; c++) r[c] = rhs_of(a, k, c);
        } else {
            const double *rr = a.ls[i].rhs + 3 * q;
            r[0] = rr[0]; r[1] = rr[1]; r[2] = rr[2];
        }
        double lr[12];
        load12(j.lam_rs + 12 * (size_t)i, lr);
#pragma unroll
        for (int m = 0; m < 4; m++) ls[m] += r[0] * lr[3 * m] + r[1] * lr[3 * m + 1] + r[2] * lr[3 * m + 2];
    }
    if (j.lam_u_ibm) {
        ls[1] += j.lam_u_ibm[3 * (size_t)c];
        ls[2] += j.lam_u_ibm[3 * (size_t)c + 1];
        ls[3] += j.lam_u_ibm[3 * (size_t)c + 2];
    }
    // state = (t1.w, t1.x / t1.w, t1.y / t1.w, t1.z / t1.w)
    const double4 t = a.t1[c];
    const double inv = 1.0 / t.w;
    const double u = t.x * inv, v = t.y * inv, w = t.z * inv;
    double4 l = j.lam_t1[c];
    l.x += ls[1] * inv;
    l.y += ls[2] * inv;
    l.z += ls[3] * inv;
    l.w += ls[0] - (ls[1] * u + ls[2] * v + ls[3] * w) * inv;
    j.lam_t1[c] = l;
}

// state = primitive(t1), as K3 forms it (FP64 form, rho0 = 0).
__global__ void k_adj_prim(FluidArgs<double> a) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= a.nc) return;
    const double4 t = a.t1[c];
    Vec4<double> s;
    s.rho = t.w;
    s.u = t.x / t.w;
    s.v = t.y / t.w;
    s.w = t.z / t.w;
    a.state[c] = s;
}

// lambda_t1 of the final step for J = sum_c w_c . u_c (velocity objective).
__global__ void k_adj_velocity_seed(FluidArgs<double> a, AdjointArgs j, const double *weights) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= a.nc) return;
    const double4 t = a.t1[c];
    const double inv = 1.0 / t.w;
    const double u = t.x * inv, v = t.y * inv, w = t.z * inv;
    const double wx = weights[3 * (size_t)c], wy = weights[3 * (size_t)c + 1], wz = weights[3 * (size_t)c + 2];
    double4 l = j.lam_t1[c];
    l.x += wx * inv;
    l.y += wy * inv;
    l.z += wz * inv;
    l.w += -(wx * u + wy * v + wz * w) * inv;
    j.lam_t1[c] = l;
}

}  // namespace

namespace {
__global__ void __launch_bounds__(256) k_copy_list(CopyList l) {
    const int q = blockIdx.y;
    const double *src = l.src[q];
    double *dst = l.dst[q];
    const long long n = l.n[q];
    const int stride = l.src_stride[q];
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        dst[i] = src[i * stride];
}
}  // namespace

void launch_copy_list(const CopyList &l, cudaStream_t s) {
    if (l.count <= 0) return;
    long long most = 0;
    for (int q = 0; q < l.count; q++) most = l.n[q] > most ? l.n[q] : most;
    const int bx = (int)((most + 255) / 256 < 296 ? (most + 255) / 256 : 296);
    k_copy_list<<<dim3(bx, l.count), 256, 0, s>>>(l);
}

void launch_adj_prim(const FluidArgs<double> &a, cudaStream_t s) {
    k_adj_prim<<<(a.nc + 255) / 256, 256, 0, s>>>(a);
}

void launch_adj_velocity_seed(const FluidArgs<double> &a, const AdjointArgs &j, const double *weights, cudaStream_t s) {
    k_adj_velocity_seed<<<(a.nc + 255) / 256, 256, 0, s>>>(a, j, weights);
}

void launch_adj_flux_axis(const FluidArgs<double> &a, const AdjointArgs &j, cudaStream_t s) {
    if (!a.axis_aligned || a.ni == 0) return;
    if (a.flux_tiles && a.n_tiles > 0) {  // the forward's tiles (block size tb_flux)
        if (a.tb_flux == 64) k_adj_flux_axis_tiles<64><<<a.n_tiles, 64, 0, s>>>(a, j);
        else if (a.tb_flux == 256) k_adj_flux_axis_tiles<256><<<a.n_tiles, 256, 0, s>>>(a, j);
        else k_adj_flux_axis_tiles<128><<<a.n_tiles, 128, 0, s>>>(a, j);
        return;
    }
    k_adj_flux_axis<<<(a.ni + 127) / 128, 128, 0, s>>>(a, j);
}

void launch_adj_flux_general(const FluidArgs<double> &a, const AdjointArgs &j, cudaStream_t s) {
    const int first = a.axis_aligned ? a.ni : 0;
    if (a.nf > first) k_adj_flux_general<<<(a.nf - first + 127) / 128, 128, 0, s>>>(a, j, first);
}

// pdl: a programmatic dependent launch directly behind the kernel it follows on the stream
template <typename... KArgs, typename... Args>
void launch_adj_kernel(void (*kernel)(KArgs...), int g, int tb, cudaStream_t s, bool pdl, Args... args) {
    if (!pdl) {
        kernel<<<g, tb, 0, s>>>(args...);
        return;
    }
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(g);
    cfg.blockDim = dim3(tb);
    cfg.stream = s;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kernel, args...);
}

void launch_adj_cells(const FluidArgs<double> &a, const AdjointArgs &j, cudaStream_t s, bool pdl) {
    launch_adj_kernel(k_adj_cell, (a.nc + 127) / 128, 128, s, pdl, a, j);
}

void launch_adj_gather(const FluidArgs<double> &a, const AdjointArgs &j, cudaStream_t s, bool pdl) {
    launch_adj_kernel(k_adj_gather, (a.nc + 127) / 128, 128, s, pdl, a, j);
}

int launch_adj_fluid(const FluidArgs<double> &a, const AdjointArgs &j, cudaStream_t s) {
    launch_adj_flux_axis(a, j, s);
    launch_adj_flux_general(a, j, s);
    launch_adj_cells(a, j, s);
    launch_adj_gather(a, j, s);
    return 4;
}

}  // namespace lbfs
