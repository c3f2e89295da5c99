// Discrete adjoint of the membrane chain (no reference counterpart).
//
// Forward, per step: x' = x + dt I(u; x) (IBM interpolation + advection),
// F = springs(x', V(x'), A(x'), MAD_n; G_s, k_b) gathered per node,
// MAD_{n+1} = sum over the first n_nodes springs of curv (A1 + A2) / 3 / A(x'),
// f_cell = sum_n F_n W(x'_n, cell) / dx^3 (spread).  Backwards, per step:
//   B1 k_adjm_spread   warp per node: lambda_F = interpolation of the cells'
//                      force adjoint at x', and the spread's dependence on x'.
//   B2 k_adjm_springs  thread per (spring, input direction): J^T lambda of
//                      the spring's 12 force outputs and its MAD term, by
//                      forward-mode dual numbers through a templated copy of
//                      the spring force (exact to rounding); 17 directions:
//                      the 4 nodes' coordinates, V, A, MAD_n, G_s, k_b.
//   B3 k_adjm_reduce   block per membrane: the V, A, MAD_n, G_s, k_b sums.
//   B4 k_adjm_nodes    thread per node: lambda_x' from its springs (in the
//                      incidence order) and its triangles' dV, dA.
//   B5 k_adjm_advect   warp per node: lambda_x = lambda_x' + dt (dI/dx)^T
//                      lambda_x'; the cells' velocity adjoint dt W lambda_x' is
//                      formed by the forward sort + spread kernels run on x
//                      (deterministic), then k_adjm_cells reads the patches.
#include <cuda_runtime.h>

#include "lbfs_adjoint.h"
#include "lbfs_b200.h"

namespace lbfs {
namespace {

// ---- dual numbers (value, derivative along one direction) -------------------
struct Dual {
    double v, d;
};
__device__ __forceinline__ Dual mk(double v, double d = 0.0) { return {v, d}; }
__device__ __forceinline__ Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.d + b.d}; }
__device__ __forceinline__ Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.d - b.d}; }
__device__ __forceinline__ Dual operator-(Dual a) { return {-a.v, -a.d}; }
__device__ __forceinline__ Dual operator*(Dual a, Dual b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
__device__ __forceinline__ Dual operator/(Dual a, Dual b) {
    const double q = a.v / b.v;
    return {q, (a.d - q * b.d) / b.v};
}
__device__ __forceinline__ Dual operator+(Dual a, double b) { return {a.v + b, a.d}; }
__device__ __forceinline__ Dual operator+(double a, Dual b) { return {a + b.v, b.d}; }
__device__ __forceinline__ Dual operator-(Dual a, double b) { return {a.v - b, a.d}; }
__device__ __forceinline__ Dual operator-(double a, Dual b) { return {a - b.v, -b.d}; }
__device__ __forceinline__ Dual operator*(Dual a, double b) { return {a.v * b, a.d * b}; }
__device__ __forceinline__ Dual operator*(double a, Dual b) { return {a * b.v, a * b.d}; }
__device__ __forceinline__ Dual operator/(Dual a, double b) { return {a.v / b, a.d / b}; }
__device__ __forceinline__ Dual operator/(double a, Dual b) {
    const double q = a / b.v;
    return {q, -q * b.d / b.v};
}
__device__ __forceinline__ Dual dsqrt(Dual a) {
    const double s = sqrt(a.v);
    return {s, 0.5 * a.d / s};
}
__device__ __forceinline__ Dual dacos(Dual a) {
    const double r = 1.0 - a.v * a.v;
    return {acos(a.v), r > 0.0 ? -a.d / sqrt(r) : 0.0};
}
__device__ __forceinline__ Dual dfmin(Dual a, double b) { return a.v <= b ? a : mk(b); }
__device__ __forceinline__ Dual dfmax(Dual a, double b) { return a.v >= b ? a : mk(b); }
__device__ __forceinline__ double val(Dual a) { return a.v; }

struct V3 {
    Dual x, y, z;
};
__device__ __forceinline__ V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ V3 operator*(V3 a, Dual s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ V3 operator/(V3 a, Dual s) { return {a.x / s, a.y / s, a.z / s}; }
__device__ __forceinline__ V3 operator/(V3 a, double s) { return {a.x / s, a.y / s, a.z / s}; }
__device__ __forceinline__ Dual dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3 cross(V3 a, V3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ V3 centroid3(V3 a, V3 b, V3 c) {
    return {(a.x + b.x + c.x) / 3.0, (a.y + b.y + c.y) / 3.0, (a.z + b.z + c.z) / 3.0};
}

// What the spring's force depends on linearly through its scalar inputs,
// filled by the value pass of spring_eval: the volume, local-area, curvature
// and length-gradient terms and the WLC polynomial.
struct ScalarTerms {
    double dvol[12], dnb[3], dnd[3], dcurve[12], dL[3], poly, curv_minus_c0;
};

// The spring force of the forward kernel (spring_forces), in dual numbers,
// step mode, membrane viscosity zero.  Outputs the 12 node-force
// contributions and the spring's MAD term curvature (A1 + A2) / 3.
__device__ void spring_eval(const MembraneArgs &A, const MembraneConst &mc, int s, V3 a, V3 b, V3 c, V3 d,
                            Dual vol_coef, Dual area_coef, Dual mad_coef, Dual kspring, Dual kb, double sfc,
                            Dual (&out)[12], Dual &mad_term, ScalarTerms *st = nullptr) {
    const V3 l = c - a;
    Dual length = dsqrt(dot(l, l));
    const V3 normal_a = cross(b - a, c - a), normal_b = cross(c - a, d - a);
    const Dual norm_1 = dsqrt(dot(normal_a, normal_a)), norm_2 = dsqrt(dot(normal_b, normal_b));
    // d_normals(a, b, c, normal_a) and d_normals(c, d, a, normal_b)
    Dual dN1[27], dN2[27], dV1[9], dV2[9];
    auto d_normals = [](V3 p, V3 q, V3 r, V3 normal, Dual (&dN)[27], Dual (&dV)[9]) {
        const V3 cen = centroid3(p, q, r);
        const Dual z = mk(0.0);
        dN[0] = z;          dN[1] = r.z - q.z;  dN[2] = q.y - r.y;
        dN[3] = q.z - r.z;  dN[4] = z;          dN[5] = r.x - q.x;
        dN[6] = r.y - q.y;  dN[7] = q.x - r.x;  dN[8] = z;
        dN[9] = z;          dN[10] = p.z - r.z; dN[11] = r.y - p.y;
        dN[12] = r.z - p.z; dN[13] = z;         dN[14] = p.x - r.x;
        dN[15] = p.y - r.y; dN[16] = r.x - p.x; dN[17] = z;
        dN[18] = z;         dN[19] = q.z - p.z; dN[20] = p.y - q.y;
        dN[21] = p.z - q.z; dN[22] = z;         dN[23] = q.x - p.x;
        dN[24] = q.y - p.y; dN[25] = p.x - q.x; dN[26] = z;
        normal = normal / 3.0;
        for (int t = 0; t < 3; t++) {
            dV[3 * t + 0] = normal.x + dN[9 * t + 1] * cen.y + dN[9 * t + 2] * cen.z;
            dV[3 * t + 1] = normal.y + dN[9 * t + 3] * cen.x + dN[9 * t + 5] * cen.z;
            dV[3 * t + 2] = normal.z + dN[9 * t + 6] * cen.x + dN[9 * t + 7] * cen.y;
        }
    };
    d_normals(a, b, c, normal_a, dN1, dV1);
    d_normals(c, d, a, normal_b, dN2, dV2);
    Dual dn1[9], dn2[9];
    {
        const V3 u1 = normal_a / norm_1, u2 = normal_b / norm_2;
        for (int i = 0; i < 9; i++) {
            dn1[i] = dN1[3 * i] * u1.x + dN1[3 * i + 1] * u1.y + dN1[3 * i + 2] * u1.z;
            dn2[i] = dN2[3 * i] * u2.x + dN2[3 * i + 1] * u2.y + dN2[3 * i + 2] * u2.z;
        }
    }
    auto merge12 = [](Dual (&o)[12], const Dual (&t1)[9], const Dual (&t2)[9]) {
        for (int j = 0; j < 9; j++) o[j] = t1[j];
        for (int j = 0; j < 3; j++) o[j + 6] = o[j + 6] + t2[j];
        for (int j = 3; j < 6; j++) o[j + 6] = t2[j];
        for (int j = 6; j < 9; j++) o[j - 6] = o[j - 6] + t2[j];
    };
    Dual d_area[12], d_volume[12];
    merge12(d_area, dn1, dn2);
    for (int j = 0; j < 12; j++) d_area[j] = d_area[j] * 0.166666666666666666666666666666666666666666;
    merge12(d_volume, dV1, dV2);
    for (int j = 0; j < 12; j++) d_volume[j] = d_volume[j] * (1.0 / 18.0);
    Dual cos_angle = dot(normal_a, normal_b) / (norm_1 * norm_2);
    cos_angle = dfmin(cos_angle, 1.0);
    cos_angle = dfmax(cos_angle, -1.0);
    const V3 centroid_1 = centroid3(a, b, c);
    const V3 centroid_2 = centroid3(a, c, d) - centroid_1;
    const double angle_direction = val(dot(normal_a, centroid_2));
    Dual angle = dacos(cos_angle);
    angle = angle * (double)((angle_direction < 0) - (angle_direction > 0));
    Dual d_angle[12];
    {
        Dual d_angle_1[9], d_angle_2[9];
        const V3 h = cross(normal_a / norm_1, l / length);
        for (int j = 0; j < 9; j++)
            d_angle_1[j] = -1.0 / norm_1 * (h.x * dN1[j * 3] + h.y * dN1[j * 3 + 1] + h.z * dN1[j * 3 + 2]);
        const V3 h2 = cross(l / length, normal_b / norm_2);
        for (int j = 0; j < 9; j++)
            d_angle_2[j] = -1.0 / norm_2 * (h2.x * dN2[j * 3] + h2.y * dN2[j * 3 + 1] + h2.z * dN2[j * 3 + 2]);
        merge12(d_angle, d_angle_1, d_angle_2);
    }
    c = c - a;
    length = dsqrt(dot(c, c));
    const V3 dL_ds = c / length;
    Dual d_curve[12];
    for (int j = 0; j < 12; j++) d_curve[j] = d_angle[j] * length;
    d_curve[0] = d_curve[0] - dL_ds.x * angle;
    d_curve[1] = d_curve[1] - dL_ds.y * angle;
    d_curve[2] = d_curve[2] - dL_ds.z * angle;
    d_curve[6] = d_curve[6] + dL_ds.x * angle;
    d_curve[7] = d_curve[7] + dL_ds.y * angle;
    d_curve[8] = d_curve[8] + dL_ds.z * angle;
    V3 fa = {mk(0), mk(0), mk(0)}, fb = fa, fc = fa, fd = fa;
    Dual lac = -1.0 * mc.local_area_modulus * (norm_1 / A.area0[2 * s] - 1.0) + area_coef;
    fb = fb + V3{lac * dn1[3], lac * dn1[4], lac * dn1[5]};
    lac = -1.0 * mc.local_area_modulus * (norm_2 / A.area0[2 * s + 1] - 1.0) + area_coef;
    fd = fd + V3{lac * dn2[3], lac * dn2[4], lac * dn2[5]};
    fa = fa + V3{vol_coef * d_volume[0], vol_coef * d_volume[1], vol_coef * d_volume[2]};
    fb = fb + V3{vol_coef * d_volume[3], vol_coef * d_volume[4], vol_coef * d_volume[5]};
    fc = fc + V3{vol_coef * d_volume[6], vol_coef * d_volume[7], vol_coef * d_volume[8]};
    fd = fd + V3{vol_coef * d_volume[9], vol_coef * d_volume[10], vol_coef * d_volume[11]};
    const Dual spring_area_total = (norm_1 + norm_2) / 6.0;
    const Dual curvature = angle * length / spring_area_total;
    const double c0 = A.curv0[s];
    const Dual lbc = -0.5 * mc.local_bending_modulus * (c0 - curvature) * (c0 - curvature);
    fa = fa + V3{lbc * d_area[0], lbc * d_area[1], lbc * d_area[2]};
    fb = fb + V3{lbc * d_area[3], lbc * d_area[4], lbc * d_area[5]};
    fc = fc + V3{lbc * d_area[6], lbc * d_area[7], lbc * d_area[8]};
    fd = fd + V3{lbc * d_area[9], lbc * d_area[10], lbc * d_area[11]};
    const Dual cc = -1.0 * kb * (curvature - c0) + mad_coef;
    fa = fa + V3{cc * d_curve[0], cc * d_curve[1], cc * d_curve[2]};
    fb = fb + V3{cc * d_curve[3], cc * d_curve[4], cc * d_curve[5]};
    fc = fc + V3{cc * d_curve[6], cc * d_curve[7], cc * d_curve[8]};
    fd = fd + V3{cc * d_curve[9], cc * d_curve[10], cc * d_curve[11]};
    const Dual sr = length / A.contour[s];
    const Dual fcoef = -1.0 * kspring * ((0.25 / ((1.0 - sr) * (1.0 - sr))) - 0.25 + sr - sfc);
    fc = fc + dL_ds * fcoef;
    fa = fa - dL_ds * fcoef;
    out[0] = fa.x; out[1] = fa.y; out[2] = fa.z;
    out[3] = fb.x; out[4] = fb.y; out[5] = fb.z;
    out[6] = fc.x; out[7] = fc.y; out[8] = fc.z;
    out[9] = fd.x; out[10] = fd.y; out[11] = fd.z;
    mad_term = curvature * (norm_1 + norm_2) * 1.0 / 3.0;
    if (st) {
        for (int j = 0; j < 12; j++) { st->dvol[j] = val(d_volume[j]); st->dcurve[j] = val(d_curve[j]); }
        for (int j = 0; j < 3; j++) { st->dnb[j] = val(dn1[3 + j]); st->dnd[j] = val(dn2[3 + j]); }
        st->dL[0] = val(dL_ds.x); st->dL[1] = val(dL_ds.y); st->dL[2] = val(dL_ds.z);
        st->poly = val((0.25 / ((1.0 - sr) * (1.0 - sr))) - 0.25 + sr - sfc);
        st->curv_minus_c0 = val(curvature) - c0;
    }
}

// ---- IBM stencil weights and their derivatives ------------------------------
__device__ __forceinline__ double peskin4_w(double r) {
    r = fabs(r);
    if (r < 1.0) return (3.0 - 2.0 * r + sqrt(1.0 + 4.0 * r - 4.0 * r * r)) * 0.125;
    if (r < 2.0) return (5.0 - 2.0 * r - sqrt(-7.0 + 12.0 * r - 4.0 * r * r)) * 0.125;
    return 0.0;
}
// d phi / d r of the 4-point delta and of the 2-point hat.
__device__ __forceinline__ double weight_deriv(int stencil, double r) {
    const double sg = r < 0 ? -1.0 : 1.0, q = fabs(r);
    if (stencil == LBFS_IBM_PESKIN4) {
        if (q < 1.0) return sg * (-2.0 + (4.0 - 8.0 * q) / (2.0 * sqrt(1.0 + 4.0 * q - 4.0 * q * q))) * 0.125;
        if (q < 2.0) return sg * (-2.0 - (12.0 - 8.0 * q) / (2.0 * sqrt(-7.0 + 12.0 * q - 4.0 * q * q))) * 0.125;
        return 0.0;
    }
    return q < 1.0 ? -sg : 0.0;
}
__device__ __forceinline__ double weight(int stencil, double r) {
    return stencil == LBFS_IBM_PESKIN4 ? peskin4_w(r) : 1 - fabs(r);
}

// Stencil of a node on its membrane's grid (node_stencil of the forward) with
// d r / d position per axis (y and z are mirrored with fabs).
struct StencilD {
    double r[3], dr[3];
    int b[3];
};
__device__ __forceinline__ StencilD stencil_d(int stencil, const MembraneConst &mc, double x, double y, double z) {
    StencilD s;
    const double p[3] = {x, y, z};
    for (int c = 0; c < 3; c++) {
        const double q = (p[c] - mc.gorigin[c]) / mc.gdx;
        s.r[c] = c == 0 ? q : fabs(q);
        s.dr[c] = (c == 0 || q >= 0) ? 1.0 / mc.gdx : -1.0 / mc.gdx;
        s.b[c] = stencil == LBFS_IBM_PESKIN4 ? (int)floor(s.r[c] - 0.5) - 1 : (int)round(s.r[c]) - 1;
    }
    return s;
}

// ---- B1: spread adjoint at x' -------------------------------------------------
__global__ void __launch_bounds__(256) k_adjm_spread(MembraneArgs A, MemAdjArgs J) {
    pdl_trigger();
    const int lane = threadIdx.x & 31;
    const int n = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (n >= A.total_nodes) return;
    const MembraneConst &mc = A.mc[A.node_mem[n]];
    const int S = A.ibm_stencil == LBFS_IBM_PESKIN4 ? 4 : 2;
    const StencilD st = stencil_d(A.ibm_stencil, mc, A.x[n], A.y[n], A.z[n]);
    const double F[3] = {A.fx[n], A.fy[n], A.fz[n]};
    const double inv3 = 1 / mc.gdx / mc.gdx / mc.gdx;
    double lF[3] = {0, 0, 0}, lx[3] = {0, 0, 0};
    for (int c = lane; c < S * S * S; c += 32) {
        const int di = c / (S * S), dj = (c / S) % S, dk = c % S;
        const int i = st.b[0] + di, jj = st.b[1] + dj, k = st.b[2] + dk;
        if (i < 0 || jj < 0 || k < 0 || i >= mc.gnx || jj >= mc.gny || k >= mc.gnz) continue;
        const int idx = mc.cell0 + i + mc.gnx * (jj + mc.gny * k);
        const double4 lt = J.lam_t1[idx];
        const double lf[3] = {J.dt * lt.x, J.dt * lt.y, J.dt * lt.z};
        const double d[3] = {i + 0.5 - st.r[0], jj + 0.5 - st.r[1], k + 0.5 - st.r[2]};
        const double w[3] = {weight(A.ibm_stencil, d[0]), weight(A.ibm_stencil, d[1]), weight(A.ibm_stencil, d[2])};
        const double dw[3] = {-weight_deriv(A.ibm_stencil, d[0]) * st.dr[0],
                              -weight_deriv(A.ibm_stencil, d[1]) * st.dr[1],
                              -weight_deriv(A.ibm_stencil, d[2]) * st.dr[2]};
        const double W = w[0] * w[1] * w[2] * inv3;
        const double g = (F[0] * lf[0] + F[1] * lf[1] + F[2] * lf[2]) * inv3;
        for (int q = 0; q < 3; q++) lF[q] += W * lf[q];
        lx[0] += g * dw[0] * w[1] * w[2];
        lx[1] += g * w[0] * dw[1] * w[2];
        lx[2] += g * w[0] * w[1] * dw[2];
    }
    for (int q = 0; q < 3; q++)
        for (int o = 16; o > 0; o >>= 1) {
            lF[q] += __shfl_down_sync(0xffffffffu, lF[q], o);
            lx[q] += __shfl_down_sync(0xffffffffu, lx[q], o);
        }
    if (lane == 0) {
        for (int q = 0; q < 3; q++) {
            J.lam_F[3 * (size_t)n + q] = lF[q];
            J.lam_xp[3 * (size_t)n + q] = J.lam_x[3 * (size_t)n + q] + lx[q];
        }
    }
}

// ---- B2: spring adjoint by dual numbers ---------------------------------------
constexpr int kDirs = 17;   // 12 coordinates, V, A, MAD_n, G_s, k_b
constexpr int kPasses = 13; // the 12 coordinate directions in dual numbers, then one value pass for the 5 scalars

__global__ void __launch_bounds__(128) k_adjm_springs(MembraneArgs A, MemAdjArgs J) {
    pdl_trigger();
    pdl_wait();
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    const int k = blockIdx.y;
    if (s >= A.total_springs) return;
    const int m = A.spring_mem[s];
    const MembraneConst &mc = A.mc[m];
    const MembraneScalars &ms = A.ms[m];
    int node[4];
    V3 p[4];
    for (int q = 0; q < 4; q++) {
        node[q] = A.spring[4 * s + q];
        const int n = node[q];
        p[q] = {mk(A.x[n], k == 3 * q ? 1.0 : 0.0), mk(A.y[n], k == 3 * q + 1 ? 1.0 : 0.0),
                mk(A.z[n], k == 3 * q + 2 ? 1.0 : 0.0)};
    }
    const double ks = A.kspring[s];
    const double wr = mc.wlc_ratio;
    const double sfc = (0.25 * wr * wr / ((wr - 1.0) * (wr - 1.0)) - 0.25 + 1.0 / wr);
    const Dual vol_coef = mk(-1.0 * mc.volume_modulus * (ms.V / ms.V0 - 1.0) / 6.0);
    const Dual area_coef = mk(-1.0 * mc.global_area_modulus * (ms.A / ms.A0 - 1.0));
    const Dual mad_coef = mk(-1.0 * 2.0 * mc.global_bending_modulus * (J.mad_n[m] - ms.MAD0) / ms.A0);
    Dual out[12], term;
    if (k < 12) {  // node coordinate 3 q + c: J^T lambda by one forward-mode pass
        spring_eval(A, mc, s, p[0], p[1], p[2], p[3], vol_coef, area_coef, mad_coef, mk(ks),
                    mk(mc.global_bending_modulus), sfc, out, term);
        double acc = 0.0;
        for (int q = 0; q < 4; q++)
            for (int c = 0; c < 3; c++) acc += J.lam_F[3 * (size_t)node[q] + c] * out[3 * q + c].d;
        if (s - mc.spring0 < mc.n_nodes) acc += J.lam_mad[m] / ms.A * term.d;
        J.adjm[kDirs * (size_t)s + k] = acc;
        return;
    }
    // V, A, MAD_n, G_s and k_b enter the force linearly, through vol_coef,
    // area_coef (the local-area terms of nodes b and d), mad_coef and k_b (the
    // curvature term) and the spring constant (the WLC term of a and c); the
    // spring's MAD term does not depend on them.  One value pass gives them all.
    ScalarTerms st;
    spring_eval(A, mc, s, p[0], p[1], p[2], p[3], vol_coef, area_coef, mad_coef, mk(ks),
                mk(mc.global_bending_modulus), sfc, out, term, &st);
    double lf[12];
    for (int q = 0; q < 4; q++)
        for (int c = 0; c < 3; c++) lf[3 * q + c] = J.lam_F[3 * (size_t)node[q] + c];
    double dv = 0.0, dc = 0.0;
    for (int j = 0; j < 12; j++) { dv += lf[j] * st.dvol[j]; dc += lf[j] * st.dcurve[j]; }
    const double da = lf[3] * st.dnb[0] + lf[4] * st.dnb[1] + lf[5] * st.dnb[2] + lf[9] * st.dnd[0] +
                      lf[10] * st.dnd[1] + lf[11] * st.dnd[2];
    const double dl = (lf[6] - lf[0]) * st.dL[0] + (lf[7] - lf[1]) * st.dL[1] + (lf[8] - lf[2]) * st.dL[2];
    double *o = J.adjm + kDirs * (size_t)s + 12;
    o[0] = -mc.volume_modulus / (6.0 * ms.V0) * dv;                              // V
    o[1] = -mc.global_area_modulus / ms.A0 * da;                                 // A
    o[2] = -2.0 * mc.global_bending_modulus / ms.A0 * dc;                        // MAD_n
    o[3] = -(ks / mc.shear_modulus) * st.poly * dl;                              // G_s (k_spring proportional to G_s)
    o[4] = (-st.curv_minus_c0 - 2.0 * (J.mad_n[m] - ms.MAD0) / ms.A0) * dc;     // k_b
}

// ---- B3: per-membrane sums ----------------------------------------------------
__global__ void __launch_bounds__(1024) k_adjm_reduce(MembraneArgs A, MemAdjArgs J) {
    __shared__ double sh[32][5];
    pdl_trigger();
    pdl_wait();
    const int m = blockIdx.x;
    const MembraneConst &mc = A.mc[m];
    double v[5] = {0, 0, 0, 0, 0};
    for (int ls = threadIdx.x; ls < mc.n_springs; ls += blockDim.x) {
        const double *r = J.adjm + kDirs * (size_t)(mc.spring0 + ls) + 12;
        for (int q = 0; q < 5; q++) v[q] += r[q];
    }
    // the five sums in one pass: warp trees, then the warps in order
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int q = 0; q < 5; q++) {
        for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
        if (lane == 0) sh[warp][q] = v[q];
    }
    __syncthreads();
    double t[5] = {0, 0, 0, 0, 0};
    if (threadIdx.x == 0)
        for (int w = 0; w < (int)(blockDim.x >> 5); w++)
            for (int q = 0; q < 5; q++) t[q] += sh[w][q];
    if (threadIdx.x == 0) {
        const MembraneScalars &ms = A.ms[m];
        const double lam_mad_next = J.lam_mad[m];
        J.red[5 * m + 0] = t[0];                                       // lambda V
        J.red[5 * m + 1] = t[1] - lam_mad_next * ms.MAD / ms.A;       // lambda A (forces and MAD / A)
        J.lam_mad[m] = t[2];                                           // lambda MAD_n (carried)
        J.gs_acc[m] += t[3];
        J.kb_acc[m] += t[4];
    }
}

// ---- B4: node gather of the spring and totals adjoints -------------------------
__global__ void __launch_bounds__(128) k_adjm_nodes(MembraneArgs A, MemAdjArgs J) {
    pdl_trigger();
    pdl_wait();
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= A.total_nodes) return;
    const int m = A.node_mem[n];
    double g[3] = {0, 0, 0};
    for (int e = A.inc_start[n]; e < A.inc_start[n + 1]; e++) {
        const int code = A.inc[e];
        const double *r = J.adjm + kDirs * (size_t)(code >> 2) + 3 * (code & 3);
        g[0] += r[0];
        g[1] += r[1];
        g[2] += r[2];
    }
    const double lV = J.red[5 * m], lA = J.red[5 * m + 1];
    for (int e = J.tri_start[n]; e < J.tri_start[n + 1]; e++) {
        const int code = J.tri_inc[e];
        const int t = code >> 2, v = code & 3;
        const int i0 = A.tri[3 * t], i1 = A.tri[3 * t + 1], i2 = A.tri[3 * t + 2];
        const double a[3] = {A.x[i0], A.y[i0], A.z[i0]}, b[3] = {A.x[i1], A.y[i1], A.z[i1]},
                     c[3] = {A.x[i2], A.y[i2], A.z[i2]};
        // V_t = a . (b x c) / 6;  A_t = |(b - a) x (c - a)| / 2
        const double *P = v == 0 ? b : (v == 1 ? c : a), *Q = v == 0 ? c : (v == 1 ? a : b);
        const double dV[3] = {(P[1] * Q[2] - P[2] * Q[1]) / 6, (P[2] * Q[0] - P[0] * Q[2]) / 6,
                              (P[0] * Q[1] - P[1] * Q[0]) / 6};
        const double e1[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]}, e2[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
        double N[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
        const double nn = sqrt(N[0] * N[0] + N[1] * N[1] + N[2] * N[2]);
        N[0] /= nn; N[1] /= nn; N[2] /= nn;
        // d|N|/d node: a -> (b - c) x n, b -> (c - a) x n, c -> (a - b) x n
        const double *U = v == 0 ? b : (v == 1 ? c : a), *W = v == 0 ? c : (v == 1 ? a : b);
        const double dd[3] = {U[0] - W[0], U[1] - W[1], U[2] - W[2]};
        const double dA[3] = {0.5 * (dd[1] * N[2] - dd[2] * N[1]), 0.5 * (dd[2] * N[0] - dd[0] * N[2]),
                              0.5 * (dd[0] * N[1] - dd[1] * N[0])};
        for (int q = 0; q < 3; q++) g[q] += lV * dV[q] + lA * dA[q];
    }
    for (int q = 0; q < 3; q++) J.lam_xp[3 * (size_t)n + q] += g[q];
}

// ---- B5: advection adjoint at x_n -------------------------------------------------
template <typename R>
__global__ void __launch_bounds__(256) k_adjm_advect(MembraneArgs A, MemAdjArgs J) {
    pdl_trigger();
    pdl_wait();
    const int lane = threadIdx.x & 31;
    const int n = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (n >= A.total_nodes) return;
    const MembraneConst &mc = A.mc[A.node_mem[n]];
    const int S = A.ibm_stencil == LBFS_IBM_PESKIN4 ? 4 : 2;
    const StencilD st = stencil_d(A.ibm_stencil, mc, J.xn[n], J.yn[n], J.zn[n]);
    const double lxp[3] = {J.lam_xp[3 * (size_t)n], J.lam_xp[3 * (size_t)n + 1], J.lam_xp[3 * (size_t)n + 2]};
    const int n_inst = mc.gnx * mc.gny * mc.gnz;
    double lx[3] = {0, 0, 0};
    for (int c = lane; c < S * S * S; c += 32) {
        const int di = c / (S * S), dj = (c / S) % S, dk = c % S;
        const int i = st.b[0] + di, jj = st.b[1] + dj, k = st.b[2] + dk;
        const int lidx = i + jj * mc.gnx + k * mc.gny * mc.gnx;
        if (lidx < 0 || lidx >= n_inst) continue;
        const Vec4<R> sv = reinterpret_cast<const Vec4<R> *>(A.state)[mc.cell0 + lidx];
        const double u[3] = {(double)sv.u, (double)sv.v, (double)sv.w};
        const double d[3] = {i + 0.5 - st.r[0], jj + 0.5 - st.r[1], k + 0.5 - st.r[2]};
        const double w[3] = {weight(A.ibm_stencil, d[0]), weight(A.ibm_stencil, d[1]), weight(A.ibm_stencil, d[2])};
        const double dw[3] = {-weight_deriv(A.ibm_stencil, d[0]) * st.dr[0],
                              -weight_deriv(A.ibm_stencil, d[1]) * st.dr[1],
                              -weight_deriv(A.ibm_stencil, d[2]) * st.dr[2]};
        const double g = J.dt * (u[0] * lxp[0] + u[1] * lxp[1] + u[2] * lxp[2]);
        lx[0] += g * dw[0] * w[1] * w[2];
        lx[1] += g * w[0] * dw[1] * w[2];
        lx[2] += g * w[0] * w[1] * dw[2];
    }
    for (int q = 0; q < 3; q++)
        for (int o = 16; o > 0; o >>= 1) lx[q] += __shfl_down_sync(0xffffffffu, lx[q], o);
    if (lane == 0) {
        for (int q = 0; q < 3; q++) J.lam_x[3 * (size_t)n + q] = lxp[q] + lx[q];
        // dt lambda_x' as the "force" the spread kernel distributes over the cells
        // (x dx^3, which its 1 / dx^3 removes)
        const double sc = J.dt * mc.gdx * mc.gdx * mc.gdx;
        J.mb.fx[n] = sc * lxp[0];
        J.mb.fy[n] = sc * lxp[1];
        J.mb.fz[n] = sc * lxp[2];
    }
}

// Cells' velocity adjoint from the patches of the second spread.
__global__ void __launch_bounds__(256) k_adjm_cells(MemAdjArgs J, int nc, const int *cell_instance,
                                                     const InstanceGrid *instances) {
    pdl_wait();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nc) return;
    const int inst = cell_instance ? cell_instance[i] : 0;
    const InstanceGrid g = instances[inst];
    const int li = i - g.cell0;
    const int ci = li % g.nx, cj = (li / g.nx) % g.ny, ck = li / (g.nx * g.ny);
    double f[3] = {0, 0, 0};
    for (int m = g.mem0; m < g.mem1; m++) {
        const MembraneScalars &ms = J.mb.ms[m];
        const int px = ci - ms.patch_lo[0], py = cj - ms.patch_lo[1], pz = ck - ms.patch_lo[2];
        if (ms.patch_cells > 0 && px >= 0 && py >= 0 && pz >= 0 && px < ms.patch_dim[0] && py < ms.patch_dim[1] &&
            pz < ms.patch_dim[2]) {
            const double *pf =
                J.mb.patch_force + ((size_t)ms.patch_off + (px + ms.patch_dim[0] * (py + ms.patch_dim[1] * pz))) * 3;
            f[0] += pf[0];
            f[1] += pf[1];
            f[2] += pf[2];
        }
    }
    J.lam_u_ibm[3 * (size_t)i] = f[0];
    J.lam_u_ibm[3 * (size_t)i + 1] = f[1];
    J.lam_u_ibm[3 * (size_t)i + 2] = f[2];
}

__global__ void k_adjm_get_mad(MembraneArgs A, double *out) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m < A.n_membranes) out[m] = A.ms[m].MAD;
}
__global__ void k_adjm_set_mad(MembraneArgs A, const double *in) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m < A.n_membranes) A.ms[m].MAD = in[m];
}

}  // namespace

void launch_adjm_get_mad(const MembraneArgs &A, double *out, cudaStream_t s) {
    k_adjm_get_mad<<<(A.n_membranes + 127) / 128, 128, 0, s>>>(A, out);
}
void launch_adjm_set_mad(const MembraneArgs &A, const double *in, cudaStream_t s) {
    k_adjm_set_mad<<<(A.n_membranes + 127) / 128, 128, 0, s>>>(A, in);
}

// The interpolation transpose's stencil tables and node sort at x_n
// (J.mb.x): independent of the adjoints, so they may run ahead of the step's
// other membrane kernels (which must follow them on the same stream).
void launch_adj_membrane_sort(const MemAdjArgs &J, cudaStream_t s) {
    launch_membrane_tables(J.mb, s);
    launch_membrane_sort(J.mb, s);
}

// Membrane part of one backward step, after launch_adj_membrane_sort: A holds
// the step's x', node forces, totals and MAD_{n+1}.
// Each kernel after the first directly behind its predecessor on the stream,
// as a programmatic dependent launch (it waits in pdl_wait for the
// predecessor's results).
template <typename... KArgs, typename... Args>
void launch_chained(void (*kernel)(KArgs...), dim3 grid, dim3 block, cudaStream_t s, Args... args) {
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.stream = s;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kernel, args...);
}

int launch_adj_membrane(const MembraneArgs &A, const MemAdjArgs &J, int nc, const int *cell_instance,
                        const InstanceGrid *instances, cudaStream_t s) {
    const int node_blocks = (A.total_nodes * 32 + 255) / 256;
    k_adjm_spread<<<node_blocks, 256, 0, s>>>(A, J);
    launch_chained(k_adjm_springs, dim3((A.total_springs + 127) / 128, kPasses), dim3(128), s, A, J);
    launch_chained(k_adjm_reduce, dim3(A.n_membranes), dim3(1024), s, A, J);
    launch_chained(k_adjm_nodes, dim3((A.total_nodes + 127) / 128), dim3(128), s, A, J);
    if (A.state_is_float) launch_chained(k_adjm_advect<float>, dim3(node_blocks), dim3(256), s, A, J);
    else launch_chained(k_adjm_advect<double>, dim3(node_blocks), dim3(256), s, A, J);
    launch_membrane_spread(J.mb, s);
    launch_chained(k_adjm_cells, dim3((nc + 255) / 256), dim3(256), s, J, nc, cell_instance, instances);
    return 7;
}

}  // namespace lbfs
