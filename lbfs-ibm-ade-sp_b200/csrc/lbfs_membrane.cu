// Membrane side of one time step, five kernels:
//
//   M1 k_mem_advect    (one warp per node)                           P0
//   M2 k_mem_springs   (one thread per spring; totals per block)     P1, P2, P4
//   M3 k_mem_nodeforce (one thread per node)                         P3
//   M4 k_mem_sort      (one CTA per membrane, on a side stream)      P5
//   k_mem_totals       (one CTA per membrane: V, A)                  P1
//   M5 k_mem_spread    (one warp per patch cell, all membranes)      P6
//   k_mem_step         (one thread-block cluster per membrane)       P1-P5 in one launch
//
//   P0  IBM velocity interpolation at the nodes + explicit node advection
//       (interpolate_velocities_on_nodes, immersed_boundary_method.cu:14-97;
//        update_node_positions, :234-264), FP64 positions.
//   P1  triangle normals / areas / signed volumes and the membrane totals V, A
//       (update_spring_network_tet_parameters, spring_network.cu:1186-1238, and
//        the host sums of total<128> partials, lagrangian_object.cpp:601-630),
//       reduced with warp shuffles in a fixed order.
//   P2  per-spring WLC, local/global area, volume, bending, ADE (MAD) and
//       membrane-viscosity forces (get_spring_forces_atomics,
//       spring_network.cu:613-971), written per spring instead of 12 atomics.
//   P3  node forces: each node sums its springs' contributions in spring order
//       (deterministic; replaces the CAS atomics).
//   P4  MAD = sum over the first n_nodes springs of c (A1 + A2) / 3, / A
//       (sum_product_curvature<128> + lagrangian_object::add_MAD).
//   P5  nodes sorted by the Eulerian cell at the base of their IBM stencil
//       (counting sort over the stencil bins of the membrane's patch, each
//       bin's nodes in index order).
//   P6  force spreading as a per-cell segmented reduction over the sorted
//       nodes into a dense patch around the membrane (replaces
//       spread_forces_on_structured_grid, :947-1024, and its CAS atomics).
#include <cooperative_groups.h>
#include <cuda_runtime.h>
#include <cstdint>

#include "lbfs_fluid.cuh"
#include "lbfs_internal.h"
#include "lbfs_kernels.h"

namespace lbfs {
namespace {

// Node sort: two int arrays of sort_capacity (bins, sorted list), then the bin
// counts of a patch with at most kSortBinsSmem - 1 bins (larger patches count
// in global memory).
constexpr int kSortBinsSmem = 12288;
size_t sort_smem_bytes(int sort_capacity) {
    return (size_t)(sort_capacity > 0 ? sort_capacity : 1) * 2 * sizeof(int) + kSortBinsSmem * sizeof(int);
}

struct D3 {
    double x, y, z;
};
__device__ __forceinline__ D3 d3(double x, double y, double z) { return {x, y, z}; }
__device__ __forceinline__ D3 operator+(D3 a, D3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ D3 operator-(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ D3 operator*(D3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ double dot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ D3 cross(D3 a, D3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
// Divisions by constants and repeated divisors are products with the
// reciprocal in the membrane kernels (an FP64 division is a dependent
// sequence of about ten instructions, and the spring forces are a chain of
// them): results differ from the reference's divisions by rounding only.
constexpr double kThird = 1.0 / 3.0, kSixth = 1.0 / 6.0;
__device__ __forceinline__ D3 tri_centroid(D3 a, D3 b, D3 c) {
    return {(a.x + b.x + c.x) * kThird, (a.y + b.y + c.y) * kThird, (a.z + b.z + c.z) * kThird};
}

// Deterministic block reductions: warp shuffle tree, then the warp results
// in warp order by one thread.  `sh` holds 33 doubles.
__device__ double block_sum(double v, double *sh) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += sh[w];
        sh[32] = s;
    }
    __syncthreads();
    const double r = sh[32];
    __syncthreads();
    return r;
}

// Peskin's 4-point delta, phi(r) for |r| < 2 (Peskin, Acta Numerica 2002, eq. 6.27).
__device__ __forceinline__ double peskin4(double r) {
    r = fabs(r);
    if (r < 1.0) return (3.0 - 2.0 * r + sqrt(1.0 + 4.0 * r - 4.0 * r * r)) * 0.125;
    if (r < 2.0) return (5.0 - 2.0 * r - sqrt(-7.0 + 12.0 * r - 4.0 * r * r)) * 0.125;
    return 0.0;
}

// Stencil reference coordinates of a node (immersed_boundary_method.cu:45-58:
// y and z are mirrored with fabs as in the reference) and the first stencil
// cell per axis: round(r) - 1 for the 2-point hat, floor(r - 0.5) - 1 for the
// 4-point delta.
struct Stencil {
    double rx, ry, rz;
    int i0, j0, k0;
};

// Index of the vertex closest to t in the increasing array v[0..n), ties to
// the upper vertex; t outside the array gives its end (find_index_closest,
// immersed_boundary_method.cu:588-630).
__device__ __forceinline__ int closest_vertex(const double *v, int n, double t) {
    if (t <= v[0]) return 0;
    if (t >= v[n - 1]) return n - 1;
    int lo = 0, hi = n - 1;  // v[lo] < t < v[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (v[mid] == t) return mid;
        if (v[mid] < t) lo = mid;
        else hi = mid;
    }
    return (t - v[lo] >= v[hi] - t) ? hi : lo;
}

// Weights at 0 of the Lagrange polynomials through x1..x4: the first column
// of the inverse Vandermonde matrix as vandemonde_inverse forms it
// (immersed_boundary_method.cu:919-941).
__device__ __forceinline__ double lagrange4_at0(const double (&x)[4], int q) {
    const double sxy = 1 / (x[0] - x[1]), sxz = 1 / (x[0] - x[2]), sxw = 1 / (x[0] - x[3]);
    const double syz = 1 / (x[1] - x[2]), syw = 1 / (x[1] - x[3]), szw = 1 / (x[2] - x[3]);
    if (q == 0) return -1 * x[1] * x[2] * x[3] * sxy * sxz * sxw;
    if (q == 1) return x[0] * x[2] * x[3] * sxy * syz * syw;
    if (q == 2) return -1 * x[0] * x[1] * x[3] * sxz * syz * szw;
    return x[0] * x[1] * x[2] * sxw * syw * szw;
}

// One-dimensional weight q of the 4x4x4 stencil on a rectilinear mesh along
// axis ax: cells b .. b + 3 of the row, offsets of their centroids from p.  A
// stencil that leaves the mesh gets zero weights (the node sort raises
// LBFS_FLAG_IBM_RANGE; the reference reads outside its arrays there).
__device__ __forceinline__ double vandermonde_weight(const MembraneArgs &a, const MembraneConst &mc, int ax, int b,
                                                     double p, int q) {
    const int n = ax == 0 ? mc.gnx : (ax == 1 ? mc.gny : mc.gnz);
    if (b < 0 || b + 3 >= n) return 0.0;
    const double *c = a.grid_c[ax] + b;
    const double x[4] = {c[0] - p, c[1] - p, c[2] - p, c[3] - p};
    return lagrange4_at0(x, q);
}

__device__ __forceinline__ Stencil node_stencil(const MembraneArgs &a, const MembraneConst &mc, double x, double y,
                                                double z) {
    Stencil s;
    if (a.ibm_stencil == LBFS_IBM_VANDERMONDE4) {
        // the closest vertex, minus 2: the first of the 4 cells per axis
        // (interpolate_velocities_on_nodes_non_uniform_grid, immersed_boundary_method.cu:685-711)
        s.rx = x; s.ry = y; s.rz = z;
        s.i0 = closest_vertex(a.grid_v[0], mc.gnx + 1, x) - 2;
        s.j0 = closest_vertex(a.grid_v[1], mc.gny + 1, y) - 2;
        s.k0 = closest_vertex(a.grid_v[2], mc.gnz + 1, z) - 2;
        return s;
    }
    s.rx = (x - mc.gorigin[0]) / mc.gdx;
    s.ry = fabs((y - mc.gorigin[1]) / mc.gdx);
    s.rz = fabs((z - mc.gorigin[2]) / mc.gdx);
    if (a.ibm_stencil == LBFS_IBM_PESKIN4) {
        s.i0 = (int)floor(s.rx - 0.5) - 1;
        s.j0 = (int)floor(s.ry - 0.5) - 1;
        s.k0 = (int)floor(s.rz - 0.5) - 1;
    } else {
        s.i0 = (int)round(s.rx) - 1;
        s.j0 = (int)round(s.ry) - 1;
        s.k0 = (int)round(s.rz) - 1;
    }
    return s;
}
__device__ __forceinline__ double stencil_weight(int stencil, double d) {
    return stencil == LBFS_IBM_PESKIN4 ? peskin4(d) : 1 - fabs(d);
}

template <typename R>
__device__ __forceinline__ void read_velocity(const void *state, int idx, double &u, double &v, double &w) {
    const Vec4<R> s = ((const Vec4<R> *)state)[idx];
    u = (double)s.u;
    v = (double)s.v;
    w = (double)s.w;
}

// ---- per-spring force (get_spring_forces_atomics, spring_network.cu:613-971) ----

// Derivatives of the triangle normal N = (q - p) x (r - p) with respect to the
// coordinates of p, q, r (get_d_normals, spring_network.cu:1348-1414):
// dN[9 s + 3 c + k] = dN_k / d(node s)_c, s = 0 p, 1 q, 2 r; and the derivative
// of the signed volume term N . centroid / 6 scaled by 6: dV[3 s + c].
__device__ __forceinline__ void d_normals(D3 a, D3 b, D3 c, D3 normal, double *dN, double *dV) {
    const D3 cen = tri_centroid(a, b, c);
    dN[0] = 0.0;        dN[1] = c.z - b.z;  dN[2] = b.y - c.y;
    dN[3] = b.z - c.z;  dN[4] = 0.0;        dN[5] = c.x - b.x;
    dN[6] = c.y - b.y;  dN[7] = b.x - c.x;  dN[8] = 0.0;
    dN[9] = 0.0;        dN[10] = a.z - c.z; dN[11] = c.y - a.y;
    dN[12] = c.z - a.z; dN[13] = 0.0;       dN[14] = a.x - c.x;
    dN[15] = a.y - c.y; dN[16] = c.x - a.x; dN[17] = 0.0;
    dN[18] = 0.0;       dN[19] = b.z - a.z; dN[20] = a.y - b.y;
    dN[21] = a.z - b.z; dN[22] = 0.0;       dN[23] = b.x - a.x;
    dN[24] = b.y - a.y; dN[25] = a.x - b.x; dN[26] = 0.0;
    normal = normal * kThird;
#pragma unroll
    for (int s = 0; s < 3; s++) {
        dV[3 * s + 0] = normal.x + dN[9 * s + 1] * cen.y + dN[9 * s + 2] * cen.z;
        dV[3 * s + 1] = normal.y + dN[9 * s + 3] * cen.x + dN[9 * s + 5] * cen.z;
        dV[3 * s + 2] = normal.z + dN[9 * s + 6] * cen.x + dN[9 * s + 7] * cen.y;
    }
}
// Projection of dN on the unit normal (get_d_norms, spring_network.cu:1419-1428).
__device__ __forceinline__ void d_norms(double *dn, const double *dN, double norm, D3 normal) {
    normal = normal * (1.0 / norm);
#pragma unroll
    for (int i = 0; i < 9; i++) dn[i] = dN[3 * i] * normal.x + dN[3 * i + 1] * normal.y + dN[3 * i + 2] * normal.z;
}
// Merge the two triangles' 9-vectors (nodes a,b,c and c,d,a) into the 12-vector
// over nodes (a, b, c, d) the way the reference assembles d_area / d_volume / d_angle.
__device__ __forceinline__ void merge12(double *out, const double *t1, const double *t2) {
#pragma unroll
    for (int j = 0; j < 9; j++) out[j] = t1[j];
#pragma unroll
    for (int j = 0; j < 3; j++) out[j + 6] += t2[j];
#pragma unroll
    for (int j = 3; j < 6; j++) out[j + 6] = t2[j];
#pragma unroll
    for (int j = 6; j < 9; j++) out[j - 6] += t2[j];
}

struct SpringGeom {
    D3 a, b, c, d, normal_a, normal_b;
    double norm_1, norm_2, length;
};

// What one spring's force needs besides the positions of its nodes a, b, c, d:
// the velocities of a and c, and its stress-free constants.
struct SpringConst {
    double area0_1, area0_2, curv0, contour, kspring;
};
__device__ __forceinline__ SpringConst spring_const(const MembraneArgs &A, int s) {
    return {A.area0[2 * s], A.area0[2 * s + 1], A.curv0[s], A.contour[s], A.kspring[s]};
}

// One spring's contributions to its four nodes (o[12]: a, b, c, d), its two
// triangle areas (doubled) and its curvature.  With `initials` the reference
// areas are the current ones (the initial pass writes them first).
__device__ __forceinline__ void spring_core(const MembraneConst &mc, D3 a, D3 b, D3 c, D3 d, D3 va, D3 vcn,
                                            const SpringConst &k, bool initials, double sfc, double vol_coef,
                                            double area_coef, double mad_coef, double *o, double &area_1,
                                            double &area_2, double &curvature_out, double &angle_out) {
    const D3 l = c - a;
    double length = sqrt(dot(l, l));
    const D3 normal_a = cross(b - a, c - a), normal_b = cross(c - a, d - a);
    const double norm_1 = sqrt(dot(normal_a, normal_a)), norm_2 = sqrt(dot(normal_b, normal_b));
    double dN1[27], dN2[27], dV1[9], dV2[9], dn1[9], dn2[9];
    d_normals(a, b, c, normal_a, dN1, dV1);
    d_normals(c, d, a, normal_b, dN2, dV2);
    d_norms(dn1, dN1, norm_1, normal_a);
    d_norms(dn2, dN2, norm_2, normal_b);
    double d_area[12], d_volume[12];
    merge12(d_area, dn1, dn2);
#pragma unroll
    for (int j = 0; j < 12; j++) d_area[j] *= 0.166666666666666666666666666666666666666666;
    merge12(d_volume, dV1, dV2);
#pragma unroll
    for (int j = 0; j < 12; j++) d_volume[j] *= (1.0 / 18.0);
    double cos_angle = dot(normal_a, normal_b) / (norm_1 * norm_2);
    cos_angle = fmin(cos_angle, 1.0);
    cos_angle = fmax(cos_angle, -1.0);
    const D3 centroid_1 = tri_centroid(a, b, c);
    const D3 centroid_2 = tri_centroid(a, c, d) - centroid_1;
    const double angle_direction = dot(normal_a, centroid_2);
    double angle = acos(cos_angle);
    angle = ((angle_direction < 0) - (angle_direction > 0)) * angle;
    angle_out = angle;
    double d_angle_1[9], d_angle_2[9], d_angle[12];
    {
        const double inv_n1 = 1.0 / norm_1, inv_n2 = 1.0 / norm_2, inv_len = 1.0 / length;
        const D3 h = cross(normal_a * inv_n1, l * inv_len);
#pragma unroll
        for (int j = 0; j < 9; j++)
            d_angle_1[j] = -inv_n1 * (h.x * dN1[j * 3] + h.y * dN1[j * 3 + 1] + h.z * dN1[j * 3 + 2]);
        const D3 h2 = cross(l * inv_len, normal_b * inv_n2);
#pragma unroll
        for (int j = 0; j < 9; j++)
            d_angle_2[j] = -inv_n2 * (h2.x * dN2[j * 3] + h2.y * dN2[j * 3 + 1] + h2.z * dN2[j * 3 + 2]);
    }
    merge12(d_angle, d_angle_1, d_angle_2);
    c = c - a;
    length = sqrt(dot(c, c));
    const D3 dL_ds = c * (1.0 / length);
    double d_curve[12];
#pragma unroll
    for (int j = 0; j < 12; j++) d_curve[j] = d_angle[j] * length;
    d_curve[0] = d_curve[0] - dL_ds.x * angle;
    d_curve[1] = d_curve[1] - dL_ds.y * angle;
    d_curve[2] = d_curve[2] - dL_ds.z * angle;
    d_curve[6] = d_curve[6] + dL_ds.x * angle;
    d_curve[7] = d_curve[7] + dL_ds.y * angle;
    d_curve[8] = d_curve[8] + dL_ds.z * angle;

    D3 fa = {0, 0, 0}, fb = {0, 0, 0}, fc = {0, 0, 0}, fd = {0, 0, 0};
    // local + global area
    double lac = -1 * mc.local_area_modulus * (norm_1 / (initials ? norm_1 : k.area0_1) - 1) + area_coef;
    fb.x += lac * dn1[3]; fb.y += lac * dn1[4]; fb.z += lac * dn1[5];
    lac = -1 * mc.local_area_modulus * (norm_2 / (initials ? norm_2 : k.area0_2) - 1) + area_coef;
    fd.x += lac * dn2[3]; fd.y += lac * dn2[4]; fd.z += lac * dn2[5];
    // volume
    fa.x += vol_coef * d_volume[0]; fa.y += vol_coef * d_volume[1]; fa.z += vol_coef * d_volume[2];
    fb.x += vol_coef * d_volume[3]; fb.y += vol_coef * d_volume[4]; fb.z += vol_coef * d_volume[5];
    fc.x += vol_coef * d_volume[6]; fc.y += vol_coef * d_volume[7]; fc.z += vol_coef * d_volume[8];
    fd.x += vol_coef * d_volume[9]; fd.y += vol_coef * d_volume[10]; fd.z += vol_coef * d_volume[11];
    // membrane viscosity (Osay form)
    {
        const D3 vc = vcn - va;
        const D3 visc = dL_ds * (-dot(dL_ds, vc) * (4.0 / 1.7320508075688772) * mc.viscosity);  // 4 / sqrt(3)
        fc = fc + visc;
        fa = fa - visc;
    }
    // curvature and bending
    const double spring_area_total = (norm_1 + norm_2) * kSixth;
    area_1 = norm_1;
    area_2 = norm_2;
    const double curvature = angle * length / spring_area_total;
    curvature_out = curvature;
    const double c0 = k.curv0;
    const double lbc = -0.5 * mc.local_bending_modulus * (c0 - curvature) * (c0 - curvature);
    fa.x += lbc * d_area[0]; fa.y += lbc * d_area[1]; fa.z += lbc * d_area[2];
    fb.x += lbc * d_area[3]; fb.y += lbc * d_area[4]; fb.z += lbc * d_area[5];
    fc.x += lbc * d_area[6]; fc.y += lbc * d_area[7]; fc.z += lbc * d_area[8];
    fd.x += lbc * d_area[9]; fd.y += lbc * d_area[10]; fd.z += lbc * d_area[11];
    const double cc = -1 * mc.global_bending_modulus * (curvature - c0) + mad_coef;
    fa.x += cc * d_curve[0]; fa.y += cc * d_curve[1]; fa.z += cc * d_curve[2];
    fb.x += cc * d_curve[3]; fb.y += cc * d_curve[4]; fb.z += cc * d_curve[5];
    fc.x += cc * d_curve[6]; fc.y += cc * d_curve[7]; fc.z += cc * d_curve[8];
    fd.x += cc * d_curve[9]; fd.y += cc * d_curve[10]; fd.z += cc * d_curve[11];
    // WLC stretching
    const double sr = length / k.contour;
    const double fcoef = -1 * k.kspring * ((0.25 / ((1.0 - sr) * (1.0 - sr))) - 0.25 + sr - sfc);
    fc = fc + dL_ds * fcoef;
    fa = fa - dL_ds * fcoef;
    o[0] = fa.x; o[1] = fa.y; o[2] = fa.z;
    o[3] = fb.x; o[4] = fb.y; o[5] = fb.z;
    o[6] = fc.x; o[7] = fc.y; o[8] = fc.z;
    o[9] = fd.x; o[10] = fd.y; o[11] = fd.z;
}

// Spring s from the node arrays: forces into contrib[12 s], areas and
// curvature into area / curv; the initial pass also records the reference
// angle and areas.
__device__ void spring_forces(const MembraneArgs &A, const MembraneConst &mc, const MembraneScalars &ms, int s,
                              bool initials, double sfc, double vol_coef, double area_coef, double mad_coef) {
    const int na = A.spring[4 * s], nb = A.spring[4 * s + 1], ncn = A.spring[4 * s + 2], nd = A.spring[4 * s + 3];
    const D3 a = d3(A.x[na], A.y[na], A.z[na]), b = d3(A.x[nb], A.y[nb], A.z[nb]);
    const D3 c = d3(A.x[ncn], A.y[ncn], A.z[ncn]), d = d3(A.x[nd], A.y[nd], A.z[nd]);
    const D3 va = d3(A.vx[na], A.vy[na], A.vz[na]), vc = d3(A.vx[ncn], A.vy[ncn], A.vz[ncn]);
    const SpringConst k = initials ? SpringConst{0.0, 0.0, A.curv0[s], A.contour[s], A.kspring[s]} : spring_const(A, s);
    double area_1, area_2, curvature, angle;
    spring_core(mc, a, b, c, d, va, vc, k, initials, sfc, vol_coef, area_coef, mad_coef, A.contrib + 12 * (size_t)s,
                area_1, area_2, curvature, angle);
    if (initials) {
        A.angle0[s] = angle;
        A.area0[2 * s] = area_1;
        A.area0[2 * s + 1] = area_2;
    }
    A.area[2 * s] = area_1;
    A.area[2 * s + 1] = area_2;
    A.curv[s] = curvature;
}

// Stress-free reference pass: get_contour_lengths (spring_network.cu:516-604)
// with get_spring_constant / get_pivkin_spring_constant (:1600-1634), and
// get_reference_curvatures (:389-513).
__device__ void spring_reference(const MembraneArgs &A, const MembraneConst &mc, int s) {
    const int na = A.spring[4 * s], nb = A.spring[4 * s + 1], ncn = A.spring[4 * s + 2], nd = A.spring[4 * s + 3];
    const D3 a = d3(A.x[na], A.y[na], A.z[na]), b = d3(A.x[nb], A.y[nb], A.z[nb]);
    D3 c = d3(A.x[ncn], A.y[ncn], A.z[ncn]);
    const D3 d = d3(A.x[nd], A.y[nd], A.z[nd]);
    D3 l = c - a;
    double length = sqrt(dot(l, l));
    const double cons_wlc = (0.5 * pow(1.0 - 1 / mc.wlc_ratio, -3.0) + 1.0);
    if (mc.pivkin_length) {
        A.kspring[s] = ((4.0 * mc.wlc_ratio * mc.reference_length * mc.shear_modulus) / (sqrt(3.0) * cons_wlc));
        A.contour[s] = mc.reference_length * mc.wlc_ratio;
    } else {
        A.kspring[s] = ((4.0 * mc.wlc_ratio * length * mc.shear_modulus) / (sqrt(3.0) * cons_wlc));
        A.contour[s] = length * mc.wlc_ratio;
    }
    const D3 normal_a = cross(b - a, c - a), normal_b = cross(c - a, d - a);
    const double norm_1 = sqrt(dot(normal_a, normal_a)), norm_2 = sqrt(dot(normal_b, normal_b));
    double cos_angle = dot(normal_a, normal_b) / (norm_1 * norm_2);
    cos_angle = fmin(cos_angle, 1.0);
    cos_angle = fmax(cos_angle, -1.0);
    const D3 centroid_1 = tri_centroid(a, b, c);
    const D3 centroid_2 = tri_centroid(a, c, d) - centroid_1;
    const D3 normal_ba = normal_b - normal_a;
    const double angle_direction = dot(normal_ba, centroid_2);
    double angle = acos(cos_angle);
    angle = ((angle_direction > 0) - (angle_direction < 0)) * angle;
    c = c - a;
    length = sqrt(dot(c, c));
    const double spring_area_total = (norm_1 + norm_2) / 6.0;
    A.curv[s] = angle * length / spring_area_total;
    A.area[2 * s] = norm_1;
    A.area[2 * s + 1] = norm_2;
    A.curv0[s] = mc.sphere_reference ? mc.curvature_ratio / 3.265483301 : 0.0;
    A.angle0[s] = angle;
    A.area0[2 * s] = norm_1;
    A.area0[2 * s + 1] = norm_2;
}

// Stencil tables of node n at position p, by the lanes of one warp: lane l < 12
// writes weight slot l (axis l / 4, offset l % 4; 0 beyond the stencil) and
// lanes 0..2 the first stencil cell per axis.  The sort and the spread read
// them instead of evaluating the delta kernel again.
__device__ __forceinline__ void write_stencil_tables(const MembraneArgs &A, const MembraneConst &mc, int n,
                                                     double x, double y, double z, int lane) {
    const int S = stencil_width(A.ibm_stencil);
    const Stencil st = node_stencil(A, mc, x, y, z);
    if (lane < 12) {
        const int ax = lane >> 2, q = lane & 3;
        const int b = ax == 0 ? st.i0 : (ax == 1 ? st.j0 : st.k0);
        const double r = ax == 0 ? st.rx : (ax == 1 ? st.ry : st.rz);
        A.node_w[12 * (size_t)n + lane] =
            q >= S ? 0.0
                   : (A.ibm_stencil == LBFS_IBM_VANDERMONDE4 ? vandermonde_weight(A, mc, ax, b, r, q)
                                                              : stencil_weight(A.ibm_stencil, b + q + 0.5 - r));
    }
    if (lane < 3) A.node_base[3 * (size_t)n + lane] = lane == 0 ? st.i0 : (lane == 1 ? st.j0 : st.k0);
}

// Tables at the current positions (the adjoint's interpolation transpose).
__global__ void __launch_bounds__(256) k_mem_tables(MembraneArgs A) {
    const int lane = threadIdx.x & 31;
    const int n = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (n >= A.total_nodes) return;
    write_stencil_tables(A, A.mc[A.node_mem[n]], n, A.x[n], A.y[n], A.z[n], lane);
}

// ---- M1: IBM interpolation + advection, one warp per node ----------------
template <typename R>
__global__ void __launch_bounds__(256) k_mem_advect(MembraneArgs A) {
    pdl_trigger();
    const int lane = threadIdx.x & 31;
    const int n = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (n >= A.total_nodes) return;
    const MembraneConst &mc = A.mc[A.node_mem[n]];
    const double x = A.x[n], y = A.y[n], z = A.z[n];
    const Stencil st = node_stencil(A, mc, x, y, z);
    const int n_inst = mc.gnx * mc.gny * mc.gnz;
    const int S = stencil_width(A.ibm_stencil);
    const int cells = S * S * S;
    // the 3 S one-dimensional weights, one per lane (lane = axis * S + offset)
    double w1 = 0.0;
    if (lane < 3 * S) {
        const int ax = lane / S, q = lane - ax * S;
        const int b = ax == 0 ? st.i0 : (ax == 1 ? st.j0 : st.k0);
        const double r = ax == 0 ? st.rx : (ax == 1 ? st.ry : st.rz);
        w1 = A.ibm_stencil == LBFS_IBM_VANDERMONDE4 ? vandermonde_weight(A, mc, ax, b, r, q)
                                                    : stencil_weight(A.ibm_stencil, b + q + 0.5 - r);
    }
    double v[3] = {0.0, 0.0, 0.0};
    for (int c0 = 0; c0 < cells; c0 += 32) {
        // cell c of the stencil, z fastest as in the reference's i, j, k loop nest
        const int c = c0 + lane;
        const int di = (c / (S * S)) % S, dj = (c / S) % S, dk = c % S;
        const double wx = __shfl_sync(0xffffffffu, w1, di);
        const double wy = __shfl_sync(0xffffffffu, w1, S + dj);
        const double wz = __shfl_sync(0xffffffffu, w1, 2 * S + dk);
        if (c >= cells) continue;
        const int i = st.i0 + di, j = st.j0 + dj, k = st.k0 + dk;
        const int lidx = i + j * mc.gnx + k * mc.gny * mc.gnx;
        if (lidx < n_inst && lidx >= 0) {
            const int idx = mc.cell0 + lidx;
            double u, vv, w;
            read_velocity<R>(A.state, idx, u, vv, w);
            v[0] += u * wx * wy * wz;
            v[1] += vv * wx * wy * wz;
            v[2] += w * wx * wy * wz;
        }
    }
#pragma unroll
    for (int c = 0; c < 3; c++)
        for (int o = 16; o > 0; o >>= 1) v[c] += __shfl_down_sync(0xffffffffu, v[c], o);
    const double dt = A.dt_dev ? __ldcg(A.dt_dev) : A.delta_t;
    const double xp = x + v[0] * dt, yp = y + v[1] * dt, zp = z + v[2] * dt;
    if (lane == 0) {
        A.vx[n] = v[0];
        A.vy[n] = v[1];
        A.vz[n] = v[2];
        A.x[n] = xp;
        A.y[n] = yp;
        A.z[n] = zp;
    }
    // stencil tables at the advected position (lane 0 holds the sums)
    write_stencil_tables(A, mc, n, __shfl_sync(0xffffffffu, xp, 0), __shfl_sync(0xffffffffu, yp, 0),
                         __shfl_sync(0xffffffffu, zp, 0), lane);
}

// ---- M2: spring forces, one thread per spring, blocks per membrane ----------
// Every block first forms its membrane's totals V and A over all triangles (the
// same fixed-order sum in every block, so all blocks agree bit for bit), then
// its springs' forces; the per-block MAD partials (curvature x area over the
// first n_nodes springs) are summed by the membrane's last block to finish.
// Reference mode: the stress-free pass (contour lengths, spring constants,
// reference curvatures).
// ---- M2: membrane totals, one CTA per membrane ------------------------------
// Volume and area: per-thread sums over triangles t, t + blockDim, ..., then
// the block tree (fixed order).  Written to ms.Vc / ms.Ac for the spring
// kernel, which every spring block reads instead of forming them again.
constexpr int kTotalsThreads = 512;
__global__ void __launch_bounds__(kTotalsThreads) k_mem_totals(MembraneArgs A) {
    __shared__ double sh[33];
    pdl_trigger();
    const int m = blockIdx.x;
    const MembraneConst mc = A.mc[m];
    // four triangles per round; the first round's indices (constant) are loaded
    // before the wait for the advected positions
    int tn[4][3];
    auto load_tris = [&](int l0) {
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const int t = mc.tri0 + (l0 + k * (int)blockDim.x < mc.n_tris ? l0 + k * (int)blockDim.x : 0);
#pragma unroll
            for (int q = 0; q < 3; q++) tn[k][q] = A.tri[3 * (size_t)t + q];
        }
    };
    load_tris(threadIdx.x);
    pdl_wait();
    double pv = 0.0, pa = 0.0;
    for (int l0 = threadIdx.x; l0 < mc.n_tris; l0 += 4 * blockDim.x) {
        if (l0 != (int)threadIdx.x) load_tris(l0);
        D3 p[4][3];
#pragma unroll
        for (int k = 0; k < 4; k++)
#pragma unroll
            for (int q = 0; q < 3; q++) p[k][q] = d3(A.x[tn[k][q]], A.y[tn[k][q]], A.z[tn[k][q]]);
#pragma unroll
        for (int k = 0; k < 4; k++) {
            if (l0 + k * (int)blockDim.x >= mc.n_tris) break;
            const D3 a = p[k][0], b = p[k][1], c = p[k][2];
            const D3 normal = cross(b - a, c - a);
            pv += dot(normal, tri_centroid(a, b, c)) * kSixth;
            pa += sqrt(dot(normal, normal)) * 0.5;
        }
    }
    const double V = block_sum(pv, sh), Ar = block_sum(pa, sh);
    if (threadIdx.x == 0) {
        A.ms[m].Vc = V;
        A.ms[m].Ac = Ar;
    }
}

__global__ void __launch_bounds__(128) k_mem_springs(MembraneArgs A) {
    __shared__ double sh[33];
    __shared__ bool last_block;
    pdl_trigger();
    const int m = blockIdx.y;
    const MembraneConst mc = A.mc[m];
    const int first = blockIdx.x * blockDim.x;
    if (first >= mc.n_springs) return;  // whole block idle for this membrane
    const int ls = first + threadIdx.x;
    const int s = mc.spring0 + ls;
    if (A.mode == kModeReference) {
        if (ls < mc.n_springs) spring_reference(A, mc, s);
        return;
    }
    MembraneScalars *ms = A.ms + m;
    const bool initials = A.mode == kModeInitial;
    // the spring's nodes and stress-free constants (not written during a step)
    // before the wait for the totals and the advected positions
    int sn[4] = {0, 0, 0, 0};
    SpringConst sk{};
    if (ls < mc.n_springs && !initials) {
#pragma unroll
        for (int q = 0; q < 4; q++) sn[q] = A.spring[4 * (size_t)s + q];
        sk = spring_const(A, s);
    }
    pdl_wait();
    const double V = ms->Vc, Ar = ms->Ac;  // k_mem_totals of this launch sequence
    const double V0 = initials ? V * mc.volume_ratio : ms->V0;
    const double A0 = initials ? Ar : ms->A0;
    const double MADp = initials ? 0.0 : ms->MAD, MAD0p = initials ? 0.0 : ms->MAD0;
    const double wr = mc.wlc_ratio;
    const double sfc = (0.25 * wr * wr / ((wr - 1.0) * (wr - 1.0)) - 0.25 + 1.0 / wr);
    const double vol_coef = -1 * mc.volume_modulus * (V / V0 - 1.0) / 6.0;
    const double area_coef = -1 * mc.global_area_modulus * (Ar / A0 - 1.0);
    const double mad_coef = -1 * 2.0 * mc.global_bending_modulus * (MADp - MAD0p) / A0;
    double pm = 0.0;
    if (ls < mc.n_springs) {
        if (initials) {
            MembraneScalars cur = *ms;
            spring_forces(A, mc, cur, s, initials, sfc, vol_coef, area_coef, mad_coef);
        } else {
            const D3 a = d3(A.x[sn[0]], A.y[sn[0]], A.z[sn[0]]), b = d3(A.x[sn[1]], A.y[sn[1]], A.z[sn[1]]);
            const D3 c = d3(A.x[sn[2]], A.y[sn[2]], A.z[sn[2]]), d = d3(A.x[sn[3]], A.y[sn[3]], A.z[sn[3]]);
            const D3 va = d3(A.vx[sn[0]], A.vy[sn[0]], A.vz[sn[0]]), vc = d3(A.vx[sn[2]], A.vy[sn[2]], A.vz[sn[2]]);
            double area_1, area_2, curvature, angle;
            spring_core(mc, a, b, c, d, va, vc, sk, false, sfc, vol_coef, area_coef, mad_coef, A.contrib + 12 * (size_t)s,
                        area_1, area_2, curvature, angle);
            A.area[2 * s] = area_1;
            A.area[2 * s + 1] = area_2;
            A.curv[s] = curvature;
        }
        if (ls < mc.n_nodes) pm = A.curv[s] * (A.area[2 * s] + A.area[2 * s + 1]) * 1 / 3;
    }
    const double part = block_sum(pm, sh);
    double *partials = A.mad_partials + (size_t)m * kMaxSpringBlocks;
    if (threadIdx.x == 0) {
        partials[blockIdx.x] = part;
        __threadfence();
        const int nblk = (mc.n_springs + blockDim.x - 1) / blockDim.x;
        last_block = atomicAdd(A.mad_ticket + m, 1u) == (unsigned)(nblk - 1);
    }
    __syncthreads();
    if (!last_block) return;
    __threadfence();
    if (threadIdx.x == 0) {
        const int nblk = (mc.n_springs + blockDim.x - 1) / blockDim.x;
        double sum = 0.0;
        for (int b = 0; b < nblk; b++) sum += __ldcg(partials + b);
        const double MAD = sum / Ar;
        ms->V = V;
        ms->A = Ar;
        ms->MAD = MAD;
        if (initials) { ms->V0 = V0; ms->A0 = A0; ms->MAD0 = MAD; }
        A.mad_ticket[m] = 0u;
    }
}

// ---- M3: node forces, one thread per node, contributions in spring order ----
__global__ void __launch_bounds__(128) k_mem_nodeforce(MembraneArgs A) {
    pdl_trigger();
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= A.total_nodes) return;
    // the node's incidence (constant) before the wait for the spring kernel's contributions
    const int e0 = A.inc_start[n], e1 = A.inc_start[n + 1];
    int code[16];
#pragma unroll
    for (int q = 0; q < 16; q++) code[q] = (e0 + q < e1) ? __ldg(A.inc + e0 + q) : -1;
    pdl_wait();
    double f[3] = {0.0, 0.0, 0.0};
    for (int c0 = e0; c0 < e1; c0 += 16) {
        if (c0 != e0) {
#pragma unroll
            for (int q = 0; q < 16; q++) code[q] = (c0 + q < e1) ? __ldg(A.inc + c0 + q) : -1;
        }
        double d[16][3];
#pragma unroll
        for (int q = 0; q < 16; q++) {
            if (code[q] >= 0) {
                const double *o = A.contrib + 12 * (size_t)(code[q] >> 2) + 3 * (code[q] & 3);
                d[q][0] = o[0]; d[q][1] = o[1]; d[q][2] = o[2];
            }
        }
#pragma unroll
        for (int q = 0; q < 16; q++)
            if (code[q] >= 0) { f[0] += d[q][0]; f[1] += d[q][1]; f[2] += d[q][2]; }
    }
    A.fx[n] = f[0];
    A.fy[n] = f[1];
    A.fz[n] = f[2];
}

// ---- M4: node bounds, nodes sorted by stencil base cell ---------------------
// One CTA per membrane; needs only the advected positions, so it runs beside
// M2.  Finds the patch (bounding box of the stencils), counts the nodes per
// stencil bin in shared memory, writes for every bin b of the patch the first
// sorted position whose bin is >= b, and the nodes in (bin, node) order.  The
// last CTA of the launch writes the prefix of patch cells over the membranes
// (the spread kernel's work list).
// The membrane's nodes in sorted order (global node indices): the spread reads
// each contribution's stencil weights and force through it.
__device__ __forceinline__ void write_sorted_nodes(const MembraneArgs &A, const MembraneConst &mc, const int *list) {
    for (int e = threadIdx.x; e < mc.n_nodes; e += blockDim.x) A.sorted_node[mc.node0 + e] = mc.node0 + list[e];
}

// Exclusive prefix sum of one int per thread over the CTA, and the CTA's
// total: a shuffle scan within each warp, the warp totals scanned by warp 0,
// two barriers (in place of a Hillis-Steele scan over the whole CTA, whose
// 2 log2(threads) barriers dominated the node sort).
__device__ int block_exclusive_scan(int v, int *total) {
    __shared__ int warp_sum[kMembraneThreads / 32 + 1];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, n_warps = (blockDim.x + 31) >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sum[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int w = lane < n_warps ? warp_sum[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < n_warps) warp_sum[lane] = w;  // inclusive prefix of the warp totals
    }
    __syncthreads();
    const int before = warp == 0 ? 0 : warp_sum[warp - 1];
    *total = warp_sum[n_warps - 1];
    const int r = before + x - v;
    __syncthreads();  // warp_sum is reused by the next call
    return r;
}

// Node bounds of a membrane for the patch and the sort: per thread over
// nodes ln = first, first + stride, ... (min of positions, minus max of
// positions, min and minus max of the first stencil cells), the range flag,
// and whether every first cell is sane; then reduced over the CTA
// (minima are exact, so any order gives the same result).  out[12] valid in
// every thread on return.
// One node's position p and first stencil cells b into the running bounds v[12].
__device__ __forceinline__ void bounds_add(double (&v)[12], const double (&p)[3], const int (&b)[3], int S,
                                           const MembraneConst &mc, unsigned int &range_flag, bool &base_range) {
    const int gn[3] = {mc.gnx, mc.gny, mc.gnz};
    for (int c = 0; c < 3; c++) {
        v[c] = fmin(v[c], p[c]);            // lower bound
        v[3 + c] = fmin(v[3 + c], -p[c]);   // minus upper bound
        v[6 + c] = fmin(v[6 + c], (double)b[c]);
        v[9 + c] = fmin(v[9 + c], -(double)b[c]);
        if (b[c] < 0 || b[c] + S > gn[c]) range_flag = LBFS_FLAG_IBM_RANGE;
        if (b[c] < -(1 << 19) || b[c] > (1 << 19)) base_range = false;
    }
}

// The threads' bounds v[12], range flags and sanity reduced over the CTA;
// out[12] valid in every thread on return.
__device__ void bounds_reduce(const double (&v)[12], unsigned int range_flag, bool base_range, double *out,
                              unsigned int *flag_out, int *sane_out) {
    __shared__ double shv[kMembraneThreads / 32][12];
    __shared__ unsigned int sflag;
    __shared__ int ssane;
    if (threadIdx.x == 0) { sflag = 0u; ssane = 1; }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < 12; q++) {
        double x = v[q];
        for (int o = 16; o > 0; o >>= 1) x = fmin(x, __shfl_down_sync(0xffffffffu, x, o));
        if (lane == 0) shv[warp][q] = x;
    }
    __syncthreads();
    if (range_flag) atomicOr(&sflag, range_flag);
    if (!base_range) ssane = 0;
    if (threadIdx.x < 12) {
        double x = shv[0][threadIdx.x];
        for (int w = 1; w < (int)(blockDim.x >> 5); w++) x = fmin(x, shv[w][threadIdx.x]);
        shv[0][threadIdx.x] = x;
    }
    __syncthreads();
    for (int q = 0; q < 12; q++) out[q] = shv[0][q];
    *flag_out = sflag;
    *sane_out = ssane;
    __syncthreads();
}

__device__ void node_bounds(const MembraneArgs &A, const MembraneConst &mc, int first, int stride, double *out,
                            unsigned int *flag_out, int *sane_out) {
    const int S = stencil_width(A.ibm_stencil);
    double v[12];
    for (int c = 0; c < 12; c++) v[c] = 1e300;
    unsigned int range_flag = 0;
    bool base_range = true;
    // four nodes per round: their loads are issued together
    for (int l0 = first; l0 < mc.n_nodes; l0 += 4 * stride) {
        double p[4][3];
        int b[4][3];
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const int ln = l0 + k * stride;
            const int n = mc.node0 + (ln < mc.n_nodes ? ln : 0);
            p[k][0] = A.x[n]; p[k][1] = A.y[n]; p[k][2] = A.z[n];
            b[k][0] = A.node_base[3 * (size_t)n]; b[k][1] = A.node_base[3 * (size_t)n + 1];
            b[k][2] = A.node_base[3 * (size_t)n + 2];
        }
#pragma unroll
        for (int k = 0; k < 4; k++)
            if (l0 + k * stride < mc.n_nodes) bounds_add(v, p[k], b[k], S, mc, range_flag, base_range);
    }
    bounds_reduce(v, range_flag, base_range, out, flag_out, sane_out);
}

// Patch of a membrane from its node bounds red[12], the prefix of patch
// cells over the membranes (by the last of the n_sorters CTAs to get here),
// and the counting sort of its nodes by stencil bin; one CTA.  `skeys` is the dynamic shared memory of sort_smem_bytes.
__device__ void sort_patch(const MembraneArgs &A, int m, const double *red, bool bases_sane, unsigned int range_flag,
                           int n_sorters, unsigned long long *skeys) {
    __shared__ bool last_sorted;
    const MembraneConst mc = A.mc[m];
    MembraneScalars *ms = A.ms + m;
    const int S = stencil_width(A.ibm_stencil);
    int plo[3], bdim[3], pdim[3];
    for (int c = 0; c < 3; c++) {
        plo[c] = (int)red[6 + c];
        bdim[c] = (int)(-red[9 + c]) - plo[c] + 1;
        pdim[c] = bdim[c] + S - 1;
    }
    const long long pcells = (long long)pdim[0] * pdim[1] * pdim[2];
    const bool overflow = pcells > mc.patch_bound || mc.n_nodes == 0 || !bases_sane || plo[2] < A.ibm_z_lo ||
                          plo[2] + pdim[2] > A.ibm_z_hi;
    if (threadIdx.x == 0) {
        if (range_flag) atomicOr(A.flags, range_flag);
        for (int c = 0; c < 3; c++) {
            ms->bbox_lo[c] = red[c];
            ms->bbox_hi[c] = -red[3 + c];
            ms->patch_lo[c] = plo[c];
            ms->patch_dim[c] = pdim[c];
        }
        ms->patch_cells = overflow ? 0 : (int)pcells;
        if (overflow) atomicOr(A.flags, LBFS_FLAG_IBM_RANGE);
        __threadfence();
        last_sorted = atomicAdd(A.sort_ticket, 1u) == (unsigned)(n_sorters - 1);
    }
    __syncthreads();
    if (last_sorted) {
        // every patch is known: prefix of patch cells over the membranes
        __threadfence();
        const int M = n_sorters;
        const int per = (M + blockDim.x - 1) / blockDim.x;
        const int m0 = min(M, (int)threadIdx.x * per), m1 = min(M, m0 + per);
        int local = 0;
        for (int q = m0; q < m1; q++) local += __ldcg(&A.ms[q].patch_cells);
        int total = 0;
        int run = block_exclusive_scan(local, &total);
        for (int q = m0; q < m1; q++) {
            A.cell_start[q] = run;
            run += __ldcg(&A.ms[q].patch_cells);
        }
        if (threadIdx.x == 0) {
            A.cell_start[M] = total;
            *A.sort_ticket = 0u;
        }
    }
    if (overflow) return;
    // counting sort of the nodes by stencil bin: counts, exclusive prefix
    // (bin_start), placement, then each bin's few nodes in index order, so the
    // result is the (bin, node) order whatever order the atomics took
    const int nbins = bdim[0] * bdim[1] * bdim[2];
    int *bin_start = A.bin_start + (size_t)ms->patch_off + m;
    int *cursor = A.bin_cursor + (size_t)ms->patch_off + m;
    int *bins = reinterpret_cast<int *>(skeys);
    int *list = bins + A.sort_capacity;
    const bool in_smem = nbins + 1 <= kSortBinsSmem;
    // counts and cursors in shared memory when the patch's bins fit, else in global memory
    int *cnt = in_smem ? list + A.sort_capacity : bin_start;
    for (int b = threadIdx.x; b <= nbins; b += blockDim.x) cnt[b] = 0;
    __syncthreads();
    for (int l0 = threadIdx.x; l0 < mc.n_nodes; l0 += 4 * blockDim.x) {  // four nodes' loads per round
        int bb[4][3];
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const int ln = l0 + k * blockDim.x;
            const int *src = A.node_base + 3 * (size_t)(mc.node0 + (ln < mc.n_nodes ? ln : 0));
#pragma unroll
            for (int q = 0; q < 3; q++) bb[k][q] = __ldcg(src + q);
        }
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const int ln = l0 + k * blockDim.x;
            if (ln >= mc.n_nodes) break;
            const int bin = (bb[k][0] - plo[0]) + bdim[0] * ((bb[k][1] - plo[1]) + bdim[1] * (bb[k][2] - plo[2]));
            bins[ln] = bin;
            atomicAdd(cnt + bin, 1);
        }
    }
    __syncthreads();
    {
        const int count = nbins + 1;
        const int per = (count + blockDim.x - 1) / blockDim.x;
        const int b0 = min(count, (int)threadIdx.x * per), b1 = min(count, b0 + per);
        int local = 0;
        // global counts were formed by atomics: L2 loads
        for (int b = b0; b < b1; b++) local += in_smem ? cnt[b] : __ldcg(cnt + b);
        int total_unused = 0;
        int run = block_exclusive_scan(local, &total_unused);
        int *cur = in_smem ? cnt : cursor;
        for (int b = b0; b < b1; b++) {
            const int c = in_smem ? cnt[b] : __ldcg(cnt + b);
            bin_start[b] = run;  // the spread's bin table
            cur[b] = run;        // placement cursor
            run += c;
        }
    }
    __syncthreads();
    int *cur = in_smem ? cnt : cursor;
    for (int ln = threadIdx.x; ln < mc.n_nodes; ln += blockDim.x) list[atomicAdd(cur + bins[ln], 1)] = ln;
    __syncthreads();
    // each bin in node-index order; after the placement cur[b] is the end of
    // bin b, the start of bin b + 1
    for (int b = threadIdx.x; b < nbins; b += blockDim.x) {
        const int lo = b == 0 ? 0 : (in_smem ? cur[b - 1] : __ldcg(cur + b - 1));
        const int hi = in_smem ? cur[b] : __ldcg(cur + b);  // global cursors were moved by atomics
        for (int i = lo + 1; i < hi; i++) {
            const int v = list[i];
            int j = i - 1;
            while (j >= lo && list[j] > v) {
                list[j + 1] = list[j];
                j--;
            }
            list[j + 1] = v;
        }
    }
    __syncthreads();
    write_sorted_nodes(A, mc, list);
}

constexpr int kSortThreads = kMembraneThreads;
__global__ void __launch_bounds__(kSortThreads) k_mem_sort(MembraneArgs A) {
    extern __shared__ unsigned long long skeys[];  // 2 int arrays of sort_capacity: bins, sorted list
    const int m = blockIdx.x;
    double red[12];
    unsigned int flag;
    int sane;
    node_bounds(A, A.mc[m], threadIdx.x, blockDim.x, red, &flag, &sane);
    sort_patch(A, m, red, sane != 0, flag, gridDim.x, skeys);
}

// ---- the membrane step as one thread-block cluster per membrane -------------
// After the advection kernel, one cluster of CL CTAs of TPB threads per
// membrane does the work of k_mem_totals, k_mem_springs, k_mem_nodeforce and
// k_mem_sort (four launches whose phases are each a few dependent memory round
// trips, so that the launches and the waits between them set the chain's
// length); the spread follows.
//  rank 0: node bounds, the patch and the node sort.
//  ranks 1..: every node position into shared memory, V and A over all
//     triangles (each CTA the same fixed-order sum, so they agree bit for
//     bit), the spring forces and the MAD terms.
//  -- cluster barrier (release / acquire): contributions and MAD partials
//  all: MAD, the node forces in spring order.
// Every sum has a fixed order that does not depend on the membrane's place in
// an ensemble.  Shared memory: step_smem_bytes.
constexpr int kStepMaxNodes = 8192;  // 24 bytes of shared memory per node
constexpr int kStepThreads = 128;

__device__ __forceinline__ void prefetch_l2(const void *p) {
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

template <int CL, int TPB>
__global__ void __launch_bounds__(TPB) k_mem_step(MembraneArgs A) {
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    extern __shared__ unsigned long long sdyn[];  // rank 0: the node sort's arrays; ranks 1..: node positions
    __shared__ double sh[33];
    __shared__ double part_va[2], part_mad[1], mad_all;
    const int m = blockIdx.y;
    const int rank = (int)cluster.block_rank();
    const int nth = CL * TPB, tid = rank * TPB + threadIdx.x;
    const MembraneConst mc = A.mc[m];
    MembraneScalars *ms = A.ms + m;
    // no early trigger: the spread behind it is a full-GPU grid whose waiting
    // blocks would hold SMs the fluid kernels use; it launches at completion
    double pm = 0.0;
    if (rank == 0) {
        double red[12];
        unsigned int flag;
        int sane;
        pdl_wait();
        node_bounds(A, mc, threadIdx.x, TPB, red, &flag, &sane);
        sort_patch(A, m, red, sane != 0, flag, gridDim.y, sdyn);
    } else {
        // this thread's first spring (ls0), its nodes, constants and end velocities
        const int spring_stride = (CL - 1) * TPB;
        const int ls0 = tid - TPB;
        int sn[4] = {0, 0, 0, 0};
        SpringConst sk{};
        D3 va{0.0, 0.0, 0.0}, vc{0.0, 0.0, 0.0};
        if (ls0 < mc.n_springs) {  // spring tables: not written during a step
            const int sp = mc.spring0 + ls0;
#pragma unroll
            for (int q = 0; q < 4; q++) sn[q] = A.spring[4 * (size_t)sp + q];
            sk = spring_const(A, sp);
        }
        pdl_wait();  // the advected positions and velocities
        if (ls0 < mc.n_springs) {
            va = d3(A.vx[sn[0]], A.vy[sn[0]], A.vz[sn[0]]);
            vc = d3(A.vx[sn[2]], A.vy[sn[2]], A.vz[sn[2]]);
        }
        {   // the incidence table for the node forces into L2 meanwhile
            const char *i0 = reinterpret_cast<const char *>(A.inc + mc.inc0);
            const char *i1 = reinterpret_cast<const char *>(A.inc + mc.inc0 + 4 * (size_t)mc.n_springs);
            for (const char *p = i0 + 128 * (size_t)(tid - TPB); p < i1; p += 128 * (size_t)(nth - TPB)) prefetch_l2(p);
        }
        const double V0 = ms->V0, A0 = ms->A0, MADp = ms->MAD, MAD0p = ms->MAD0;
        double *px = reinterpret_cast<double *>(sdyn), *py = px + mc.n_nodes, *pz = py + mc.n_nodes;
#pragma unroll 4
        for (int ln = threadIdx.x; ln < mc.n_nodes; ln += TPB) {
            const int n = mc.node0 + ln;
            px[ln] = A.x[n];
            py[ln] = A.y[n];
            pz[ln] = A.z[n];
        }
        __syncthreads();
        // volume and area (update_spring_network_tet_parameters + total<128>)
        double pv = 0.0, pa = 0.0;
        for (int l0 = threadIdx.x; l0 < mc.n_tris; l0 += 4 * TPB) {  // four triangles' indices per round
            int tn[4][3];
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const int t = mc.tri0 + (l0 + k * TPB < mc.n_tris ? l0 + k * TPB : 0);
#pragma unroll
                for (int q = 0; q < 3; q++) tn[k][q] = A.tri[3 * (size_t)t + q] - mc.node0;
            }
#pragma unroll
            for (int k = 0; k < 4; k++) {
                if (l0 + k * TPB >= mc.n_tris) break;
                const int na = tn[k][0], nb = tn[k][1], nc = tn[k][2];
                const D3 a = d3(px[na], py[na], pz[na]), b = d3(px[nb], py[nb], pz[nb]), c = d3(px[nc], py[nc], pz[nc]);
                const D3 normal = cross(b - a, c - a);
                pv += dot(normal, tri_centroid(a, b, c)) * kSixth;
                pa += sqrt(dot(normal, normal)) * 0.5;
            }
        }
        const double V = block_sum(pv, sh), Ar = block_sum(pa, sh);
        if (threadIdx.x == 0) {
            part_va[0] = V;
            part_va[1] = Ar;
        }
        // spring forces (get_spring_forces_atomics) and the MAD terms of the first n_nodes springs
        const double wr = mc.wlc_ratio;
        const double sfc = (0.25 * wr * wr / ((wr - 1.0) * (wr - 1.0)) - 0.25 + 1.0 / wr);
        const double vol_coef = -1 * mc.volume_modulus * (V / V0 - 1.0) / 6.0;
        const double area_coef = -1 * mc.global_area_modulus * (Ar / A0 - 1.0);
        const double mad_coef = -1 * 2.0 * mc.global_bending_modulus * (MADp - MAD0p) / A0;
        for (int ls = ls0; ls < mc.n_springs; ls += spring_stride) {
            const int sp = mc.spring0 + ls;
            if (ls != ls0) {  // springs past the first pass: loaded now
#pragma unroll
                for (int q = 0; q < 4; q++) sn[q] = A.spring[4 * (size_t)sp + q];
                sk = spring_const(A, sp);
                va = d3(A.vx[sn[0]], A.vy[sn[0]], A.vz[sn[0]]);
                vc = d3(A.vx[sn[2]], A.vy[sn[2]], A.vz[sn[2]]);
            }
            const int la = sn[0] - mc.node0, lb = sn[1] - mc.node0, lc = sn[2] - mc.node0, ld = sn[3] - mc.node0;
            double area_1, area_2, curvature, angle;
            spring_core(mc, d3(px[la], py[la], pz[la]), d3(px[lb], py[lb], pz[lb]), d3(px[lc], py[lc], pz[lc]),
                        d3(px[ld], py[ld], pz[ld]), va, vc, sk, false, sfc, vol_coef, area_coef, mad_coef,
                        A.contrib + 12 * (size_t)sp, area_1, area_2, curvature, angle);
            A.area[2 * sp] = area_1;
            A.area[2 * sp + 1] = area_2;
            A.curv[sp] = curvature;
            if (ls < mc.n_nodes) pm += curvature * (area_1 + area_2) * 1 / 3;
        }
    }
    const double bm = block_sum(pm, sh);
    if (threadIdx.x == 0) part_mad[0] = bm;
    cluster.sync();

    // MAD: one warp reads the CL partials (lane r from rank r) and adds them in rank order
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        const double v = lane < CL ? *cluster.map_shared_rank(part_mad, lane) : 0.0;
        double mad = 0.0;
        for (int r = 0; r < CL; r++) mad += __shfl_sync(0xffffffffu, v, r);
        if (lane == 0) mad_all = mad;
    }
    // node forces: each node's contributions in spring order
    for (int ln = tid; ln < mc.n_nodes; ln += nth) {
        const int n = mc.node0 + ln;
        double f[3] = {0.0, 0.0, 0.0};
        const int e0 = A.inc_start[n], e1 = A.inc_start[n + 1];
        for (int c0 = e0; c0 < e1; c0 += 8) {
            int code[8];
#pragma unroll
            for (int q = 0; q < 8; q++) code[q] = (c0 + q < e1) ? __ldg(A.inc + c0 + q) : -1;
            double d[8][3];
#pragma unroll
            for (int q = 0; q < 8; q++) {
                if (code[q] >= 0) {  // written by other CTAs of this launch: L2 loads
                    const double *o = A.contrib + 12 * (size_t)(code[q] >> 2) + 3 * (code[q] & 3);
                    d[q][0] = __ldcg(o);
                    d[q][1] = __ldcg(o + 1);
                    d[q][2] = __ldcg(o + 2);
                }
            }
#pragma unroll
            for (int q = 0; q < 8; q++)
                if (code[q] >= 0) { f[0] += d[q][0]; f[1] += d[q][1]; f[2] += d[q][2]; }
        }
        A.fx[n] = f[0];
        A.fy[n] = f[1];
        A.fz[n] = f[2];
    }
    __syncthreads();
    if (rank == 0 && threadIdx.x == 0) {
        const double *va = cluster.map_shared_rank(part_va, 1);  // V and A as every rank 1.. formed them
        const double V = va[0], Ar = va[1];
        ms->Vc = V;
        ms->Ac = Ar;
        ms->V = V;
        ms->A = Ar;
        ms->MAD = mad_all / Ar;
    }
    cluster.sync();  // no CTA leaves while another may still read its shared memory
}

size_t step_smem_bytes(int sort_capacity, int max_nodes) {
    const size_t sort = sort_smem_bytes(sort_capacity), pos = 3 * sizeof(double) * (size_t)(max_nodes > 0 ? max_nodes : 1);
    return sort > pos ? sort : pos;
}

// ---- M5: spread as a per-cell reduction over the sorted nodes -------------
// One warp per patch cell.  The cell's contributions are the nodes of S*S rows
// of bins (rows in (z, y) order, each row a contiguous range of the sorted
// nodes); lane q of the warp takes contributions q, q + 32, ... of that list,
// then the warp adds the lanes in a fixed tree.  All nodes of a row share the
// stencil's y and z offsets, and a node's record carries its first x cell, so
// the loads of one contribution do not wait on each other.
template <int S>
__global__ void __launch_bounds__(256) k_mem_spread(MembraneArgs A) {
    pdl_wait();
    const int lane = threadIdx.x & 31;
    const int M = A.n_membranes;
    const int total = __ldg(A.cell_start + M);
    const int n_warps = (gridDim.x * blockDim.x) >> 5;
    for (int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < total; t += n_warps) {
        // membrane m with cell_start[m] <= t < cell_start[m + 1]: the warp probes
        // 32 evenly spaced entries of [lo_m, hi_m) per round (one load per lane)
        int lo_m = 0, hi_m = M;
        while (hi_m - lo_m > 1) {
            const int step = (hi_m - lo_m + 31) / 32;
            const int probe = lo_m + lane * step;
            const bool le = probe < hi_m && __ldg(A.cell_start + probe) <= t;
            const unsigned ballot = __ballot_sync(0xffffffffu, le);
            const int last = 31 - __clz(ballot);  // lane 0 always qualifies: cell_start[lo_m] <= t
            lo_m = lo_m + last * step;
            hi_m = min(hi_m, lo_m + step);
        }
        const int m = lo_m;
        const MembraneScalars &ms = A.ms[m];
        const MembraneConst &mc = A.mc[m];
        const int pc = t - __ldg(A.cell_start + m);
        const int pdim[3] = {ms.patch_dim[0], ms.patch_dim[1], ms.patch_dim[2]};
        const int bdim[3] = {pdim[0] - S + 1, pdim[1] - S + 1, pdim[2] - S + 1};
        const int px = pc % pdim[0], py = (pc / pdim[0]) % pdim[1], pz = pc / (pdim[0] * pdim[1]);
        const int ci = ms.patch_lo[0] + px;
        const int *bin_start = A.bin_start + (size_t)ms.patch_off + m;
        const int bx0 = max(px - S + 1, 0), bx1 = min(px, bdim[0] - 1);
        // lane r < S*S: sorted range of row r
        int lo = 0, len = 0;
        if (lane < S * S) {
            const int by = py - S + 1 + lane % S, bz = pz - S + 1 + lane / S;
            if (by >= 0 && by < bdim[1] && bz >= 0 && bz < bdim[2] && bx0 <= bx1) {
                const int row = bdim[0] * (by + bdim[1] * bz);
                lo = __ldg(bin_start + row + bx0);
                len = __ldg(bin_start + row + bx1 + 1) - lo;
            }
        }
        int end = len;  // inclusive prefix of the row lengths
#pragma unroll
        for (int o = 1; o < S * S; o <<= 1) {
            const int x = __shfl_up_sync(0xffffffffu, end, o);
            if (lane >= o) end += x;
        }
        const int count = __shfl_sync(0xffffffffu, end, S * S - 1);
        const int *sorted = A.sorted_node + mc.node0;

        double inv3 = 1 / mc.gdx / mc.gdx / mc.gdx;
        if (A.ibm_stencil == LBFS_IBM_VANDERMONDE4) {
            // divided by the cell's volume (spread_forces_on_non_uniform_grid, immersed_boundary_method.cu:851)
            const int cj = ms.patch_lo[1] + py, ck = ms.patch_lo[2] + pz;
            const int lidx = ci + mc.gnx * (cj + mc.gny * ck);
            inv3 = (ci >= 0 && ci < mc.gnx && cj >= 0 && cj < mc.gny && ck >= 0 && ck < mc.gnz)
                       ? 1.0 / __ldg(A.cell_volume + mc.cell0 + lidx)
                       : 0.0;
        }
        double f[3] = {0.0, 0.0, 0.0};
        for (int q0 = 0; q0 < count; q0 += 32) {
            const int q = q0 + lane;
            int r = 0;  // row of contribution q: rows whose prefix end is <= q come before it
#pragma unroll
            for (int k = 0; k < S * S; k++) r += (__shfl_sync(0xffffffffu, end, k) <= q) ? 1 : 0;
            r = min(r, S * S - 1);
            const int r_end = __shfl_sync(0xffffffffu, end, r), r_len = __shfl_sync(0xffffffffu, len, r);
            const int r_lo = __shfl_sync(0xffffffffu, lo, r);
            if (q < count) {
                const int e = r_lo + q - (r_end - r_len);
                const int node = __ldg(sorted + e);
                const double *w = A.node_w + 12 * (size_t)node;
                const double3 F = make_double3(__ldg(A.fx + node), __ldg(A.fy + node), __ldg(A.fz + node));
                const double wy = __ldg(w + 4 + S - 1 - r % S), wz = __ldg(w + 8 + S - 1 - r / S);
                const double wx = __ldg(w + ci - __ldg(A.node_base + 3 * (size_t)node));
                f[0] += F.x * wx * wy * wz * inv3;
                f[1] += F.y * wx * wy * wz * inv3;
                f[2] += F.z * wx * wy * wz * inv3;
            }
        }
#pragma unroll
        for (int c = 0; c < 3; c++)
            for (int o = 16; o > 0; o >>= 1) f[c] += __shfl_down_sync(0xffffffffu, f[c], o);
        if (lane == 0) {
            double *pf = A.patch_force + ((size_t)ms.patch_off + pc) * 3;
            pf[0] = f[0];
            pf[1] = f[1];
            pf[2] = f[2];
        }
    }
}

// ---- energy diagnostics (Solver_gpu.cu:1073-1136) ------------------------
// One CTA per membrane: the sums over its springs of get_area_energy,
// get_bending_energy and get_spring_energy (spring_network.cu:1687-1768),
// each a fixed-order block sum.  out[3 m + 0..2]: local area, local bending,
// spring (WLC) energy.  As the reference launches them: the area energy uses
// the global area modulus, the bending energy divides by spring_area[i] (the
// i-th entry of the two-per-spring array), the WLC constants take
// 1 / wlc_ratio.
__global__ void __launch_bounds__(kTotalsThreads) k_mem_energies(MembraneArgs A, double *out) {
    __shared__ double sh[33];
    const int m = blockIdx.x;
    const MembraneConst &mc = A.mc[m];
    const double r = 1 / mc.wlc_ratio;
    const double c1 = (0.25 / (1 - r) / (1 - r) - 0.25 + r);
    const double c2 = r * r * (3.0 - 2.0 * r) / (1.0 - r) - 4 * c1 * r;
    double ea = 0.0, eb = 0.0, es = 0.0;
    for (int ls = threadIdx.x; ls < mc.n_springs; ls += blockDim.x) {
        const int i = mc.spring0 + ls;
        const double a0 = A.area[2 * i] - A.area0[2 * i], a1 = A.area[2 * i + 1] - A.area0[2 * i + 1];
        ea += mc.global_area_modulus * 0.5 * (a0 * a0 / A.area0[2 * i] + a1 * a1 / A.area0[2 * i + 1]);
        const double dc = A.curv[i] - A.curv0[i];
        eb += 0.5 * mc.local_bending_modulus * dc * dc / A.area[i];
        const int na = A.spring[4 * i], nc = A.spring[4 * i + 2];
        const D3 d = d3(A.x[nc], A.y[nc], A.z[nc]) - d3(A.x[na], A.y[na], A.z[na]);
        const double len = sqrt(dot(d, d)), L0 = A.contour[i], sr = len / L0;
        es += 0.5 * A.kspring[i] * fabs(0.25 * L0 * (sr * sr * (3.0 - 2.0 * sr) / (1.0 - sr) - 4 * sr * c1 - c2));
    }
    const double ta = block_sum(ea, sh), tb = block_sum(eb, sh), ts = block_sum(es, sh);
    if (threadIdx.x == 0) {
        out[3 * m] = ta;
        out[3 * m + 1] = tb;
        out[3 * m + 2] = ts;
    }
}

// ---- periodic object (gpu_solver::check_periodic_object, Solver_gpu.cu:1277-1304) ----
// One CTA of 128 threads per membrane flagged periodic (LBFS_WRAP_OWN), or
// one CTA for all membranes together (LBFS_WRAP_ALL on membrane 0: the
// reference's object_z array holds every object's nodes).  The mean z of the
// nodes is summed as total<128> does (common_kernels.hpp:71-94: every 256
// consecutive nodes tree-summed, stride 128 down to 1) with the chunk sums
// added in order from 0, as the host adds the block partials; a mean above
// origin_z + 0.75 Z moves every node by -0.5 Z (add_double).
__global__ void __launch_bounds__(128) k_mem_wrap(MembraneArgs A) {
    __shared__ double part[256];
    __shared__ bool shift;
    const int m = blockIdx.x;
    const MembraneConst &mc = A.mc[m];
    if (!mc.periodic) return;
    const bool all = A.mc[0].periodic == LBFS_WRAP_ALL;
    if (all && m > 0) return;  // membrane 0's CTA moves them all
    const int n_nodes = all ? A.total_nodes : mc.n_nodes;
    const int t = threadIdx.x;
    double *z = A.z + (all ? 0 : mc.node0);
    double sum = 0.0;
    for (int s0 = 0; s0 < n_nodes; s0 += 256) {
        part[t] = s0 + t < n_nodes ? z[s0 + t] : 0.0;
        part[128 + t] = s0 + 128 + t < n_nodes ? z[s0 + 128 + t] : 0.0;
        for (int stride = 128; stride >= 1; stride >>= 1) {
            __syncthreads();
            if (t < stride) part[t] += part[t + stride];
        }
        __syncthreads();
        if (t == 0) sum = sum + part[0];
        __syncthreads();
    }
    if (t == 0) shift = sum / n_nodes > mc.domain_z0 + 0.75 * mc.domain_Z;
    __syncthreads();
    if (!shift) return;
    const double dz = -0.5 * mc.domain_Z;
    for (int n = t; n < n_nodes; n += blockDim.x) z[n] = z[n] + dz;
}

// ---- interior viscosity (update_interior_viscosities_plucker, immersed_boundary_method.cu:389-527) ----
//
// The reference tests every cell of the membrane's box (+- 2 delta_h) against
// every triangle: the parity of the crossings of the +x ray from the cell's
// centroid (Plucker side tests, triangles entirely ahead of the cell) and
// the smallest distance to a vertex of those triangles, which enters the
// smoothed step (d / dh + sin(pi d / dh) / pi) / 2 capped at 1/2.  Here the
// triangles are first binned by their y-z boxes (V1, one CTA per membrane),
// so a cell tests only the triangles of the bin holding its (y, z) for
// crossings (a crossed triangle's y-z box holds the point) and those of the
// bins within 2 delta_h for the distance (the smoothed step is exactly 1 at
// distances >= delta_h, so a distance needs to be exact only below that).
// Counts and minima do not depend on the order of the candidates: the result
// is the same as testing every triangle.

__device__ __forceinline__ int visc_bin(double v, double v0, double inv_b, int n) {
    const int b = (int)floor((v - v0) * inv_b);
    return b < 0 ? 0 : (b >= n ? n - 1 : b);
}

// V1: bins of one membrane's triangles (counting sort in shared memory).
__global__ void __launch_bounds__(512) k_visc_bins(ViscArgs a) {
    __shared__ int cnt[kViscBins];
    __shared__ double shd[33];
    __shared__ ViscBins g;
    const int m = blockIdx.x;
    const MembraneConst mc = a.mc[m];
    const MembraneScalars ms = a.ms[m];
    const double dh = mc.gdh;
    double ext = 4.0 * dh;
    for (int lt = threadIdx.x; lt < mc.n_tris; lt += blockDim.x) {
        const int t = mc.tri0 + lt;
        const int n0 = a.tri[3 * t], n1 = a.tri[3 * t + 1], n2 = a.tri[3 * t + 2];
        const double ey = fmax(a.y[n0], fmax(a.y[n1], a.y[n2])) - fmin(a.y[n0], fmin(a.y[n1], a.y[n2]));
        const double ez = fmax(a.z[n0], fmax(a.z[n1], a.z[n2])) - fmin(a.z[n0], fmin(a.z[n1], a.z[n2]));
        ext = fmax(ext, fmax(ey, ez));
    }
    // block maximum
    for (int o = 16; o > 0; o >>= 1) ext = fmax(ext, __shfl_down_sync(0xffffffffu, ext, o));
    if ((threadIdx.x & 31) == 0) shd[threadIdx.x >> 5] = ext;
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = shd[0];
        for (int w = 1; w < (int)(blockDim.x >> 5); w++) b = fmax(b, shd[w]);
        const double y0 = ms.bbox_lo[1] - 2 * dh, y1 = ms.bbox_hi[1] + 2 * dh;
        const double z0 = ms.bbox_lo[2] - 2 * dh, z1 = ms.bbox_hi[2] + 2 * dh;
        int ny = (int)((y1 - y0) / b) + 1, nz = (int)((z1 - z0) / b) + 1;
        while (ny * nz > kViscBins) {
            b *= 1.5;
            ny = (int)((y1 - y0) / b) + 1;
            nz = (int)((z1 - z0) / b) + 1;
        }
        g = {y0, z0, 1.0 / b, ny, nz};
        a.bins[m] = g;
    }
    __syncthreads();
    const int nb = g.ny * g.nz;
    for (int q = threadIdx.x; q < nb; q += blockDim.x) cnt[q] = 0;
    __syncthreads();
    // each triangle goes to every bin its y-z box overlaps (at most 2 x 2)
    for (int pass = 0; pass < 2; pass++) {
        for (int lt = threadIdx.x; lt < mc.n_tris; lt += blockDim.x) {
            const int t = mc.tri0 + lt;
            const int n0 = a.tri[3 * t], n1 = a.tri[3 * t + 1], n2 = a.tri[3 * t + 2];
            const int y_lo = visc_bin(fmin(a.y[n0], fmin(a.y[n1], a.y[n2])), g.y0, g.inv_b, g.ny);
            const int y_hi = visc_bin(fmax(a.y[n0], fmax(a.y[n1], a.y[n2])), g.y0, g.inv_b, g.ny);
            const int z_lo = visc_bin(fmin(a.z[n0], fmin(a.z[n1], a.z[n2])), g.z0, g.inv_b, g.nz);
            const int z_hi = visc_bin(fmax(a.z[n0], fmax(a.z[n1], a.z[n2])), g.z0, g.inv_b, g.nz);
            for (int iz = z_lo; iz <= z_hi; iz++)
                for (int iy = y_lo; iy <= y_hi; iy++) {
                    const int bin = iy + g.ny * iz;
                    if (pass == 0) atomicAdd(&cnt[bin], 1);
                    else a.bin_list[4 * (size_t)mc.tri0 + atomicAdd(&cnt[bin], 1)] = t;
                }
        }
        __syncthreads();
        if (pass == 0) {
            // exclusive prefix of the counts (one thread: at most 4096 bins, once per 10^4 steps)
            if (threadIdx.x == 0) {
                int run = 0;
                int *start = a.bin_start + (size_t)m * (kViscBins + 1);
                for (int q = 0; q < nb; q++) {
                    const int c = cnt[q];
                    start[q] = run;
                    cnt[q] = run;  // placement cursor
                    run += c;
                }
                start[nb] = run;
            }
            __syncthreads();
        }
    }
}

template <typename R>
__global__ void k_interior_viscosity(ViscArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.nc) return;
    const int inst = a.cell_instance ? a.cell_instance[i] : 0;
    const InstanceGrid g = a.instances[inst];
    // update_viscosities fills every cell with 1 before the ray test (fill_double, Solver_gpu.cu:2194):
    // cells outside every membrane's box, and cell 0, which the test skips, end at 1
    double out = 1.0;
    const D3 cc = d3(a.centroid[3 * i], a.centroid[3 * i + 1], a.centroid[3 * i + 2]);
    const double pi = acos(-1.0);
    for (int m = g.mem0; m < g.mem1 && i != g.cell0; m++) {
        const MembraneScalars ms = a.ms[m];
        const MembraneConst mc = a.mc[m];
        const double dh = mc.gdh;
        const double xl = ms.bbox_lo[0] - 2 * dh, xh = ms.bbox_hi[0] + 2 * dh;
        const double yl = ms.bbox_lo[1] - 2 * dh, yh = ms.bbox_hi[1] + 2 * dh;
        const double zl = ms.bbox_lo[2] - 2 * dh, zh = ms.bbox_hi[2] + 2 * dh;
        if (!(cc.x >= xl && cc.x <= xh && cc.y >= yl && cc.y <= yh && cc.z >= zl && cc.z <= zh)) continue;
        // ray from the centroid along +x to x = xh; Plucker side tests against each triangle edge
        const double pc0 = cc.x * cc.y - xh * cc.y, pc1 = cc.x * cc.z - xh * cc.z, pc2 = cc.x - xh;
        const ViscBins bg = a.bins[m];
        const int *start = a.bin_start + (size_t)m * (kViscBins + 1);
        const int *list = a.bin_list + 4 * (size_t)mc.tri0;
        const int by = visc_bin(cc.y, bg.y0, bg.inv_b, bg.ny), bz = visc_bin(cc.z, bg.z0, bg.inv_b, bg.nz);
        const int dy0 = visc_bin(cc.y - 2 * dh, bg.y0, bg.inv_b, bg.ny), dy1 = visc_bin(cc.y + 2 * dh, bg.y0, bg.inv_b, bg.ny);
        const int dz0 = visc_bin(cc.z - 2 * dh, bg.z0, bg.inv_b, bg.nz), dz1 = visc_bin(cc.z + 2 * dh, bg.z0, bg.inv_b, bg.nz);
        int crossings = 0;
        double min_distance = 1000000000;
        for (int iz = dz0; iz <= dz1; iz++)
            for (int iy = dy0; iy <= dy1; iy++) {
                const int bin = iy + bg.ny * iz;
                const bool own_bin = iy == by && iz == bz;  // crossings from this bin only (each triangle once)
                for (int e0 = start[bin]; e0 < start[bin + 1]; e0++) {
                    const int t = list[e0];
                    const int na = a.tri[3 * t], nb = a.tri[3 * t + 1], nc = a.tri[3 * t + 2];
                    const D3 A = d3(a.x[na], a.y[na], a.z[na]), B = d3(a.x[nb], a.y[nb], a.z[nb]),
                             C = d3(a.x[nc], a.y[nc], a.z[nc]);
                    if (!(A.x > cc.x && B.x > cc.x && C.x > cc.x)) continue;
                    if (own_bin) {
                        const D3 P[3] = {A, B, C};
                        double side[3];
                        for (int e = 0; e < 3; e++) {
                            const D3 p = P[e], q = P[(e + 1) % 3];
                            const double e0v = p.y * q.z - q.y * p.z, e1 = p.z - q.z, e2 = q.y - p.y;
                            side[e] = pc0 * e1 + pc1 * e2 + pc2 * e0v;
                        }
                        if ((side[0] < 0 && side[1] < 0 && side[2] < 0) || (side[0] > 0 && side[1] > 0 && side[2] > 0))
                            crossings++;
                    }
                    min_distance = fmin(sqrt(dot(cc - A, cc - A)), min_distance);
                    min_distance = fmin(sqrt(dot(cc - B, cc - B)), min_distance);
                    min_distance = fmin(sqrt(dot(cc - C, cc - C)), min_distance);
                }
            }
        const bool inside = (crossings % 2) != 0;
        const double r = mc.internal_viscosity_ratio;
        const double factor = 2.0 * fmin(0.5, (min_distance * 0.5 / dh + 1.0 / pi * sin(pi * min_distance / dh) * 0.5));
        const double visc = inside ? (r + 1.0) + (r - 1.0) * factor : (r + 1.0) + (1.0 - r) * factor;
        out = visc * 0.5;
    }
    ((R *)a.visc_factor)[i] = (R)out;
}

}  // namespace

namespace {
template <int CL, int TPB> void prepare_step(int smem) {
    cudaFuncSetAttribute(k_mem_step<CL, TPB>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (CL > 8) cudaFuncSetAttribute(k_mem_step<CL, TPB>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
}
}  // namespace

bool membrane_cluster_fits(int max_nodes) { return max_nodes <= kStepMaxNodes; }

void membrane_prepare(int sort_capacity, int max_nodes) {
    const size_t smem = sort_smem_bytes(sort_capacity);
    cudaFuncSetAttribute(k_mem_sort, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (!membrane_cluster_fits(max_nodes)) return;
    const int fs = (int)step_smem_bytes(sort_capacity, max_nodes);
    prepare_step<8, kStepThreads>(fs);
    prepare_step<16, kStepThreads>(fs);
}

namespace {
// Launch with the device's greatest scheduling priority: the membrane chain is
// the critical path of a step and runs beside the fluid kernels on a second
// stream, so its blocks are placed ahead of pending fluid blocks.
template <typename... Args>
void launch_hi(void (*kernel)(Args...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, const MembraneArgs &a,
               int cluster_x = 0, bool after_kernel = false) {
    int lo = 0, hi = 0;
    cudaDeviceGetStreamPriorityRange(&lo, &hi);
    cudaLaunchAttribute attr[3];
    attr[0].id = cudaLaunchAttributePriority;
    attr[0].val.priority = hi;
    int n_attr = 1;
    if (cluster_x > 0) {  // thread-block clusters of cluster_x CTAs along x
        attr[n_attr].id = cudaLaunchAttributeClusterDimension;
        attr[n_attr].val.clusterDim.x = cluster_x;
        attr[n_attr].val.clusterDim.y = 1;
        attr[n_attr].val.clusterDim.z = 1;
        n_attr++;
    }
    if (after_kernel) {  // directly behind a kernel of the chain on the same stream: programmatic launch
        attr[n_attr].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[n_attr].val.programmaticStreamSerializationAllowed = 1;
        n_attr++;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cfg.attrs = attr;
    cfg.numAttrs = n_attr;
    cudaLaunchKernelEx(&cfg, kernel, a);
}
}  // namespace

int launch_membrane(const MembraneArgs &a, cudaStream_t s, cudaStream_t s_side, cudaEvent_t ev_advected,
                    cudaEvent_t ev_sorted, bool without_spread) {
    const size_t smem = sort_smem_bytes(a.sort_capacity);
    const dim3 spring_grid((a.max_springs + 127) / 128, a.n_membranes);
    if (a.mode == kModeReference) {  // stress-free reference pass
        launch_hi(k_mem_springs, spring_grid, dim3(128), 0, s, a);
        return 1;
    }
    if (a.mode == kModeInitial) {  // initial pass: V0, A0, MAD0, areas, angles
        launch_hi(k_mem_totals, dim3(a.n_membranes), dim3(kTotalsThreads), 0, s, a);
        launch_hi(k_mem_springs, spring_grid, dim3(128), 0, s, a);
        return 2;
    }
    const int blocks = (a.total_nodes * 32 + 255) / 256;
    if (a.state_is_float) launch_hi(k_mem_advect<float>, dim3(blocks), dim3(256), 0, s, a);
    else launch_hi(k_mem_advect<double>, dim3(blocks), dim3(256), 0, s, a);
    const dim3 spread_grid(a.spread_blocks);
    if (a.force_cluster == 8 || a.force_cluster == 16) {
        // totals, sort, spring and node forces as one cluster per membrane, then the spread
        const size_t fs = step_smem_bytes(a.sort_capacity, a.max_nodes);
        const dim3 grid(a.force_cluster, a.n_membranes), block(kStepThreads);
        if (a.force_cluster == 16) launch_hi(k_mem_step<16, kStepThreads>, grid, block, fs, s, a, 16, true);
        else launch_hi(k_mem_step<8, kStepThreads>, grid, block, fs, s, a, 8, true);
        if (without_spread) return 2;
        if (stencil_width(a.ibm_stencil) == 4) launch_hi(k_mem_spread<4>, spread_grid, dim3(256), 0, s, a, 0, true);
        else launch_hi(k_mem_spread<2>, spread_grid, dim3(256), 0, s, a, 0, true);
        return 3;
    }
    // the node sort needs only the advected positions: side stream
    const bool side = s_side != nullptr && ev_advected != nullptr && ev_sorted != nullptr;
    if (side) {
        cudaEventRecord(ev_advected, s);
        cudaStreamWaitEvent(s_side, ev_advected, 0);
    }
    launch_hi(k_mem_sort, dim3(a.n_membranes), dim3(kSortThreads), smem, side ? s_side : s, a);
    if (side) cudaEventRecord(ev_sorted, s_side);
    // separate kernels for the totals, the spring forces and the node forces
    launch_hi(k_mem_totals, dim3(a.n_membranes), dim3(kTotalsThreads), 0, s, a, 0, true);
    launch_hi(k_mem_springs, spring_grid, dim3(128), 0, s, a, 0, true);
    launch_hi(k_mem_nodeforce, dim3((a.total_nodes + 127) / 128), dim3(128), 0, s, a, 0, true);
    const int n = 6;
    // the spread reads the sorted node list and the node forces
    if (side) cudaStreamWaitEvent(s, ev_sorted, 0);
    if (without_spread) return n - 1;
    if (stencil_width(a.ibm_stencil) == 4) launch_hi(k_mem_spread<4>, spread_grid, dim3(256), 0, s, a);
    else launch_hi(k_mem_spread<2>, spread_grid, dim3(256), 0, s, a);
    return n;
}

void launch_membrane_tables(const MembraneArgs &a, cudaStream_t s) {
    launch_hi(k_mem_tables, dim3((a.total_nodes * 32 + 255) / 256), dim3(256), 0, s, a);
}

// Advection, totals, spring forces and node forces of a step (no sort, no
// spread): what the adjoint's recomputation of a step needs.
void launch_membrane_forces(const MembraneArgs &a, cudaStream_t s) {
    const dim3 spring_grid((a.max_springs + 127) / 128, a.n_membranes);
    const int blocks = (a.total_nodes * 32 + 255) / 256;
    if (a.state_is_float) launch_hi(k_mem_advect<float>, dim3(blocks), dim3(256), 0, s, a);
    else launch_hi(k_mem_advect<double>, dim3(blocks), dim3(256), 0, s, a);
    launch_hi(k_mem_totals, dim3(a.n_membranes), dim3(kTotalsThreads), 0, s, a);
    launch_hi(k_mem_springs, spring_grid, dim3(128), 0, s, a);
    launch_hi(k_mem_nodeforce, dim3((a.total_nodes + 127) / 128), dim3(128), 0, s, a);
}

void launch_membrane_sort(const MembraneArgs &a, cudaStream_t s) {
    const size_t smem = sort_smem_bytes(a.sort_capacity);
    launch_hi(k_mem_sort, dim3(a.n_membranes), dim3(kSortThreads), smem, s, a);
}

void launch_membrane_energies(const MembraneArgs &a, double *out, cudaStream_t s) {
    if (a.n_membranes > 0) k_mem_energies<<<a.n_membranes, kTotalsThreads, 0, s>>>(a, out);
}

void launch_membrane_wrap(const MembraneArgs &a, cudaStream_t s) {
    if (a.n_membranes > 0) k_mem_wrap<<<a.n_membranes, 128, 0, s>>>(a);
}

void launch_membrane_spread(const MembraneArgs &a, cudaStream_t s, bool programmatic) {
    const dim3 grid(a.spread_blocks);
    if (stencil_width(a.ibm_stencil) == 4) launch_hi(k_mem_spread<4>, grid, dim3(256), 0, s, a, 0, programmatic);
    else launch_hi(k_mem_spread<2>, grid, dim3(256), 0, s, a, 0, programmatic);
}

void launch_interior_viscosity(const ViscArgs &a, cudaStream_t s) {
    if (a.n_membranes > 0) k_visc_bins<<<a.n_membranes, 512, 0, s>>>(a);
    const int blocks = (a.nc + 255) / 256;
    if (a.visc_is_float) k_interior_viscosity<float><<<blocks, 256, 0, s>>>(a);
    else k_interior_viscosity<double><<<blocks, 256, 0, s>>>(a);
}

}  // namespace lbfs
