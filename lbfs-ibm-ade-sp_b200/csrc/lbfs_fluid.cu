// Fluid kernels of one LBFS time step; see lbfs_fluid.cuh for the mapping to
// the reference kernels they replace.
#include <cuda_runtime.h>

#include <algorithm>

#include "lbfs_fluid.cuh"
#include "lbfs_internal.h"
#include "lbfs_kernels.h"

namespace lbfs {

// ------------------------------------------------------------------ K1 ----

// Ghost-cell macros from the owner state (update_unstructured_bcs,
// LBFS.cu:1868-1918).  Type 3 (periodic) takes the partner cell's state, as
// the reference's CPU solver does (Solution::update_unstructured_bcs,
// Solution.cpp:777-803).  Types outside {1,2,3} / {1,2,3,9,10} are rejected at
// creation, so every branch here assigns.
template <typename R>
__device__ __forceinline__ Vec4<R> ghost_state(const FluidArgs<R> &a, int b, const Vec4<R> &own) {
    const Vec4<R> bc = a.bc_val[b];
    Vec4<R> g;
    const int rt = a.bc_rho_type[b], vt = a.bc_vel_type[b];
    const Vec4<R> p = (rt == 3 || vt == 3) ? a.state[a.bc_periodic[b]] : own;
    if (rt == 1) g.rho = bc.rho - (own.rho - bc.rho);
    else if (rt == 2) g.rho = own.rho;
    else g.rho = p.rho;
    if (vt == 3) {
        g.u = p.u; g.v = p.v; g.w = p.w;
    } else if (vt == 2) {
        g.u = own.u; g.v = own.v; g.w = own.w;
    } else {
        R ut = bc.u;
        if (vt == 9) {
            const BcRec<R> r = a.bc_rec[b];
            ut = (R)(16 * (double)bc.u * (a.H2 + r.gy) * (a.H2 - r.gy) * (a.H2 + r.gz) * (a.H2 - r.gz) / a.H4);
        } else if (vt == 10) {
            ut = a.bc_rec[b].gy * bc.u;
        }
        g.u = ut - (own.u - ut);
        g.v = bc.v - (own.v - bc.v);
        g.w = bc.w - (own.w - bc.w);
    }
    return g;
}

template <typename R, int TB>
__global__ void __launch_bounds__(TB, TB == 128 ? 5 : 1) k_cell_gradients(FluidArgs<R> a, int begin, int end) {
    const int i = begin + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= end) return;
    const Vec4<R> own = a.state[i];
    int st[6];
#pragma unroll
    for (int q = 0; q < 3; q++) {
        const int2 p = __ldg(a.stencil + 3 * i + q);
        st[2 * q] = p.x;
        st[2 * q + 1] = p.y;
    }
    const LsW<R> W = a.lsw[i];
    GradRec<R> gr;
    R *g = gr.g;
#pragma unroll
    for (int t = 0; t < 12; t++) g[t] = R(0);
#pragma unroll
    for (int q = 0; q < 6; q++) {
        const int j = st[q];
        Vec4<R> s;
        if (j < a.nc) {
            s = a.state[j];
        } else {
            s = ghost_state(a, j - a.nc, own);
        }
        // add_LS_contributions (LBFS.cu:2051-2083) with LHS^-1 folded in
        const R d[4] = {s.rho - own.rho, s.u - own.u, s.v - own.v, s.w - own.w};
#pragma unroll
        for (int m = 0; m < 4; m++)
#pragma unroll
            for (int r = 0; r < 3; r++) g[3 * m + r] = g[3 * m + r] + W.w[3 * q + r] * d[m];
    }
    reinterpret_cast<GradRec<R> *>(a.grad)[i] = gr;
}

// ------------------------------------------------------------------ K2 ----

struct Dir {
    int ex, ey, ez;
};
__device__ __forceinline__ Dir dir_of(int k) { return {c_ex(k), c_ey(k), c_ez(k)}; }

// Moments of the reconstructed populations, accumulated direction by
// direction in the order k = 0..14 (the same sums and order as over a stored
// fl[15], with 8-16 accumulators live instead of 15 populations).
template <typename R> struct Moments {
    R rho, m[3], F[3][4];  // F[c][.] over the directions crossing the face (c = axis, or all c)
};
template <typename R> __device__ __forceinline__ void moments_init(Moments<R> &M) {
    M.rho = R(0);
#pragma unroll
    for (int c = 0; c < 3; c++) {
        M.m[c] = R(0);
#pragma unroll
        for (int j = 0; j < 4; j++) M.F[c][j] = R(0);
    }
}
template <typename R>
__device__ __forceinline__ void moments_add(Moments<R> &M, int k, R f, int axis) {
    M.rho = (k == 0) ? f : M.rho + f;
    if (k == 0) return;
    const Dir e = dir_of(k);
    if (e.ex) M.m[0] = (e.ex > 0) ? M.m[0] + f : M.m[0] - f;
    if (e.ey) M.m[1] = (e.ey > 0) ? M.m[1] + f : M.m[1] - f;
    if (e.ez) M.m[2] = (e.ez > 0) ? M.m[2] + f : M.m[2] - f;
    if (axis == 0 && !e.ex) return;
    if (axis == 1 && !e.ey) return;
    if (axis == 2 && !e.ez) return;
    const int ee[3] = {e.ex, e.ey, e.ez};
#pragma unroll
    for (int c = 0; c < 3; c++) {
        if (axis >= 0 && c != axis) continue;
        if (!ee[c]) continue;
        M.F[c][0] = (ee[c] > 0) ? M.F[c][0] + f : M.F[c][0] - f;
#pragma unroll
        for (int q = 0; q < 3; q++) {
            if (!ee[q]) continue;
            M.F[c][1 + q] = (ee[c] * ee[q] > 0) ? M.F[c][1 + q] + f : M.F[c][1 + q] - f;
        }
    }
}

// Interface equilibrium, BGK relaxation towards the lattice equilibria and
// the flux through the face: calculate_flux_at_interface (LBFS.cu:1462-1648)
// and its axis-aligned forms (LBFS.cu:3648-4092).  `axis` < 0 selects the
// general three-component form with the face normal; otherwise only the
// face-normal component is formed.
//
// The relaxed populations are f_k - tau (f_k - fl_k), f_k the interface
// equilibrium, so the flux tensor is (1 - tau) F_eq + tau F_fl, F_fl the
// first and second moments of the reconstructed fl_k over the directions
// crossing the face and F_eq those of the equilibrium.  The D3Q15 weights
// make the equilibrium moments exact closed forms (sum w e = 0,
// sum w e e = I / 3, sum w e e e e = (dd + dd + dd) / 9):
//   sum_k e_c f_k = rho u_c,  sum_k e_c e_m f_k = rho (q u_c u_m + d_cm / 3)
// (q the preconditioning factor); in the deviation form (f' = f - w rho0)
// the second moment's d_cm term is rho' / 3.  The reference sums the 15
// equilibria explicitly; the closed form is the same quantity with fewer
// roundings.
template <typename R>
__device__ __forceinline__ Vec4<R> interface_flux(Moments<R> &M, R rho0, R tau, R qscale, R area, int axis, R nx,
                                                  R ny, R nz) {
    const R rho_dev = M.rho;
    const R rho_i = rho_dev + rho0;
    const R inv = R(1) / rho_i;
    const R u[3] = {inv * M.m[0], inv * M.m[1], inv * M.m[2]};
    const R keep = R(1) - tau;
#pragma unroll
    for (int c = 0; c < 3; c++) {
        if (axis >= 0 && c != axis) continue;
        M.F[c][0] = keep * (rho_i * u[c]) + tau * M.F[c][0];
#pragma unroll
        for (int m = 0; m < 3; m++) {
            R eq = rho_i * (qscale * u[c] * u[m]);
            if (m == c) eq = eq + rho_dev * R(1.0 / 3.0);
            M.F[c][1 + m] = keep * eq + tau * M.F[c][1 + m];
        }
    }
    Vec4<R> out;
    if (axis >= 0) {
        out.rho = M.F[axis][0] * area;
        out.u = M.F[axis][1] * area;
        out.v = M.F[axis][2] * area;
        out.w = M.F[axis][3] * area;
    } else {
        out.rho = (M.F[0][0] * nx + M.F[1][0] * ny + M.F[2][0] * nz) * area;
        out.u = (M.F[0][1] * nx + M.F[1][1] * ny + M.F[2][1] * nz) * area;
        out.v = (M.F[0][2] * nx + M.F[1][2] * ny + M.F[2][2] * nz) * area;
        out.w = (M.F[0][3] * nx + M.F[1][3] * ny + M.F[2][3] * nz) * area;
    }
    return out;
}

template <typename R> __device__ __forceinline__ void load_grad(const R *g, R (&o)[12]) {
    const GradRec<R> r = *reinterpret_cast<const GradRec<R> *>(g);
#pragma unroll
    for (int t = 0; t < 12; t++) o[t] = r.g[t];
}

// Axis-aligned face: populate_lattice_macros_uniform_{x,y,z} (LBFS.cu:2939-3644).
// For direction k the lattice node sits at x_f - e_k dt; directions with
// e_k[axis] = +1 extrapolate from the owner, -1 from the neighbour, 0 from the
// face centre with the distance-weighted gradient.
template <typename R, int axis>
__device__ __forceinline__ Vec4<R> axis_face_flux(const FluidArgs<R> &a, int f) {
    const int2 oc = __ldg(a.face_cells + f);
    const AxisFace<R> geo = a.axis_face[f];
    const Vec4<R> s1 = a.state[oc.x], s2 = a.state[oc.y];
    R g1[12], g2[12];
    load_grad(a.grad + (size_t)12 * oc.x, g1);
    load_grad(a.grad + (size_t)12 * oc.y, g2);
    const R dt = geo.dt, t1 = geo.t1, t2 = geo.t2;
    const R c = t2 - t1;
    const R wa = fabs(t2 / c), wb = fabs(t1 / c);
    const R S1[4] = {s1.rho, s1.u, s1.v, s1.w}, S2[4] = {s2.rho, s2.u, s2.v, s2.w};
    R pi[4], pn[4], p0[4];
#pragma unroll
    for (int m = 0; m < 4; m++) {
        pi[m] = S1[m] - t1 * g1[3 * m + axis];
        pn[m] = S2[m] - (t2 * g2[3 * m + axis]);
        p0[m] = (pi[m] + pn[m]) * R(0.5);
    }
    constexpr int ob = axis == 0 ? 1 : 0;  // other axes in increasing order
    constexpr int oc2 = axis == 2 ? 1 : 2;
    Moments<R> M;
    moments_init(M);
#pragma unroll
    for (int k = 0; k < 15; k++) {
        const Dir e = dir_of(k);
        const int ee[3] = {e.ex, e.ey, e.ez};
        R L[4];
#pragma unroll
        for (int m = 0; m < 4; m++) {
            R val;
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
                    const R gi = g1[3 * m + ob] * wa + g2[3 * m + ob] * wb;
                    val = (ee[ob] > 0) ? val - gi * dt : val + gi * dt;
                }
                if (ee[oc2]) {
                    const R gi = g1[3 * m + oc2] * wa + g2[3 * m + oc2] * wb;
                    val = (ee[oc2] > 0) ? val - gi * dt : val + gi * dt;
                }
            }
            L[m] = val;
        }
        moments_add(M, k, feq_dev<R>(k, L[0], L[1], L[2], L[3], a.rho0, R(1)), axis);
    }
    const R vf = a.visc_factor[oc.x];
    const R tau = (a.testcase == 8) ? R(0) : (a.visc * vf * R(3) / dt * a.gamma_inv);
    return interface_flux<R>(M, a.rho0, tau, R(1), geo.area, axis, 0, 0, 0);
}

// General face: populate_lattice_macros (LBFS.cu:323-936).  Boundary faces
// take the boundary branch except the face of the first ghost (LBFS.cu tests
// neighbour > n_cells), which the host marks per instance in bc_branch.
// Ghost of boundary face f (ghost cell g = its neighbour): its state
// (update_unstructured_bcs, LBFS.cu:1843-1928) and its gradients
// (get_bc_gradients, LBFS.cu:1933-2048): Dirichlet components the difference
// to the owner over the owner-ghost distance along that direction, the others
// the owner's gradient without its face-normal part; a periodic component
// (type 3) the partner cell's gradient (gradients::Get_LS_Gradients,
// gradients.cpp:428-440).  Formed here, once every cell's gradients exist,
// and stored in the ghost's records for the fields and the adjoint.
template <typename R>
__device__ __forceinline__ void boundary_ghost(const FluidArgs<R> &a, int g, const Vec4<R> &own, const R (&go)[12],
                                               Vec4<R> &gs, R (&gg)[12]) {
    const int b = g - a.nc;
    gs = ghost_state(a, b, own);
    const BcRec<R> r = a.bc_rec[b];
    const int rt = a.bc_rho_type[b], vt = a.bc_vel_type[b];
    const R d[4] = {gs.rho - own.rho, gs.u - own.u, gs.v - own.v, gs.w - own.w};
#pragma unroll
    for (int m = 0; m < 4; m++) {
        const bool dirichlet = (m == 0) ? rt == 1 : (vt != 2 && vt != 3);
        if (dirichlet) {
            gg[3 * m + 0] = d[m] / r.dmag * r.dnx;
            gg[3 * m + 1] = d[m] / r.dmag * r.dny;
            gg[3 * m + 2] = d[m] / r.dmag * r.dnz;
        } else {
            gg[3 * m + 0] = go[3 * m + 0] * r.mx;
            gg[3 * m + 1] = go[3 * m + 1] * r.my;
            gg[3 * m + 2] = go[3 * m + 2] * r.mz;
        }
    }
    if (rt == 3 || vt == 3) {
        R gp[12];
        load_grad(a.grad + (size_t)12 * a.bc_periodic[b], gp);
#pragma unroll
        for (int t = 0; t < 12; t++)
            if ((t < 3) ? rt == 3 : vt == 3) gg[t] = gp[t];
    }
    a.state[g] = gs;
    GradRec<R> gr;
#pragma unroll
    for (int t = 0; t < 12; t++) gr.g[t] = gg[t];
    reinterpret_cast<GradRec<R> *>(a.grad)[g] = gr;
}

template <typename R>
__device__ __forceinline__ Vec4<R> general_face_flux(const FluidArgs<R> &a, int f, bool is_bc) {
    const int2 oc = __ldg(a.face_cells + f);
    const GenFace<R> geo = a.gen_face[a.axis_aligned ? f - a.ni : f];
    const Vec4<R> s1 = a.state[oc.x];
    Vec4<R> s2;
    R g1[12], g2[12];
    load_grad(a.grad + (size_t)12 * oc.x, g1);
    if (is_bc) {
        boundary_ghost(a, oc.y, s1, g1, s2, g2);
    } else {
        s2 = a.state[oc.y];
        load_grad(a.grad + (size_t)12 * oc.y, g2);
    }
    const R dt = geo.dt;
    const R S1[4] = {s1.rho, s1.u, s1.v, s1.w}, S2[4] = {s2.rho, s2.u, s2.v, s2.w};
    R pi[4], pn[4], p0[4], g3[12];
    if (geo.bc_branch != R(0)) {
        const int b = oc.y - a.nc;
        const Vec4<R> bc = a.bc_val[b];
        const bool rd = a.bc_rho_type[b] == 1, vd = a.bc_vel_type[b] == 1;
        const R bcv[4] = {bc.rho, bc.u, bc.v, bc.w};
#pragma unroll
        for (int m = 0; m < 4; m++) {
            const bool dir = (m == 0) ? rd : vd;
            p0[m] = dir ? bcv[m]
                        : S1[m] - (geo.t1x * g2[3 * m] + geo.t1y * g2[3 * m + 1] + geo.t1z * g2[3 * m + 2]);
            pi[m] = p0[m];
            pn[m] = p0[m];
        }
#pragma unroll
        for (int t = 0; t < 12; t++) { g3[t] = g2[t]; g1[t] = g2[t]; }
    } else {
#pragma unroll
        for (int m = 0; m < 4; m++) {
            pi[m] = S1[m] - (geo.t1x * g1[3 * m] + geo.t1y * g1[3 * m + 1] + geo.t1z * g1[3 * m + 2]);
            pn[m] = S2[m] - (geo.t2x * g2[3 * m] + geo.t2y * g2[3 * m + 1] + geo.t2z * g2[3 * m + 2]);
            p0[m] = (pi[m] + pn[m]) * R(0.5);
        }
#pragma unroll
        for (int t = 0; t < 12; t++) g3[t] = (g1[t] + g2[t]) * R(0.5);
    }
    // Upwind selection by the sign of n.e_k with the threshold 0.001 dt
    // (LBFS.cu:351-352 override the sin(pi/14) arguments).
    const R thr = R(0.001) * dt;
    Moments<R> M;
    moments_init(M);
    moments_add(M, 0, feq_dev<R>(0, p0[0], p0[1], p0[2], p0[3], a.rho0, a.recon_q), -1);
#pragma unroll
    for (int k = 1; k < 15; k += 2) {
        const Dir e = dir_of(k);
        const R s = (k < 7) ? (e.ex ? geo.nx : (e.ey ? geo.ny : geo.nz))
                            : (R(e.ex) * geo.nx + R(e.ey) * geo.ny + R(e.ez) * geo.nz);
        // side of direction k and of its opposite k+1: 0 owner, 1 neighbour, 2 centre
        const int side_k = (s > thr) ? 0 : ((s < -thr) ? 1 : 2);
        const int side_o = (side_k == 2) ? 2 : 1 - side_k;
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int kk = k + h;
            const int side = h ? side_o : side_k;
            const int ee[3] = {h ? -e.ex : e.ex, h ? -e.ey : e.ey, h ? -e.ez : e.ez};
            R L[4];
#pragma unroll
            for (int m = 0; m < 4; m++) {
                R val = side == 0 ? pi[m] : (side == 1 ? pn[m] : p0[m]);
#pragma unroll
                for (int d = 0; d < 3; d++) {
                    if (!ee[d]) continue;
                    const R gd = side == 0 ? g1[3 * m + d] : (side == 1 ? g2[3 * m + d] : g3[3 * m + d]);
                    val = (ee[d] > 0) ? val - gd * dt : val + gd * dt;
                }
                L[m] = val;
            }
            moments_add(M, kk, feq_dev<R>(kk, L[0], L[1], L[2], L[3], a.rho0, a.recon_q), -1);
        }
    }
    const R vf = is_bc ? R(1) : a.visc_factor[oc.x];
    const R tau = (a.testcase == 8) ? R(0) : (a.visc * vf * R(3) / dt * a.gamma_inv);
    return interface_flux<R>(M, a.rho0, tau, a.gamma_inv, geo.area, -1, geo.nx, geo.ny, geo.nz);
}

// Interior faces of an axis-aligned mesh: faces [0, nfx) x, [nfx, nfx+nfy) y,
// the rest z; warps never mix axes except at the two range boundaries.
// TB threads per block, 640 / TB blocks per SM (at most 102 registers a thread).
template <typename R, int TB>
__global__ void __launch_bounds__(TB, 640 / TB) k_face_flux(FluidArgs<R> a, FaceRanges r) {
    int t = blockIdx.x * blockDim.x + threadIdx.x, f;
    if (t < r.count[0]) f = r.start[0] + t;
    else if ((t -= r.count[0]) < r.count[1]) f = r.start[1] + t;
    else if ((t -= r.count[1]) < r.count[2]) f = r.start[2] + t;
    else return;
    Vec4<R> out;
    if (f < a.nfx) out = axis_face_flux<R, 0>(a, f);
    else if (f < a.nfx + a.nfy) out = axis_face_flux<R, 1>(a, f);
    else out = axis_face_flux<R, 2>(a, f);
    a.flux[f] = out;
}

// Boundary faces (always) and the interior faces of meshes that are not axis
// aligned: the general-normal reconstruction.  `first` is ni (axis-aligned
// meshes) or 0.
template <typename R, int TB>
__global__ void __launch_bounds__(TB) k_face_flux_general(FluidArgs<R> a, int first) {
    const int f = first + blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= a.nf) return;
    a.flux[f] = general_face_flux<R>(a, f, f >= a.ni);
}

// ----------------------------------------------------------------- CFL ----
// get_cfl_device (LBFS.cu:2868-2932) per cell, then the minimum over the cells
// (min<128> + min_block, common_kernels.hpp:147-170, Solver_gpu.cu:57-66):
// block minima, the last block takes the minimum of the block minima.  A
// minimum is exact, so the result does not depend on the grid.  The effective
// speed of sound (a constant of the step) is formed on the host.  Products and
// sums use explicitly rounded intrinsics so no multiply-add is contracted,
// as in the reference's evaluation.
template <typename R>
__global__ void __launch_bounds__(256) k_cfl(FluidArgs<R> a) {
    __shared__ double sh[8];
    __shared__ bool last_block;
    double mn = 100000000.0;  // min<128> pads its blocks with 1e8
    const double ce = __dadd_rn(a.cfl_max_velocity, a.cfl_esos);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.nc; i += gridDim.x * blockDim.x) {
        const double4 c = a.cfl[i];  // area x, y, z, volume
        const double rho = (double)a.state[i].rho + (double)a.rho0;
        double eig = __dadd_rn(__dadd_rn(__dmul_rn(ce, c.x), __dmul_rn(ce, c.y)), __dmul_rn(ce, c.z));
        eig = eig / a.cfl_gamma;
        double ve = 2.0 * a.cfl_visc / a.cfl_gamma / rho / c.w;
        ve = __dmul_rn(ve, __dadd_rn(__dadd_rn(__dmul_rn(c.x, c.x), __dmul_rn(c.y, c.y)), __dmul_rn(c.z, c.z)));
        eig = __dadd_rn(eig, __dmul_rn(4.0, ve));
        const double dt = __dmul_rn(a.cfl_factor, c.w) / eig;
        a.dt_local[i] = dt;
        mn = fmin(mn, dt);
    }
    for (int o = 16; o > 0; o >>= 1) mn = fmin(mn, __shfl_down_sync(0xffffffffu, mn, o));
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) sh[warp] = mn;
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = sh[0];
        for (int w = 1; w < (int)(blockDim.x >> 5); w++) b = fmin(b, sh[w]);
        a.dt_partials[blockIdx.x] = b;
        __threadfence();
        last_block = atomicAdd(a.dt_ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (last_block && threadIdx.x == 0) {
        __threadfence();
        double b = 100000000.0;
        for (int k = 0; k < (int)gridDim.x; k++) b = fmin(b, __ldcg(a.dt_partials + k));
        *a.dt_min = b;
        *a.dt_ticket = 0u;
    }
}

// ------------------------------------------------------------------ K3 ----

template <typename R, int TB>
__global__ void __launch_bounds__(TB) k_cell_update(FluidArgs<R> a) {
    __shared__ double sh[4][TB / 32];
    __shared__ bool last_block;
    double sq[4] = {0, 0, 0, 0};
    unsigned int flag = 0;
    // the step: constant, or the minimum per-cell step, or each cell's own (LBFS_DT_LOCAL)
    const bool local_dt = a.time_stepping == LBFS_DT_LOCAL;
    const double dt_all = (a.time_stepping == LBFS_DT_MIN || a.time_stepping == LBFS_DT_TALTS) ? __ldcg(a.dt_min)
                                                                                                 : a.delta_t;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.nc; i += gridDim.x * blockDim.x) {
        const double iv = __ldg(a.cell_inv_volume + i);  // 1 / volume: products instead of 24 divisions
        double r[4] = {0, 0, 0, 0};  // rho, u, v, w
        int cfl[6];
#pragma unroll
        for (int q = 0; q < 3; q++) {
            const int2 p = __ldg(reinterpret_cast<const int2 *>(a.cell_faces) + 3 * i + q);
            cfl[2 * q] = p.x;
            cfl[2 * q + 1] = p.y;
        }
#pragma unroll
        for (int q = 0; q < 6; q++) {
            const int e = cfl[q];
            const int f = (e > 0 ? e : -e) - 1;
            const Vec4<R> fx = a.flux[f];
            const double fv[4] = {(double)fx.rho, (double)fx.u, (double)fx.v, (double)fx.w};
#pragma unroll
            for (int m = 0; m < 4; m++) r[m] = (e > 0) ? r[m] + (-fv[m] * iv) : r[m] + fv[m] * iv;
        }
        if (a.closure) {
#pragma unroll
            for (int m = 0; m < 3; m++) r[1 + m] = r[1 + m] + __ldg(a.closure + 3 * (size_t)i + m);
        }
        double fx = a.force[0], fy = a.force[1], fz = a.force[2];
        if (a.n_membranes > 0) {
            const int inst = a.cell_instance ? __ldg(a.cell_instance + i) : 0;
            const InstanceGrid g = reinterpret_cast<const InstanceGrid *>(a.instances)[inst];
            const int li = i - g.cell0;
            const int ci = li % g.nx, cj = (li / g.nx) % g.ny, ck = li / (g.nx * g.ny);
            const MembraneScalars *ms = (const MembraneScalars *)a.membrane_scalars;
            for (int m = g.mem0; m < g.mem1; m++) {
                const int px = ci - ms[m].patch_lo[0], py = cj - ms[m].patch_lo[1], pz = ck - ms[m].patch_lo[2];
                if (ms[m].patch_cells > 0 && px >= 0 && py >= 0 && pz >= 0 && px < ms[m].patch_dim[0] &&
                    py < ms[m].patch_dim[1] && pz < ms[m].patch_dim[2]) {
                    const double *pf = a.patch_force + ((size_t)ms[m].patch_off +
                                                        (px + ms[m].patch_dim[0] * (py + ms[m].patch_dim[1] * pz))) * 3;
                    fx = fx + pf[0];
                    fy = fy + pf[1];
                    fz = fz + pf[2];
                }
            }
        }
        r[1] = r[1] + fx;
        r[2] = r[2] + fy;
        r[3] = r[3] + fz;
        double4 t = a.t1[i];
        const double dt = local_dt ? a.dt_local[i] : dt_all;
        t.w = t.w + dt * r[0];
        t.x = t.x + dt * r[1];
        t.y = t.y + dt * r[2];
        t.z = t.z + dt * r[3];
        a.t1[i] = t;
        Vec4<R> s;
        s.rho = (R)(t.w - (double)a.rho0);
        s.u = (R)(t.x / t.w);
        s.v = (R)(t.y / t.w);
        s.w = (R)(t.z / t.w);
        a.state[i] = s;
        if (a.res_out) {
            a.res_out[4 * i] = r[0]; a.res_out[4 * i + 1] = r[1];
            a.res_out[4 * i + 2] = r[2]; a.res_out[4 * i + 3] = r[3];
        }
#pragma unroll
        for (int m = 0; m < 4; m++) sq[m] = sq[m] + r[m] * r[m];
        if (!(isfinite(t.w) && isfinite(t.x) && isfinite(t.y) && isfinite(t.z))) flag |= LBFS_FLAG_NONFINITE;
        else if (!(t.w > 0.0) || t.w > 1000.0) flag |= LBFS_FLAG_RHO_RANGE;
    }
    if (flag) atomicOr(a.flags, flag);
    // Block partial sums of the squared residuals (fixed order: warp tree, then warps in order).
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int m = 0; m < 4; m++) {
        double v = sq[m];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) sh[m][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int m = 0; m < 4; m++) {
            double v = 0;
            for (int w = 0; w < (int)(blockDim.x >> 5); w++) v += sh[m][w];
            a.partials[4 * blockIdx.x + m] = v;
        }
        __threadfence();
        const unsigned int prev = atomicAdd(a.ticket, 1u);
        last_block = (prev == gridDim.x - 1);
    }
    __syncthreads();
    if (last_block) {
        // Final sum of the block partials by the whole last block: thread t
        // adds partials t, t + blockDim, ... (fixed assignment), then the same
        // warp/block tree as above.  Deterministic for a fixed grid.
        __threadfence();
        double acc[4] = {0, 0, 0, 0};
        for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x)
#pragma unroll
            for (int m = 0; m < 4; m++) acc[m] += __ldcg(a.partials + 4 * b + m);
#pragma unroll
        for (int m = 0; m < 4; m++) {
            double v = acc[m];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
            if (lane == 0) sh[m][warp] = v;
        }
        __syncthreads();
        if (threadIdx.x < 4) {
            double v = 0;
            for (int w = 0; w < (int)(blockDim.x >> 5); w++) v += sh[threadIdx.x][w];
            a.residual_sums[threadIdx.x] = v;
        }
        if (threadIdx.x == 0) *a.ticket = 0u;
    }
}

// ------------------------------------------------------- state transfer ----

template <typename R>
__global__ void k_pack_state(FluidArgs<R> a, const double *__restrict__ stage) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.nc) return;
    const size_t n = (size_t)a.nc;
    const double rho = stage[i], u = stage[n + i], v = stage[2 * n + i], w = stage[3 * n + i];
    Vec4<R> s;
    s.u = (R)u; s.v = (R)v; s.w = (R)w; s.rho = (R)(rho - (double)a.rho0);
    a.state[i] = s;
    a.t1[i] = make_double4(u, v, w, rho);
}

template <typename R>
__global__ void k_unpack_state(FluidArgs<R> a, double *__restrict__ stage) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.nc) return;
    const size_t n = (size_t)a.nc;
    const Vec4<R> s = a.state[i];
    stage[i] = (double)s.rho + (double)a.rho0;
    stage[n + i] = (double)s.u;
    stage[2 * n + i] = (double)s.v;
    stage[3 * n + i] = (double)s.w;
}

// ------------------------------------------------------------ launchers ----

template <typename R> int k3_grid(const FluidArgs<R> &a) {
    const int g = (a.nc + a.tb_update - 1) / a.tb_update;
    return g < a.update_blocks ? g : a.update_blocks;
}

template <typename R> void launch_fluid_gradients_range(const FluidArgs<R> &a, int begin, int end, cudaStream_t s) {
    if (end <= begin) return;
    const int tb = a.tb_grad, g = (end - begin + tb - 1) / tb;
    if (tb == 128) k_cell_gradients<R, 128><<<g, 128, 0, s>>>(a, begin, end);
    else if (tb == 512) k_cell_gradients<R, 512><<<g, 512, 0, s>>>(a, begin, end);
    else k_cell_gradients<R, 256><<<g, 256, 0, s>>>(a, begin, end);
}
template <typename R> void launch_fluid_gradients(const FluidArgs<R> &a, cudaStream_t s) {
    launch_fluid_gradients_range<R>(a, 0, a.nc, s);
}
template <typename R> void launch_fluid_flux_axis_ranges(const FluidArgs<R> &a, const FaceRanges &r, cudaStream_t s) {
    const int n = r.count[0] + r.count[1] + r.count[2];
    if (!a.axis_aligned || n == 0) return;
    const int tb = a.tb_flux, g = (n + tb - 1) / tb;
    if (tb == 64) k_face_flux<R, 64><<<g, 64, 0, s>>>(a, r);
    else if (tb == 256) k_face_flux<R, 256><<<g, 256, 0, s>>>(a, r);
    else k_face_flux<R, 128><<<g, 128, 0, s>>>(a, r);
}
template <typename R> void launch_fluid_flux_axis(const FluidArgs<R> &a, cudaStream_t s) {
    const FaceRanges r = {{0, a.nfx, a.nfx + a.nfy}, {a.nfx, a.nfy, a.ni - a.nfx - a.nfy}};
    launch_fluid_flux_axis_ranges<R>(a, r, s);
}
template <typename R> void launch_fluid_flux_general(const FluidArgs<R> &a, cudaStream_t s) {
    const int first = a.axis_aligned ? a.ni : 0;
    if (a.nf <= first) return;
    const int tb = a.tb_gen, g = (a.nf - first + tb - 1) / tb;
    if (tb == 64) k_face_flux_general<R, 64><<<g, 64, 0, s>>>(a, first);
    else if (tb == 256) k_face_flux_general<R, 256><<<g, 256, 0, s>>>(a, first);
    else k_face_flux_general<R, 128><<<g, 128, 0, s>>>(a, first);
}
template <typename R> void launch_fluid_flux(const FluidArgs<R> &a, cudaStream_t s) {
    launch_fluid_flux_axis<R>(a, s);
    launch_fluid_flux_general<R>(a, s);
}
template <typename R> void launch_fluid_update(const FluidArgs<R> &a, cudaStream_t s) {
    const int tb = a.tb_update, g = k3_grid(a);
    if (tb == 128) k_cell_update<R, 128><<<g, 128, 0, s>>>(a);
    else if (tb == 512) k_cell_update<R, 512><<<g, 512, 0, s>>>(a);
    else k_cell_update<R, 256><<<g, 256, 0, s>>>(a);
}

template <typename R> void launch_fluid_cfl(const FluidArgs<R> &a, cudaStream_t s) {
    const int g = std::min(kCflBlocks, (a.nc + 255) / 256);
    k_cfl<R><<<g, 256, 0, s>>>(a);
}

template <typename R> void launch_pack_state(const FluidArgs<R> &a, const double *stage, cudaStream_t s) {
    k_pack_state<R><<<(a.nc + 255) / 256, 256, 0, s>>>(a, stage);
}
template <typename R> void launch_unpack_state(const FluidArgs<R> &a, double *stage, cudaStream_t s) {
    k_unpack_state<R><<<(a.nc + 255) / 256, 256, 0, s>>>(a, stage);
}
template void launch_pack_state<double>(const FluidArgs<double> &, const double *, cudaStream_t);
template void launch_pack_state<float>(const FluidArgs<float> &, const double *, cudaStream_t);
template void launch_unpack_state<double>(const FluidArgs<double> &, double *, cudaStream_t);
template void launch_unpack_state<float>(const FluidArgs<float> &, double *, cudaStream_t);

template void launch_fluid_gradients<double>(const FluidArgs<double> &, cudaStream_t);
template void launch_fluid_flux<double>(const FluidArgs<double> &, cudaStream_t);
template void launch_fluid_flux_axis<double>(const FluidArgs<double> &, cudaStream_t);
template void launch_fluid_flux_general<double>(const FluidArgs<double> &, cudaStream_t);
template void launch_fluid_flux_axis<float>(const FluidArgs<float> &, cudaStream_t);
template void launch_fluid_flux_general<float>(const FluidArgs<float> &, cudaStream_t);
template void launch_fluid_update<double>(const FluidArgs<double> &, cudaStream_t);
template void launch_fluid_gradients<float>(const FluidArgs<float> &, cudaStream_t);
template void launch_fluid_flux<float>(const FluidArgs<float> &, cudaStream_t);
template void launch_fluid_update<float>(const FluidArgs<float> &, cudaStream_t);
template void launch_fluid_cfl<double>(const FluidArgs<double> &, cudaStream_t);
template void launch_fluid_gradients_range<double>(const FluidArgs<double> &, int, int, cudaStream_t);
template void launch_fluid_gradients_range<float>(const FluidArgs<float> &, int, int, cudaStream_t);
template void launch_fluid_flux_axis_ranges<double>(const FluidArgs<double> &, const FaceRanges &, cudaStream_t);
template void launch_fluid_flux_axis_ranges<float>(const FluidArgs<float> &, const FaceRanges &, cudaStream_t);
template void launch_fluid_cfl<float>(const FluidArgs<float> &, cudaStream_t);

}  // namespace lbfs
