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
    pdl_trigger();  // the interior-face kernel may be scheduled behind the last wave
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
    LsW<R> W;
    if (a.lsw_code) {  // the weights from the per-mesh table by the cell's six 3-bit codes
        const unsigned code = __ldg(a.lsw_code + i);
#pragma unroll
        for (int q = 0; q < 6; q++) {
            const unsigned k = (code >> (3 * q)) & 7u;
#pragma unroll
            for (int r = 0; r < 3; r++) {
                R v = a.lsw_tab[0][r];
#pragma unroll
                for (unsigned t = 1; t < 8; t++) v = (k == t) ? a.lsw_tab[t][r] : v;
                W.w[3 * q + r] = v;
            }
        }
    } else {
        W = a.lsw[i];
    }
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

// Density offset of the stored state: 0 in FP64 (a compile-time zero, so no
// add is spent on it), rho0 in the FP32-bulk form.
template <typename R> __device__ __forceinline__ R rho0_of(const FluidArgs<R> &a) {
    if constexpr (sizeof(R) == 8) return R(0);
    else return a.rho0;
}

// Lattice population divided by its weight, g_k = f_k / w_k, at a reconstructed
// state L = (rho', u, v, w):  g = rho' + (rho' + rho0) X,
// X = 3 e.u + q (4.5 (e.u)^2 - 1.5 |u|^2).  The reference's equilibrium
// w_k rho (1 + X) (populate_feq_lattice_explicit, LBFS.cu:1041-1354; populate_feq,
// LBFS.cu:940-1036 with the preconditioning factor q) with the weight applied
// later, once per group of directions that share it.
template <typename R>
__device__ __forceinline__ R pop_g(const R (&L)[4], R eu, R rho0, R q) {
    const R usq = L[1] * L[1] + L[2] * L[2] + L[3] * L[3];
    const R X = R(3) * eu + q * (R(4.5) * eu * eu - R(1.5) * usq);
    if constexpr (sizeof(R) == 8) return L[0] + L[0] * X;
    else return L[0] + (L[0] + rho0) * X;
}

// FP32-bulk (deviation) form of pop_g at a reconstructed state written as
// L = p0 + d, p0 the face-centre state and d the direction's small offset
// from it.  The population's term 3 rho0 e.p0_u is large (the velocity
// itself) and the same for every direction, so that summing the populations
// over directions would cancel it and leave its FP32 rounding in the
// cross-stream moments; it is left out here, and its moments (rho0 p0_u in
// the first moment, zero in every other) are added once, exactly, by the
// caller.  The rest is formed from small terms only:
//   g~ = rho' (1 + X) + rho0 (3 e.d_u + q (4.5 (e.u)^2 - 1.5 |u|^2)).
// eu = e.u at L, edu = e.d_u.
__device__ __forceinline__ float pop_dev(const float (&L)[4], float eu, float edu, float rho0, float q) {
    const float usq = L[1] * L[1] + L[2] * L[2] + L[3] * L[3];
    const float Q = q * (4.5f * eu * eu - 1.5f * usq);
    const float X = 3.0f * eu + Q;
    return (L[0] + L[0] * X) + rho0 * (3.0f * edu + Q);
}

// Moments of the reconstructed lattice populations that the interface flux
// needs: rho = sum f, m_c = sum e_c f, d_c = sum_{e_c != 0} f (= sum e_c e_c f),
// o_xy, o_xz, o_yz = sum e_c e_m f.  Formed from sums and differences of
// opposite directions (the D3Q15 set is symmetric), then weighted once per
// group: a few dozen adds instead of one accumulation per direction and moment.
template <typename R> struct LatMoments {
    R rho, m[3], d[3], o[3];  // o: xy, xz, yz
};
template <typename R> __device__ __forceinline__ R o_of(const LatMoments<R> &M, int c, int q) {
    // symmetric second moment e_c e_q for c != q
    return (c + q == 1) ? M.o[0] : ((c + q == 2) ? M.o[1] : M.o[2]);
}

// Interface equilibrium, BGK relaxation towards the lattice populations and
// the flux through the face: calculate_flux_at_interface (LBFS.cu:1462-1648)
// and its axis-aligned forms (LBFS.cu:3648-4092).  The relaxed populations are
// f_k - tau (f_k - fl_k), f_k the interface equilibrium, so the flux tensor is
// (1 - tau) F_eq + tau F_fl, F_fl the moments of the lattice populations fl_k.
// The D3Q15 weights make the equilibrium moments exact closed forms
// (sum w e = 0, sum w e e = I / 3, sum w e e e e = (dd + dd + dd) / 9):
//   sum_k e_c f_k = rho u_c = m_c,  sum_k e_c e_q f_k = q_s m_c m_q / rho + d_cq rho' / 3
// (q_s the preconditioning factor; in the deviation form the d_cq term is
// rho' / 3).  So the mass flux is m . n exactly, and the momentum flux is
// formed from the six distinct second moments.  The reference sums the 15
// equilibria explicitly; the closed form is the same quantity with fewer
// roundings.  `axis` >= 0: only the face-normal component (axis-aligned faces,
// n = e_axis); `axis` < 0: all three with the face normal.
template <typename R>
__device__ __forceinline__ Vec4<R> interface_flux(const LatMoments<R> &M, R rho0, R tau, R qscale, R area, int axis,
                                                  R nx, R ny, R nz) {
    const R rho_i = M.rho + rho0;
    const R inv = R(1) / rho_i;
    const R keep = R(1) - tau;
    const R third = M.rho * R(1.0 / 3.0);
    // relaxed second moment c, q
    auto T = [&](int c, int q) -> R {
        R eq = qscale * (M.m[c] * inv) * M.m[q];
        R fl;
        if (c == q) {
            eq = eq + third;
            fl = M.d[c];
        } else {
            fl = o_of(M, c, q);
        }
        return keep * eq + tau * fl;
    };
    Vec4<R> out;
    if (axis >= 0) {
        out.rho = M.m[axis] * area;
        out.u = T(axis, 0) * area;
        out.v = T(axis, 1) * area;
        out.w = T(axis, 2) * area;
    } else {
        const R Txx = T(0, 0), Tyy = T(1, 1), Tzz = T(2, 2), Txy = T(0, 1), Txz = T(0, 2), Tyz = T(1, 2);
        out.rho = (M.m[0] * nx + M.m[1] * ny + M.m[2] * nz) * area;
        out.u = (Txx * nx + Txy * ny + Txz * nz) * area;
        out.v = (Txy * nx + Tyy * ny + Tyz * nz) * area;
        out.w = (Txz * nx + Tyz * ny + Tzz * nz) * area;
    }
    return out;
}

struct Dir {
    int ex, ey, ez;
};
__device__ __forceinline__ Dir dir_of(int k) { return {c_ex(k), c_ey(k), c_ez(k)}; }

template <typename R> __device__ __forceinline__ void load_grad(const R *g, R (&o)[12]) {
    const GradRec<R> r = *reinterpret_cast<const GradRec<R> *>(g);
#pragma unroll
    for (int t = 0; t < 12; t++) o[t] = r.g[t];
}

// The five directions of one side of an axis-A face: e_A = s (s = +1 owner
// side, -1 neighbour side) with (e_B, e_C) in {(0,0), (+,+), (+,-), (-,+), (-,-)}
// (B < C the other two axes).  populate_lattice_macros_uniform_{x,y,z}
// (LBFS.cu:2939-3644): the lattice node sits at x_f - e dt and is extrapolated
// from the side's cell: L = p - dt (e . g).  With a = p - s dt g_A,
// b = dt g_B, c = dt g_C the four corners are (a -+ b) -+ c.  Returns the
// side's weighted sums S = sum f, YB = sum e_B f, YC = sum e_C f.
template <typename R, int A>
__device__ __forceinline__ void axis_side(const R (&p)[4], const R (&g)[12], R s, R dt, R rho0, R &S, R &YB,
                                          R &YC) {
    constexpr int B = A == 0 ? 1 : 0, C = A == 2 ? 1 : 2;
    R av[4], amb[4], apb[4], cv[4];
#pragma unroll
    for (int m = 0; m < 4; m++) {
        av[m] = p[m] - s * dt * g[3 * m + A];
        const R b = dt * g[3 * m + B];
        cv[m] = dt * g[3 * m + C];
        amb[m] = av[m] - b;  // e_B = +1
        apb[m] = av[m] + b;  // e_B = -1
    }
    // e = (s e_A, e_B, e_C) in (A, B, C) order; e.u = s u_A + e_B u_B + e_C u_C
    const R g0 = pop_g<R>(av, s * av[1 + A], rho0, R(1));
    R Lc[4], gpp, gpm, gmp, gmm;
#pragma unroll
    for (int m = 0; m < 4; m++) Lc[m] = amb[m] - cv[m];
    gpp = pop_g<R>(Lc, s * Lc[1 + A] + Lc[1 + B] + Lc[1 + C], rho0, R(1));
#pragma unroll
    for (int m = 0; m < 4; m++) Lc[m] = amb[m] + cv[m];
    gpm = pop_g<R>(Lc, s * Lc[1 + A] + Lc[1 + B] - Lc[1 + C], rho0, R(1));
#pragma unroll
    for (int m = 0; m < 4; m++) Lc[m] = apb[m] - cv[m];
    gmp = pop_g<R>(Lc, s * Lc[1 + A] - Lc[1 + B] + Lc[1 + C], rho0, R(1));
#pragma unroll
    for (int m = 0; m < 4; m++) Lc[m] = apb[m] + cv[m];
    gmm = pop_g<R>(Lc, s * Lc[1 + A] - Lc[1 + B] - Lc[1 + C], rho0, R(1));
    const R bp = gpp + gpm, bm = gmp + gmm, cp = gpp - gpm, cm = gmp - gmm;
    constexpr R w_axis = R(1.0 / 9.0), w_corner = R(1.0 / 72.0);
    S = w_axis * g0 + w_corner * (bp + bm);
    YB = w_corner * (bp - bm);
    YC = w_corner * (cp + cm);
}

// The same five directions in the deviation form: the side's offsets from
// the face centre, d = s (hdp - dt g_A) -+ dt g_B -+ dt g_C (hdp half the
// owner-neighbour difference of the reconstructed states), and L = p0 + d.
template <int A>
__device__ __forceinline__ void axis_side_dev(const float (&p0)[4], const float (&hdp)[4], const float (&g)[12],
                                              float s, float dt, float rho0, float &S, float &YB, float &YC) {
    constexpr int B = A == 0 ? 1 : 0, C = A == 2 ? 1 : 2;
    float ad[4], amb[4], apb[4], cv[4];
#pragma unroll
    for (int m = 0; m < 4; m++) {
        ad[m] = s * (hdp[m] - dt * g[3 * m + A]);
        const float b = dt * g[3 * m + B];
        cv[m] = dt * g[3 * m + C];
        amb[m] = ad[m] - b;
        apb[m] = ad[m] + b;
    }
    float L[4], d[4];
#pragma unroll
    for (int m = 0; m < 4; m++) L[m] = p0[m] + ad[m];
    const float g0 = pop_dev(L, s * L[1 + A], s * ad[1 + A], rho0, 1.0f);
    float gq[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const float eb = (q < 2) ? 1.0f : -1.0f, ec = (q & 1) ? -1.0f : 1.0f;  // (+,+), (+,-), (-,+), (-,-)
#pragma unroll
        for (int m = 0; m < 4; m++) {
            d[m] = ((q < 2) ? amb[m] : apb[m]) - ec * cv[m];
            L[m] = p0[m] + d[m];
        }
        gq[q] = pop_dev(L, s * L[1 + A] + eb * L[1 + B] + ec * L[1 + C], s * d[1 + A] + eb * d[1 + B] + ec * d[1 + C],
                        rho0, 1.0f);
    }
    const float bp = gq[0] + gq[1], bm = gq[2] + gq[3], cp = gq[0] - gq[1], cm = gq[2] - gq[3];
    S = (1.0f / 9.0f) * g0 + (1.0f / 72.0f) * (bp + bm);
    YB = (1.0f / 72.0f) * (bp - bm);
    YC = (1.0f / 72.0f) * (cp + cm);
}

// Axis-aligned interior face of axis A (calc_face_flux_x/_y/_z, LBFS.cu:2283-2569):
// directions with e_A = +1 extrapolate from the owner, -1 from the neighbour,
// 0 from the face centre with the distance-weighted gradient.
template <typename R, int A>
__device__ __forceinline__ Vec4<R> axis_face_flux(const FluidArgs<R> &a, int f) {
    constexpr int B = A == 0 ? 1 : 0, C = A == 2 ? 1 : 2;
    const int2 oc = __ldg(a.face_cells + f);
    AxisFace<R> geo;
    R wa, wb;
    if (a.axis_uniform) {
        geo = {a.axis_geo[A][0], a.axis_geo[A][1], a.axis_geo[A][2], a.axis_geo[A][3]};
        wa = a.axis_wa[A];
        wb = a.axis_wb[A];
    } else {
        geo = a.axis_face[f];
        const R ic = R(1) / (geo.t2 - geo.t1);
        wa = fabs(geo.t2 * ic);
        wb = fabs(geo.t1 * ic);
    }
    const Vec4<R> s1 = a.state[oc.x], s2 = a.state[oc.y];
    R g1[12], g2[12];
    load_grad(a.grad + (size_t)12 * oc.x, g1);
    load_grad(a.grad + (size_t)12 * oc.y, g2);
    const R rho0 = rho0_of(a);
    const R dt = geo.dt, t1 = geo.t1, t2 = geo.t2;
    const R S1[4] = {s1.rho, s1.u, s1.v, s1.w}, S2[4] = {s2.rho, s2.u, s2.v, s2.w};
    R pi[4], pn[4], p0[4];
#pragma unroll
    for (int m = 0; m < 4; m++) {
        pi[m] = S1[m] - t1 * g1[3 * m + A];
        pn[m] = S2[m] - t2 * g2[3 * m + A];
        p0[m] = (pi[m] + pn[m]) * R(0.5);
    }
    LatMoments<R> M;
    R Sp, Bp, Cp, Sn, Bn, Cn;
    if constexpr (sizeof(R) == 8) {
        axis_side<R, A>(pi, g1, R(1), dt, rho0, Sp, Bp, Cp);
        axis_side<R, A>(pn, g2, R(-1), dt, rho0, Sn, Bn, Cn);
    } else {
        // half the owner-neighbour difference, from the states' difference (exact for close values)
        R hdp[4];
#pragma unroll
        for (int m = 0; m < 4; m++) hdp[m] = ((S1[m] - S2[m]) - (t1 * g1[3 * m + A] - t2 * g2[3 * m + A])) * R(0.5);
        axis_side_dev<A>(p0, hdp, g1, 1.0f, dt, rho0, Sp, Bp, Cp);
        axis_side_dev<A>(p0, hdp, g2, -1.0f, dt, rho0, Sn, Bn, Cn);
    }
    // centre directions (e_A = 0): rest, +-B, +-C, from p0 with gi = wa g1 + wb g2
    R gz0, gbp, gbm, gcp, gcm;
    if constexpr (sizeof(R) == 4) {
        R bv[4], cv[4], L[4];
#pragma unroll
        for (int m = 0; m < 4; m++) {
            bv[m] = dt * (g1[3 * m + B] * wa + g2[3 * m + B] * wb);
            cv[m] = dt * (g1[3 * m + C] * wa + g2[3 * m + C] * wb);
        }
        gz0 = pop_dev(p0, R(0), R(0), rho0, R(1));
#pragma unroll
        for (int m = 0; m < 4; m++) L[m] = p0[m] - bv[m];
        gbp = pop_dev(L, L[1 + B], -bv[1 + B], rho0, R(1));
#pragma unroll
        for (int m = 0; m < 4; m++) L[m] = p0[m] + bv[m];
        gbm = pop_dev(L, -L[1 + B], -bv[1 + B], rho0, R(1));
#pragma unroll
        for (int m = 0; m < 4; m++) L[m] = p0[m] - cv[m];
        gcp = pop_dev(L, L[1 + C], -cv[1 + C], rho0, R(1));
#pragma unroll
        for (int m = 0; m < 4; m++) L[m] = p0[m] + cv[m];
        gcm = pop_dev(L, -L[1 + C], -cv[1 + C], rho0, R(1));
    } else {
        R bv[4], cv[4], L[4];
#pragma unroll
        for (int m = 0; m < 4; m++) {
            bv[m] = dt * (g1[3 * m + B] * wa + g2[3 * m + B] * wb);
            cv[m] = dt * (g1[3 * m + C] * wa + g2[3 * m + C] * wb);
        }
        gz0 = pop_g<R>(p0, R(0), rho0, R(1));
#pragma unroll
        for (int m = 0; m < 4; m++) L[m] = p0[m] - bv[m];
        gbp = pop_g<R>(L, L[1 + B], rho0, R(1));
#pragma unroll
        for (int m = 0; m < 4; m++) L[m] = p0[m] + bv[m];
        gbm = pop_g<R>(L, -L[1 + B], rho0, R(1));
#pragma unroll
        for (int m = 0; m < 4; m++) L[m] = p0[m] - cv[m];
        gcp = pop_g<R>(L, L[1 + C], rho0, R(1));
#pragma unroll
        for (int m = 0; m < 4; m++) L[m] = p0[m] + cv[m];
        gcm = pop_g<R>(L, -L[1 + C], rho0, R(1));
    }
    constexpr R w_rest = R(2.0 / 9.0), w_axis = R(1.0 / 9.0);
    const R Sz = w_rest * gz0 + w_axis * ((gbp + gbm) + (gcp + gcm));
    const R Bz = w_axis * (gbp - gbm), Cz = w_axis * (gcp - gcm);
    M.rho = (Sp + Sn) + Sz;
    M.m[A] = Sp - Sn;
    M.d[A] = Sp + Sn;
    M.m[B] = (Bp + Bn) + Bz;
    M.m[C] = (Cp + Cn) + Cz;
    M.o[A + B - 1] = Bp - Bn;  // o index of the pair (A, B): xy 0, xz 1, yz 2
    M.o[A + C - 1] = Cp - Cn;
    M.d[B] = M.d[C] = M.o[B + C - 1] = R(0);  // not read by the axis-A flux
    if constexpr (sizeof(R) == 4) {
        // first moments of the left-out term 3 rho0 e.p0_u (pop_dev)
#pragma unroll
        for (int c = 0; c < 3; c++) M.m[c] = M.m[c] + rho0 * p0[1 + c];
    }
    const R vf = a.visc_factor[oc.x];
    const R tau = (a.testcase == 8) ? R(0) : (a.visc * vf * R(3) / dt * a.gamma_inv);
    return interface_flux<R>(M, rho0, tau, R(1), geo.area, A, 0, 0, 0);
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
    const R rho0 = rho0_of(a);
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
    R pi[4], pn[4], p0[4];
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
        for (int t = 0; t < 12; t++) g1[t] = g2[t];
    } else {
#pragma unroll
        for (int m = 0; m < 4; m++) {
            pi[m] = S1[m] - (geo.t1x * g1[3 * m] + geo.t1y * g1[3 * m + 1] + geo.t1z * g1[3 * m + 2]);
            pn[m] = S2[m] - (geo.t2x * g2[3 * m] + geo.t2y * g2[3 * m + 1] + geo.t2z * g2[3 * m + 2]);
            p0[m] = (pi[m] + pn[m]) * R(0.5);
        }
    }
    // FP32 deviation form: offsets from the face centre (pop_dev); hdp is half
    // the owner-neighbour difference of the reconstructed states
    R hdp[4] = {R(0), R(0), R(0), R(0)};
    if constexpr (sizeof(R) == 4) {
        if (geo.bc_branch == R(0)) {
#pragma unroll
            for (int m = 0; m < 4; m++)
                hdp[m] = ((S1[m] - S2[m]) - ((geo.t1x * g1[3 * m] + geo.t1y * g1[3 * m + 1] + geo.t1z * g1[3 * m + 2]) -
                                             (geo.t2x * g2[3 * m] + geo.t2y * g2[3 * m + 1] + geo.t2z * g2[3 * m + 2]))) *
                         R(0.5);
        }
    }
    // Upwind selection by the sign of n.e_k with the threshold 0.001 dt
    // (LBFS.cu:351-352 override the sin(pi/14) arguments).  Directions come in
    // opposite pairs (k, k + 1): sum and difference of the pair's populations
    // feed the moments.
    const R thr = R(0.001) * dt;
    const R q = a.recon_q;
    R g0;
    if constexpr (sizeof(R) == 4) g0 = pop_dev(p0, R(0), R(0), rho0, q);
    else g0 = pop_g<R>(p0, R(0), rho0, q);
    R sax[3], dax[3];          // axis pairs (+e_c, -e_c): sum and difference
    R sc, mcor[3], ocor[3];    // corner pairs: sum of sums; sum of e_c x difference; of e_c e_q x sum
#pragma unroll
    for (int k = 1; k < 15; k += 2) {
        const Dir e = dir_of(k);  // odd k: e_k; k + 1: -e_k
        const int ee[3] = {e.ex, e.ey, e.ez};
        const R s = (k < 7) ? (e.ex ? geo.nx : (e.ey ? geo.ny : geo.nz))
                            : (R(e.ex) * geo.nx + R(e.ey) * geo.ny + R(e.ez) * geo.nz);
        // Upwind sides.  With sg = -1 where n.e < -thr and +1 otherwise, the population of
        // direction sg e comes from the owner and that of -sg e from the neighbour, each
        // extrapolated along its own direction: Lo = p_owner - sg dt (e . g_owner),
        // Ln = p_neighbour + sg dt (e . g_neighbour).  Where |n.e| <= thr (cen) both come from
        // the face centre with the mean gradient C (sg = +1: +e at Lo, -e at Ln).  Only warps
        // with such a lane take the selects; in the others the side is a sign of dt.
        const bool neg = s < -thr, cen = !(s > thr) && !neg;
        const R sg = neg ? R(-1) : R(1);
        const R sdt = sg * dt;
        R A[4], B[4];  // e . gradient per component, owner (A) and neighbour (B)
#pragma unroll
        for (int m = 0; m < 4; m++) {
            bool first = true;
#pragma unroll
            for (int d = 0; d < 3; d++) {
                if (!ee[d]) continue;
                const R ga = ee[d] > 0 ? g1[3 * m + d] : -g1[3 * m + d];
                const R gb = ee[d] > 0 ? g2[3 * m + d] : -g2[3 * m + d];
                A[m] = first ? ga : A[m] + ga;
                B[m] = first ? gb : B[m] + gb;
                first = false;
            }
        }
        R Lo[4], Ln[4], Do[4], Dn[4];
        if (__any_sync(__activemask(), cen)) {
#pragma unroll
            for (int m = 0; m < 4; m++) {
                const R C = (A[m] + B[m]) * R(0.5);
                const R Xo = cen ? C : A[m], Xn = cen ? C : B[m];
                if constexpr (sizeof(R) == 8) {
                    Lo[m] = (cen ? p0[m] : pi[m]) - sdt * Xo;
                    Ln[m] = (cen ? p0[m] : pn[m]) + sdt * Xn;
                } else {
                    // FP32: offsets from the face centre (+hdp owner, -hdp neighbour, 0 centre)
                    Do[m] = (cen ? R(0) : hdp[m]) - sdt * Xo;
                    Dn[m] = (cen ? R(0) : -hdp[m]) + sdt * Xn;
                    Lo[m] = p0[m] + Do[m];
                    Ln[m] = p0[m] + Dn[m];
                }
            }
        } else {
#pragma unroll
            for (int m = 0; m < 4; m++) {
                if constexpr (sizeof(R) == 8) {
                    Lo[m] = pi[m] - sdt * A[m];
                    Ln[m] = pn[m] + sdt * B[m];
                } else {
                    Do[m] = hdp[m] - sdt * A[m];
                    Dn[m] = -hdp[m] + sdt * B[m];
                    Lo[m] = p0[m] + Do[m];
                    Ln[m] = p0[m] + Dn[m];
                }
            }
        }
        // e . u at both states (and e . d, FP32); the owner's direction is sg e, the neighbour's -sg e
        R Eo, En, Edo = R(0), Edn = R(0);
        {
            bool first = true;
#pragma unroll
            for (int d = 0; d < 3; d++) {
                if (!ee[d]) continue;
                const R uo = ee[d] > 0 ? Lo[1 + d] : -Lo[1 + d], un = ee[d] > 0 ? Ln[1 + d] : -Ln[1 + d];
                Eo = first ? uo : Eo + uo;
                En = first ? un : En + un;
                if constexpr (sizeof(R) == 4) {
                    const R dO = ee[d] > 0 ? Do[1 + d] : -Do[1 + d], dN = ee[d] > 0 ? Dn[1 + d] : -Dn[1 + d];
                    Edo = first ? dO : Edo + dO;
                    Edn = first ? dN : Edn + dN;
                }
                first = false;
            }
        }
        R go, gn;
        if constexpr (sizeof(R) == 4) {
            go = pop_dev(Lo, sg * Eo, sg * Edo, rho0, q);
            gn = pop_dev(Ln, -sg * En, -sg * Edn, rho0, q);
        } else {
            go = pop_g<R>(Lo, sg * Eo, rho0, q);
            gn = pop_g<R>(Ln, -sg * En, rho0, q);
        }
        // the pair's sum and its (+e) - (-e) difference
        const R sig = go + gn, del = sg * (go - gn);
        if (k < 7) {
            const int c = e.ex ? 0 : (e.ey ? 1 : 2);
            sax[c] = sig;
            dax[c] = del;
        } else if (k == 7) {  // (+,+,+): first corner pair
            sc = sig;
#pragma unroll
            for (int d = 0; d < 3; d++) { mcor[d] = del; ocor[d] = sig; }
        } else {
            sc = sc + sig;
#pragma unroll
            for (int d = 0; d < 3; d++) mcor[d] = (ee[d] > 0) ? mcor[d] + del : mcor[d] - del;
            ocor[0] = (ee[0] * ee[1] > 0) ? ocor[0] + sig : ocor[0] - sig;
            ocor[1] = (ee[0] * ee[2] > 0) ? ocor[1] + sig : ocor[1] - sig;
            ocor[2] = (ee[1] * ee[2] > 0) ? ocor[2] + sig : ocor[2] - sig;
        }
    }
    constexpr R w_rest = R(2.0 / 9.0), w_axis = R(1.0 / 9.0), w_corner = R(1.0 / 72.0);
    LatMoments<R> M;
    M.rho = w_rest * g0 + w_axis * ((sax[0] + sax[1]) + sax[2]) + w_corner * sc;
#pragma unroll
    for (int c = 0; c < 3; c++) {
        M.m[c] = w_axis * dax[c] + w_corner * mcor[c];
        M.d[c] = w_axis * sax[c] + w_corner * sc;
        M.o[c] = w_corner * ocor[c];
        if constexpr (sizeof(R) == 4) M.m[c] = M.m[c] + rho0 * p0[1 + c];  // the term pop_dev leaves out
    }
    const R vf = is_bc ? R(1) : a.visc_factor[oc.x];
    const R tau = (a.testcase == 8) ? R(0) : (a.visc * vf * R(3) / dt * a.gamma_inv);
    return interface_flux<R>(M, rho0, tau, a.gamma_inv, geo.area, -1, geo.nx, geo.ny, geo.nz);
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

// Interior faces of an axis-aligned mesh, tile by tile: block b takes the
// faces owned by the TB cells of tile tile0 + b -- the x, y and z faces whose
// owner lies in the tile, three contiguous ranges of the face list
// (tiles[3 t + axis] = first face of that axis owned by tile t) -- so the
// tile's cell states and gradients come from DRAM once for all three axes
// instead of once per axis sweep.  Warps take the x faces, then the y, then
// the z faces: one axis per warp at a time.  Load-latency bound: FP64 fits 96
// registers (20 warps per SM; at 80 it spills), FP32 64 (32 warps per SM).
template <typename R, int TB>
__global__ void __launch_bounds__(TB, (sizeof(R) == 4 ? 1024 : 640) / TB) k_face_flux_tiles(FluidArgs<R> a, int tile0) {
    pdl_trigger();
    const int *tp = a.flux_tiles + 3 * (tile0 + (int)blockIdx.x);
    const int f0x = __ldg(tp), f0y = __ldg(tp + 1), f0z = __ldg(tp + 2);
    const int f1x = __ldg(tp + 3), f1y = __ldg(tp + 4), f1z = __ldg(tp + 5);
    pdl_wait();  // the gradients
    for (int f = f0x + (int)threadIdx.x; f < f1x; f += TB) a.flux[f] = axis_face_flux<R, 0>(a, f);
    for (int f = f0y + (int)threadIdx.x; f < f1y; f += TB) a.flux[f] = axis_face_flux<R, 1>(a, f);
    for (int f = f0z + (int)threadIdx.x; f < f1z; f += TB) a.flux[f] = axis_face_flux<R, 2>(a, f);
}

// Interior faces of a mesh that is not axis aligned (every face takes the
// general-normal reconstruction), tile by tile as k_face_flux_tiles: block b
// takes the faces owned by the TB cells of tile tile0 + b, in up to three
// face ranges ordered by owner (the generator's x, y, z faces; an imported
// mesh's internal faces, which OpenFOAM orders by owner, form one range).
// FP64 at 128 registers (16 warps per SM; at 96 it spills 1.4 KB a thread), FP32 at 64 (32 warps
// per SM, 44 B spilled; 6 % faster than at 80 registers and 24 warps).
template <typename R, int TB>
__global__ void __launch_bounds__(TB, (sizeof(R) == 4 ? 1024 : 512) / TB) k_face_flux_general_tiles(FluidArgs<R> a, int tile0) {
    pdl_trigger();
    pdl_wait();  // the gradients
    const int *tp = a.flux_tiles + 3 * (tile0 + (int)blockIdx.x);
#pragma unroll 1
    for (int r = 0; r < 3; r++) {
        const int f0 = __ldg(tp + r), f1 = __ldg(tp + 3 + r);
        for (int f = f0 + (int)threadIdx.x; f < f1; f += TB) a.flux[f] = general_face_flux<R>(a, f, false);
    }
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
    // one instance with few membranes: its grid and the membranes' patches cached per block,
    // with each patch's first and last linear cell (cells outside skip the i, j, k split)
    __shared__ int s_grid[6];                 // cell0, nx, ny, nz, mem0, mem1
    __shared__ int s_patch[kK3PatchCache][10];  // lo[3], dim[3], cells, off, first, last linear cell
    pdl_wait();  // the face fluxes
    const bool cached = a.n_membranes > 0 && a.n_membranes <= kK3PatchCache && !a.cell_instance;
    if (cached) {
        const InstanceGrid g0 = reinterpret_cast<const InstanceGrid *>(a.instances)[0];
        if (threadIdx.x == 0) {
            s_grid[0] = g0.cell0; s_grid[1] = g0.nx; s_grid[2] = g0.ny; s_grid[3] = g0.nz;
            s_grid[4] = g0.mem0; s_grid[5] = g0.mem1;
        }
        const MembraneScalars *ms = (const MembraneScalars *)a.membrane_scalars;
        if ((int)threadIdx.x < a.n_membranes) {
            const MembraneScalars &q = ms[threadIdx.x];
            int *e = s_patch[threadIdx.x];
            for (int c = 0; c < 3; c++) { e[c] = q.patch_lo[c]; e[3 + c] = q.patch_dim[c]; }
            e[6] = q.patch_cells;
            e[7] = q.patch_off;
            e[8] = q.patch_lo[0] + g0.nx * (q.patch_lo[1] + g0.ny * q.patch_lo[2]);
            e[9] = (q.patch_lo[0] + q.patch_dim[0] - 1) +
                   g0.nx * ((q.patch_lo[1] + q.patch_dim[1] - 1) + g0.ny * (q.patch_lo[2] + q.patch_dim[2] - 1));
        }
        __syncthreads();
    }
    double sq[4] = {0, 0, 0, 0};
    unsigned int flag = 0;
    // the step: constant, or the minimum per-cell step, or each cell's own (LBFS_DT_LOCAL)
    const bool local_dt = a.time_stepping == LBFS_DT_LOCAL;
    const double dt_all = (a.time_stepping == LBFS_DT_MIN || a.time_stepping == LBFS_DT_TALTS) ? __ldcg(a.dt_min)
                                                                                                 : a.delta_t;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.nc; i += gridDim.x * blockDim.x) {
        // 1 / volume: products instead of 24 divisions
        const double iv = a.inv_volume_uniform ? a.inv_volume_all : __ldg(a.cell_inv_volume + i);
        double r[4] = {0, 0, 0, 0};  // rho, u, v, w
        int cfl[6];
        if (a.grid_faces) {  // the structured mesh's faces, formed (no dependent load before the fluxes)
            grid_cell_faces(i, a.grid_n[0], a.grid_n[1], a.grid_n[2], cfl);
        } else {
#pragma unroll
            for (int q = 0; q < 3; q++) {
                const int2 p = __ldg(reinterpret_cast<const int2 *>(a.cell_faces) + 3 * i + q);
                cfl[2 * q] = p.x;
                cfl[2 * q + 1] = p.y;
            }
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
        if (cached) {
            const int li = i - s_grid[0];
            for (int m = s_grid[4]; m < s_grid[5]; m++) {
                const int *e = s_patch[m];
                if (e[6] <= 0 || li < e[8] || li > e[9]) continue;
                const int nx = s_grid[1], ny = s_grid[2];
                const int ci = li % nx, cj = (li / nx) % ny, ck = li / (nx * ny);
                const int px = ci - e[0], py = cj - e[1], pz = ck - e[2];
                if (px >= 0 && py >= 0 && pz >= 0 && px < e[3] && py < e[4] && pz < e[5]) {
                    const double *pf = a.patch_force + ((size_t)e[7] + (px + e[3] * (py + e[4] * pz))) * 3;
                    fx = fx + pf[0];
                    fy = fy + pf[1];
                    fz = fz + pf[2];
                }
            }
        } else if (a.n_membranes > 0) {
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
// A launch with the programmatic-serialization attribute when `pdl` (the
// kernel directly behind the kernel whose output it reads, on the same stream).
template <typename... KArgs, typename... Args>
void launch_maybe_pdl(void (*kernel)(KArgs...), int g, int tb, cudaStream_t s, bool pdl, Args... args) {
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
template <typename R>
void launch_fluid_flux_tiles(const FluidArgs<R> &a, int tile0, int tile1, cudaStream_t s, bool pdl) {
    const int g = tile1 - tile0;
    if (g <= 0) return;
    if (!a.axis_aligned) {
        if (a.tb_gen == 64) launch_maybe_pdl(k_face_flux_general_tiles<R, 64>, g, 64, s, pdl, a, tile0);
        else if (a.tb_gen == 256) launch_maybe_pdl(k_face_flux_general_tiles<R, 256>, g, 256, s, pdl, a, tile0);
        else launch_maybe_pdl(k_face_flux_general_tiles<R, 128>, g, 128, s, pdl, a, tile0);
        return;
    }
    if (a.tb_flux == 64) launch_maybe_pdl(k_face_flux_tiles<R, 64>, g, 64, s, pdl, a, tile0);
    else if (a.tb_flux == 256) launch_maybe_pdl(k_face_flux_tiles<R, 256>, g, 256, s, pdl, a, tile0);
    else launch_maybe_pdl(k_face_flux_tiles<R, 128>, g, 128, s, pdl, a, tile0);
}
template <typename R> void launch_fluid_flux_axis(const FluidArgs<R> &a, cudaStream_t s, bool pdl) {
    if (a.flux_tiles) {  // interior faces by tiles (axis-aligned or general-normal kernel)
        launch_fluid_flux_tiles<R>(a, 0, a.n_tiles, s, pdl);
        return;
    }
    const FaceRanges r = {{0, a.nfx, a.nfx + a.nfy}, {a.nfx, a.nfy, a.ni - a.nfx - a.nfy}};
    launch_fluid_flux_axis_ranges<R>(a, r, s);
}
// Boundary faces of an axis-aligned mesh: a short launch of long threads (a
// one-wave grid that forms ghost records and general-normal fluxes) that runs
// beside the interior-face tiles on another stream.  Launched with the
// device's greatest scheduling priority so that its blocks are placed first
// and finish under the interior faces instead of after them (the step graph is
// instantiated with per-node priorities).
template <typename R, int TB> void launch_general(const FluidArgs<R> &a, int first, int g, cudaStream_t s, bool hi) {
    if (!hi) {
        k_face_flux_general<R, TB><<<g, TB, 0, s>>>(a, first);
        return;
    }
    int lo = 0, top = 0;
    cudaDeviceGetStreamPriorityRange(&lo, &top);
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributePriority;
    attr[0].val.priority = top;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(g);
    cfg.blockDim = dim3(TB);
    cfg.stream = s;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, k_face_flux_general<R, TB>, a, first);
}
template <typename R> void launch_fluid_flux_general(const FluidArgs<R> &a, cudaStream_t s) {
    // boundary faces only when the interior faces have a kernel of their own (axis faces, or tiles)
    const bool bc_only = a.axis_aligned || a.flux_tiles;
    const int first = bc_only ? a.ni : 0;
    if (a.nf <= first) return;
    const int tb = a.tb_gen, g = (a.nf - first + tb - 1) / tb;
    const bool hi = bc_only;  // beside the interior-face kernel
    if (tb == 64) launch_general<R, 64>(a, first, g, s, hi);
    else if (tb == 256) launch_general<R, 256>(a, first, g, s, hi);
    else launch_general<R, 128>(a, first, g, s, hi);
}
template <typename R> void launch_fluid_flux(const FluidArgs<R> &a, cudaStream_t s) {
    launch_fluid_flux_axis<R>(a, s);
    launch_fluid_flux_general<R>(a, s);
}
template <typename R> void launch_fluid_update(const FluidArgs<R> &a, cudaStream_t s, bool pdl) {
    const int tb = a.tb_update, g = k3_grid(a);
    if (tb == 128) launch_maybe_pdl(k_cell_update<R, 128>, g, 128, s, pdl, a);
    else if (tb == 512) launch_maybe_pdl(k_cell_update<R, 512>, g, 512, s, pdl, a);
    else launch_maybe_pdl(k_cell_update<R, 256>, g, 256, s, pdl, a);
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
template void launch_fluid_flux_axis<double>(const FluidArgs<double> &, cudaStream_t, bool);
template void launch_fluid_flux_general<double>(const FluidArgs<double> &, cudaStream_t);
template void launch_fluid_flux_axis<float>(const FluidArgs<float> &, cudaStream_t, bool);
template void launch_fluid_flux_general<float>(const FluidArgs<float> &, cudaStream_t);
template void launch_fluid_update<double>(const FluidArgs<double> &, cudaStream_t, bool);
template void launch_fluid_gradients<float>(const FluidArgs<float> &, cudaStream_t);
template void launch_fluid_flux<float>(const FluidArgs<float> &, cudaStream_t);
template void launch_fluid_update<float>(const FluidArgs<float> &, cudaStream_t, bool);
template void launch_fluid_cfl<double>(const FluidArgs<double> &, cudaStream_t);
template void launch_fluid_gradients_range<double>(const FluidArgs<double> &, int, int, cudaStream_t);
template void launch_fluid_gradients_range<float>(const FluidArgs<float> &, int, int, cudaStream_t);
template void launch_fluid_flux_axis_ranges<double>(const FluidArgs<double> &, const FaceRanges &, cudaStream_t);
template void launch_fluid_flux_axis_ranges<float>(const FluidArgs<float> &, const FaceRanges &, cudaStream_t);
template void launch_fluid_flux_tiles<double>(const FluidArgs<double> &, int, int, cudaStream_t, bool);
template void launch_fluid_flux_tiles<float>(const FluidArgs<float> &, int, int, cudaStream_t, bool);
template void launch_fluid_cfl<float>(const FluidArgs<float> &, cudaStream_t);

}  // namespace lbfs
