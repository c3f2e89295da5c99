// The generator's hex meshes built on a GPU: vertices, faces, cell geometry,
// ghost cells and least-squares matrices, one thread per vertex, face or cell,
// with the same arithmetic as the host builder (host_setup.cpp) in the same
// order: every product, sum, quotient and square root is an explicitly rounded
// intrinsic (no multiply-add contraction), the host compiles with
// -ffp-contract=off, and glibc's pow(x, 2) equals x * x, so the arrays come
// out bit for bit those of lbfs_mesh_build_rectilinear / _jittered.  Sums over
// a cell's faces, which the host accumulates face by face, are gathered per
// cell in increasing face order.  Imported meshes (an OpenFOAM polyMesh) take
// the same kernels with their topology from lists instead of the generator's
// closed forms: the arrays of lbfs_mesh_import_openfoam bit for bit.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "lbfs_b200.h"
#include "lbfs_internal.h"
#include "lbfs_mesh_common.h"

namespace lbfs {
namespace {

struct D3 {
    double x, y, z;
};
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dvd(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ D3 sub3(D3 a, D3 b) { return {sub(a.x, b.x), sub(a.y, b.y), sub(a.z, b.z)}; }
__device__ __forceinline__ D3 add3(D3 a, D3 b) { return {add(a.x, b.x), add(a.y, b.y), add(a.z, b.z)}; }
__device__ __forceinline__ D3 cross3(D3 a, D3 b) {
    return {sub(mul(a.y, b.z), mul(a.z, b.y)), sub(mul(a.z, b.x), mul(a.x, b.z)), sub(mul(a.x, b.y), mul(a.y, b.x))};
}
__device__ __forceinline__ double dot3(D3 a, D3 b) { return add(add(mul(a.x, b.x), mul(a.y, b.y)), mul(a.z, b.z)); }
// vector_var::Magnitude: sqrt(pow(x, 2) + pow(y, 2) + pow(z, 2))
__device__ __forceinline__ double mag3(D3 a) {
    return __dsqrt_rn(add(add(mul(a.x, a.x), mul(a.y, a.y)), mul(a.z, a.z)));
}

struct MeshDims {
    int nx, ny, nz, nvx, nvy, nvz;
    int nc, nf, ni, nfx, nfy;
    double dx, dy, dz, jitter, reference_dt;
    unsigned long long seed;
    int closed_faces, hybrid;
};

// Vertices (float, as unstructured_mesh.h:59 stores them): the axis
// coordinates, interior ones moved by jitter * spacing * jitter_unit.
__global__ void k_mesh_vertices(MeshDims m, const double *ax, const double *ay, const double *az, float *vx,
                                float *vy, float *vz) {
    const long long nv = (long long)m.nvx * m.nvy * m.nvz;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nv; t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t % m.nvx), j = (int)((t / m.nvx) % m.nvy), k = (int)(t / ((long long)m.nvx * m.nvy));
        double px = ax[i], py = ay[j], pz = az[k];
        if (m.jitter > 0 && i > 0 && j > 0 && k > 0 && i < m.nvx - 1 && j < m.nvy - 1 && k < m.nvz - 1) {
            px = add(px, mul(mul(m.jitter, m.dx), jitter_unit(m.seed, (unsigned long long)t, 0)));
            py = add(py, mul(mul(m.jitter, m.dy), jitter_unit(m.seed, (unsigned long long)t, 1)));
            pz = add(pz, mul(mul(m.jitter, m.dz), jitter_unit(m.seed, (unsigned long long)t, 2)));
        }
        vx[t] = __double2float_rn(px);
        vy[t] = __double2float_rn(py);
        vz[t] = __double2float_rn(pz);
    }
}

// Face f of the generator (unstructured_mesh.cpp:415-664): its four vertices
// in winding order and its owner; interior faces also their neighbour.  x,
// y, z interior faces, then the patches left, right, bottom, top, back,
// front, each in the generator's loop order.
__device__ void face_topology(const MeshDims &m, int f, int (&v)[4], int &own, int &nb) {
    const int sxy = m.nvx * m.nvy, nxy = m.nx * m.ny;
    nb = -1;
    if (f < m.nfx) {  // i in 1 .. nvx-2 fastest, then j, k
        const int i = 1 + f % (m.nx - 1), j = (f / (m.nx - 1)) % m.ny, k = f / ((m.nx - 1) * m.ny);
        const int a = k * sxy + j * m.nvx + i, b = a + m.nvx;
        v[0] = a; v[1] = b; v[2] = b + sxy; v[3] = a + sxy;
        own = (i - 1) + j * m.nx + k * nxy;
        nb = own + 1;
        return;
    }
    f -= m.nfx;
    if (f < m.nfy) {  // i fastest, j in 1 .. nvy-2, k
        const int i = f % m.nx, j = 1 + (f / m.nx) % (m.ny - 1), k = f / (m.nx * (m.ny - 1));
        const int a = k * sxy + j * m.nvx + i, b = a + sxy;
        v[0] = a; v[1] = b; v[2] = b + 1; v[3] = a + 1;
        own = i + (j - 1) * m.nx + k * nxy;
        nb = own + m.nx;
        return;
    }
    f -= m.nfy;
    const int nfz = m.ni - m.nfx - m.nfy;
    if (f < nfz) {  // i fastest, j, k in 1 .. nvz-2
        const int i = f % m.nx, j = (f / m.nx) % m.ny, k = 1 + f / nxy;
        const int a = k * sxy + j * m.nvx + i, b = a + 1, c = b + m.nvx;
        v[0] = a; v[1] = b; v[2] = c; v[3] = c - 1;
        own = i + j * m.nx + (k - 1) * nxy;
        nb = own + nxy;
        return;
    }
    f -= nfz;
    const int nyz = m.ny * m.nz, nxz = m.nx * m.nz;
    if (f < 2 * nyz) {  // left, right: j fastest, k
        const bool right = f >= nyz;
        const int r = right ? f - nyz : f, j = r % m.ny, k = r / m.ny;
        const int i = right ? m.nvx - 1 : 0, a = k * sxy + j * m.nvx + i;
        if (!right) {
            v[0] = a; v[1] = a + sxy; v[2] = a + m.nvx + sxy; v[3] = a + m.nvx;
            own = j * m.nx + k * nxy;
        } else {
            const int b = a + m.nvx;
            v[0] = a; v[1] = b; v[2] = b + sxy; v[3] = a + sxy;
            own = (i - 1) + j * m.nx + k * nxy;
        }
        return;
    }
    f -= 2 * nyz;
    if (f < 2 * nxz) {  // bottom, top: i fastest, k
        const bool top = f >= nxz;
        const int r = top ? f - nxz : f, i = r % m.nx, k = r / m.nx;
        const int j = top ? m.nvy - 1 : 0, a = k * sxy + j * m.nvx + i;
        if (!top) {
            v[0] = a; v[1] = a + 1; v[2] = a + sxy + 1; v[3] = a + sxy;
            own = i + k * nxy;
        } else {
            const int b = a + sxy;
            v[0] = a; v[1] = b; v[2] = b + 1; v[3] = a + 1;
            own = i + (j - 1) * m.nx + k * nxy;
        }
        return;
    }
    f -= 2 * nxz;
    {  // back, front: i fastest, j
        const bool front = f >= nxy;
        const int r = front ? f - nxy : f, i = r % m.nx, j = r / m.nx;
        const int k = front ? m.nvz - 1 : 0, a = k * sxy + j * m.nvx + i;
        if (!front) {
            const int b = a + m.nvx;
            v[0] = a; v[1] = b; v[2] = b + 1; v[3] = a + 1;
            own = i + j * m.nx;
        } else {
            const int b = a + 1, c = b + m.nvx;
            v[0] = a; v[1] = b; v[2] = c; v[3] = c - 1;
            own = i + j * m.nx + (k - 1) * nxy;
        }
    }
}

// Topology of an imported mesh (device arrays): four vertex ids per face in
// winding order, the owner of every face, the neighbour of every interior
// face; cell_face / cell_count receive each cell's faces (six slots per cell,
// in arrival order) from k_mesh_cell_faces.
struct FaceLists {
    const int *fv, *owner, *neighbour;
    int *cell_face, *cell_count;
};

// Per face: owner / neighbour (ghost nc + f - ni for boundary faces), area,
// centroid, normal and streaming dt (unstructured_mesh.cpp:1592-1692), and
// for the cells' sums the two triangles' volumes, the face's triangle-area
// sum and its area-weighted centroid sum.  kList: the topology from L (an
// imported mesh), otherwise the generator's.
template <bool kList>
__global__ void k_mesh_faces(MeshDims m, FaceLists L, const float *vx, const float *vy, const float *vz, int *owner,
                             int *neighbour, double *face_area, double *face_normal, double *face_centroid,
                             double *streaming_dt, double *tvol, double *tarea, double *tcen) {
    for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < m.nf; f += gridDim.x * blockDim.x) {
        int v[4], own, nb;
        if (kList) {
#pragma unroll
            for (int q = 0; q < 4; q++) v[q] = L.fv[4 * (size_t)f + q];
            own = L.owner[f];
            nb = f < m.ni ? L.neighbour[f] : -1;
        } else {
            face_topology(m, f, v, own, nb);
        }
        owner[f] = own;
        neighbour[f] = f < m.ni ? nb : m.nc + f - m.ni;
        D3 nd[4];
#pragma unroll
        for (int q = 0; q < 4; q++) nd[q] = {(double)vx[v[q]], (double)vy[v[q]], (double)vz[v[q]]};
#pragma unroll
        for (int t = 0; t < 2; t++) {  // tet_volume
            const D3 a = nd[0], b = sub3(nd[t + 1], a), c = sub3(nd[t + 2], a);
            tvol[2 * (size_t)f + t] = dvd(dot3(a, cross3(b, c)), 6.0);
        }
        double area_f = 0.0;
        D3 fcen = {0, 0, 0}, fnorm = {0, 0, 0};
#pragma unroll
        for (int t = 0; t < 2; t++) {  // cell_tet_area
            const D3 a = nd[0], b = nd[t + 1], c = nd[t + 2];
            D3 cen = {dvd(add(add(a.x, b.x), c.x), 3.0), dvd(add(add(a.y, b.y), c.y), 3.0),
                      dvd(add(add(a.z, b.z), c.z), 3.0)};
            const D3 n = cross3(sub3(b, a), sub3(c, a));
            const double ar = mul(0.5, mag3(n));
            area_f = add(area_f, ar);
            const double inv = dvd(1.0, ar);  // vector_var::factor divides by its argument
            cen = {dvd(cen.x, inv), dvd(cen.y, inv), dvd(cen.z, inv)};
            fcen = add3(fcen, cen);
            fnorm = add3(fnorm, n);
        }
        face_area[f] = m.closed_faces ? mul(0.5, mag3(fnorm)) : area_f;
        face_centroid[3 * (size_t)f] = dvd(fcen.x, area_f);
        face_centroid[3 * (size_t)f + 1] = dvd(fcen.y, area_f);
        face_centroid[3 * (size_t)f + 2] = dvd(fcen.z, area_f);
        const double nm = mag3(fnorm);
        face_normal[3 * (size_t)f] = dvd(fnorm.x, nm);
        face_normal[3 * (size_t)f + 1] = dvd(fnorm.y, nm);
        face_normal[3 * (size_t)f + 2] = dvd(fnorm.z, nm);
        const double face_dt = mul(0.5, __dsqrt_rn(area_f));
        streaming_dt[f] = m.reference_dt < face_dt ? m.reference_dt : face_dt;  // std::min
        tarea[f] = area_f;
        tcen[3 * (size_t)f] = fcen.x;
        tcen[3 * (size_t)f + 1] = fcen.y;
        tcen[3 * (size_t)f + 2] = fcen.z;
    }
}

// The six faces of cell c (i, j, k) in increasing face index, with the cell
// on their other side (a ghost for boundary faces): the order in which the
// generator's face loop reaches the cell, and the order of its gradient
// stencil (unstructured_mesh.cpp:1645-1665).
__device__ void cell_faces(const MeshDims &m, int c, int (&face)[6], int (&other)[6]) {
    const int i = c % m.nx, j = (c / m.nx) % m.ny, k = c / (m.nx * m.ny);
    const int nyz = m.ny * m.nz, nxz = m.nx * m.nz, nxy = m.nx * m.ny;
    const int bl = m.ni, br = bl + nyz, bb = br + nyz, bt = bb + nxz, bk = bt + nxz, bf = bk + nxy;
    const int z0 = m.nfx + m.nfy;
    face[0] = i > 0 ? (i - 1) + (m.nx - 1) * (j + m.ny * k) : bl + j + m.ny * k;
    other[0] = i > 0 ? c - 1 : -1;
    face[1] = i < m.nx - 1 ? i + (m.nx - 1) * (j + m.ny * k) : br + j + m.ny * k;
    other[1] = i < m.nx - 1 ? c + 1 : -1;
    face[2] = j > 0 ? m.nfx + i + m.nx * ((j - 1) + (m.ny - 1) * k) : bb + i + m.nx * k;
    other[2] = j > 0 ? c - m.nx : -1;
    face[3] = j < m.ny - 1 ? m.nfx + i + m.nx * (j + (m.ny - 1) * k) : bt + i + m.nx * k;
    other[3] = j < m.ny - 1 ? c + m.nx : -1;
    face[4] = k > 0 ? z0 + i + m.nx * (j + m.ny * (k - 1)) : bk + i + m.nx * j;
    other[4] = k > 0 ? c - nxy : -1;
    face[5] = k < m.nz - 1 ? z0 + i + m.nx * (j + m.ny * k) : bf + i + m.nx * j;
    other[5] = k < m.nz - 1 ? c + nxy : -1;
#pragma unroll
    for (int q = 0; q < 6; q++)
        if (other[q] < 0) other[q] = m.nc + face[q] - m.ni;
    for (int a = 1; a < 6; a++)  // insertion sort by face index
        for (int b = a; b > 0 && face[b] < face[b - 1]; b--) {
            const int tf = face[b], to = other[b];
            face[b] = face[b - 1]; other[b] = other[b - 1];
            face[b - 1] = tf; other[b - 1] = to;
        }
}

// Each face of an imported mesh into the slot lists of its owner and (interior
// faces) its neighbour.  The host has checked that every cell has six faces;
// the slot bound keeps the writes inside the lists regardless.
__global__ void k_mesh_cell_faces(MeshDims m, FaceLists L) {
    for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < m.nf; f += gridDim.x * blockDim.x) {
        const int o = L.owner[f];
        int s = atomicAdd(&L.cell_count[o], 1);
        if (s < 6) L.cell_face[6 * (size_t)o + s] = f;
        if (f < m.ni) {
            const int n = L.neighbour[f];
            s = atomicAdd(&L.cell_count[n], 1);
            if (s < 6) L.cell_face[6 * (size_t)n + s] = f;
        }
    }
}

// Per interior cell: volume (signed tet volumes, + as owner, - as neighbour),
// the area-weighted centroid, and its stencil (sorted faces, other cells).
// kList: the cell's faces from L's slots, sorted by face index (the order of
// the host's face loop), the other cell from owner / neighbour (neighbour
// already holds the ghost of a boundary face).
template <bool kList>
__global__ void k_mesh_cells(MeshDims m, FaceLists L, const int *owner, const int *neighbour, const double *tvol,
                             const double *tarea, const double *tcen, double *cell_volume, double *cell_centroid,
                             int *stencil, int *stencil_face) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < m.nc; c += gridDim.x * blockDim.x) {
        int face[6], other[6];
        if (kList) {
#pragma unroll
            for (int q = 0; q < 6; q++) face[q] = L.cell_face[6 * (size_t)c + q];
            for (int a = 1; a < 6; a++)  // insertion sort by face index
                for (int b = a; b > 0 && face[b] < face[b - 1]; b--) {
                    const int t = face[b];
                    face[b] = face[b - 1];
                    face[b - 1] = t;
                }
#pragma unroll
            for (int q = 0; q < 6; q++) other[q] = owner[face[q]] == c ? neighbour[face[q]] : owner[face[q]];
        } else {
            cell_faces(m, c, face, other);
        }
        double vol = 0.0, csum = 0.0, cx = 0.0, cy = 0.0, cz = 0.0;
#pragma unroll
        for (int q = 0; q < 6; q++) {
            const int f = face[q];
            const bool own = owner[f] == c;
#pragma unroll
            for (int t = 0; t < 2; t++) vol = own ? add(vol, tvol[2 * (size_t)f + t]) : sub(vol, tvol[2 * (size_t)f + t]);
            csum = add(csum, tarea[f]);
            cx = add(cx, tcen[3 * (size_t)f]);
            cy = add(cy, tcen[3 * (size_t)f + 1]);
            cz = add(cz, tcen[3 * (size_t)f + 2]);
            stencil[6 * (size_t)c + q] = other[q];
            stencil_face[6 * (size_t)c + q] = f;
        }
        cell_volume[c] = vol;
        cell_centroid[3 * (size_t)c] = dvd(cx, csum);
        cell_centroid[3 * (size_t)c + 1] = dvd(cy, csum);
        cell_centroid[3 * (size_t)c + 2] = dvd(cz, csum);
    }
}

// Ghost cells: the owner's centroid reflected through the face centroid
// (populate_ghost_cell_from_foam_face, unstructured_mesh.cpp:1963-1996);
// their volumes stay 0.
__global__ void k_mesh_ghosts(MeshDims m, const int *owner, const double *face_centroid, double *cell_volume,
                              double *cell_centroid) {
    for (int f = m.ni + blockIdx.x * blockDim.x + threadIdx.x; f < m.nf; f += gridDim.x * blockDim.x) {
        const size_t g = (size_t)m.nc + f - m.ni, o = owner[f];
#pragma unroll
        for (int a = 0; a < 3; a++) {
            const double e = dvd(sub(face_centroid[3 * (size_t)f + a], cell_centroid[3 * o + a]), 0.5);
            cell_centroid[3 * g + a] = add(cell_centroid[3 * o + a], e);
        }
        cell_volume[g] = 0.0;
    }
}

// Least-squares / hybrid gradient geometry per cell: gradients::
// pre_fill_LHS_and_RHS_matrix (gradients.cpp:214-315) and
// add_non_macrovariable_contributions (:149-211), with the reference's
// determinant formula.
__global__ void k_mesh_ls(MeshDims m, const int *owner, const double *face_area, const double *face_normal,
                          const double *face_centroid, const double *cell_volume, const double *cell_centroid,
                          const int *stencil, const int *stencil_face, double *lhs_inverse, double *rhs) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m.nc; i += gridDim.x * blockDim.x) {
        const double cxi = cell_centroid[3 * (size_t)i], cyi = cell_centroid[3 * (size_t)i + 1],
                     czi = cell_centroid[3 * (size_t)i + 2];
        const double cvol = cell_volume[i];
        double max_area = 0.0, max_disp = 0.0;
        for (int q = 0; q < 6; q++) {
            const size_t i1 = stencil[6 * (size_t)i + q];
            const int f = stencil_face[6 * (size_t)i + q];
            max_area = max_area < face_area[f] ? face_area[f] : max_area;  // std::max(max_area, area)
            const double ddx = sub(cell_centroid[3 * i1], cxi), ddy = sub(cell_centroid[3 * i1 + 1], cyi),
                         ddz = sub(cell_centroid[3 * i1 + 2], czi);
            const double disp = __dsqrt_rn(add(add(mul(ddx, ddx), mul(ddy, ddy)), mul(ddz, ddz)));
            max_disp = disp < max_disp ? max_disp : disp;  // std::max(disp, max_disp)
        }
        const double aspect = dvd(mul(mul(2.0, fabs(max_disp)), max_area), cvol);
        const double two_over = dvd(2.0, aspect);
        const double beta = m.hybrid ? (two_over < 1.0 ? two_over : 1.0) : 1.0;  // std::min(1.0, 2 / aspect)
        double L[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        const double gg = mul(mul(2.0, sub(1.0, beta)), cvol);
        L[0] = add(L[0], gg);
        L[4] = add(L[4], gg);
        L[8] = add(L[8], gg);
        for (int q = 0; q < 6; q++) {
            const size_t i1 = stencil[6 * (size_t)i + q];
            const int f = stencil_face[6 * (size_t)i + q];
            const double fi = face_normal[3 * (size_t)f], fj = face_normal[3 * (size_t)f + 1],
                         fk = face_normal[3 * (size_t)f + 2];
            double ddx = sub(face_centroid[3 * (size_t)f], cxi), ddy = sub(face_centroid[3 * (size_t)f + 1], cyi),
                   ddz = sub(face_centroid[3 * (size_t)f + 2], czi);
            const double l_norm = add(add(mul(ddx, fi), mul(ddy, fj)), mul(ddz, fk));
            ddx = sub(cell_centroid[3 * i1], cxi);
            ddy = sub(cell_centroid[3 * i1 + 1], cyi);
            ddz = sub(cell_centroid[3 * i1 + 2], czi);
            const double Ld = __dsqrt_rn(add(add(mul(ddx, ddx), mul(ddy, ddy)), mul(ddz, ddz)));
            const double s = face_area[f];
            const double L_norm = add(add(mul(ddx, fi), mul(ddy, fj)), mul(ddz, fk));
            const double ratio = dvd(mul(2.0, l_norm), L_norm);
            const double alpha_w = mul(ratio, ratio);
            const double w = dvd(mul(alpha_w, s), Ld);
            const double d3[3] = {ddx, ddy, ddz};
#pragma unroll
            for (int r = 0; r < 3; r++)
#pragma unroll
                for (int c = 0; c < 3; c++) L[3 * r + c] = add(L[3 * r + c], mul(mul(mul(w, d3[r]), d3[c]), beta));
            const double n3[3] = {fi, fj, fk};
            const bool own = owner[f] == i;
            double *R = rhs + 18 * (size_t)i + 3 * q;
#pragma unroll
            for (int r = 0; r < 3; r++) {
                const double ls = mul(mul(beta, w), d3[r]);
                double gt = mul(mul(mul(2.0, sub(1.0, beta)), 0.5), n3[r]);
                if (!own) gt = mul(gt, -1.0);
                R[r] = add(ls, mul(gt, s));
            }
        }
        const double a = L[0], b = L[1], c = L[2], dd = L[3], e = L[4], ff = L[5], g = L[6], h = L[7], k = L[8];
        const double det = add(add(mul(a, sub(mul(e, k), mul(ff, h))), mul(b, sub(sub(mul(dd, k), ff), g))),
                               mul(c, sub(mul(dd, h), mul(e, g))));
        const double id = dvd(1.0, det);
        double *I = lhs_inverse + 9 * (size_t)i;
        I[0] = mul(id, sub(mul(e, k), mul(ff, h)));
        I[1] = mul(id, sub(mul(c, h), mul(b, k)));
        I[2] = mul(id, sub(mul(b, ff), mul(c, e)));
        I[3] = mul(id, sub(mul(ff, g), mul(dd, k)));
        I[4] = mul(id, sub(mul(a, k), mul(c, g)));
        I[5] = mul(id, sub(mul(c, dd), mul(a, ff)));
        I[6] = mul(id, sub(mul(dd, h), mul(e, g)));
        I[7] = mul(id, sub(mul(b, g), mul(a, h)));
        I[8] = mul(id, sub(mul(a, e), mul(b, dd)));
    }
}

// Device buffers of one build, released on every return path.
struct Scratch {
    std::vector<void *> p;
    template <typename T> int get(T **out, size_t n) {
        void *q = nullptr;
        cudaError_t e = cudaMalloc(&q, (n > 0 ? n : 1) * sizeof(T));
        if (e != cudaSuccess) return set_error(LBFS_ERR_NOMEM, std::string("mesh build on the GPU: ") + cudaGetErrorString(e));
        p.push_back(q);
        *out = static_cast<T *>(q);
        return LBFS_OK;
    }
    ~Scratch() {
        for (void *q : p) cudaFree(q);
    }
};

int grid_for(long long n) { return (int)std::min<long long>((n + 255) / 256, 148LL * 16); }

}  // namespace
}  // namespace lbfs

extern "C" int lbfs_mesh_build_gpu(double X, double Y, double Z, double dt, const double *origin, double visc,
                                   double fneq_min, int32_t gradient_hybrid, int32_t mesh_type, double plateau_width,
                                   double plateau_slope, double jitter, uint64_t seed, int32_t closed_faces,
                                   int32_t device, int32_t *owner, int32_t *neighbour, double *face_area,
                                   double *face_normal, double *face_centroid, double *streaming_dt,
                                   double *cell_volume, double *cell_centroid, int32_t *gradient_stencil,
                                   double *lhs_inverse, double *rhs, int32_t *bc_patch, double *delta_h,
                                   double *grid_xyz) {
    using namespace lbfs;
    int32_t cnt[8];
    int rc = lbfs_mesh_uniform_counts(X, Y, Z, dt, cnt);
    if (rc) return rc;
    if (mesh_type != 4 && mesh_type != 5 && mesh_type != 6 && mesh_type != 7)
        return set_error(LBFS_ERR_ARG, "mesh_type must be 4 (plateau), 5, 6 (uniform) or 7 (cosine)");
    if (!(jitter >= 0.0 && jitter < 0.25)) return set_error(LBFS_ERR_ARG, "jitter must be in [0, 0.25) of the cell spacing");
    if (!origin || !owner || !neighbour || !face_area || !face_normal || !face_centroid || !streaming_dt ||
        !cell_volume || !cell_centroid || !gradient_stencil || !lhs_inverse || !rhs || !bc_patch || !delta_h)
        return set_error(LBFS_ERR_ARG, "null output buffer");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return set_error(LBFS_ERR_CUDA, "no CUDA device: this library has no CPU path");
    if (device < 0 || device >= ndev) return set_error(LBFS_ERR_ARG, "bad device index");
    LBFS_CUDA(cudaSetDevice(device));
    const UniformDims d = uniform_dims(X, Y, Z, dt);
    MeshDims m;
    m.nx = d.nx; m.ny = d.ny; m.nz = d.nz;
    m.nvx = d.nx + 1; m.nvy = d.ny + 1; m.nvz = d.nz + 1;
    m.nc = d.n_cells; m.nf = d.n_faces; m.ni = d.n_interior; m.nfx = d.n_fx; m.nfy = d.n_fy;
    m.dx = d.dx; m.dy = d.dy; m.dz = d.dz;
    m.jitter = jitter;
    m.seed = seed;
    m.closed_faces = (jitter > 0 && closed_faces) ? 1 : 0;
    m.hybrid = gradient_hybrid ? 1 : 0;
    m.reference_dt = visc * 3 / 1.0 / fneq_min;  // pre_conditioned_gamma = 1, as the host builder
    const bool cl = mesh_type == 5 || mesh_type == 7;
    const std::vector<double> ax = axis_vertices(mesh_type, cl, d.nx, origin[0], X, d.dx, plateau_width, plateau_slope),
                              ay = axis_vertices(mesh_type, cl, d.ny, origin[1], Y, d.dy, plateau_width, plateau_slope),
                              az = axis_vertices(mesh_type, mesh_type == 5, d.nz, origin[2], Z, d.dz, plateau_width,
                                                 plateau_slope);
    if (grid_xyz) {
        std::copy(ax.begin(), ax.end(), grid_xyz);
        std::copy(ay.begin(), ay.end(), grid_xyz + m.nvx);
        std::copy(az.begin(), az.end(), grid_xyz + m.nvx + m.nvy);
    }
    {  // patches in face order: left, right (ny nz each), bottom, top (nx nz), back, front (nx ny)
        const int sizes[6] = {d.ny * d.nz, d.ny * d.nz, d.nx * d.nz, d.nx * d.nz, d.nx * d.ny, d.nx * d.ny};
        int b = 0;
        for (int p = 0; p < 6; p++)
            for (int q = 0; q < sizes[p]; q++) bc_patch[b++] = p;
    }
    *delta_h = std::min(std::min(d.dx, std::min(d.dy, d.dz)) * 0.5, 0.1);
    const size_t nc = m.nc, nf = m.nf, nt = nc + (nf - m.ni), nv = (size_t)m.nvx * m.nvy * m.nvz;
    Scratch S;
    double *dax, *day, *daz, *d_area, *d_normal, *d_fcen, *d_sdt, *d_vol, *d_cen, *d_lhs, *d_rhs, *tvol, *tarea, *tcen;
    float *vx, *vy, *vz;
    int *d_owner, *d_nb, *d_st, *d_stf;
    if ((rc = S.get(&dax, ax.size())) || (rc = S.get(&day, ay.size())) || (rc = S.get(&daz, az.size())) ||
        (rc = S.get(&vx, nv)) || (rc = S.get(&vy, nv)) || (rc = S.get(&vz, nv)) || (rc = S.get(&d_owner, nf)) ||
        (rc = S.get(&d_nb, nf)) || (rc = S.get(&d_area, nf)) || (rc = S.get(&d_normal, 3 * nf)) ||
        (rc = S.get(&d_fcen, 3 * nf)) || (rc = S.get(&d_sdt, nf)) || (rc = S.get(&tvol, 2 * nf)) ||
        (rc = S.get(&tarea, nf)) || (rc = S.get(&tcen, 3 * nf)) || (rc = S.get(&d_vol, nt)) ||
        (rc = S.get(&d_cen, 3 * nt)) || (rc = S.get(&d_st, 6 * nc)) || (rc = S.get(&d_stf, 6 * nc)) ||
        (rc = S.get(&d_lhs, 9 * nc)) || (rc = S.get(&d_rhs, 18 * nc)))
        return rc;
    LBFS_CUDA(cudaMemcpy(dax, ax.data(), sizeof(double) * ax.size(), cudaMemcpyHostToDevice));
    LBFS_CUDA(cudaMemcpy(day, ay.data(), sizeof(double) * ay.size(), cudaMemcpyHostToDevice));
    LBFS_CUDA(cudaMemcpy(daz, az.data(), sizeof(double) * az.size(), cudaMemcpyHostToDevice));
    k_mesh_vertices<<<grid_for((long long)nv), 256>>>(m, dax, day, daz, vx, vy, vz);
    const FaceLists none = {nullptr, nullptr, nullptr, nullptr, nullptr};
    k_mesh_faces<false><<<grid_for((long long)nf), 256>>>(m, none, vx, vy, vz, d_owner, d_nb, d_area, d_normal, d_fcen,
                                                          d_sdt, tvol, tarea, tcen);
    k_mesh_cells<false><<<grid_for((long long)nc), 256>>>(m, none, d_owner, d_nb, tvol, tarea, tcen, d_vol, d_cen, d_st,
                                                          d_stf);
    k_mesh_ghosts<<<grid_for((long long)(nf - m.ni)), 256>>>(m, d_owner, d_fcen, d_vol, d_cen);
    k_mesh_ls<<<grid_for((long long)nc), 256>>>(m, d_owner, d_area, d_normal, d_fcen, d_vol, d_cen, d_st, d_stf,
                                                d_lhs, d_rhs);
    LBFS_CUDA(cudaGetLastError());
    LBFS_CUDA(cudaDeviceSynchronize());
    LBFS_CUDA(cudaMemcpy(owner, d_owner, sizeof(int) * nf, cudaMemcpyDeviceToHost));
    LBFS_CUDA(cudaMemcpy(neighbour, d_nb, sizeof(int) * nf, cudaMemcpyDeviceToHost));
    LBFS_CUDA(cudaMemcpy(face_area, d_area, sizeof(double) * nf, cudaMemcpyDeviceToHost));
    LBFS_CUDA(cudaMemcpy(face_normal, d_normal, sizeof(double) * 3 * nf, cudaMemcpyDeviceToHost));
    LBFS_CUDA(cudaMemcpy(face_centroid, d_fcen, sizeof(double) * 3 * nf, cudaMemcpyDeviceToHost));
    LBFS_CUDA(cudaMemcpy(streaming_dt, d_sdt, sizeof(double) * nf, cudaMemcpyDeviceToHost));
    LBFS_CUDA(cudaMemcpy(cell_volume, d_vol, sizeof(double) * nt, cudaMemcpyDeviceToHost));
    LBFS_CUDA(cudaMemcpy(cell_centroid, d_cen, sizeof(double) * 3 * nt, cudaMemcpyDeviceToHost));
    LBFS_CUDA(cudaMemcpy(gradient_stencil, d_st, sizeof(int) * 6 * nc, cudaMemcpyDeviceToHost));
    LBFS_CUDA(cudaMemcpy(lhs_inverse, d_lhs, sizeof(double) * 9 * nc, cudaMemcpyDeviceToHost));
    LBFS_CUDA(cudaMemcpy(rhs, d_rhs, sizeof(double) * 18 * nc, cudaMemcpyDeviceToHost));
    return LBFS_OK;
}

// The geometry of a hex mesh given as lists, on GPU `device`: the kernels
// above with the topology from the lists, so every array equals the host
// routine's (host_setup.cpp mesh_geometry) bit for bit.  The host has
// checked the indices (vertices < np, cells < nc); this checks that no face
// has its owner as neighbour and that every cell has six faces, as the host
// routine's stencil check does.
int lbfs::mesh_geometry_gpu(int device, int np, int nc, int nf, int ni, const float *vx, const float *vy,
                            const float *vz, const int *fv, const int32_t *owner, int32_t *neighbour, double visc,
                            double fneq_min, int32_t gradient_hybrid, bool closed_faces, double *face_area,
                            double *face_normal, double *face_centroid, double *streaming_dt, double *cell_volume,
                            double *cell_centroid, int32_t *gradient_stencil, double *lhs_inverse, double *rhs) {
    if (np <= 0 || nc <= 0 || ni < 0 || ni > nf) return set_error(LBFS_ERR_ARG, "mesh_geometry_gpu: bad sizes");
    {
        std::vector<int> count(nc, 0);
        for (int f = 0; f < nf; f++) {
            count[owner[f]]++;
            if (f < ni) {
                if (neighbour[f] == owner[f]) return set_error(LBFS_ERR_ARG, "face with its owner as neighbour");
                count[neighbour[f]]++;
            }
        }
        for (int c = 0; c < nc; c++)
            if (count[c] != 6) return set_error(LBFS_ERR_ARG, "hex cell without 6 stencil entries");
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return set_error(LBFS_ERR_CUDA, "no CUDA device: this library has no CPU path");
    if (device < 0 || device >= ndev) return set_error(LBFS_ERR_ARG, "bad device index");
    LBFS_CUDA(cudaSetDevice(device));
    MeshDims m = {};
    m.nc = nc; m.nf = nf; m.ni = ni;
    m.closed_faces = closed_faces ? 1 : 0;
    m.hybrid = gradient_hybrid ? 1 : 0;
    m.reference_dt = visc * 3 / 1.0 / fneq_min;  // pre_conditioned_gamma = 1, as the host routine
    const size_t unc = nc, unf = nf, nt = unc + (unf - ni);
    Scratch S;
    double *d_area, *d_normal, *d_fcen, *d_sdt, *d_vol, *d_cen, *d_lhs, *d_rhs, *tvol, *tarea, *tcen;
    float *d_vx, *d_vy, *d_vz;
    int *d_fv, *d_own_in, *d_nb_in, *d_owner, *d_nb, *d_st, *d_stf, *d_cf, *d_cc;
    int rc;
    if ((rc = S.get(&d_vx, np)) || (rc = S.get(&d_vy, np)) || (rc = S.get(&d_vz, np)) || (rc = S.get(&d_fv, 4 * unf)) ||
        (rc = S.get(&d_own_in, unf)) || (rc = S.get(&d_nb_in, (size_t)ni)) || (rc = S.get(&d_owner, unf)) ||
        (rc = S.get(&d_nb, unf)) || (rc = S.get(&d_area, unf)) || (rc = S.get(&d_normal, 3 * unf)) ||
        (rc = S.get(&d_fcen, 3 * unf)) || (rc = S.get(&d_sdt, unf)) || (rc = S.get(&tvol, 2 * unf)) ||
        (rc = S.get(&tarea, unf)) || (rc = S.get(&tcen, 3 * unf)) || (rc = S.get(&d_vol, nt)) ||
        (rc = S.get(&d_cen, 3 * nt)) || (rc = S.get(&d_st, 6 * unc)) || (rc = S.get(&d_stf, 6 * unc)) ||
        (rc = S.get(&d_lhs, 9 * unc)) || (rc = S.get(&d_rhs, 18 * unc)) || (rc = S.get(&d_cf, 6 * unc)) ||
        (rc = S.get(&d_cc, unc)))
        return rc;
    LBFS_CUDA(cudaMemcpy(d_vx, vx, sizeof(float) * np, cudaMemcpyHostToDevice));
    LBFS_CUDA(cudaMemcpy(d_vy, vy, sizeof(float) * np, cudaMemcpyHostToDevice));
    LBFS_CUDA(cudaMemcpy(d_vz, vz, sizeof(float) * np, cudaMemcpyHostToDevice));
    LBFS_CUDA(cudaMemcpy(d_fv, fv, sizeof(int) * 4 * unf, cudaMemcpyHostToDevice));
    LBFS_CUDA(cudaMemcpy(d_own_in, owner, sizeof(int) * unf, cudaMemcpyHostToDevice));
    if (ni > 0) LBFS_CUDA(cudaMemcpy(d_nb_in, neighbour, sizeof(int) * ni, cudaMemcpyHostToDevice));
    LBFS_CUDA(cudaMemset(d_cc, 0, sizeof(int) * unc));
    const FaceLists L = {d_fv, d_own_in, d_nb_in, d_cf, d_cc};
    k_mesh_faces<true><<<grid_for((long long)nf), 256>>>(m, L, d_vx, d_vy, d_vz, d_owner, d_nb, d_area, d_normal, d_fcen,
                                                         d_sdt, tvol, tarea, tcen);
    k_mesh_cell_faces<<<grid_for((long long)nf), 256>>>(m, L);
    k_mesh_cells<true><<<grid_for((long long)nc), 256>>>(m, L, d_owner, d_nb, tvol, tarea, tcen, d_vol, d_cen, d_st,
                                                         d_stf);
    if (nf > ni) k_mesh_ghosts<<<grid_for((long long)(nf - ni)), 256>>>(m, d_owner, d_fcen, d_vol, d_cen);
    k_mesh_ls<<<grid_for((long long)nc), 256>>>(m, d_owner, d_area, d_normal, d_fcen, d_vol, d_cen, d_st, d_stf,
                                                d_lhs, d_rhs);
    LBFS_CUDA(cudaGetLastError());
    LBFS_CUDA(cudaDeviceSynchronize());
    LBFS_CUDA(cudaMemcpy(neighbour, d_nb, sizeof(int) * unf, cudaMemcpyDeviceToHost));
    LBFS_CUDA(cudaMemcpy(face_area, d_area, sizeof(double) * unf, cudaMemcpyDeviceToHost));
    LBFS_CUDA(cudaMemcpy(face_normal, d_normal, sizeof(double) * 3 * unf, cudaMemcpyDeviceToHost));
    LBFS_CUDA(cudaMemcpy(face_centroid, d_fcen, sizeof(double) * 3 * unf, cudaMemcpyDeviceToHost));
    LBFS_CUDA(cudaMemcpy(streaming_dt, d_sdt, sizeof(double) * unf, cudaMemcpyDeviceToHost));
    LBFS_CUDA(cudaMemcpy(cell_volume, d_vol, sizeof(double) * nt, cudaMemcpyDeviceToHost));
    LBFS_CUDA(cudaMemcpy(cell_centroid, d_cen, sizeof(double) * 3 * nt, cudaMemcpyDeviceToHost));
    LBFS_CUDA(cudaMemcpy(gradient_stencil, d_st, sizeof(int) * 6 * unc, cudaMemcpyDeviceToHost));
    LBFS_CUDA(cudaMemcpy(lhs_inverse, d_lhs, sizeof(double) * 9 * unc, cudaMemcpyDeviceToHost));
    LBFS_CUDA(cudaMemcpy(rhs, d_rhs, sizeof(double) * 18 * unc, cudaMemcpyDeviceToHost));
    return LBFS_OK;
}
