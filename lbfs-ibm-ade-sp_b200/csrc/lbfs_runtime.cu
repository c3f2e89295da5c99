// Host runtime behind the C ABI of include/lbfs_b200.h.
//
// One handle = one solver instance on one GPU: mesh geometry and membranes are
// uploaded once, the state stays resident in HBM, and each time step is four
// kernels (membrane kernel on a forked stream, overlapping the gradient and
// face-flux kernels, then the cell update), optionally replayed from a CUDA
// graph.  This replaces gpu_solver::General_Purpose_Solver_mk_i's set-up
// (Solver_gpu.cu:178-746) and loop body (Solver_gpu.cu:749-1046), which issue
// 20-30 synchronising launches per step on managed memory.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdint>
#include <initializer_list>
#include <cstdlib>
#include <functional>
#include <cstring>
#include <string>
#include <vector>

#include "lbfs_adjoint.h"
#include "lbfs_b200.h"
#include "lbfs_fluid.cuh"
#include "lbfs_internal.h"
#include "lbfs_kernels.h"

namespace lbfs {

static thread_local std::string g_last_error;
constexpr int kPhases = 6;  // 5 kernels + the whole step

int set_error(int code, const std::string &msg) {
    g_last_error = msg;
    return code;
}

}  // namespace lbfs

using namespace lbfs;

struct lbfs_solver {
    int device = 0;
    cudaStream_t stream = nullptr, stream2 = nullptr, stream3 = nullptr, stream4 = nullptr;
    // pipelined K1 -> K2 (axis-aligned meshes): chunk c covers cells [chunk_cell[c], chunk_cell[c + 1])
    // and the interior faces chunk_faces[c] (every face whose cells lie in chunks <= c)
    int flux_chunks = 1;
    // membrane kernels of a captured step behind the gradient kernel's launch completion (launch shape)
    bool membrane_after_k1 = false;
    bool chunkable = false;
    std::vector<int> chunk_nb;   // neighbours of the interior faces (for the plan)
    int chunk_start[3] = {0, 0, 0}, chunk_count[3] = {0, 0, 0};
    std::vector<int> chunk_cell;
    std::vector<FaceRanges> chunk_faces;
    // tiles of the face kernel (interior faces ordered by owner within each axis), one table per flux
    // block size 64 / 128 / 256: tiles_h[b] = first face of each axis owned by tile t (3 ints per
    // tile, n_tiles + 1 rows), tile_maxnb[b][t] = largest neighbour of the faces of tiles <= t
    bool tiled = false;
    std::vector<int> tiles_h[3], tile_maxnb[3];
    int *d_tiles[3] = {};
    std::vector<int> chunk_tile;  // K + 1 tile splits of the pipelined K2
    cudaEvent_t ev_chunk[kMaxFluxChunks] = {}, ev_flux = nullptr, ev_bnd = nullptr;
    cudaEvent_t ev_advected = nullptr, ev_sorted = nullptr;
    bool own_stream = true;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    lbfs_params params{};
    bool fp32 = false;
    bool periodic = false;  // some boundary has type 3
    bool wrap_membranes = false;  // some membrane is periodic (check_periodic_object)
    int nc = 0, nf = 0, ni = 0, nb = 0;
    int n_membranes = 0, total_nodes = 0, total_springs = 0, total_tris = 0;
    std::vector<void *> allocs;
    FluidArgs<double> f64{};
    FluidArgs<float> f32{};
    MembraneArgs ma{};
    ViscArgs va{};
    double *d_centroid = nullptr;
    double *d_res_out = nullptr;
    bool keep_residuals = false;
    long long t = 0;  // time-step counter (the reference's loop index)
    cudaGraphExec_t graph = nullptr;
    int graph_steps = 0;
    // lbfs_step_until: one graph whose while node repeats the step and a convergence check
    cudaGraphExec_t loop_graph = nullptr;
    bool loop_unavailable = false;  // the loop graph could not be built (steps go one at a time)
    struct UntilState *d_until = nullptr;
    int launches_per_step = 0;
    // per-kernel timing: start/stop events per phase (membrane, gradients, flux, update, viscosity)
    bool profiling = false;    // step events (level >= 1)
    bool kernel_events = false; // per-kernel events too (level 2)
    cudaEvent_t ev_phase[kPhases][2] = {};
    bool phase_recorded[kPhases] = {};
    bool graph_phase_recorded[kPhases] = {};  // phases recorded by one replay of the graph
    // staging buffer for host <-> device state transfers: rho, u, v, w planes
    double *d_stage = nullptr;
    // ensemble instances (one when the mesh is a single case)
    std::vector<lbfs_grid_desc> grids;
    std::vector<InstanceGrid> inst;
    long long total_patch = 0;  // cells of all IBM patch slices
    // discrete adjoint: persistent buffers (allocated on first use)
    AdjointArgs adj{};
    bool adj_ready = false;
    MemAdjArgs madj{};
    bool madj_ready = false;

    template <typename T> int alloc(T **p, size_t count) {
        void *q = nullptr;
        if (count == 0) count = 1;
        cudaError_t e = cudaMalloc(&q, count * sizeof(T));
        if (e != cudaSuccess)
            return set_error(LBFS_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
        allocs.push_back(q);
        *p = (T *)q;
        return LBFS_OK;
    }
    template <typename T> int upload(T **p, const std::vector<T> &h) {
        int rc = alloc(p, h.size());
        if (rc) return rc;
        if (!h.empty()) {
            cudaError_t e = cudaMemcpy(*p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice);
            if (e != cudaSuccess) return set_error(LBFS_ERR_CUDA, std::string("upload: ") + cudaGetErrorString(e));
        }
        return LBFS_OK;
    }
};

// Device record of lbfs_step_until's loop: steps taken in this launch, their limit, the tolerance,
// the last step's residual norms and why the loop stopped (0 limit, 1 converged, 2 diverged).
struct UntilState {
    int count, limit, stop, pad;
    double tol;
    double res[4];
};

namespace {

// time stepping other than constant (lbfs_params.time_stepping 1, 3, 4)
bool dynamic_dt(const lbfs_params &p) { return p.time_stepping != 0 && p.time_stepping != LBFS_DT_CONSTANT; }

// The cached graphs of a step hold the launch shape, the stream and the kernel arguments: dropped
// whenever one of those changes.
void drop_step_graphs(lbfs_solver *s) {
    if (s->graph) { cudaGraphExecDestroy(s->graph); s->graph = nullptr; s->graph_steps = 0; }
    if (s->loop_graph) { cudaGraphExecDestroy(s->loop_graph); s->loop_graph = nullptr; }
}

// The convergence test of the reference's loop (Solver_gpu.cu:1206-1208:
// convergence_residual.max_error() < tolerance) on the step's residual norms,
// formed as lbfs_get_residuals forms them, and the drop-in's divergence test
// (non-finite state or density out of range); sets the while node's condition.
__global__ void k_until_check(cudaGraphConditionalHandle h, UntilState *u, const double *sums, const unsigned int *flags,
                              double nc, double ref_rho, double ref_mom) {
    if (threadIdx.x != 0) return;
    double r[4];
    for (int k = 0; k < 4; k++) {
        r[k] = sqrt(sums[k] / nc) / (k == 0 ? ref_rho : ref_mom);
        u->res[k] = r[k];
    }
    const double m01 = r[0] < r[1] ? r[1] : r[0], m23 = r[2] < r[3] ? r[3] : r[2];  // std::max
    const double mx = m01 < m23 ? m23 : m01;
    const bool converged = mx < u->tol;
    const bool diverged = (*flags & (LBFS_FLAG_NONFINITE | LBFS_FLAG_RHO_RANGE)) != 0u;
    const int c = u->count + 1;
    u->count = c;
    u->stop = converged ? 1 : (diverged ? 2 : 0);
    cudaGraphSetConditional(h, (!converged && !diverged && c < u->limit) ? 1u : 0u);
}

// Device buffer freed when it leaves scope (temporary storage).
struct DevBuf {
    void *p = nullptr;
    ~DevBuf() { if (p) cudaFree(p); }
};

template <typename R> FluidArgs<R> &fluid(lbfs_solver *s);
template <> FluidArgs<double> &fluid<double>(lbfs_solver *s) { return s->f64; }
template <> FluidArgs<float> &fluid<float>(lbfs_solver *s) { return s->f32; }

int check_mesh(const lbfs_mesh_desc *m) {
    if (!m) return set_error(LBFS_ERR_ARG, "mesh descriptor is null");
    if (m->n_cells <= 0 || m->n_bc < 0 || m->n_interior < 0 || m->n_faces != m->n_interior + m->n_bc)
        return set_error(LBFS_ERR_ARG, "inconsistent mesh sizes");
    if (!m->owner || !m->neighbour || !m->face_area || !m->face_normal || !m->face_centroid || !m->streaming_dt ||
        !m->cell_volume || !m->cell_centroid || !m->gradient_stencil || !m->lhs_inverse || !m->rhs ||
        (m->n_bc > 0 && (!m->bc_rho_type || !m->bc_vel_type || !m->bc_values)))
        return set_error(LBFS_ERR_ARG, "mesh descriptor has a null array");
    if (m->axis_aligned && m->n_face_x + m->n_face_y + m->n_face_z != m->n_interior)
        return set_error(LBFS_ERR_ARG, "axis-aligned face ranges do not cover the interior faces");
    const int nt = m->n_cells + m->n_bc;
    for (int f = 0; f < m->n_faces; f++) {
        if (m->owner[f] < 0 || m->owner[f] >= m->n_cells || m->neighbour[f] < 0 || m->neighbour[f] >= nt)
            return set_error(LBFS_ERR_ARG, "face cell index out of range");
        if (f >= m->n_interior && m->neighbour[f] != m->n_cells + f - m->n_interior)
            return set_error(LBFS_ERR_ARG, "boundary face neighbour is not its ghost cell");
        if (!(m->streaming_dt[f] > 0) || !(m->face_area[f] > 0))
            return set_error(LBFS_ERR_ARG, "face area and streaming dt must be positive");
    }
    for (int i = 0; i < 6 * m->n_cells; i++)
        if (m->gradient_stencil[i] < 0 || m->gradient_stencil[i] >= nt)
            return set_error(LBFS_ERR_ARG, "gradient stencil index out of range");
    for (int b = 0; b < m->n_bc; b++) {
        const int rt = m->bc_rho_type[b], vt = m->bc_vel_type[b];
        if (!(rt == 1 || rt == 2 || rt == 3) || !(vt == 1 || vt == 2 || vt == 3 || vt == 9 || vt == 10))
            return set_error(LBFS_ERR_UNSUPPORTED,
                             "boundary types: rho must be 1, 2 or 3, velocity 1, 2, 3, 9 or 10 (the reference GPU "
                             "kernels implement 1, 2, 9 and 10, LBFS.cu:1872-1918; 3 is its CPU solver's periodic)");
        if (rt == 3 || vt == 3) {
            if (!m->periodic_node) return set_error(LBFS_ERR_ARG, "periodic boundary without periodic_node");
            if (m->periodic_node[b] < 0 || m->periodic_node[b] >= m->n_cells)
                return set_error(LBFS_ERR_ARG, "periodic_node must be an interior cell");
        }
    }
    for (int i = 0; i < m->n_cells; i++)
        if (!(m->cell_volume[i] > 0)) return set_error(LBFS_ERR_ARG, "cell volume must be positive");
    return LBFS_OK;
}

template <typename R> int setup_fluid(lbfs_solver *s, const lbfs_mesh_desc *m) {
    FluidArgs<R> &a = fluid<R>(s);
    const lbfs_params &p = s->params;
    const int nc = m->n_cells, nf = m->n_faces, ni = m->n_interior, nb = m->n_bc, nt = nc + nb;
    const double rho0 = s->fp32 ? p.rho0 : 0.0;
    a.nc = nc; a.nf = nf; a.ni = ni; a.nb = nb;
    a.nfx = m->n_face_x; a.nfy = m->n_face_y; a.nfz = m->n_face_z;
    a.axis_aligned = m->axis_aligned ? 1 : 0;
    a.testcase = p.testcase;
    a.rho0 = (R)rho0;
    a.gamma_inv = (R)p.gamma_inv;
    a.recon_q = p.preconditioning ? (R)p.gamma_inv : R(1);
    a.visc = (R)p.visc;
    a.delta_t = p.delta_t;
    a.H2 = p.channel_diameter * 0.5;
    a.H4 = p.channel_diameter * p.channel_diameter * p.channel_diameter * p.channel_diameter;
    for (int c = 0; c < 3; c++) a.force[c] = p.body_force[c];
    const double *cen = m->cell_centroid, *fc = m->face_centroid, *fn = m->face_normal;
    // K1 geometry
    std::vector<int2> stencil(3 * (size_t)nc);
    for (size_t q = 0; q < 3 * (size_t)nc; q++) stencil[q] = make_int2(m->gradient_stencil[2 * q], m->gradient_stencil[2 * q + 1]);
    std::vector<LsRec<R>> ls(s->fp32 ? 0 : nc);  // the adjoint's (FP64 handles)
    for (size_t i = 0; i < ls.size(); i++) {
        for (int q = 0; q < 18; q++) ls[i].rhs[q] = (R)m->rhs[18 * i + q];
        for (int q = 0; q < 9; q++) ls[i].lhs[q] = (R)m->lhs_inverse[9 * i + q];
        ls[i].pad = 0;
    }
    std::vector<LsW<R>> lsw(nc);  // W_q = LHS^-1 RHS_q, formed in FP64
    for (int i = 0; i < nc; i++) {
        const double *L = m->lhs_inverse + 9 * (size_t)i, *rh = m->rhs + 18 * (size_t)i;
        for (int q = 0; q < 6; q++)
            for (int r = 0; r < 3; r++)
                lsw[i].w[3 * q + r] = (R)(L[3 * r] * rh[3 * q] + L[3 * r + 1] * rh[3 * q + 1] + L[3 * r + 2] * rh[3 * q + 2]);
    }
    // at most 8 distinct weight vectors over all cells and slots: 3-bit codes per slot
    // (LBFS_GENERIC_GEOMETRY set: never, nor one geometry per axis below; a diagnostic switch)
    const bool generic = std::getenv("LBFS_GENERIC_GEOMETRY") != nullptr;
    std::vector<unsigned> lcode(nc);
    int n_tab = 0;
    bool coded = nc > 0 && !generic;
    for (int i = 0; i < nc && coded; i++) {
        unsigned c = 0;
        for (int q = 0; q < 6 && coded; q++) {
            const R *v = lsw[i].w + 3 * q;
            int k = 0;
            while (k < n_tab && std::memcmp(a.lsw_tab[k], v, 3 * sizeof(R)) != 0) k++;
            if (k == n_tab) {
                if (n_tab == 8) { coded = false; break; }
                std::memcpy(a.lsw_tab[n_tab++], v, 3 * sizeof(R));
            }
            c |= (unsigned)k << (3 * q);
        }
        lcode[i] = c;
    }
    for (int k = n_tab; k < 8; k++) a.lsw_tab[k][0] = a.lsw_tab[k][1] = a.lsw_tab[k][2] = R(0);
    // the adjoint's LHS^-1 and RHS by the same codes: one LHS^-1 for all cells, one RHS vector per code
    a.ls_coded = 0;
    if (coded && !ls.empty()) {
        bool ok = true, seen[8] = {false, false, false, false, false, false, false, false};
        std::memcpy(a.ls_lhs, ls[0].lhs, 9 * sizeof(R));
        for (int i = 0; i < nc && ok; i++) {
            ok = std::memcmp(ls[i].lhs, a.ls_lhs, 9 * sizeof(R)) == 0;
            for (int q = 0; q < 6 && ok; q++) {
                const unsigned k = (lcode[i] >> (3 * q)) & 7u;
                if (!seen[k]) {
                    std::memcpy(a.ls_rhs_tab[k], ls[i].rhs + 3 * q, 3 * sizeof(R));
                    seen[k] = true;
                } else {
                    ok = std::memcmp(a.ls_rhs_tab[k], ls[i].rhs + 3 * q, 3 * sizeof(R)) == 0;
                }
            }
        }
        for (int k = 0; k < 8; k++)
            if (!seen[k]) a.ls_rhs_tab[k][0] = a.ls_rhs_tab[k][1] = a.ls_rhs_tab[k][2] = R(0);
        a.ls_coded = ok ? 1 : 0;
    }
    std::vector<int> rt(nb), vt(nb), per(nb, 0);
    std::vector<Vec4<R>> bcv(nb);
    std::vector<BcRec<R>> bcr(nb);
    for (int b = 0; b < nb; b++) {
        rt[b] = m->bc_rho_type[b];
        vt[b] = m->bc_vel_type[b];
        if (rt[b] == 3 || vt[b] == 3) {
            per[b] = m->periodic_node[b];
            s->periodic = true;
        }
        const double *v = m->bc_values + 4 * b;
        bcv[b] = {(R)v[0], (R)v[1], (R)v[2], (R)(v[3] - rho0)};
        const int f = ni + b, g = nc + b, o = m->owner[f];
        // get_bc_gradients, LBFS.cu:1968-1979
        const double dx = cen[3 * g] - cen[3 * o], dy = cen[3 * g + 1] - cen[3 * o + 1], dz = cen[3 * g + 2] - cen[3 * o + 2];
        const double dmag = std::sqrt(std::pow(dx, 2.0) + std::pow(dy, 2.0) + std::pow(dz, 2.0));
        bcr[b] = {(R)dmag, (R)(dx / dmag), (R)(dy / dmag), (R)(dz / dmag), (R)(1 - std::fabs(fn[3 * f])),
                  (R)(1 - std::fabs(fn[3 * f + 1])), (R)(1 - std::fabs(fn[3 * f + 2])), (R)cen[3 * g + 1],
                  (R)cen[3 * g + 2]};
    }
    // K2 geometry
    std::vector<int2> fcells(nf);
    for (int f = 0; f < nf; f++) fcells[f] = make_int2(m->owner[f], m->neighbour[f]);
    std::vector<AxisFace<R>> axf;
    if (a.axis_aligned) {
        axf.resize(ni);
        for (int f = 0; f < ni; f++) {
            const int ax = (f < a.nfx) ? 0 : ((f < a.nfx + a.nfy) ? 1 : 2);
            const int o = m->owner[f], n = m->neighbour[f];
            axf[f] = {(R)m->face_area[f], (R)m->streaming_dt[f], (R)(cen[3 * o + ax] - fc[3 * f + ax]),
                      (R)(cen[3 * n + ax] - fc[3 * f + ax])};
        }
    }
    const int gf0 = a.axis_aligned ? ni : 0;
    // first ghost of every instance: its face takes the interior branch
    std::vector<char> first_ghost(nb, 0);
    {
        std::vector<int> starts;
        for (const lbfs_grid_desc &g : s->grids) starts.push_back(g.cell0);
        std::vector<char> seen(starts.size(), 0);
        for (int b = 0; b < nb; b++) {
            const int o = m->owner[ni + b];
            const size_t k = std::upper_bound(starts.begin(), starts.end(), o) - starts.begin() - 1;
            if (!seen[k]) { seen[k] = 1; first_ghost[b] = 1; }
        }
    }
    std::vector<GenFace<R>> gen(nf - gf0);
    for (int f = gf0; f < nf; f++) {
        const int o = m->owner[f], n = m->neighbour[f];
        GenFace<R> g;
        g.area = (R)m->face_area[f];
        g.dt = (R)m->streaming_dt[f];
        g.nx = (R)fn[3 * f]; g.ny = (R)fn[3 * f + 1]; g.nz = (R)fn[3 * f + 2];
        g.t1x = (R)(cen[3 * o] - fc[3 * f]); g.t1y = (R)(cen[3 * o + 1] - fc[3 * f + 1]); g.t1z = (R)(cen[3 * o + 2] - fc[3 * f + 2]);
        g.t2x = (R)(cen[3 * n] - fc[3 * f]); g.t2y = (R)(cen[3 * n + 1] - fc[3 * f + 1]); g.t2z = (R)(cen[3 * n + 2] - fc[3 * f + 2]);
        g.bc_branch = (R)((f >= ni && !first_ghost[f - ni]) ? 1 : 0);
        gen[f - gf0] = g;
    }
    // K3: signed face list per cell, faces in increasing index order
    std::vector<int> cf(6 * (size_t)nc, 0), cnt(nc, 0);
    for (int f = 0; f < nf; f++) {
        const int o = m->owner[f];
        if (cnt[o] >= 6) return set_error(LBFS_ERR_UNSUPPORTED, "cell with more than 6 faces (hexahedra only)");
        cf[6 * (size_t)o + cnt[o]++] = f + 1;
        if (f < ni) {
            const int n = m->neighbour[f];
            if (cnt[n] >= 6) return set_error(LBFS_ERR_UNSUPPORTED, "cell with more than 6 faces (hexahedra only)");
            cf[6 * (size_t)n + cnt[n]++] = -(f + 1);
        }
    }
    for (int i = 0; i < nc; i++)
        if (cnt[i] != 6) return set_error(LBFS_ERR_UNSUPPORTED, "cell without 6 faces (hexahedra only)");
    std::vector<double> vol(m->cell_volume, m->cell_volume + nc), inv_vol(nc);
    for (int i = 0; i < nc; i++) inv_vol[i] = 1.0 / vol[i];
    // FP32 bulk: the per-cell residual of the constant flux rho0/3 n area the
    // deviation form leaves out; zero on cells whose faces close
    std::vector<double> closure;
    if (s->fp32) {
        closure.assign(3 * (size_t)nc, 0.0);
        double amax = 0.0, cmax = 0.0;
        for (int f = 0; f < nf; f++) {
            const double c = rho0 / 3.0 * m->face_area[f];
            amax = std::max(amax, std::fabs(c));
            for (int q = 0; q < 3; q++) {
                const double v = c * fn[3 * f + q];
                closure[3 * (size_t)m->owner[f] + q] -= v;
                if (f < ni) closure[3 * (size_t)m->neighbour[f] + q] += v;
            }
        }
        for (int i = 0; i < nc; i++)
            for (int q = 0; q < 3; q++) cmax = std::max(cmax, std::fabs(closure[3 * (size_t)i + q]));
        if (cmax <= 1e-12 * amax) closure.clear();  // every cell closes
        else
            for (int i = 0; i < nc; i++)
                for (int q = 0; q < 3; q++) closure[3 * (size_t)i + q] *= inv_vol[i];
    }
    std::vector<R> visc(nc, (R)p.visc_factor_initial);
    int rc = 0;
    int *d_rt, *d_vt, *d_per, *d_cf;
    int2 *d_stencil;
    LsRec<R> *d_ls = nullptr;
    LsW<R> *d_lsw;
    R *d_visc;
    Vec4<R> *d_bcv;
    BcRec<R> *d_bcr;
    int2 *d_fcells;
    AxisFace<R> *d_axf = nullptr;
    GenFace<R> *d_gen;
    double *d_vol, *d_ivol;
    if ((rc = s->upload(&d_stencil, stencil)) || (rc = s->upload(&d_lsw, lsw)) ||
        (!ls.empty() && (rc = s->upload(&d_ls, ls))) ||
        (rc = s->upload(&d_rt, rt)) || (rc = s->upload(&d_vt, vt)) || (rc = s->upload(&d_per, per)) ||
        (rc = s->upload(&d_bcv, bcv)) ||
        (rc = s->upload(&d_bcr, bcr)) || (rc = s->upload(&d_fcells, fcells)) || (rc = s->upload(&d_gen, gen)) ||
        (rc = s->upload(&d_cf, cf)) || (rc = s->upload(&d_vol, vol)) || (rc = s->upload(&d_ivol, inv_vol)) ||
        (rc = s->upload(&d_visc, visc)))
        return rc;
    if (a.axis_aligned && (rc = s->upload(&d_axf, axf))) return rc;
    // one geometry per axis (bit for bit) on the generator's uniform meshes
    a.axis_uniform = 0;
    if (a.axis_aligned && ni > 0 && !generic) {
        const int first[3] = {0, a.nfx, a.nfx + a.nfy}, count[3] = {a.nfx, a.nfy, ni - a.nfx - a.nfy};
        bool uniform = true;
        for (int ax = 0; ax < 3 && uniform; ax++) {
            if (count[ax] == 0) continue;
            const AxisFace<R> &r = axf[first[ax]];
            for (int f = first[ax]; f < first[ax] + count[ax] && uniform; f++)
                uniform = std::memcmp(&axf[f], &r, sizeof(AxisFace<R>)) == 0;
            if (!uniform) break;
            a.axis_geo[ax][0] = r.area; a.axis_geo[ax][1] = r.dt; a.axis_geo[ax][2] = r.t1; a.axis_geo[ax][3] = r.t2;
            const R ic = R(1) / (r.t2 - r.t1);  // as the kernel forms it (IEEE division and product)
            a.axis_wa[ax] = std::fabs(r.t2 * ic);
            a.axis_wb[ax] = std::fabs(r.t1 * ic);
        }
        a.axis_uniform = uniform ? 1 : 0;
    }
    // K3 on the generator's structured meshes (one instance): the face table in closed form when it
    // equals the table entry for entry, and one 1 / volume when every cell has it
    a.grid_faces = 0;
    a.inv_volume_uniform = 0;
    if (a.axis_aligned && !generic && m->n_instances == 0 && m->delta_x > 0) {
        int n3[3];
        bool dims = true;
        for (int d = 0; d < 3; d++) {
            const double q = m->length[d] / m->delta_x;
            n3[d] = (int)std::llround(q);
            dims = dims && n3[d] > 0 && std::fabs(q - n3[d]) < 1e-9 * q;
        }
        dims = dims && (long long)n3[0] * n3[1] * n3[2] == nc && (long long)(n3[0] - 1) * n3[1] * n3[2] == a.nfx &&
               (long long)n3[0] * (n3[1] - 1) * n3[2] == a.nfy;
        bool same = dims;
        for (int c = 0; c < nc && same; c++) {
            int g[6];
            grid_cell_faces(c, n3[0], n3[1], n3[2], g);
            same = std::memcmp(g, &cf[6 * (size_t)c], sizeof g) == 0;
        }
        if (same) {
            a.grid_faces = 1;
            for (int d = 0; d < 3; d++) a.grid_n[d] = n3[d];
        }
        bool one = nc > 0;
        for (int c = 1; c < nc && one; c++) one = std::memcmp(&inv_vol[c], &inv_vol[0], sizeof(double)) == 0;
        if (one) {
            a.inv_volume_uniform = 1;
            a.inv_volume_all = inv_vol[0];
        }
    }
    a.closure = nullptr;
    if (!closure.empty()) {
        double *d_cl;
        if ((rc = s->upload(&d_cl, closure))) return rc;
        a.closure = d_cl;
    }
    a.lsw_code = nullptr;
    if (coded) {
        unsigned *d_code;
        if ((rc = s->upload(&d_code, lcode))) return rc;
        a.lsw_code = d_code;
    }
    a.stencil = d_stencil; a.ls = d_ls; a.lsw = d_lsw; a.bc_rho_type = d_rt; a.bc_vel_type = d_vt; a.bc_periodic = d_per;
    a.bc_val = d_bcv; a.bc_rec = d_bcr; a.face_cells = d_fcells; a.axis_face = d_axf; a.gen_face = d_gen;
    a.visc_factor = d_visc; a.cell_faces = d_cf; a.cell_volume = d_vol; a.cell_inv_volume = d_ivol;
    Vec4<R> *d_state, *d_flux;
    R *d_grad;
    double4 *d_t1;
    if ((rc = s->alloc(&d_state, nt)) || (rc = s->alloc(&d_grad, 12 * (size_t)nt)) || (rc = s->alloc(&d_flux, nf)) ||
        (rc = s->alloc(&d_t1, nc)))
        return rc;
    LBFS_CUDA(cudaMemset(d_state, 0, sizeof(Vec4<R>) * nt));
    LBFS_CUDA(cudaMemset(d_grad, 0, sizeof(R) * 12 * (size_t)nt));
    LBFS_CUDA(cudaMemset(d_flux, 0, sizeof(Vec4<R>) * nf));
    LBFS_CUDA(cudaMemset(d_t1, 0, sizeof(double4) * nc));
    a.state = d_state; a.grad = d_grad; a.flux = d_flux; a.t1 = d_t1;
    double *d_partials, *d_rsum;
    unsigned int *d_ticket, *d_flags;
    if ((rc = s->alloc(&d_partials, 4 * (size_t)kK3BlocksLimit)) || (rc = s->alloc(&d_rsum, 4)) ||
        (rc = s->alloc(&d_ticket, 1)) || (rc = s->alloc(&d_flags, 1)))
        return rc;
    LBFS_CUDA(cudaMemset(d_ticket, 0, sizeof(unsigned int)));
    LBFS_CUDA(cudaMemset(d_flags, 0, sizeof(unsigned int)));
    LBFS_CUDA(cudaMemset(d_rsum, 0, 4 * sizeof(double)));
    a.partials = d_partials; a.residual_sums = d_rsum; a.ticket = d_ticket; a.flags = d_flags;
    a.res_out = nullptr;
    a.tb_grad = 256; a.tb_flux = 128; a.tb_gen = 128; a.tb_update = 256; a.update_blocks = kK3MaxBlocks;
    a.n_membranes = 0;
    a.instances = nullptr;
    a.cell_instance = nullptr;
    return LBFS_OK;
}

// Time stepping other than constant: the per-cell CFL areas (populate_cfl_areas,
// Solver_gpu.cu:1657-1687: half the sums of |n_c| * area over the cell's faces,
// in the order of gradient_faces, i.e. the face loop of
// unstructured_mesh.cpp:1645-1665) with the cell volume, the per-cell steps,
// their minimum, and the constants of get_cfl_device.
template <typename R> int setup_time_stepping(lbfs_solver *s, const lbfs_mesh_desc *m) {
    FluidArgs<R> &a = fluid<R>(s);
    const lbfs_params &p = s->params;
    a.time_stepping = p.time_stepping;
    a.cfl = nullptr; a.dt_local = nullptr; a.dt_min = nullptr; a.dt_partials = nullptr; a.dt_ticket = nullptr;
    s->ma.dt_dev = nullptr;
    if (!dynamic_dt(p)) return LBFS_OK;
    const int nc = m->n_cells;
    std::vector<double4> cfl(nc, make_double4(0, 0, 0, 0));
    for (int f = 0; f < m->n_faces; f++) {
        const double *n = m->face_normal + 3 * (size_t)f;
        const double ar = m->face_area[f];
        const int cells[2] = {m->owner[f], f < m->n_interior ? m->neighbour[f] : -1};
        for (int c : cells) {
            if (c < 0 || c >= nc) continue;
            cfl[c].x = cfl[c].x + std::fabs(n[0] * ar);
            cfl[c].y = cfl[c].y + std::fabs(n[1] * ar);
            cfl[c].z = cfl[c].z + std::fabs(n[2] * ar);
        }
    }
    for (int i = 0; i < nc; i++) {
        cfl[i].x = cfl[i].x / 2;
        cfl[i].y = cfl[i].y / 2;
        cfl[i].z = cfl[i].z / 2;
        cfl[i].w = m->cell_volume[i];
    }
    double4 *d_cfl;
    double *d_dtl, *d_min, *d_part;
    unsigned int *d_ticket;
    int rc;
    if ((rc = s->upload(&d_cfl, cfl)) || (rc = s->alloc(&d_dtl, nc)) || (rc = s->alloc(&d_min, 1)) ||
        (rc = s->alloc(&d_part, kCflBlocks)) || (rc = s->alloc(&d_ticket, 1)))
        return rc;
    LBFS_CUDA(cudaMemset(d_ticket, 0, sizeof(unsigned int)));
    LBFS_CUDA(cudaMemcpy(d_min, &p.delta_t, sizeof(double), cudaMemcpyHostToDevice));
    LBFS_CUDA(cudaMemset(d_dtl, 0, sizeof(double) * nc));
    a.cfl = d_cfl; a.dt_local = d_dtl; a.dt_min = d_min; a.dt_partials = d_part; a.dt_ticket = d_ticket;
    const double g = p.pre_conditioned_gamma > 0 ? p.pre_conditioned_gamma : 1.0 / p.gamma_inv;
    const double mv = p.max_velocity;
    // effective speed of sound of get_cfl_device (LBFS.cu:2888-2889), a constant of the run
    a.cfl_esos = mv * std::sqrt(1 - g + std::pow(g / std::sqrt(3.0) / mv, 2));
    a.cfl_gamma = g;
    a.cfl_visc = p.visc;
    a.cfl_max_velocity = mv;
    a.cfl_factor = p.delta_t;  // globals.time_marching_step
    s->ma.dt_dev = d_min;      // node advection moves by the minimum step (Solver_gpu.cu:827)
    return LBFS_OK;
}

// LBFS_IBM_VANDERMONDE4: the vertex coordinates per axis (plateau_x/y/z), the
// centroid coordinate of each cell row (the cells the reference indexes,
// centroid[i].x, centroid[j nx].y, centroid[k nx ny].z,
// immersed_boundary_method.cu:718-740) and the cell volumes.
int setup_rectilinear_ibm(lbfs_solver *s, const lbfs_mesh_desc *m) {
    MembraneArgs &ma = s->ma;
    for (int q = 0; q < 3; q++) { ma.grid_v[q] = nullptr; ma.grid_c[q] = nullptr; }
    ma.cell_volume = s->fp32 ? s->f32.cell_volume : s->f64.cell_volume;
    if (s->params.ibm_stencil != LBFS_IBM_VANDERMONDE4 || s->n_membranes == 0) return LBFS_OK;
    const InstanceGrid &g = s->inst[0];
    const int n[3] = {g.nx, g.ny, g.nz};
    const double *gv[3] = {m->grid_x, m->grid_y, m->grid_z};
    const long long stride[3] = {1, (long long)g.nx, (long long)g.nx * g.ny};
    int rc;
    for (int q = 0; q < 3; q++) {
        std::vector<double> v(gv[q], gv[q] + n[q] + 1), c(n[q]);
        for (int i = 1; i < n[q] + 1; i++)
            if (!(v[i] > v[i - 1])) return set_error(LBFS_ERR_ARG, "grid vertex coordinates must increase");
        for (int i = 0; i < n[q]; i++) c[i] = m->cell_centroid[3 * (g.cell0 + i * stride[q]) + q];
        double *dv, *dc;
        if ((rc = s->upload(&dv, v)) || (rc = s->upload(&dc, c))) return rc;
        ma.grid_v[q] = dv;
        ma.grid_c[q] = dc;
    }
    return LBFS_OK;
}

// Ensemble instance table: the descriptor's instances, or one instance covering
// the whole mesh from origin/length/delta_x/delta_h.
int setup_instances(lbfs_solver *s, const lbfs_mesh_desc *m) {
    std::vector<lbfs_grid_desc> gd;
    if (m->n_instances < 0) return set_error(LBFS_ERR_ARG, "negative instance count");
    if (m->n_instances > 0) {
        if (!m->instances) return set_error(LBFS_ERR_ARG, "instance table is null");
        gd.assign(m->instances, m->instances + m->n_instances);
    } else {
        lbfs_grid_desc g{};
        g.cell0 = 0; g.n_cells = m->n_cells;
        for (int c = 0; c < 3; c++) { g.origin[c] = m->origin[c]; g.length[c] = m->length[c]; }
        g.delta_x = m->delta_x; g.delta_h = m->delta_h;
        gd.push_back(g);
    }
    int next = 0;
    s->grids = gd;
    s->inst.resize(gd.size());
    for (size_t k = 0; k < gd.size(); k++) {
        const lbfs_grid_desc &g = gd[k];
        if (g.cell0 != next || g.n_cells <= 0)
            return set_error(LBFS_ERR_ARG, "instances must be contiguous, non-empty cell ranges in order");
        next += g.n_cells;
        InstanceGrid &q = s->inst[k];
        q.cell0 = g.cell0;
        q.nx = g.delta_x > 0 ? (int)(g.length[0] / g.delta_x) : 0;
        q.ny = g.delta_x > 0 ? (int)(g.length[1] / g.delta_x) : 0;
        q.nz = g.delta_x > 0 ? (int)(g.length[2] / g.delta_x) : 0;
        q.mem0 = q.mem1 = 0;
        q.pad0 = q.pad1 = 0;
    }
    if (next != m->n_cells) return set_error(LBFS_ERR_ARG, "instances do not cover the interior cells");
    return LBFS_OK;
}

int setup_membranes(lbfs_solver *s, const lbfs_mesh_desc *m, const lbfs_rbc_desc *rbc, int n_rbc) {
    const lbfs_params &p = s->params;
    MembraneArgs &ma = s->ma;
    ma.n_membranes = n_rbc;
    ma.ibm_stencil = p.ibm_stencil;
    ma.delta_t = p.delta_t;
    ma.force_cluster = 0;  // separate kernels; lbfs_autotune may choose a cluster of 8 or 16
    ma.nc = m->n_cells;
    ma.state_is_float = s->fp32 ? 1 : 0;
    if (n_rbc == 0) return LBFS_OK;
    const int n_inst = (int)s->inst.size();
    for (int r = 0; r < n_rbc; r++) {
        const int k = rbc[r].instance;
        if (k < 0 || k >= n_inst) return set_error(LBFS_ERR_ARG, "membrane instance out of range");
        if (r > 0 && k < rbc[r - 1].instance)
            return set_error(LBFS_ERR_ARG, "membranes must be grouped by instance, in increasing order");
        const InstanceGrid &g = s->inst[k];
        if (!(s->grids[k].delta_x > 0) || (long long)g.nx * g.ny * g.nz != s->grids[k].n_cells)
            return set_error(LBFS_ERR_ARG, "membranes need the lexicographic uniform grid the IBM stencils index "
                                           "(length / delta_x cells per axis)");
    }
    std::vector<MembraneConst> mc(n_rbc);
    std::vector<int> tri, spr;
    std::vector<double> sf, init;
    int cap = 1, maxn = 0;
    for (int r = 0; r < n_rbc; r++) {
        const lbfs_rbc_desc &d = rbc[r];
        if (d.n_nodes <= 3 || d.n_tris <= 0 || d.n_springs <= 0 || !d.tri || !d.spring || !d.xyz_stress_free ||
            !d.xyz_initial)
            return set_error(LBFS_ERR_ARG, "bad membrane descriptor");
        if (d.n_nodes > kMaxMembraneNodes) return set_error(LBFS_ERR_LIMIT, "membrane has more nodes than one CTA handles");
        MembraneConst &c = mc[r];
        c.node0 = s->total_nodes; c.n_nodes = d.n_nodes;
        c.tri0 = s->total_tris; c.n_tris = d.n_tris;
        c.spring0 = s->total_springs; c.n_springs = d.n_springs;
        c.inc0 = 4 * s->total_springs;
        c.volume_modulus = d.volume_modulus; c.local_area_modulus = d.local_area_modulus;
        c.global_area_modulus = d.global_area_modulus; c.shear_modulus = d.shear_modulus;
        c.global_bending_modulus = d.global_bending_modulus; c.local_bending_modulus = d.local_bending_modulus;
        c.membrane_thickness = d.membrane_thickness; c.viscosity = d.viscosity; c.wlc_ratio = d.wlc_ratio;
        c.curvature_ratio = d.curvature_ratio; c.volume_ratio = d.volume_ratio;
        c.internal_viscosity_ratio = d.internal_viscosity_ratio; c.reference_length = d.reference_length;
        c.pivkin_length = d.pivkin_length; c.sphere_reference = d.sphere_reference;
        const InstanceGrid &g = s->inst[d.instance];
        const lbfs_grid_desc &gd = s->grids[d.instance];
        c.instance = d.instance;
        c.cell0 = g.cell0; c.gnx = g.nx; c.gny = g.ny; c.gnz = g.nz;
        for (int q = 0; q < 3; q++) c.gorigin[q] = gd.origin[q];
        c.gdx = gd.delta_x; c.gdh = gd.delta_h;
        if (d.periodic < 0 || d.periodic > LBFS_WRAP_ALL || (d.periodic == LBFS_WRAP_ALL && r > 0 && rbc[0].periodic != LBFS_WRAP_ALL))
            return set_error(LBFS_ERR_ARG, "periodic: 0, LBFS_WRAP_OWN, or LBFS_WRAP_ALL on membrane 0 (it decides for all)");
        c.periodic = rbc[0].periodic == LBFS_WRAP_ALL ? LBFS_WRAP_ALL : d.periodic;
        c.domain_z0 = gd.origin[2];
        c.domain_Z = gd.length[2];
        if (c.periodic) s->wrap_membranes = true;
        {
            // a patch of in-range stencils lies inside the instance's grid
            const int S = stencil_width(p.ibm_stencil);
            const long long cells = (long long)(g.nx + S - 1) * (g.ny + S - 1) * (g.nz + S - 1);
            c.patch_bound = (int)std::min<long long>(kMaxPatchCells, cells);
        }
        if (s->inst[d.instance].mem1 == 0) s->inst[d.instance].mem0 = r;
        s->inst[d.instance].mem1 = r + 1;
        for (int i = 0; i < 3 * d.n_tris; i++) {
            if (d.tri[i] < 0 || d.tri[i] >= d.n_nodes) return set_error(LBFS_ERR_ARG, "triangle index out of range");
            tri.push_back(d.tri[i] + s->total_nodes);
        }
        for (int i = 0; i < 4 * d.n_springs; i++) {
            if (d.spring[i] < 0 || d.spring[i] >= d.n_nodes) return set_error(LBFS_ERR_ARG, "spring index out of range");
            spr.push_back(d.spring[i] + s->total_nodes);
        }
        sf.insert(sf.end(), d.xyz_stress_free, d.xyz_stress_free + 3 * d.n_nodes);
        init.insert(init.end(), d.xyz_initial, d.xyz_initial + 3 * d.n_nodes);
        s->total_nodes += d.n_nodes;
        s->total_tris += d.n_tris;
        s->total_springs += d.n_springs;
        maxn = std::max(maxn, d.n_nodes);
    }
    while (cap < maxn) cap <<= 1;
    ma.sort_capacity = cap;
    ma.max_nodes = maxn;
    membrane_prepare(cap, maxn);
    // node -> (spring, slot) incidence in spring order
    const int N = s->total_nodes, S = s->total_springs;
    std::vector<int> inc_start(N + 1, 0), inc(4 * (size_t)S);
    for (int i = 0; i < 4 * S; i++) inc_start[spr[i] + 1]++;
    for (int n = 0; n < N; n++) inc_start[n + 1] += inc_start[n];
    std::vector<int> fill(inc_start.begin(), inc_start.end() - 1);
    for (int sp = 0; sp < S; sp++)
        for (int q = 0; q < 4; q++) inc[fill[spr[4 * sp + q]]++] = 4 * sp + q;
    std::vector<double> x(N), y(N), z(N);
    for (int n = 0; n < N; n++) { x[n] = sf[3 * n]; y[n] = sf[3 * n + 1]; z[n] = sf[3 * n + 2]; }
    std::vector<double> zeros_n(N, 0.0), zeros_s(S, 0.0), zeros_2s(2 * (size_t)S, 0.0);
    std::vector<MembraneScalars> msz(n_rbc);
    std::memset(msz.data(), 0, sizeof(MembraneScalars) * n_rbc);
    long long total_patch = 0;
    for (int r = 0; r < n_rbc; r++) {
        msz[r].patch_off = (int)total_patch;
        total_patch += mc[r].patch_bound;
    }
    if (total_patch + n_rbc > INT32_MAX) return set_error(LBFS_ERR_LIMIT, "IBM patches exceed 2^31 cells in total");
    s->total_patch = total_patch;
    // one warp per patch cell, 8 warps a block, grid-stride
    ma.spread_blocks = (int)std::max<long long>(1, std::min<long long>((total_patch + 7) / 8, kSpreadMaxBlocks));
    ma.ibm_z_lo = 0;
    ma.ibm_z_hi = INT32_MAX;
    int rc = 0;
    std::vector<int> spring_mem(S), node_mem(N), identity(N);
    for (int n = 0; n < N; n++) identity[n] = n;
    for (int r = 0; r < n_rbc; r++) {
        for (int q = 0; q < mc[r].n_springs; q++) spring_mem[mc[r].spring0 + q] = r;
        for (int q = 0; q < mc[r].n_nodes; q++) node_mem[mc[r].node0 + q] = r;
    }
    std::vector<int> cell_inst;
    if (n_inst > 1) {
        cell_inst.resize(m->n_cells);
        for (int k = 0; k < n_inst; k++)
            for (int i = 0; i < s->grids[k].n_cells; i++) cell_inst[s->inst[k].cell0 + i] = k;
    }
    ma.total_nodes = N;
    ma.total_springs = S;
    MembraneConst *d_mc; MembraneScalars *d_ms; int *d_tri, *d_spr, *d_inc, *d_incs, *d_smem, *d_nmem;
    InstanceGrid *d_inst; int *d_cinst = nullptr;
    if ((rc = s->upload(&d_inst, s->inst)) || (rc = s->upload(&d_nmem, node_mem)) ||
        (n_inst > 1 && (rc = s->upload(&d_cinst, cell_inst))))
        return rc;
    if ((rc = s->upload(&d_mc, mc)) || (rc = s->upload(&d_ms, msz)) || (rc = s->upload(&d_tri, tri)) ||
        (rc = s->upload(&d_spr, spr)) || (rc = s->upload(&d_inc, inc)) || (rc = s->upload(&d_incs, inc_start)) ||
        (rc = s->upload(&ma.x, x)) || (rc = s->upload(&ma.y, y)) || (rc = s->upload(&ma.z, z)) ||
        (rc = s->upload(&ma.vx, zeros_n)) || (rc = s->upload(&ma.vy, zeros_n)) || (rc = s->upload(&ma.vz, zeros_n)) ||
        (rc = s->upload(&ma.fx, zeros_n)) || (rc = s->upload(&ma.fy, zeros_n)) || (rc = s->upload(&ma.fz, zeros_n)) ||
        (rc = s->upload(&ma.contour, zeros_s)) || (rc = s->upload(&ma.kspring, zeros_s)) ||
        (rc = s->upload(&ma.curv, zeros_s)) || (rc = s->upload(&ma.curv0, zeros_s)) ||
        (rc = s->upload(&ma.angle0, zeros_s)) || (rc = s->upload(&ma.area0, zeros_2s)) ||
        (rc = s->upload(&ma.area, zeros_2s)) || (rc = s->alloc(&ma.contrib, 12 * (size_t)S)) ||
        (rc = s->alloc(&ma.keys, N)) || (rc = s->alloc(&ma.patch_force, (size_t)total_patch * 3)) ||
        (rc = s->upload(&d_smem, spring_mem)) ||
        (rc = s->alloc(&ma.bin_start, (size_t)total_patch + n_rbc)) ||
        (rc = s->alloc(&ma.bin_cursor, (size_t)total_patch + n_rbc)) ||
        (rc = s->alloc(&ma.cell_start, (size_t)n_rbc + 1)) || (rc = s->alloc(&ma.sort_ticket, 1)) ||
        (rc = s->upload(&ma.sorted_node, identity)) ||
        (rc = s->alloc(&ma.node_base, 3 * (size_t)N)) ||
        (rc = s->alloc(&ma.node_w, 12 * (size_t)N)) ||
        (rc = s->alloc(&ma.mad_partials, (size_t)n_rbc * kMaxSpringBlocks)) ||
        (rc = s->alloc(&ma.mad_ticket, (size_t)n_rbc)))
        return rc;
    LBFS_CUDA(cudaMemset(ma.mad_ticket, 0, sizeof(unsigned int) * n_rbc));
    LBFS_CUDA(cudaMemset(ma.sort_ticket, 0, sizeof(unsigned int)));
    LBFS_CUDA(cudaMemset(ma.cell_start, 0, sizeof(int) * (n_rbc + 1)));
    LBFS_CUDA(cudaMemset(ma.patch_force, 0, sizeof(double) * 3 * (size_t)total_patch));
    ma.max_springs = 0;
    ma.max_patch_bound = 0;
    for (int r = 0; r < n_rbc; r++) {
        ma.max_springs = std::max(ma.max_springs, mc[r].n_springs);
        ma.max_patch_bound = std::max(ma.max_patch_bound, mc[r].patch_bound);
    }
    ma.node_mem = d_nmem;

    ma.spring_mem = d_smem;
    ma.mc = d_mc; ma.ms = d_ms; ma.tri = d_tri; ma.spring = d_spr; ma.inc = d_inc; ma.inc_start = d_incs;
    ma.flags = s->fp32 ? s->f32.flags : s->f64.flags;
    ma.state = s->fp32 ? (const void *)s->f32.state : (const void *)s->f64.state;
    // reference pass on the stress-free mesh, then the initial mesh
    ma.mode = kModeReference;
    launch_membrane(ma, s->stream);
    LBFS_CUDA(cudaGetLastError());
    for (int n = 0; n < N; n++) { x[n] = init[3 * n]; y[n] = init[3 * n + 1]; z[n] = init[3 * n + 2]; }
    LBFS_CUDA(cudaMemcpyAsync(ma.x, x.data(), N * sizeof(double), cudaMemcpyHostToDevice, s->stream));
    LBFS_CUDA(cudaMemcpyAsync(ma.y, y.data(), N * sizeof(double), cudaMemcpyHostToDevice, s->stream));
    LBFS_CUDA(cudaMemcpyAsync(ma.z, z.data(), N * sizeof(double), cudaMemcpyHostToDevice, s->stream));
    ma.mode = kModeInitial;
    launch_membrane(ma, s->stream);
    launch_membrane_tables(ma, s->stream);  // stencil tables at the initial positions
    LBFS_CUDA(cudaGetLastError());
    LBFS_CUDA(cudaStreamSynchronize(s->stream));
    ma.mode = kModeStep;
    // FluidArgs see the patches
    s->f64.n_membranes = s->f32.n_membranes = n_rbc;
    s->f64.membrane_scalars = s->f32.membrane_scalars = d_ms;
    s->f64.patch_force = s->f32.patch_force = ma.patch_force;
    s->f64.instances = s->f32.instances = d_inst;
    s->f64.cell_instance = s->f32.cell_instance = d_cinst;
    // interior viscosity
    ViscArgs &va = s->va;
    va.nc = m->n_cells; va.n_membranes = n_rbc; va.centroid = s->d_centroid; va.mc = d_mc; va.ms = d_ms;
    va.tri = d_tri; va.x = ma.x; va.y = ma.y; va.z = ma.z;
    va.instances = d_inst; va.cell_instance = d_cinst;
    va.visc_factor = s->fp32 ? (void *)s->f32.visc_factor : (void *)s->f64.visc_factor;
    va.visc_is_float = s->fp32 ? 1 : 0;
    va.total_tris = s->total_tris;
    if ((rc = s->alloc(&va.bins, n_rbc)) || (rc = s->alloc(&va.bin_start, (size_t)n_rbc * (kViscBins + 1))) ||
        (rc = s->alloc(&va.bin_list, 4 * (size_t)s->total_tris)))
        return rc;
    return LBFS_OK;
}

// Records `ev` on `st`; inside stream capture as an external event node (so the
// graph replay records it), outside capture as a plain record.
cudaError_t record_event(cudaEvent_t ev, cudaStream_t st) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(st, &cs);
    if (cs == cudaStreamCaptureStatusActive) return cudaEventRecordWithFlags(ev, st, cudaEventRecordExternal);
    return cudaEventRecord(ev, st);
}

// The chunk plan of the pipelined K1 -> K2.  It needs an axis-aligned mesh
// whose interior faces have owner < neighbour and, within each axis range,
// non-decreasing neighbours (the generator's order; ensembles keep it): then
// the faces whose neighbour lies below a split form a prefix of each range,
// and the faces of chunk c need the gradients of chunks <= c only.
//
// Tiles of the face kernel need in addition owners that do not decrease within
// each axis range (the generator's order; ensembles keep it): the faces owned
// by a tile of cells are then a contiguous range of each axis.
//
// Meshes that are not axis aligned take tiles too (their interior faces in the
// general-normal kernel): the generator's face ranges when the x, y, z counts
// cover the interior faces, else one range of all interior faces (an imported
// polyMesh, whose internal faces OpenFOAM orders by owner); no chunking.
int plan_chunks(lbfs_solver *s, const int *owner, const int *neighbour, int nfx, int nfy, int nfz, bool axis_aligned) {
    s->chunkable = false;
    s->tiled = false;
    const int ni = s->ni, nc = s->nc;
    if (ni == 0 || !owner) return LBFS_OK;
    if (nfx < 0 || nfy < 0 || nfz < 0 || (long long)nfx + nfy + nfz != ni) {
        if (axis_aligned) return LBFS_OK;
        nfx = ni; nfy = 0; nfz = 0;
    }
    const int start[3] = {0, nfx, nfx + nfy}, count[3] = {nfx, nfy, nfz};
    bool ordered = true, owners_ordered = true;
    for (int ax = 0; ax < 3; ax++)
        for (int f = start[ax]; f < start[ax] + count[ax]; f++) {
            if (!(owner[f] < neighbour[f]) || (f > start[ax] && neighbour[f] < neighbour[f - 1])) ordered = false;
            if (f > start[ax] && owner[f] < owner[f - 1]) owners_ordered = false;
        }
    if (owners_ordered) {
        for (int b = 0; b < 3; b++) {
            const int T = 64 << b, nt = (nc + T - 1) / T;
            std::vector<int> &tt = s->tiles_h[b];
            std::vector<int> &mx = s->tile_maxnb[b];
            tt.assign(3 * (size_t)(nt + 1), 0);
            mx.assign(nt, -1);
            for (int ax = 0; ax < 3; ax++) {
                const int *ow = owner + start[ax];
                for (int t = 0; t <= nt; t++)
                    tt[3 * (size_t)t + ax] =
                        start[ax] + (int)(std::lower_bound(ow, ow + count[ax], (int)std::min<long long>((long long)t * T, nc)) - ow);
            }
            int run = -1;
            for (int t = 0; t < nt; t++) {
                for (int ax = 0; ax < 3; ax++) {
                    const int f1 = tt[3 * (size_t)(t + 1) + ax];
                    if (f1 > tt[3 * (size_t)t + ax]) run = std::max(run, neighbour[f1 - 1]);
                }
                mx[t] = run;
            }
            int rc = s->upload(&s->d_tiles[b], tt);
            if (rc) return rc;
        }
        s->tiled = true;
    }
    if (!ordered || !axis_aligned || nc < 2 * kMaxFluxChunks * 256) return LBFS_OK;
    s->chunkable = true;
    s->chunk_nb.assign(neighbour, neighbour + ni);
    for (int ax = 0; ax < 3; ax++) { s->chunk_start[ax] = start[ax]; s->chunk_count[ax] = count[ax]; }
    return LBFS_OK;
}

// Face-kernel tiles of the current flux block size into the kernel arguments.
template <typename R> void apply_tiles(lbfs_solver *s, FluidArgs<R> &a) {
    const int tb = a.axis_aligned ? a.tb_flux : a.tb_gen;  // the tile kernel's block size
    const int b = tb == 64 ? 0 : (tb == 256 ? 2 : 1);
    a.flux_tiles = s->tiled ? s->d_tiles[b] : nullptr;
    a.n_tiles = s->tiled ? (int)s->tile_maxnb[b].size() : 0;
}

// Cell splits and face ranges for K chunks (chunk_cell has K + 1 entries).
void set_chunks(lbfs_solver *s, int K) {
    if (!s->chunkable || K < 2) K = 1;
    s->flux_chunks = K;
    if (s->fp32) apply_tiles<float>(s, s->f32);
    else apply_tiles<double>(s, s->f64);
    const bool aa = s->fp32 ? s->f32.axis_aligned : s->f64.axis_aligned;
    const int tb = s->fp32 ? (aa ? s->f32.tb_flux : s->f32.tb_gen) : (aa ? s->f64.tb_flux : s->f64.tb_gen);
    const std::vector<int> &mx = s->tile_maxnb[tb == 64 ? 0 : (tb == 256 ? 2 : 1)];
    // gradients and interior fluxes (K each), boundary fluxes, update; membrane kernels; CFL
    s->launches_per_step = 2 * K + 2 + (s->n_membranes > 0 ? (s->ma.force_cluster > 0 ? 3 : 6) : 0) + (dynamic_dt(s->params) ? 1 : 0);
    s->chunk_cell.assign(K + 1, 0);
    s->chunk_faces.assign(K, FaceRanges{});
    for (int c = 0; c <= K; c++) s->chunk_cell[c] = (int)((long long)s->nc * c / K);
    // tiles of chunk c: those whose faces' neighbours all lie below the chunk's upper split
    s->chunk_tile.assign(K + 1, 0);
    if (s->tiled) {
        const int nt = (int)mx.size();
        for (int c = 1; c < K; c++)
            s->chunk_tile[c] = std::max(s->chunk_tile[c - 1],
                                        (int)(std::lower_bound(mx.begin(), mx.end(), s->chunk_cell[c]) - mx.begin()));
        s->chunk_tile[K] = nt;
    }
    if (K == 1) return;
    int prev[3] = {0, 0, 0};
    for (int c = 0; c < K; c++) {
        FaceRanges &r = s->chunk_faces[c];
        for (int ax = 0; ax < 3; ax++) {
            const int *b = s->chunk_nb.data() + s->chunk_start[ax], n = s->chunk_count[ax];
            // faces of this axis whose neighbour lies below the chunk's upper split
            const int end = c == K - 1 ? n : (int)(std::lower_bound(b, b + n, s->chunk_cell[c + 1]) - b);
            r.start[ax] = s->chunk_start[ax] + prev[ax];
            r.count[ax] = end - prev[ax];
            prev[ax] = end;
        }
    }
}

struct PhaseMark {
    lbfs_solver *s;
    int phase;
    cudaStream_t st;
    PhaseMark(lbfs_solver *s_, int ph, cudaStream_t st_) : s(s_), phase(ph), st(st_) {
        if (s->kernel_events) record_event(s->ev_phase[phase][0], st);
    }
    ~PhaseMark() {
        if (s->kernel_events) {
            record_event(s->ev_phase[phase][1], st);
            s->phase_recorded[phase] = true;
        }
    }
};

// K1 and K2 of a step: in sequence on the handle's stream, or pipelined in
// chunks of cells: the gradients of each chunk on the handle's stream, the
// interior-face fluxes of that chunk on a second stream as soon as they (and
// the chunks before) are done, so the FP64-heavy fluxes of one chunk run beside
// the load-latency-bound gradients of the next; the boundary faces (which read
// ghost gradients) follow every K1, and the handle's stream joins the second.
//
// Unpipelined, the boundary faces (a short kernel of long threads that would
// otherwise add its whole latency after the interior faces) run on the second
// stream beside the interior faces, which follow the gradients on the
// handle's stream as a programmatic dependent launch (their CTAs are placed
// behind the gradients' last wave and wait there for its results) unless
// per-kernel events sit between the two.
//
// spread_here: the membrane chain (on its own stream, recorded in ev_join)
// left its spread out; it runs on the boundary-face stream after the boundary
// faces, so the cell update depends on two kernels, the interior faces (a
// programmatic edge, which lets it be placed behind their last wave) and that
// stream's last one, as without membranes.  With the membrane stream joined to
// the handle's stream directly the update started only after the interior
// faces had finished.
template <typename R> bool spread_with_faces(const lbfs_solver *s, const FluidArgs<R> &a) {
    const int K = a.axis_aligned ? s->flux_chunks : 1;
    return s->n_membranes > 0 && K <= 1 && (a.axis_aligned || a.flux_tiles) && !s->kernel_events;
}
//
// after_k1 (may be null): enqueued right behind the gradient launch (the last
// chunk's), before anything that waits for the membrane stream.  With it and
// spread_here, the spread instead follows the membrane kernels on their own
// stream as a programmatic launch, joined by the boundary faces (which then
// end long before the membrane kernels): the cell update still has one other
// dependency, and the spread starts behind the last membrane kernel's last
// wave instead of a launch after it.
template <typename R>
int enqueue_k1_k2(lbfs_solver *s, FluidArgs<R> &a, int *n, bool spread_here,
                  const std::function<int()> *after_k1 = nullptr) {
    const int K = a.axis_aligned ? s->flux_chunks : 1;
    if (K <= 1) {
        { PhaseMark m(s, 1, s->stream); launch_fluid_gradients<R>(a, s->stream); }
        if (after_k1) {
            int rc = (*after_k1)();
            if (rc) return rc;
        }
        {
            PhaseMark m(s, 2, s->stream);
            const bool fork = a.axis_aligned || a.flux_tiles;  // interior faces in their own kernel
            if (fork) {
                LBFS_CUDA(cudaEventRecord(s->ev_chunk[0], s->stream));
                LBFS_CUDA(cudaStreamWaitEvent(s->stream4, s->ev_chunk[0], 0));
                launch_fluid_flux_general<R>(a, s->stream4);
                if (spread_here && after_k1) {
                    LBFS_CUDA(cudaEventRecord(s->ev_bnd, s->stream4));
                    LBFS_CUDA(cudaStreamWaitEvent(s->stream2, s->ev_bnd, 0));
                    launch_membrane_spread(s->ma, s->stream2, true);
                    *n += 1;
                    LBFS_CUDA(cudaEventRecord(s->ev_flux, s->stream2));
                } else {
                    if (spread_here) {
                        LBFS_CUDA(cudaStreamWaitEvent(s->stream4, s->ev_join, 0));
                        launch_membrane_spread(s->ma, s->stream4);
                        *n += 1;
                    }
                    LBFS_CUDA(cudaEventRecord(s->ev_flux, s->stream4));
                }
                launch_fluid_flux_axis<R>(a, s->stream, !s->kernel_events);
                LBFS_CUDA(cudaStreamWaitEvent(s->stream, s->ev_flux, 0));
            } else {
                launch_fluid_flux_general<R>(a, s->stream);
            }
        }
        *n += 2;
        return LBFS_OK;
    }
    {
        PhaseMark m(s, 1, s->stream);
        for (int c = 0; c < K; c++) {
            launch_fluid_gradients_range<R>(a, s->chunk_cell[c], s->chunk_cell[c + 1], s->stream);
            LBFS_CUDA(cudaEventRecord(s->ev_chunk[c], s->stream));
        }
    }
    if (after_k1) {
        int rc = (*after_k1)();
        if (rc) return rc;
    }
    for (int c = 0; c < K; c++) {
        LBFS_CUDA(cudaStreamWaitEvent(s->stream4, s->ev_chunk[c], 0));
        if (c == 0 && s->kernel_events) LBFS_CUDA(record_event(s->ev_phase[2][0], s->stream4));
        if (a.flux_tiles) launch_fluid_flux_tiles<R>(a, s->chunk_tile[c], s->chunk_tile[c + 1], s->stream4);
        else launch_fluid_flux_axis_ranges<R>(a, s->chunk_faces[c], s->stream4);
    }
    if (s->kernel_events) {
        LBFS_CUDA(record_event(s->ev_phase[2][1], s->stream4));
        s->phase_recorded[2] = true;
    }
    LBFS_CUDA(cudaEventRecord(s->ev_flux, s->stream4));
    launch_fluid_flux_general<R>(a, s->stream);
    LBFS_CUDA(cudaStreamWaitEvent(s->stream, s->ev_flux, 0));
    *n += 2 * K + 1;
    return LBFS_OK;
}

template <typename R> int enqueue_step(lbfs_solver *s, bool visc_update, int *launches) {
    FluidArgs<R> &a = fluid<R>(s);
    int n = 0;
    for (int p = 0; p < kPhases; p++) s->phase_recorded[p] = false;
    if (s->profiling) LBFS_CUDA(record_event(s->ev_phase[5][0], s->stream));
    if (a.time_stepping != 0 && a.time_stepping != LBFS_DT_CONSTANT) {
        // the step's time step from the state at its start (Solver_gpu.cu:767-787)
        launch_fluid_cfl<R>(a, s->stream);
        n += 1;
    }
    if (s->n_membranes > 0) {
        if (visc_update) {
            { PhaseMark m(s, 0, s->stream); n += launch_membrane(s->ma, s->stream); }
            { PhaseMark m(s, 4, s->stream); launch_interior_viscosity(s->va, s->stream); }
            { PhaseMark m(s, 1, s->stream); launch_fluid_gradients<R>(a, s->stream); }
            { PhaseMark m(s, 2, s->stream); launch_fluid_flux<R>(a, s->stream); }
            n += 3;
        } else {
            const bool spread_here = spread_with_faces<R>(s, a);
            auto membranes = [&]() -> int {
                {
                    PhaseMark m(s, 0, s->stream2);
                    n += launch_membrane(s->ma, s->stream2, s->stream3, s->ev_advected, s->ev_sorted, spread_here);
                }
                LBFS_CUDA(cudaEventRecord(s->ev_join, s->stream2));
                return LBFS_OK;
            };
            cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
            LBFS_CUDA(cudaStreamIsCapturing(s->stream, &cap));
            int rc;
            if (s->membrane_after_k1 && cap == cudaStreamCaptureStatusActive && !s->kernel_events) {
                // The membrane kernels beside the gradient kernel from the step's start compete with its
                // blocks for the SMs' registers as they are placed.  Here the membrane stream joins the
                // capture behind the gradient kernel's launch-completion port (every block has begun;
                // the advection kernel reads nothing the gradients write and does not wait on its
                // programmatic predecessor), so its kernels are placed behind the gradients' last wave.
                const std::function<int()> after_k1 = [&]() -> int {
                    cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
                    const cudaGraphNode_t *deps = nullptr;
                    const cudaGraphEdgeData *edges = nullptr;
                    size_t nd = 0;
                    LBFS_CUDA(cudaStreamGetCaptureInfo_v3(s->stream, &st, nullptr, nullptr, &deps, &edges, &nd));
                    cudaGraphNode_t k1 = nullptr;
                    cudaGraphNodeType type;
                    if (st == cudaStreamCaptureStatusActive && nd == 1 &&
                        cudaGraphNodeGetType(deps[0], &type) == cudaSuccess && type == cudaGraphNodeTypeKernel)
                        k1 = deps[0];
                    LBFS_CUDA(cudaEventRecord(s->ev_fork, s->stream));
                    LBFS_CUDA(cudaStreamWaitEvent(s->stream2, s->ev_fork, 0));
                    if (k1) {  // otherwise the membrane stream stays behind the gradient kernel's end
                        cudaGraphEdgeData e = {};
                        e.from_port = cudaGraphKernelNodePortLaunchCompletion;
                        e.type = cudaGraphDependencyTypeProgrammatic;
                        LBFS_CUDA(cudaStreamUpdateCaptureDependencies_v2(s->stream2, &k1, &e, 1,
                                                                         cudaStreamSetCaptureDependencies));
                    }
                    return membranes();
                };
                rc = enqueue_k1_k2<R>(s, a, &n, spread_here, &after_k1);
            } else {
                LBFS_CUDA(cudaEventRecord(s->ev_fork, s->stream));
                LBFS_CUDA(cudaStreamWaitEvent(s->stream2, s->ev_fork, 0));
                if ((rc = membranes())) return rc;
                rc = enqueue_k1_k2<R>(s, a, &n, spread_here);
            }
            if (rc) return rc;
            if (!spread_here) LBFS_CUDA(cudaStreamWaitEvent(s->stream, s->ev_join, 0));
        }
    } else {
        int rc = enqueue_k1_k2<R>(s, a, &n, false);
        if (rc) return rc;
    }
    // behind the face kernels as a programmatic dependent launch (its wait also covers the joined streams)
    { PhaseMark m(s, 3, s->stream); launch_fluid_update<R>(a, s->stream, !s->kernel_events); }
    n += 1;
    if (s->profiling) {
        LBFS_CUDA(record_event(s->ev_phase[5][1], s->stream));
        s->phase_recorded[5] = true;
    }
    LBFS_CUDA(cudaGetLastError());
    if (launches) *launches = n;
    return LBFS_OK;
}

int enqueue(lbfs_solver *s, bool visc_update, int *launches) {
    return s->fp32 ? enqueue_step<float>(s, visc_update, launches) : enqueue_step<double>(s, visc_update, launches);
}

bool visc_due(const lbfs_solver *s, long long t) {
    return s->n_membranes > 0 && s->params.viscosity_period > 0 && t % s->params.viscosity_period == 1;
}

// gpu_solver::check_periodic_object at t % 5000 == 1 (Solver_gpu.cu:1027-1029),
// after the step's fluid update: enqueued behind the step on the solver stream.
constexpr int kWrapPeriod = 5000;
bool wrap_due(const lbfs_solver *s, long long t) { return s->wrap_membranes && t % kWrapPeriod == 1; }
int after_step(lbfs_solver *s) {
    if (!wrap_due(s, s->t)) return LBFS_OK;
    launch_membrane_wrap(s->ma, s->stream);
    LBFS_CUDA(cudaGetLastError());
    return LBFS_OK;
}

void free_all(lbfs_solver *s) {
    if (s->graph) cudaGraphExecDestroy(s->graph);
    if (s->loop_graph) cudaGraphExecDestroy(s->loop_graph);
    for (int p = 0; p < kPhases; p++)
        for (int e = 0; e < 2; e++)
            if (s->ev_phase[p][e]) cudaEventDestroy(s->ev_phase[p][e]);
    for (void *p : s->allocs) cudaFree(p);
    s->allocs.clear();
    if (s->ev_fork) cudaEventDestroy(s->ev_fork);
    if (s->ev_join) cudaEventDestroy(s->ev_join);
    if (s->ev_advected) cudaEventDestroy(s->ev_advected);
    if (s->ev_sorted) cudaEventDestroy(s->ev_sorted);
    if (s->stream3) cudaStreamDestroy(s->stream3);
    if (s->stream4) cudaStreamDestroy(s->stream4);
    if (s->ev_flux) cudaEventDestroy(s->ev_flux);
    if (s->ev_bnd) cudaEventDestroy(s->ev_bnd);
    for (cudaEvent_t e : s->ev_chunk)
        if (e) cudaEventDestroy(e);
    if (s->stream2) cudaStreamDestroy(s->stream2);
    if (s->stream && s->own_stream) cudaStreamDestroy(s->stream);
}

}  // namespace

extern "C" int lbfs_create(const lbfs_mesh_desc *mesh, const lbfs_params *params, const lbfs_rbc_desc *rbc,
                           int32_t n_rbc, int32_t device, lbfs_solver **out) {
    if (!out || !params) return set_error(LBFS_ERR_ARG, "null argument");
    *out = nullptr;
    int rc = check_mesh(mesh);
    if (rc) return rc;
    if (n_rbc < 0 || (n_rbc > 0 && !rbc)) return set_error(LBFS_ERR_ARG, "bad membrane count");
    if (params->precision != LBFS_FP64 && params->precision != LBFS_FP32_BULK)
        return set_error(LBFS_ERR_ARG, "precision must be LBFS_FP64 or LBFS_FP32_BULK");
    if (params->ibm_stencil != LBFS_IBM_HAT2 && params->ibm_stencil != LBFS_IBM_PESKIN4 &&
        params->ibm_stencil != LBFS_IBM_VANDERMONDE4)
        return set_error(LBFS_ERR_ARG, "ibm_stencil must be LBFS_IBM_HAT2, LBFS_IBM_PESKIN4 or LBFS_IBM_VANDERMONDE4");
    if (params->ibm_stencil == LBFS_IBM_VANDERMONDE4 && n_rbc > 0) {
        if (!mesh->grid_x || !mesh->grid_y || !mesh->grid_z)
            return set_error(LBFS_ERR_ARG, "LBFS_IBM_VANDERMONDE4 needs the mesh's vertex coordinates (grid_x/y/z)");
        if (mesh->n_instances > 1 || !mesh->axis_aligned)
            return set_error(LBFS_ERR_UNSUPPORTED, "LBFS_IBM_VANDERMONDE4 runs on one rectilinear mesh");
    }
    if (!(params->delta_t > 0)) return set_error(LBFS_ERR_ARG, "delta_t must be positive");
    if (params->time_stepping < 0 || params->time_stepping > LBFS_DT_TALTS)
        return set_error(LBFS_ERR_ARG, "time_stepping must be 0 or LBFS_DT_LOCAL/CONSTANT/MIN/TALTS");
    if (dynamic_dt(*params)) {
        if (mesh->n_instances > 1)
            return set_error(LBFS_ERR_UNSUPPORTED, "time stepping other than constant couples the instances of an "
                                                   "ensemble through the minimum step; use constant time stepping");
        const double g = params->pre_conditioned_gamma > 0 ? params->pre_conditioned_gamma : 1.0 / params->gamma_inv;
        if (!(g > 0) || !(params->max_velocity > 0))
            return set_error(LBFS_ERR_ARG, "time stepping other than constant needs gamma > 0 and max_velocity > 0");
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return set_error(LBFS_ERR_CUDA, "no CUDA device: this library has no CPU path");
    if (device < 0 || device >= ndev) return set_error(LBFS_ERR_ARG, "device index out of range");
    lbfs_solver *s = new lbfs_solver();
    s->device = device;
    s->params = *params;
    s->fp32 = params->precision == LBFS_FP32_BULK;
    s->nc = mesh->n_cells; s->nf = mesh->n_faces; s->ni = mesh->n_interior; s->nb = mesh->n_bc;
    s->n_membranes = n_rbc;
    auto fail = [&](int code) { free_all(s); delete s; return code; };
    if (cudaSetDevice(device) != cudaSuccess) return fail(set_error(LBFS_ERR_CUDA, "cudaSetDevice failed"));
    int prio_lo = 0, prio_hi = 0;
    cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi);
    if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithPriority(&s->stream2, cudaStreamNonBlocking, prio_hi) != cudaSuccess ||
        cudaStreamCreateWithPriority(&s->stream3, cudaStreamNonBlocking, prio_hi) != cudaSuccess ||
        cudaStreamCreateWithFlags(&s->stream4, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&s->ev_flux, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&s->ev_bnd, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&s->ev_advected, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&s->ev_sorted, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&s->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&s->ev_join, cudaEventDisableTiming) != cudaSuccess)
        return fail(set_error(LBFS_ERR_CUDA, "stream/event creation failed"));
    for (cudaEvent_t &e : s->ev_chunk)
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess)
            return fail(set_error(LBFS_ERR_CUDA, "event creation failed"));
    if ((rc = setup_instances(s, mesh))) return fail(rc);
    rc = s->fp32 ? setup_fluid<float>(s, mesh) : setup_fluid<double>(s, mesh);
    if (rc) return fail(rc);
    std::vector<double> centroid(mesh->cell_centroid, mesh->cell_centroid + 3 * (size_t)mesh->n_cells);
    if ((rc = s->upload(&s->d_centroid, centroid))) return fail(rc);
    if ((rc = setup_rectilinear_ibm(s, mesh))) return fail(rc);  // read by the stencil tables of the set-up
    rc = setup_membranes(s, mesh, rbc, n_rbc);
    if (rc) return fail(rc);
    rc = s->fp32 ? setup_time_stepping<float>(s, mesh) : setup_time_stepping<double>(s, mesh);
    if (rc) return fail(rc);
    if ((rc = plan_chunks(s, mesh->owner, mesh->neighbour, mesh->n_face_x, mesh->n_face_y, mesh->n_face_z,
                          mesh->axis_aligned != 0)))
        return fail(rc);
    set_chunks(s, 1);
    *out = s;
    return LBFS_OK;
}

extern "C" int lbfs_destroy(lbfs_solver *s) {
    if (!s) return LBFS_OK;
    cudaSetDevice(s->device);
    if (s->stream) cudaStreamSynchronize(s->stream);
    free_all(s);
    delete s;
    return LBFS_OK;
}

extern "C" int lbfs_set_stream(lbfs_solver *s, void *stream) {
    if (!s) return set_error(LBFS_ERR_ARG, "null handle");
    LBFS_CUDA(cudaStreamSynchronize(s->stream));
    if (s->own_stream) cudaStreamDestroy(s->stream);
    s->stream = (cudaStream_t)stream;
    s->own_stream = false;
    drop_step_graphs(s);
    return LBFS_OK;
}

namespace {
int ensure_stage(lbfs_solver *s) {
    if (s->d_stage) return LBFS_OK;
    return s->alloc(&s->d_stage, 4 * (size_t)s->nc);
}
}  // namespace

// Host arrays are copied as four planes into a device staging buffer (one
// cudaMemcpyAsync each: full DMA bandwidth from pinned memory) and packed into
// the resident (u, v, w, rho) records by a kernel.
extern "C" int lbfs_set_state(lbfs_solver *s, const double *rho, const double *u, const double *v, const double *w) {
    if (!s || !rho || !u || !v || !w) return set_error(LBFS_ERR_ARG, "null argument");
    LBFS_CUDA(cudaSetDevice(s->device));
    int rc = ensure_stage(s);
    if (rc) return rc;
    const size_t nc = (size_t)s->nc, bytes = nc * sizeof(double);
    const double *src[4] = {rho, u, v, w};
    for (int k = 0; k < 4; k++)
        LBFS_CUDA(cudaMemcpyAsync(s->d_stage + k * nc, src[k], bytes, cudaMemcpyHostToDevice, s->stream));
    if (s->fp32) launch_pack_state<float>(s->f32, s->d_stage, s->stream);
    else launch_pack_state<double>(s->f64, s->d_stage, s->stream);
    LBFS_CUDA(cudaGetLastError());
    LBFS_CUDA(cudaStreamSynchronize(s->stream));
    return LBFS_OK;
}

extern "C" int lbfs_get_state(lbfs_solver *s, double *rho, double *u, double *v, double *w) {
    if (!s || !rho || !u || !v || !w) return set_error(LBFS_ERR_ARG, "null argument");
    LBFS_CUDA(cudaSetDevice(s->device));
    int rc = ensure_stage(s);
    if (rc) return rc;
    const size_t nc = (size_t)s->nc, bytes = nc * sizeof(double);
    if (s->fp32) launch_unpack_state<float>(s->f32, s->d_stage, s->stream);
    else launch_unpack_state<double>(s->f64, s->d_stage, s->stream);
    LBFS_CUDA(cudaGetLastError());
    double *dst[4] = {rho, u, v, w};
    for (int k = 0; k < 4; k++)
        LBFS_CUDA(cudaMemcpyAsync(dst[k], s->d_stage + k * nc, bytes, cudaMemcpyDeviceToHost, s->stream));
    LBFS_CUDA(cudaStreamSynchronize(s->stream));
    return LBFS_OK;
}

extern "C" int lbfs_set_profiling(lbfs_solver *s, int32_t on) {
    if (!s) return set_error(LBFS_ERR_ARG, "null handle");
    LBFS_CUDA(cudaSetDevice(s->device));
    LBFS_CUDA(cudaStreamSynchronize(s->stream));
    if (on && !s->ev_phase[0][0])
        for (int p = 0; p < kPhases; p++)
            for (int e = 0; e < 2; e++) LBFS_CUDA(cudaEventCreate(&s->ev_phase[p][e]));
    s->profiling = on != 0;
    s->kernel_events = on >= 2;
    for (int p = 0; p < kPhases; p++) s->phase_recorded[p] = false;
    drop_step_graphs(s);
    return LBFS_OK;
}

extern "C" int lbfs_get_phase_times(lbfs_solver *s, double *ms) {
    if (!s || !ms) return set_error(LBFS_ERR_ARG, "null argument");
    LBFS_CUDA(cudaSetDevice(s->device));
    LBFS_CUDA(cudaStreamSynchronize(s->stream));
    for (int p = 0; p < kPhases; p++) {
        ms[p] = 0.0;
        if (!s->profiling || !s->phase_recorded[p]) continue;
        float t = 0.f;
        LBFS_CUDA(cudaEventElapsedTime(&t, s->ev_phase[p][0], s->ev_phase[p][1]));
        ms[p] = t;
    }
    return LBFS_OK;
}

extern "C" int lbfs_step(lbfs_solver *s, int32_t n_steps) {
    if (!s || n_steps < 0) return set_error(LBFS_ERR_ARG, "bad arguments");
    LBFS_CUDA(cudaSetDevice(s->device));
    for (int k = 0; k < n_steps; k++) {
        int n = 0;
        int rc = enqueue(s, visc_due(s, s->t), &n);
        if (rc || (rc = after_step(s))) return rc;
        s->t++;
    }
    return LBFS_OK;
}

extern "C" int lbfs_step_graph(lbfs_solver *s, int32_t n_steps) {
    if (!s || n_steps < 0) return set_error(LBFS_ERR_ARG, "bad arguments");
    LBFS_CUDA(cudaSetDevice(s->device));
    if (!s->graph) {
        cudaGraph_t g = nullptr;
        LBFS_CUDA(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
        int n = 0;
        int rc = enqueue(s, false, &n);
        cudaError_t e = cudaStreamEndCapture(s->stream, &g);
        if (rc || e != cudaSuccess) {
            if (g) cudaGraphDestroy(g);  // a capture that ended but whose enqueue failed
            if (rc) return rc;
            return set_error(LBFS_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
        }
        // keep the membrane kernels' launch priority inside the graph (without
        // the flag every node runs at the priority of the stream it is launched into)
        e = cudaGraphInstantiate(&s->graph, g, cudaGraphInstantiateFlagUseNodePriority);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return set_error(LBFS_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
        s->graph_steps = 1;
        for (int p = 0; p < kPhases; p++) s->graph_phase_recorded[p] = s->phase_recorded[p];
    }
    for (int k = 0; k < n_steps; k++) {
        if (visc_due(s, s->t)) {
            int rc = enqueue(s, true, nullptr);
            if (rc) return rc;
        } else {
            LBFS_CUDA(cudaGraphLaunch(s->graph, s->stream));
            for (int p = 0; p < kPhases; p++) s->phase_recorded[p] = s->graph_phase_recorded[p];
        }
        if (int rc = after_step(s)) return rc;
        s->t++;
    }
    return LBFS_OK;
}

namespace {
// The loop graph of lbfs_step_until: a while node whose body is one regular step (as the step graph
// captures it) followed by k_until_check.  Returns LBFS_OK with s->loop_unavailable set when the
// driver refuses the body (the caller then steps one graph at a time).
int build_loop_graph(lbfs_solver *s) {
    if (!s->d_until) {
        int rc = s->alloc(&s->d_until, 1);
        if (rc) return rc;
    }
    cudaGraph_t loop = nullptr;
    LBFS_CUDA(cudaGraphCreate(&loop, 0));
    cudaGraphConditionalHandle h;
    cudaError_t e = cudaGraphConditionalHandleCreate(&h, loop, 1, cudaGraphCondAssignDefault);
    cudaGraphNodeParams p = {};
    p.type = cudaGraphNodeTypeConditional;
    p.conditional.handle = h;
    p.conditional.type = cudaGraphCondTypeWhile;
    p.conditional.size = 1;
    cudaGraphNode_t node;
    if (e == cudaSuccess) e = cudaGraphAddNode(&node, loop, nullptr, 0, &p);
    if (e != cudaSuccess) {
        cudaGraphDestroy(loop);
        cudaGetLastError();
        s->loop_unavailable = true;
        return LBFS_OK;
    }
    cudaGraph_t body = p.conditional.phGraph_out[0];
    e = cudaStreamBeginCaptureToGraph(s->stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) {
        cudaGraphDestroy(loop);
        cudaGetLastError();
        s->loop_unavailable = true;
        return LBFS_OK;
    }
    int n = 0;
    int rc = enqueue(s, false, &n);
    if (!rc) {
        const double ref_mom = s->params.ref_rho * s->params.max_velocity;
        k_until_check<<<1, 32, 0, s->stream>>>(h, s->d_until, s->fp32 ? s->f32.residual_sums : s->f64.residual_sums,
                                               s->fp32 ? s->f32.flags : s->f64.flags, (double)s->nc, s->params.ref_rho,
                                               ref_mom);
    }
    cudaGraph_t captured = nullptr;
    e = cudaStreamEndCapture(s->stream, &captured);
    if (rc) {
        cudaGraphDestroy(loop);
        return rc;
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&s->loop_graph, loop, cudaGraphInstantiateFlagUseNodePriority);
    cudaGraphDestroy(loop);
    if (e != cudaSuccess) {
        cudaGetLastError();
        s->loop_graph = nullptr;
        s->loop_unavailable = true;
    }
    return LBFS_OK;
}
}  // namespace

extern "C" int lbfs_step_until(lbfs_solver *s, int32_t max_steps, double tolerance, int32_t *steps_done,
                               double *residuals) {
    if (!s || max_steps < 0 || !steps_done) return set_error(LBFS_ERR_ARG, "bad arguments");
    LBFS_CUDA(cudaSetDevice(s->device));
    int done = 0, stop = 0;
    double res[4] = {0.0, 0.0, 0.0, 0.0};
    while (done < max_steps && !stop) {
        // regular steps ahead (no interior-viscosity update, no object wrap): one launch of the loop graph
        const bool loop_ok = !s->profiling && !s->loop_unavailable;
        int chunk = 0;
        while (loop_ok && done + chunk < max_steps && !visc_due(s, s->t + chunk) && !wrap_due(s, s->t + chunk)) chunk++;
        if (chunk > 0 && !s->loop_graph) {
            int rc = build_loop_graph(s);
            if (rc) return rc;
        }
        if (chunk > 0 && s->loop_graph) {
            UntilState u = {0, chunk, 0, 0, tolerance, {0.0, 0.0, 0.0, 0.0}};
            LBFS_CUDA(cudaMemcpyAsync(s->d_until, &u, sizeof u, cudaMemcpyHostToDevice, s->stream));
            LBFS_CUDA(cudaGraphLaunch(s->loop_graph, s->stream));
            LBFS_CUDA(cudaMemcpyAsync(&u, s->d_until, sizeof u, cudaMemcpyDeviceToHost, s->stream));
            LBFS_CUDA(cudaStreamSynchronize(s->stream));
            s->t += u.count;
            done += u.count;
            for (int k = 0; k < 4; k++) res[k] = u.res[k];
            stop = u.stop;
            continue;
        }
        // one step through the step graph (or its interior-viscosity form) and the same tests on the host
        int rc = lbfs_step_graph(s, 1);
        if (rc) return rc;
        if ((rc = lbfs_get_residuals(s, res))) return rc;
        uint32_t flags = 0;
        if ((rc = lbfs_status(s, &flags))) return rc;
        done++;
        const double mx = std::max(std::max(res[0], res[1]), std::max(res[2], res[3]));
        stop = mx < tolerance ? 1 : ((flags & (LBFS_FLAG_NONFINITE | LBFS_FLAG_RHO_RANGE)) ? 2 : 0);
    }
    *steps_done = done;
    if (residuals)
        for (int k = 0; k < 4; k++) residuals[k] = res[k];
    return LBFS_OK;
}

extern "C" int lbfs_synchronize(lbfs_solver *s) {
    if (!s) return set_error(LBFS_ERR_ARG, "null handle");
    LBFS_CUDA(cudaSetDevice(s->device));
    LBFS_CUDA(cudaStreamSynchronize(s->stream));
    return LBFS_OK;
}

extern "C" int lbfs_get_nodes(lbfs_solver *s, int32_t which, double *out) {
    if (!s || !out) return set_error(LBFS_ERR_ARG, "null argument");
    if (s->n_membranes == 0) return LBFS_OK;
    LBFS_CUDA(cudaSetDevice(s->device));
    double *src[3];
    if (which == LBFS_NODES_POSITION) { src[0] = s->ma.x; src[1] = s->ma.y; src[2] = s->ma.z; }
    else if (which == LBFS_NODES_VELOCITY) { src[0] = s->ma.vx; src[1] = s->ma.vy; src[2] = s->ma.vz; }
    else if (which == LBFS_NODES_FORCE) { src[0] = s->ma.fx; src[1] = s->ma.fy; src[2] = s->ma.fz; }
    else return set_error(LBFS_ERR_ARG, "unknown node array");
    const int N = s->total_nodes;
    std::vector<double> h(3 * (size_t)N);
    for (int c = 0; c < 3; c++)
        LBFS_CUDA(cudaMemcpyAsync(h.data() + (size_t)c * N, src[c], N * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    LBFS_CUDA(cudaStreamSynchronize(s->stream));
    for (int n = 0; n < N; n++)
        for (int c = 0; c < 3; c++) out[3 * n + c] = h[(size_t)c * N + n];
    return LBFS_OK;
}

extern "C" int lbfs_set_nodes(lbfs_solver *s, const double *xyz) {
    if (!s || !xyz) return set_error(LBFS_ERR_ARG, "null argument");
    if (s->n_membranes == 0) return LBFS_OK;
    LBFS_CUDA(cudaSetDevice(s->device));
    const int N = s->total_nodes;
    std::vector<double> h(3 * (size_t)N);
    for (int n = 0; n < N; n++)
        for (int c = 0; c < 3; c++) h[(size_t)c * N + n] = xyz[3 * n + c];
    double *dst[3] = {s->ma.x, s->ma.y, s->ma.z};
    for (int c = 0; c < 3; c++)
        LBFS_CUDA(cudaMemcpyAsync(dst[c], h.data() + (size_t)c * N, N * sizeof(double), cudaMemcpyHostToDevice, s->stream));
    LBFS_CUDA(cudaStreamSynchronize(s->stream));
    return LBFS_OK;
}

extern "C" int lbfs_get_totals(lbfs_solver *s, double *out) {
    if (!s || !out) return set_error(LBFS_ERR_ARG, "null argument");
    if (s->n_membranes == 0) return LBFS_OK;
    LBFS_CUDA(cudaSetDevice(s->device));
    std::vector<MembraneScalars> h(s->n_membranes);
    LBFS_CUDA(cudaMemcpyAsync(h.data(), s->ma.ms, h.size() * sizeof(MembraneScalars), cudaMemcpyDeviceToHost, s->stream));
    LBFS_CUDA(cudaStreamSynchronize(s->stream));
    for (int m = 0; m < s->n_membranes; m++) {
        out[6 * m] = h[m].V; out[6 * m + 1] = h[m].V0; out[6 * m + 2] = h[m].A;
        out[6 * m + 3] = h[m].A0; out[6 * m + 4] = h[m].MAD; out[6 * m + 5] = h[m].MAD0;
    }
    return LBFS_OK;
}

extern "C" int lbfs_get_energies(lbfs_solver *s, double *out) {
    if (!s || !out) return set_error(LBFS_ERR_ARG, "null argument");
    const int M = s->n_membranes;
    if (M == 0) return LBFS_OK;
    LBFS_CUDA(cudaSetDevice(s->device));
    DevBuf sums;
    LBFS_CUDA(cudaMalloc(&sums.p, sizeof(double) * 3 * (size_t)M));
    launch_membrane_energies(s->ma, (double *)sums.p, s->stream);
    LBFS_CUDA(cudaGetLastError());
    std::vector<double> e(3 * (size_t)M);
    std::vector<MembraneScalars> h(M);
    std::vector<MembraneConst> c(M);
    LBFS_CUDA(cudaMemcpyAsync(e.data(), sums.p, e.size() * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    LBFS_CUDA(cudaMemcpyAsync(h.data(), s->ma.ms, h.size() * sizeof(MembraneScalars), cudaMemcpyDeviceToHost, s->stream));
    LBFS_CUDA(cudaMemcpyAsync(c.data(), s->ma.mc, c.size() * sizeof(MembraneConst), cudaMemcpyDeviceToHost, s->stream));
    LBFS_CUDA(cudaStreamSynchronize(s->stream));
    for (int m = 0; m < M; m++) {
        // Solver_gpu.cu:1073-1136
        const MembraneScalars &q = h[m];
        const double ade = 0.5 * c[m].global_bending_modulus * (q.MAD - q.MAD0) * (q.MAD - q.MAD0) / q.A0;
        const double vol = 0.5 * c[m].volume_modulus * (q.V - q.V0) * (q.V - q.V0) / q.V0;
        const double gar = 0.5 * c[m].global_area_modulus * (q.A - q.A0) * (q.A - q.A0) / q.A0;
        double *o = out + 7 * (size_t)m;
        o[0] = vol; o[1] = gar; o[2] = e[3 * m]; o[3] = e[3 * m + 1]; o[4] = ade; o[5] = e[3 * m + 2];
        o[6] = vol + gar + o[2] + o[3] + ade + o[5];
    }
    return LBFS_OK;
}

extern "C" int lbfs_get_residuals(lbfs_solver *s, double *out) {
    if (!s || !out) return set_error(LBFS_ERR_ARG, "null argument");
    LBFS_CUDA(cudaSetDevice(s->device));
    double h[4];
    LBFS_CUDA(cudaMemcpyAsync(h, s->fp32 ? s->f32.residual_sums : s->f64.residual_sums, sizeof(h),
                              cudaMemcpyDeviceToHost, s->stream));
    LBFS_CUDA(cudaStreamSynchronize(s->stream));
    const double ref_mom = s->params.ref_rho * s->params.max_velocity;
    for (int k = 0; k < 4; k++) out[k] = std::sqrt(h[k] / s->nc) / (k == 0 ? s->params.ref_rho : ref_mom);
    return LBFS_OK;
}

namespace {
template <typename R> int copy_real(lbfs_solver *s, const R *src, size_t n, double *out) {
    std::vector<R> h(n);
    LBFS_CUDA(cudaMemcpyAsync(h.data(), src, n * sizeof(R), cudaMemcpyDeviceToHost, s->stream));
    LBFS_CUDA(cudaStreamSynchronize(s->stream));
    for (size_t i = 0; i < n; i++) out[i] = (double)h[i];
    return LBFS_OK;
}
template <typename R> int get_field_t(lbfs_solver *s, int which, double *out) {
    FluidArgs<R> &a = fluid<R>(s);
    const size_t nt = (size_t)s->nc + s->nb;
    switch (which) {
    case LBFS_FIELD_GRADIENTS: return copy_real<R>(s, a.grad, 12 * nt, out);
    case LBFS_FIELD_FACE_FLUX: return copy_real<R>(s, (const R *)a.flux, 4 * (size_t)s->nf, out);
    case LBFS_FIELD_RESIDUAL:
        if (!s->d_res_out) return set_error(LBFS_ERR_STATE, "residuals are kept only after lbfs_keep_residuals(s, 1)");
        return copy_real<double>(s, s->d_res_out, 4 * (size_t)s->nc, out);
    case LBFS_FIELD_T1: return copy_real<double>(s, (const double *)a.t1, 4 * (size_t)s->nc, out);
    case LBFS_FIELD_VISC: return copy_real<R>(s, a.visc_factor, (size_t)s->nc, out);
    case LBFS_FIELD_DT_LOCAL: {
        // delta_t_local as the reference leaves it: the constant step
        // (fill_double), each cell's own step (local, talts), or the minimum
        // (min; Solver_gpu.cu:781-787)
        if (a.time_stepping == LBFS_DT_LOCAL || a.time_stepping == LBFS_DT_TALTS)
            return copy_real<double>(s, a.dt_local, (size_t)s->nc, out);
        double dt = s->params.delta_t;
        if (a.dt_min) LBFS_CUDA(cudaMemcpy(&dt, a.dt_min, sizeof(double), cudaMemcpyDeviceToHost));
        for (int i = 0; i < s->nc; i++) out[i] = dt;
        return LBFS_OK;
    }
    case LBFS_FIELD_GHOST: {
        std::vector<double> tmp(4 * nt);
        int rc = copy_real<R>(s, (const R *)a.state, 4 * nt, tmp.data());
        if (rc) return rc;
        for (int b = 0; b < s->nb; b++)
            for (int c = 0; c < 4; c++) out[4 * b + c] = tmp[4 * ((size_t)s->nc + b) + c] + (c == 3 ? (double)a.rho0 : 0.0);
        return LBFS_OK;
    }
    case LBFS_FIELD_FORCE: {
        // body force + IBM patches, evaluated on the host from the device patches
        const int nc = s->nc;
        for (int i = 0; i < nc; i++) { out[3 * i] = a.force[0]; out[3 * i + 1] = a.force[1]; out[3 * i + 2] = a.force[2]; }
        if (s->n_membranes == 0) return LBFS_OK;
        std::vector<MembraneScalars> ms(s->n_membranes);
        LBFS_CUDA(cudaMemcpy(ms.data(), s->ma.ms, ms.size() * sizeof(MembraneScalars), cudaMemcpyDeviceToHost));
        std::vector<double> pf((size_t)s->total_patch * 3);
        LBFS_CUDA(cudaMemcpy(pf.data(), s->ma.patch_force, pf.size() * sizeof(double), cudaMemcpyDeviceToHost));
        for (int k = 0; k < (int)s->inst.size(); k++) {
            const InstanceGrid &g = s->inst[k];
            for (int i = g.cell0; i < g.cell0 + s->grids[k].n_cells; i++) {
                const int li = i - g.cell0;
                const int ci = li % g.nx, cj = (li / g.nx) % g.ny, ck = li / (g.nx * g.ny);
                for (int m = g.mem0; m < g.mem1; m++) {
                    const int px = ci - ms[m].patch_lo[0], py = cj - ms[m].patch_lo[1], pz = ck - ms[m].patch_lo[2];
                    if (ms[m].patch_cells > 0 && px >= 0 && py >= 0 && pz >= 0 && px < ms[m].patch_dim[0] &&
                        py < ms[m].patch_dim[1] && pz < ms[m].patch_dim[2]) {
                        const double *p = pf.data() + ((size_t)ms[m].patch_off +
                                                        (px + ms[m].patch_dim[0] * (py + ms[m].patch_dim[1] * pz))) * 3;
                        out[3 * i] += p[0]; out[3 * i + 1] += p[1]; out[3 * i + 2] += p[2];
                    }
                }
            }
        }
        return LBFS_OK;
    }
    case LBFS_FIELD_SPRING: {
        const int S = s->total_springs;
        if (S == 0) return LBFS_OK;
        std::vector<double> c(S), k(S), cv(S), c0(S), a0(S), ar0(2 * (size_t)S), ar(2 * (size_t)S);
        LBFS_CUDA(cudaMemcpy(c.data(), s->ma.contour, S * sizeof(double), cudaMemcpyDeviceToHost));
        LBFS_CUDA(cudaMemcpy(k.data(), s->ma.kspring, S * sizeof(double), cudaMemcpyDeviceToHost));
        LBFS_CUDA(cudaMemcpy(cv.data(), s->ma.curv, S * sizeof(double), cudaMemcpyDeviceToHost));
        LBFS_CUDA(cudaMemcpy(c0.data(), s->ma.curv0, S * sizeof(double), cudaMemcpyDeviceToHost));
        LBFS_CUDA(cudaMemcpy(a0.data(), s->ma.angle0, S * sizeof(double), cudaMemcpyDeviceToHost));
        LBFS_CUDA(cudaMemcpy(ar0.data(), s->ma.area0, 2 * S * sizeof(double), cudaMemcpyDeviceToHost));
        LBFS_CUDA(cudaMemcpy(ar.data(), s->ma.area, 2 * S * sizeof(double), cudaMemcpyDeviceToHost));
        for (int i = 0; i < S; i++) {
            double *o = out + 9 * (size_t)i;
            o[0] = c[i]; o[1] = k[i]; o[2] = cv[i]; o[3] = c0[i]; o[4] = a0[i];
            o[5] = ar0[2 * i]; o[6] = ar0[2 * i + 1]; o[7] = ar[2 * i]; o[8] = ar[2 * i + 1];
        }
        return LBFS_OK;
    }
    default: return set_error(LBFS_ERR_ARG, "unknown field");
    }
}
}  // namespace

extern "C" int lbfs_get_field(lbfs_solver *s, int32_t which, double *out) {
    if (!s || !out) return set_error(LBFS_ERR_ARG, "null argument");
    LBFS_CUDA(cudaSetDevice(s->device));
    LBFS_CUDA(cudaStreamSynchronize(s->stream));
    return s->fp32 ? get_field_t<float>(s, which, out) : get_field_t<double>(s, which, out);
}

extern "C" int lbfs_get_time_step(lbfs_solver *s, double *delta_t) {
    if (!s || !delta_t) return set_error(LBFS_ERR_ARG, "null argument");
    const double *d = s->fp32 ? s->f32.dt_min : s->f64.dt_min;
    *delta_t = s->params.delta_t;
    if (!d) return LBFS_OK;
    LBFS_CUDA(cudaSetDevice(s->device));
    LBFS_CUDA(cudaMemcpyAsync(delta_t, d, sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    LBFS_CUDA(cudaStreamSynchronize(s->stream));
    return LBFS_OK;
}

// Slab decomposition: the state records and FP64 accumulators of a range of
// cells, copied device to device on the handle's stream (no synchronisation),
// so a caller can move halo planes between handles with NCCL or peer copies
// on that stream.  Layout of the buffer: the n_cells state records, then the
// n_cells accumulators.
namespace {
size_t state_record_bytes(const lbfs_solver *s) { return s->fp32 ? sizeof(Vec4<float>) : sizeof(Vec4<double>); }
int halo_range(const lbfs_solver *s, int32_t first_cell, int32_t n_cells, const void *buf) {
    if (!s || !buf) return set_error(LBFS_ERR_ARG, "null argument");
    if (first_cell < 0 || n_cells < 0 || (long long)first_cell + n_cells > (long long)s->nc)
        return set_error(LBFS_ERR_ARG, "halo cells outside the interior cells");
    return LBFS_OK;
}
}  // namespace

extern "C" int lbfs_halo_bytes(lbfs_solver *s, int32_t n_cells, uint64_t *bytes) {
    if (!s || !bytes || n_cells < 0) return set_error(LBFS_ERR_ARG, "bad argument");
    *bytes = (uint64_t)n_cells * (state_record_bytes(s) + sizeof(double4));
    return LBFS_OK;
}

extern "C" int lbfs_halo_pack(lbfs_solver *s, int32_t first_cell, int32_t n_cells, void *d_out) {
    int rc = halo_range(s, first_cell, n_cells, d_out);
    if (rc || n_cells == 0) return rc;
    LBFS_CUDA(cudaSetDevice(s->device));
    const size_t rb = state_record_bytes(s), n = (size_t)n_cells;
    const char *state = s->fp32 ? (const char *)s->f32.state : (const char *)s->f64.state;
    const double4 *t1 = s->fp32 ? s->f32.t1 : s->f64.t1;
    char *out = static_cast<char *>(d_out);
    LBFS_CUDA(cudaMemcpyAsync(out, state + rb * first_cell, rb * n, cudaMemcpyDeviceToDevice, s->stream));
    LBFS_CUDA(cudaMemcpyAsync(out + rb * n, t1 + first_cell, sizeof(double4) * n, cudaMemcpyDeviceToDevice, s->stream));
    return LBFS_OK;
}

extern "C" int lbfs_halo_unpack(lbfs_solver *s, int32_t first_cell, int32_t n_cells, const void *d_in) {
    int rc = halo_range(s, first_cell, n_cells, d_in);
    if (rc || n_cells == 0) return rc;
    LBFS_CUDA(cudaSetDevice(s->device));
    const size_t rb = state_record_bytes(s), n = (size_t)n_cells;
    char *state = s->fp32 ? (char *)s->f32.state : (char *)s->f64.state;
    double4 *t1 = s->fp32 ? s->f32.t1 : s->f64.t1;
    const char *in = static_cast<const char *>(d_in);
    LBFS_CUDA(cudaMemcpyAsync(state + rb * first_cell, in, rb * n, cudaMemcpyDeviceToDevice, s->stream));
    LBFS_CUDA(cudaMemcpyAsync(t1 + first_cell, in + rb * n, sizeof(double4) * n, cudaMemcpyDeviceToDevice, s->stream));
    return LBFS_OK;
}

extern "C" int lbfs_set_ibm_window(lbfs_solver *s, int32_t z_lo, int32_t z_hi) {
    if (!s) return set_error(LBFS_ERR_ARG, "null handle");
    if (z_lo < 0 || z_hi <= z_lo) return set_error(LBFS_ERR_ARG, "IBM window must satisfy 0 <= z_lo < z_hi");
    LBFS_CUDA(cudaSetDevice(s->device));
    LBFS_CUDA(cudaStreamSynchronize(s->stream));
    s->ma.ibm_z_lo = z_lo;
    s->ma.ibm_z_hi = z_hi;
    drop_step_graphs(s);
    return LBFS_OK;
}

extern "C" int lbfs_keep_residuals(lbfs_solver *s, int32_t on) {
    if (!s) return set_error(LBFS_ERR_ARG, "null handle");
    LBFS_CUDA(cudaSetDevice(s->device));
    if (on && !s->d_res_out) {
        int rc = s->alloc(&s->d_res_out, 4 * (size_t)s->nc);
        if (rc) return rc;
        LBFS_CUDA(cudaMemset(s->d_res_out, 0, 4 * sizeof(double) * (size_t)s->nc));
    }
    double *p = on ? s->d_res_out : nullptr;
    s->f64.res_out = p;
    s->f32.res_out = p;
    drop_step_graphs(s);
    return LBFS_OK;
}

extern "C" int lbfs_status(lbfs_solver *s, uint32_t *flags) {
    if (!s || !flags) return set_error(LBFS_ERR_ARG, "null argument");
    LBFS_CUDA(cudaSetDevice(s->device));
    unsigned int h = 0;
    LBFS_CUDA(cudaMemcpyAsync(&h, s->fp32 ? s->f32.flags : s->f64.flags, sizeof(h), cudaMemcpyDeviceToHost, s->stream));
    LBFS_CUDA(cudaStreamSynchronize(s->stream));
    *flags = h;
    return LBFS_OK;
}

extern "C" int lbfs_launches_per_step(lbfs_solver *s, int32_t *launches) {
    if (!s || !launches) return set_error(LBFS_ERR_ARG, "null argument");
    *launches = s->launches_per_step;
    return LBFS_OK;
}

extern "C" int lbfs_last_error(char *buf, int32_t len) {
    if (!buf || len <= 0) return LBFS_ERR_ARG;
    std::snprintf(buf, (size_t)len, "%s", g_last_error.c_str());
    return LBFS_OK;
}

// ---- launch shapes and the autotuner ---------------------------------------

namespace {

template <typename R> void shape_to_args(lbfs_solver *s, const lbfs_launch_shape &sh) {
    FluidArgs<R> &a = fluid<R>(s);
    a.tb_grad = sh.gradient_threads; a.tb_flux = sh.flux_threads; a.tb_gen = sh.general_flux_threads;
    a.tb_update = sh.update_threads; a.update_blocks = sh.update_blocks;
    s->ma.spread_blocks = sh.spread_blocks;
    s->ma.force_cluster = sh.membrane_cluster;
    s->membrane_after_k1 = sh.membrane_after_k1 != 0;
    set_chunks(s, sh.flux_chunks);
}

template <typename R> lbfs_launch_shape args_to_shape(lbfs_solver *s) {
    const FluidArgs<R> &a = fluid<R>(s);
    lbfs_launch_shape sh{};
    sh.gradient_threads = a.tb_grad; sh.flux_threads = a.tb_flux; sh.general_flux_threads = a.tb_gen;
    sh.update_threads = a.tb_update; sh.update_blocks = a.update_blocks;
    sh.spread_blocks = s->ma.spread_blocks > 0 ? s->ma.spread_blocks : 1;
    sh.flux_chunks = s->flux_chunks;
    sh.membrane_cluster = s->ma.force_cluster;
    sh.membrane_after_k1 = s->membrane_after_k1 ? 1 : 0;
    return sh;
}

bool one_of(int v, std::initializer_list<int> set) {
    for (int x : set) if (v == x) return true;
    return false;
}

int check_shape(const lbfs_launch_shape &sh) {
    if (!one_of(sh.gradient_threads, {128, 256, 512}) || !one_of(sh.flux_threads, {64, 128, 256}) ||
        !one_of(sh.general_flux_threads, {64, 128, 256}) || !one_of(sh.update_threads, {128, 256, 512}))
        return set_error(LBFS_ERR_ARG, "launch shape: block sizes must be 128/256/512 (gradients, update) or "
                                       "64/128/256 (flux kernels)");
    if (sh.update_blocks < 1 || sh.update_blocks > LBFS_MAX_UPDATE_BLOCKS || sh.spread_blocks < 1 ||
        sh.spread_blocks > LBFS_MAX_SPREAD_BLOCKS)
        return set_error(LBFS_ERR_ARG, "launch shape: grid caps out of range");
    if (!one_of(sh.flux_chunks, {0, 1, 2, 4, 8}))
        return set_error(LBFS_ERR_ARG, "launch shape: flux_chunks must be 1, 2, 4 or 8");
    if (!one_of(sh.membrane_cluster, {0, 8, 16}))
        return set_error(LBFS_ERR_ARG, "launch shape: membrane_cluster must be 0, 8 or 16");
    if (!one_of(sh.membrane_after_k1, {0, 1}))
        return set_error(LBFS_ERR_ARG, "launch shape: membrane_after_k1 must be 0 or 1");
    return LBFS_OK;
}

void drop_graph(lbfs_solver *s) {
    drop_step_graphs(s);
}

int autotune_steps(lbfs_solver *s, int reps, lbfs_launch_shape *out, bool fp32);

}  // namespace

extern "C" int lbfs_get_launch_shape(lbfs_solver *s, lbfs_launch_shape *shape) {
    if (!s || !shape) return set_error(LBFS_ERR_ARG, "null argument");
    *shape = s->fp32 ? args_to_shape<float>(s) : args_to_shape<double>(s);
    return LBFS_OK;
}

extern "C" int lbfs_set_launch_shape(lbfs_solver *s, const lbfs_launch_shape *shape) {
    if (!s || !shape) return set_error(LBFS_ERR_ARG, "null argument");
    int rc = check_shape(*shape);
    if (rc) return rc;
    if (shape->membrane_cluster != 0 && s->n_membranes > 0 && !membrane_cluster_fits(s->ma.max_nodes))
        return set_error(LBFS_ERR_ARG, "launch shape: membrane_cluster 8 or 16 holds membranes of at most 8192 "
                                       "nodes in shared memory");
    if (s->fp32) shape_to_args<float>(s, *shape);
    else shape_to_args<double>(s, *shape);
    drop_graph(s);
    return LBFS_OK;
}

extern "C" int lbfs_autotune(lbfs_solver *s, int32_t reps, lbfs_launch_shape *shape) {
    if (!s) return set_error(LBFS_ERR_ARG, "null handle");
    if (reps < 1 || reps > 1000) return set_error(LBFS_ERR_ARG, "reps must be in 1..1000");
    LBFS_CUDA(cudaSetDevice(s->device));
    return autotune_steps(s, reps, shape, s->fp32);
}


// ---- discrete adjoint -------------------------------------------------------

namespace {

int adj_prepare(lbfs_solver *s) {
    if (s->adj_ready) return LBFS_OK;
    AdjointArgs &j = s->adj;
    const int nc = s->nc, nf = s->nf, nb = s->nb;
    int rc;
    j.nf = nf;
    if ((rc = s->alloc(&j.lam_t1, nc)) || (rc = s->alloc(&j.lam_face, 32 * (size_t)nf)) ||
        (rc = s->alloc(&j.lam_bcv, 4 * (size_t)(nb > 0 ? nb : 1))) || (rc = s->alloc(&j.lam_rs, 12 * (size_t)nc)) ||
        (rc = s->alloc(&j.lam_state, 4 * (size_t)nc)) || (rc = s->alloc(&j.sigma_acc, nc)))
        return rc;
    LBFS_CUDA(cudaMemset(j.lam_bcv, 0, sizeof(double) * 4 * (size_t)(nb > 0 ? nb : 1)));
    // transposed gradient stencil: for each interior cell, the (cell, slot) pairs that read it
    std::vector<int2> st(3 * (size_t)nc);
    LBFS_CUDA(cudaMemcpy(st.data(), s->f64.stencil, sizeof(int2) * st.size(), cudaMemcpyDeviceToHost));
    std::vector<int> start(nc + 1, 0);
    auto entry = [&](int i, int q) { return q & 1 ? st[3 * (size_t)i + q / 2].y : st[3 * (size_t)i + q / 2].x; };
    for (int i = 0; i < nc; i++)
        for (int q = 0; q < 6; q++) {
            const int c = entry(i, q);
            if (c < nc) start[c + 1]++;
        }
    for (int c = 0; c < nc; c++) start[c + 1] += start[c];
    std::vector<int> fill(start.begin(), start.end() - 1), tst(start[nc] > 0 ? start[nc] : 1);
    for (int i = 0; i < nc; i++)
        for (int q = 0; q < 6; q++) {
            const int c = entry(i, q);
            if (c < nc) tst[fill[c]++] = 8 * i + q;
        }
    int *d_start, *d_tst;
    if ((rc = s->upload(&d_start, start)) || (rc = s->upload(&d_tst, tst))) return rc;
    j.tst_start = d_start;
    j.tst = d_tst;
    j.dt = s->params.delta_t;
    j.lam_u_ibm = nullptr;
    s->adj_ready = true;
    return LBFS_OK;
}


int run_one_step(lbfs_solver *s) {
    if (visc_due(s, s->t)) {
        int rc = enqueue(s, true, nullptr);
        if (rc || (rc = after_step(s))) return rc;
    } else {
        int rc = lbfs_step_graph(s, 1);
        if (rc) return rc;
        s->t--;  // lbfs_step_graph advanced it
    }
    s->t++;
    return LBFS_OK;
}

// Membrane adjoint buffers: the adjoints, the node -> triangle incidence, and
// a second set of sort / spread buffers (the interpolation transpose).
int adjm_prepare(lbfs_solver *s) {
    if (s->madj_ready) return LBFS_OK;
    MemAdjArgs &J = s->madj;
    const MembraneArgs &ma = s->ma;
    const int N = s->total_nodes, S = s->total_springs, M = s->n_membranes, T = s->total_tris;
    int rc;
    if ((rc = s->alloc(&J.lam_x, 3 * (size_t)N)) || (rc = s->alloc(&J.lam_xp, 3 * (size_t)N)) ||
        (rc = s->alloc(&J.lam_F, 3 * (size_t)N)) || (rc = s->alloc(&J.adjm, 17 * (size_t)S)) ||
        (rc = s->alloc(&J.lam_mad, M)) || (rc = s->alloc(&J.red, 5 * (size_t)M)) || (rc = s->alloc(&J.gs_acc, M)) ||
        (rc = s->alloc(&J.kb_acc, M)) || (rc = s->alloc(&J.lam_u_ibm, 3 * (size_t)s->nc)))
        return rc;
    std::vector<int> tri(3 * (size_t)T);
    LBFS_CUDA(cudaMemcpy(tri.data(), ma.tri, sizeof(int) * tri.size(), cudaMemcpyDeviceToHost));
    std::vector<int> start(N + 1, 0);
    for (int q = 0; q < 3 * T; q++) start[tri[q] + 1]++;
    for (int n = 0; n < N; n++) start[n + 1] += start[n];
    std::vector<int> fill(start.begin(), start.end() - 1), inc(3 * (size_t)T);
    for (int t = 0; t < T; t++)
        for (int v = 0; v < 3; v++) inc[fill[tri[3 * t + v]]++] = 4 * t + v;
    int *d_start, *d_inc;
    if ((rc = s->upload(&d_start, start)) || (rc = s->upload(&d_inc, inc))) return rc;
    J.tri_start = d_start;
    J.tri_inc = d_inc;
    // second sort / spread set
    MembraneArgs mb = ma;
    std::vector<int> identity(N);
    for (int n = 0; n < N; n++) identity[n] = n;
    MembraneScalars *ms2;
    if ((rc = s->alloc(&ms2, M)) ||
        (rc = s->alloc(&mb.bin_start, (size_t)s->total_patch + M)) || (rc = s->alloc(&mb.cell_start, (size_t)M + 1)) ||
        (rc = s->alloc(&mb.bin_cursor, (size_t)s->total_patch + M)) ||
        (rc = s->alloc(&mb.sort_ticket, 1)) || (rc = s->upload(&mb.sorted_node, identity)) ||
        (rc = s->alloc(&mb.fx, N)) || (rc = s->alloc(&mb.fy, N)) || (rc = s->alloc(&mb.fz, N)) ||
        (rc = s->alloc(&mb.patch_force, 3 * (size_t)s->total_patch)) ||
        (rc = s->alloc(&mb.node_base, 3 * (size_t)N)) || (rc = s->alloc(&mb.node_w, 12 * (size_t)N)))
        return rc;
    LBFS_CUDA(cudaMemcpy(ms2, ma.ms, sizeof(MembraneScalars) * M, cudaMemcpyDeviceToDevice));
    LBFS_CUDA(cudaMemset(mb.sort_ticket, 0, sizeof(unsigned int)));
    LBFS_CUDA(cudaMemset(mb.cell_start, 0, sizeof(int) * (M + 1)));
    // the interpolation transpose's "forces" (dt lambda_x'), which its spread reads in node order
    LBFS_CUDA(cudaMemset(mb.fx, 0, sizeof(double) * N));
    LBFS_CUDA(cudaMemset(mb.fy, 0, sizeof(double) * N));
    LBFS_CUDA(cudaMemset(mb.fz, 0, sizeof(double) * N));
    mb.ms = ms2;
    J.mb = mb;
    J.dt = s->params.delta_t;
    s->madj_ready = true;
    return LBFS_OK;
}

// Taylor deformation (L - B) / (L + B) of one membrane in the x-y plane, L and
// B the square roots of the eigenvalues of its nodes' 2-D second-moment
// tensor about their centroid; and dD / d(node positions).
double taylor_deformation(const double *x, const double *y, int n, double *gx, double *gy) {
    double cx = 0, cy = 0;
    for (int i = 0; i < n; i++) { cx += x[i]; cy += y[i]; }
    cx /= n;
    cy /= n;
    double Ixx = 0, Iyy = 0, Ixy = 0;
    for (int i = 0; i < n; i++) {
        const double dx = x[i] - cx, dy = y[i] - cy;
        Ixx += dx * dx; Iyy += dy * dy; Ixy += dx * dy;
    }
    const double T = 0.5 * (Ixx + Iyy), D = 0.5 * (Ixx - Iyy), R = std::sqrt(D * D + Ixy * Ixy);
    const double lp = T + R, lm = T - R;
    const double L = std::sqrt(lp), B = std::sqrt(lm);
    const double J = (L - B) / (L + B);
    const double dJdL = 2 * B / ((L + B) * (L + B)), dJdB = -2 * L / ((L + B) * (L + B));
    const double dJdlp = dJdL / (2 * L), dJdlm = dJdB / (2 * B);
    // d lambda+- / d(Ixx, Iyy, Ixy)
    const double dxx = dJdlp * (0.5 + 0.5 * D / R) + dJdlm * (0.5 - 0.5 * D / R);
    const double dyy = dJdlp * (0.5 - 0.5 * D / R) + dJdlm * (0.5 + 0.5 * D / R);
    const double dxy = dJdlp * (Ixy / R) - dJdlm * (Ixy / R);
    for (int i = 0; i < n; i++) {
        const double dx = x[i] - cx, dy = y[i] - cy;
        gx[i] = dxx * 2 * dx + dxy * dy;
        gy[i] = dyy * 2 * dy + dxy * dx;
    }
    return J;
}

}  // namespace

extern "C" int lbfs_adjoint(lbfs_solver *s, int32_t n_steps, int32_t checkpoint_every, const lbfs_objective *obj,
                            double *J, double *grad, double *times_ms) {
    if (!s || !obj || !J || !grad || n_steps < 1 || checkpoint_every < 1)
        return set_error(LBFS_ERR_ARG, "lbfs_adjoint: bad arguments");
    if (s->fp32) return set_error(LBFS_ERR_UNSUPPORTED, "lbfs_adjoint: FP64 handles only");
    if (s->params.gamma_inv != 1.0 || s->params.preconditioning)
        return set_error(LBFS_ERR_UNSUPPORTED, "lbfs_adjoint: no preconditioning");
    if (dynamic_dt(s->params))
        return set_error(LBFS_ERR_UNSUPPORTED, "lbfs_adjoint: constant time stepping only");
    if (s->periodic) return set_error(LBFS_ERR_UNSUPPORTED, "lbfs_adjoint: no periodic boundaries");
    if (s->params.ibm_stencil == LBFS_IBM_VANDERMONDE4 && s->n_membranes > 0)
        return set_error(LBFS_ERR_UNSUPPORTED, "lbfs_adjoint: LBFS_IBM_HAT2 or LBFS_IBM_PESKIN4 only");
    if (obj->kind == LBFS_OBJ_VELOCITY) {
        if (!obj->cell_weights) return set_error(LBFS_ERR_ARG, "lbfs_adjoint: velocity objective needs weights");
    } else if (obj->kind == LBFS_OBJ_TAYLOR) {
        if (obj->membrane < 0 || obj->membrane >= s->n_membranes)
            return set_error(LBFS_ERR_ARG, "lbfs_adjoint: objective membrane out of range");
    } else {
        return set_error(LBFS_ERR_ARG, "lbfs_adjoint: unknown objective");
    }
    LBFS_CUDA(cudaSetDevice(s->device));
    const int M = s->n_membranes, N = s->total_nodes;
    std::vector<MembraneConst> mch(M);
    if (M > 0) {
        LBFS_CUDA(cudaMemcpy(mch.data(), s->ma.mc, sizeof(MembraneConst) * M, cudaMemcpyDeviceToHost));
        bool visc_in_window = false, wrap_in_window = false;
        for (long long t = s->t; t < s->t + n_steps; t++) {
            visc_in_window = visc_in_window || visc_due(s, t);
            wrap_in_window = wrap_in_window || wrap_due(s, t);
        }
        if (wrap_in_window)
            return set_error(LBFS_ERR_UNSUPPORTED, "lbfs_adjoint: a periodic membrane's z wrap falls in the window");
        for (const MembraneConst &c : mch) {
            if (c.viscosity != 0.0) return set_error(LBFS_ERR_UNSUPPORTED, "lbfs_adjoint: membrane viscosity must be 0");
            if (!(c.shear_modulus > 0.0)) return set_error(LBFS_ERR_UNSUPPORTED, "lbfs_adjoint: shear modulus must be > 0");
            if (visc_in_window && c.internal_viscosity_ratio != 1.0)
                return set_error(LBFS_ERR_UNSUPPORTED, "lbfs_adjoint: an interior-viscosity update falls in the window "
                                                       "(its position dependence is not differentiated) unless the "
                                                       "interior viscosity ratio is 1");
        }
    }
    int rc = adj_prepare(s);
    if (rc) return rc;
    if (M > 0 && (rc = adjm_prepare(s))) return rc;
    FluidArgs<double> &a = s->f64;
    MembraneArgs &ma = s->ma;
    AdjointArgs &j = s->adj;
    MemAdjArgs &mj = s->madj;
    const int nc = s->nc, nt = s->nc + s->nb;
    const int K = checkpoint_every, n_ck = (n_steps + K - 1) / K;
    const size_t xs = 3 * (size_t)N;  // positions of one step: x, y, z planes
    cudaStream_t st = s->stream;
    DevBuf ck, st0, fin_t1, fin_state, wts, ckx, ckm, finx, finm, bst;
    // segment storage: per step t1, the gradients and ghost states of its K1,
    // x', node forces, membrane scalars and MAD.  Two sets, the re-run of one
    // segment filling one while the backward sweep of the next later segment
    // reads the other; or, when every segment's set fits in half the free
    // device memory (at most LBFS_ADJOINT_MEMORY_MB if that is set), one set per
    // segment, filled by the forward sweep itself, and the reverse sweep
    // re-runs nothing (the same kernels on the same inputs: the same results).
    struct SegStore {
        DevBuf t1, g, h, x, f, s, m;
    };
    const size_t gsz = 12 * (size_t)nt;
    const size_t nbx = s->nb > 0 ? s->nb : 1;
    const size_t set_bytes = (sizeof(double4) * (size_t)nc + sizeof(double) * gsz + sizeof(Vec4<double>) * nbx) * K +
                             (M > 0 ? sizeof(double) * xs * (2 * (size_t)K + 1) +
                                          (sizeof(MembraneScalars) + sizeof(double)) * (size_t)M * K
                                    : 0);
    bool store_all = false;
    if (n_ck > 1) {
        size_t free_b = 0, total_b = 0;
        LBFS_CUDA(cudaMemGetInfo(&free_b, &total_b));
        size_t budget = free_b / 2;
        if (const char *mb = std::getenv("LBFS_ADJOINT_MEMORY_MB")) {
            const long long v = std::atoll(mb);
            budget = std::min(budget, v > 0 ? (size_t)v << 20 : (size_t)0);
        }
        store_all = set_bytes * (size_t)n_ck <= budget;
    }
    const int n_sets = store_all ? n_ck : (n_ck > 1 ? 2 : 1);
    std::vector<SegStore> segbuf(n_sets);
    LBFS_CUDA(cudaMalloc(&ck.p, sizeof(double4) * (size_t)nc * n_ck));
    for (int b = 0; b < n_sets; b++) {
        SegStore &q = segbuf[b];
        LBFS_CUDA(cudaMalloc(&q.t1.p, sizeof(double4) * (size_t)nc * K));
        LBFS_CUDA(cudaMalloc(&q.g.p, sizeof(double) * gsz * K));
        LBFS_CUDA(cudaMalloc(&q.h.p, sizeof(Vec4<double>) * nbx * K));
        if (M > 0) {
            LBFS_CUDA(cudaMalloc(&q.x.p, sizeof(double) * xs * (K + 1)));
            LBFS_CUDA(cudaMalloc(&q.f.p, sizeof(double) * xs * K));
            LBFS_CUDA(cudaMalloc(&q.s.p, sizeof(MembraneScalars) * M * K));
            LBFS_CUDA(cudaMalloc(&q.m.p, sizeof(double) * M * K));
        }
    }
    LBFS_CUDA(cudaMalloc(&st0.p, sizeof(Vec4<double>) * (size_t)nt));
    LBFS_CUDA(cudaMalloc(&bst.p, sizeof(Vec4<double>) * (size_t)nt));
    LBFS_CUDA(cudaMalloc(&fin_t1.p, sizeof(double4) * (size_t)nc));
    LBFS_CUDA(cudaMalloc(&fin_state.p, sizeof(Vec4<double>) * (size_t)nt));
    if (obj->kind == LBFS_OBJ_VELOCITY) {
        LBFS_CUDA(cudaMalloc(&wts.p, sizeof(double) * 3 * (size_t)nc));
        LBFS_CUDA(cudaMemcpyAsync(wts.p, obj->cell_weights, sizeof(double) * 3 * (size_t)nc, cudaMemcpyHostToDevice, st));
    }
    if (M > 0) {
        LBFS_CUDA(cudaMalloc(&ckx.p, sizeof(double) * xs * n_ck));
        LBFS_CUDA(cudaMalloc(&ckm.p, sizeof(double) * M * n_ck));
        LBFS_CUDA(cudaMalloc(&finx.p, sizeof(double) * xs));
        LBFS_CUDA(cudaMalloc(&finm.p, sizeof(double) * M));
    }
    double4 *ck_t1 = (double4 *)ck.p;
    double *ck_x = (double *)ckx.p, *ck_m = (double *)ckm.p;
    Vec4<double> *bstate = (Vec4<double> *)bst.p;
    auto save_x = [&](double *dst) -> int {
        LBFS_CUDA(cudaMemcpyAsync(dst, ma.x, sizeof(double) * N, cudaMemcpyDeviceToDevice, st));
        LBFS_CUDA(cudaMemcpyAsync(dst + N, ma.y, sizeof(double) * N, cudaMemcpyDeviceToDevice, st));
        LBFS_CUDA(cudaMemcpyAsync(dst + 2 * (size_t)N, ma.z, sizeof(double) * N, cudaMemcpyDeviceToDevice, st));
        return LBFS_OK;
    };
    auto load_x = [&](const double *src) -> int {
        LBFS_CUDA(cudaMemcpyAsync(ma.x, src, sizeof(double) * N, cudaMemcpyDeviceToDevice, st));
        LBFS_CUDA(cudaMemcpyAsync(ma.y, src + N, sizeof(double) * N, cudaMemcpyDeviceToDevice, st));
        LBFS_CUDA(cudaMemcpyAsync(ma.z, src + 2 * (size_t)N, sizeof(double) * N, cudaMemcpyDeviceToDevice, st));
        return LBFS_OK;
    };
    // streams of the reverse sweep: fluid backward (sf), general faces (sg_),
    // membrane backward (sm); the re-runs stay on the handle's stream
    struct Streams {
        cudaStream_t f = nullptr, g = nullptr, m = nullptr;
        cudaEvent_t ev[8] = {};
        ~Streams() {
            for (cudaEvent_t e : ev)
                if (e) cudaEventDestroy(e);
            for (cudaStream_t x : {f, g, m})
                if (x) cudaStreamDestroy(x);
        }
    } rs;
    {
        int prio_lo = 0, prio_hi = 0;
        cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi);
        LBFS_CUDA(cudaStreamCreateWithPriority(&rs.f, cudaStreamNonBlocking, prio_hi));
        LBFS_CUDA(cudaStreamCreateWithPriority(&rs.g, cudaStreamNonBlocking, prio_hi));
        LBFS_CUDA(cudaStreamCreateWithPriority(&rs.m, cudaStreamNonBlocking, prio_hi));
        for (cudaEvent_t &e : rs.ev) LBFS_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    cudaEvent_t &ev_setup = rs.ev[0], &ev_gen = rs.ev[1], &ev_mem = rs.ev[2], &ev_start = rs.ev[3];
    cudaEvent_t *ev_rerun = rs.ev + 4, *ev_back = rs.ev + 6;  // per segment set
    const long long t_start = s->t;
    cudaEvent_t e0, e1, e2;
    cudaEventCreate(&e0); cudaEventCreate(&e1); cudaEventCreate(&e2);
    // run segment sg from the handle's state into segment set b, keeping each
    // step's inputs (t1, x, MAD) and what its backward reads (gradients, ghost
    // states, x', node forces, membrane scalars); on the handle's stream
    auto record = [&](int sg, int b) -> int {
        SegStore &q = segbuf[b];
        double4 *seg_t1 = (double4 *)q.t1.p;
        double *seg_g = (double *)q.g.p, *seg_x = (double *)q.x.p, *seg_f = (double *)q.f.p, *seg_m = (double *)q.m.p;
        Vec4<double> *seg_h = (Vec4<double> *)q.h.p;
        MembraneScalars *seg_s = (MembraneScalars *)q.s.p;
        const int n0 = sg * K, n1 = std::min(n_steps, n0 + K);
        int rc;
        // the stores of a step in one launch each (a dozen separate copies per
        // step cost more than the copies themselves): before the first step
        // t1, x and MAD; after step i its gradients, ghost states, x', node
        // forces and scalars, and t1 and MAD of step i + 1
        static_assert(sizeof(MembraneScalars) % sizeof(double) == 0, "MembraneScalars copied as doubles");
        const int mad_stride = (int)(sizeof(MembraneScalars) / sizeof(double));
        const double *mad_src = &ma.ms[0].MAD;
        const int count = n1 - n0;
        {
            CopyList pre = {};
            pre.add(a.t1, seg_t1, 4 * (long long)nc);
            if (M > 0) {
                pre.add(ma.x, seg_x, N);
                pre.add(ma.y, seg_x + N, N);
                pre.add(ma.z, seg_x + 2 * (size_t)N, N);
                pre.add(mad_src, seg_m, M, mad_stride);
            }
            launch_copy_list(pre, st);
        }
        for (int n = n0; n < n1; n++) {
            const size_t i = n - n0;
            s->t = t_start + n;
            if ((rc = run_one_step(s))) return rc;
            CopyList post = {};
            post.add(a.grad, seg_g + i * gsz, (long long)gsz);
            post.add(a.state + nc, seg_h + i * s->nb, 4 * (long long)s->nb);
            if ((int)i + 1 < count) post.add(a.t1, seg_t1 + (i + 1) * nc, 4 * (long long)nc);
            if (M > 0) {
                double *xn1 = seg_x + (i + 1) * xs, *fi = seg_f + i * xs;
                post.add(ma.x, xn1, N);
                post.add(ma.y, xn1 + N, N);
                post.add(ma.z, xn1 + 2 * (size_t)N, N);
                post.add(ma.fx, fi, N);
                post.add(ma.fy, fi + N, N);
                post.add(ma.fz, fi + 2 * (size_t)N, N);
                post.add(ma.ms, seg_s + i * M, (long long)(sizeof(MembraneScalars) / sizeof(double)) * M);
                if ((int)i + 1 < count) post.add(mad_src, seg_m + (i + 1) * M, M, mad_stride);
            }
            launch_copy_list(post, st);
            LBFS_CUDA(cudaGetLastError());
        }
        return LBFS_OK;
    };
    // the same from segment sg's checkpoint (the two-set form of the reverse sweep)
    auto rerun = [&](int sg, int b) -> int {
        const int n0 = sg * K;
        int rc;
        LBFS_CUDA(cudaMemcpyAsync(a.t1, ck_t1 + (size_t)sg * nc, sizeof(double4) * nc, cudaMemcpyDeviceToDevice, st));
        if (n0 == 0) LBFS_CUDA(cudaMemcpyAsync(a.state, st0.p, sizeof(Vec4<double>) * nt, cudaMemcpyDeviceToDevice, st));
        else launch_adj_prim(a, st);
        if (M > 0) {
            if ((rc = load_x(ck_x + (size_t)sg * xs))) return rc;
            launch_adjm_set_mad(ma, ck_m + (size_t)sg * M, st);
        }
        return record(sg, b);
    };
    // ---- forward sweep with checkpoints
    LBFS_CUDA(cudaMemcpyAsync(st0.p, a.state, sizeof(Vec4<double>) * nt, cudaMemcpyDeviceToDevice, st));
    LBFS_CUDA(cudaMemsetAsync(a.flags, 0, sizeof(unsigned int), st));
    cudaEventRecord(e0, st);
    if (store_all) {
        for (int sg = 0; sg < n_ck; sg++)
            if ((rc = record(sg, sg))) return rc;
    } else {
        for (int n = 0; n < n_steps; n++) {
            if (n % K == 0) {
                LBFS_CUDA(cudaMemcpyAsync(ck_t1 + (size_t)(n / K) * nc, a.t1, sizeof(double4) * nc, cudaMemcpyDeviceToDevice, st));
                if (M > 0) {
                    if ((rc = save_x(ck_x + (size_t)(n / K) * xs))) return rc;
                    launch_adjm_get_mad(ma, ck_m + (size_t)(n / K) * M, st);
                }
            }
            if ((rc = run_one_step(s))) return rc;
        }
    }
    cudaEventRecord(e1, st);
    LBFS_CUDA(cudaMemcpyAsync(fin_t1.p, a.t1, sizeof(double4) * nc, cudaMemcpyDeviceToDevice, st));
    LBFS_CUDA(cudaMemcpyAsync(fin_state.p, a.state, sizeof(Vec4<double>) * nt, cudaMemcpyDeviceToDevice, st));
    if (M > 0) {
        if ((rc = save_x((double *)finx.p))) return rc;
        launch_adjm_get_mad(ma, (double *)finm.p, st);
    }
    unsigned int flags = 0;
    LBFS_CUDA(cudaMemcpyAsync(&flags, a.flags, sizeof(unsigned int), cudaMemcpyDeviceToHost, st));
    LBFS_CUDA(cudaStreamSynchronize(st));
    if (flags) return set_error(LBFS_ERR_STATE, "lbfs_adjoint: the forward run raised status flags " + std::to_string(flags));
    // ---- objective and its seed
    LBFS_CUDA(cudaMemsetAsync(j.lam_t1, 0, sizeof(double4) * nc, st));
    LBFS_CUDA(cudaMemsetAsync(j.sigma_acc, 0, sizeof(double) * nc, st));
    if (M > 0) {
        LBFS_CUDA(cudaMemsetAsync(mj.lam_x, 0, sizeof(double) * xs, st));
        LBFS_CUDA(cudaMemsetAsync(mj.lam_mad, 0, sizeof(double) * M, st));
        LBFS_CUDA(cudaMemsetAsync(mj.gs_acc, 0, sizeof(double) * M, st));
        LBFS_CUDA(cudaMemsetAsync(mj.kb_acc, 0, sizeof(double) * M, st));
    }
    if (obj->kind == LBFS_OBJ_VELOCITY) {
        std::vector<double4> t1h(nc);
        LBFS_CUDA(cudaMemcpyAsync(t1h.data(), a.t1, sizeof(double4) * nc, cudaMemcpyDeviceToHost, st));
        LBFS_CUDA(cudaStreamSynchronize(st));
        double acc = 0.0;
        for (int c = 0; c < nc; c++) {
            const double *w = obj->cell_weights + 3 * (size_t)c;
            acc += w[0] * (t1h[c].x / t1h[c].w) + w[1] * (t1h[c].y / t1h[c].w) + w[2] * (t1h[c].z / t1h[c].w);
        }
        *J = acc;
        launch_adj_velocity_seed(a, j, (const double *)wts.p, st);
    } else {
        const MembraneConst &c = mch[obj->membrane];
        std::vector<double> xh(xs), g(xs, 0.0);
        LBFS_CUDA(cudaMemcpyAsync(xh.data(), finx.p, sizeof(double) * xs, cudaMemcpyDeviceToHost, st));
        LBFS_CUDA(cudaStreamSynchronize(st));
        *J = taylor_deformation(xh.data() + c.node0, xh.data() + N + c.node0, c.n_nodes, g.data() + 0,
                                g.data() + c.n_nodes);
        // lam_x is node-major (x, y, z per node)
        std::vector<double> lam(xs, 0.0);
        for (int i = 0; i < c.n_nodes; i++) {
            lam[3 * (size_t)(c.node0 + i)] = g[i];
            lam[3 * (size_t)(c.node0 + i) + 1] = g[c.n_nodes + i];
        }
        LBFS_CUDA(cudaMemcpyAsync(mj.lam_x, lam.data(), sizeof(double) * xs, cudaMemcpyHostToDevice, st));
        LBFS_CUDA(cudaStreamSynchronize(st));
    }
    // ---- reverse sweep
    j.lam_u_ibm = M > 0 ? mj.lam_u_ibm : nullptr;
    mj.lam_t1 = j.lam_t1;
    // backward sweep of segment sg from segment set b.  The kernels read the
    // stored intermediates in place (their own FluidArgs / MembraneArgs), so
    // nothing of the handle's live buffers is touched and the next re-run
    // overlaps it.  Per step: setup (state of step n) on sf; the membrane
    // backward on sm and the general faces on sg_, beside the axis faces and
    // A2 on sf; A3 (which updates lam_t1) after all of them.
    auto backward = [&](int sg, int b, cudaEvent_t ready) -> int {
        SegStore &q = segbuf[b];
        double4 *seg_t1 = (double4 *)q.t1.p;
        double *seg_g = (double *)q.g.p, *seg_x = (double *)q.x.p, *seg_f = (double *)q.f.p, *seg_m = (double *)q.m.p;
        Vec4<double> *seg_h = (Vec4<double> *)q.h.p;
        MembraneScalars *seg_s = (MembraneScalars *)q.s.p;
        const int n0 = sg * K, n1 = std::min(n_steps, n0 + K);
        if (M > 0) LBFS_CUDA(cudaStreamWaitEvent(rs.m, ready, 0));
        for (int n = n1 - 1; n >= n0; n--) {
            const size_t i = n - n0;
            FluidArgs<double> ab = a;
            ab.t1 = seg_t1 + i * nc;
            ab.grad = seg_g + i * gsz;
            ab.state = bstate;
            // the state of step n: primitive interior from t1 (the user's state at n = 0) and its ghosts
            if (n == 0) LBFS_CUDA(cudaMemcpyAsync(bstate, st0.p, sizeof(Vec4<double>) * nc, cudaMemcpyDeviceToDevice, rs.f));
            else launch_adj_prim(ab, rs.f);
            if (s->nb > 0)
                LBFS_CUDA(cudaMemcpyAsync(bstate + nc, seg_h + i * s->nb, sizeof(Vec4<double>) * s->nb,
                                          cudaMemcpyDeviceToDevice, rs.f));
            LBFS_CUDA(cudaEventRecord(ev_setup, rs.f));
            if (M > 0) {
                // after the step's membrane chain: x', forces, totals, MAD_{n+1}; x_n and MAD_n before it
                MembraneArgs mbk = ma;
                double *xp = seg_x + (i + 1) * xs, *fp = seg_f + i * xs;
                mbk.x = xp; mbk.y = xp + N; mbk.z = xp + 2 * (size_t)N;
                mbk.fx = fp; mbk.fy = fp + N; mbk.fz = fp + 2 * (size_t)N;
                mbk.ms = seg_s + i * M;
                mbk.state = bstate;
                const double *xn = seg_x + i * xs;
                mj.mad_n = seg_m + i * M;
                mj.xn = xn;
                mj.yn = xn + N;
                mj.zn = xn + 2 * (size_t)N;
                // the interpolation transpose sorts the nodes at x_n (read
                // only), ahead of the step's adjoints
                mj.mb.x = const_cast<double *>(mj.xn);
                mj.mb.y = const_cast<double *>(mj.yn);
                mj.mb.z = const_cast<double *>(mj.zn);
                launch_adj_membrane_sort(mj, rs.m);
                LBFS_CUDA(cudaStreamWaitEvent(rs.m, ev_setup, 0));
                launch_adj_membrane(mbk, mj, nc, a.cell_instance, (const InstanceGrid *)a.instances, rs.m);
                LBFS_CUDA(cudaEventRecord(ev_mem, rs.m));
            }
            LBFS_CUDA(cudaStreamWaitEvent(rs.g, ev_setup, 0));
            launch_adj_flux_general(ab, j, rs.g);
            LBFS_CUDA(cudaEventRecord(ev_gen, rs.g));
            launch_adj_flux_axis(ab, j, rs.f);
            LBFS_CUDA(cudaStreamWaitEvent(rs.f, ev_gen, 0));
            // A2 and A3 behind A1 and A2 as programmatic dependent launches (their other
            // dependency, the boundary faces / the membrane backward, is one kernel each)
            launch_adj_cells(ab, j, rs.f, a.axis_aligned && a.ni > 0);
            if (M > 0) LBFS_CUDA(cudaStreamWaitEvent(rs.f, ev_mem, 0));
            launch_adj_gather(ab, j, rs.f, true);
            LBFS_CUDA(cudaGetLastError());
        }
        return LBFS_OK;
    };
    LBFS_CUDA(cudaEventRecord(ev_start, st));
    LBFS_CUDA(cudaStreamWaitEvent(rs.f, ev_start, 0));
    if (store_all) {  // every segment recorded by the forward sweep
        LBFS_CUDA(cudaEventRecord(ev_rerun[0], st));
        for (int sg = n_ck - 1; sg >= 0; sg--)
            if ((rc = backward(sg, sg, ev_rerun[0]))) return rc;
        LBFS_CUDA(cudaEventRecord(ev_back[0], rs.f));
    } else {
    if ((rc = rerun(n_ck - 1, (n_ck - 1) % n_sets))) return rc;
    LBFS_CUDA(cudaEventRecord(ev_rerun[(n_ck - 1) % n_sets], st));
    for (int sg = n_ck - 1; sg >= 0; sg--) {
        if (sg > 0) {
            const int b = (sg - 1) % n_sets;
            // set b was last read by the backward sweep of segment sg + 1
            if (sg + 1 < n_ck) LBFS_CUDA(cudaStreamWaitEvent(st, ev_back[b], 0));
            if ((rc = rerun(sg - 1, b))) return rc;
            LBFS_CUDA(cudaEventRecord(ev_rerun[b], st));
        }
        const int b = sg % n_sets;
        LBFS_CUDA(cudaStreamWaitEvent(rs.f, ev_rerun[b], 0));
        if ((rc = backward(sg, b, ev_rerun[b]))) return rc;
        LBFS_CUDA(cudaEventRecord(ev_back[b], rs.f));
    }
    }
    LBFS_CUDA(cudaStreamWaitEvent(st, ev_back[0], 0));
    cudaEventRecord(e2, st);
    // ---- final forward state back, sensitivities
    LBFS_CUDA(cudaMemcpyAsync(a.t1, fin_t1.p, sizeof(double4) * nc, cudaMemcpyDeviceToDevice, st));
    LBFS_CUDA(cudaMemcpyAsync(a.state, fin_state.p, sizeof(Vec4<double>) * nt, cudaMemcpyDeviceToDevice, st));
    if (M > 0) {
        if ((rc = load_x((const double *)finx.p))) return rc;
        launch_adjm_set_mad(ma, (const double *)finm.p, st);
    }
    s->t = t_start + n_steps;
    std::vector<double> sig(nc), gs(M > 0 ? M : 1, 0.0), kb(M > 0 ? M : 1, 0.0);
    LBFS_CUDA(cudaMemcpyAsync(sig.data(), j.sigma_acc, sizeof(double) * nc, cudaMemcpyDeviceToHost, st));
    if (M > 0) {
        LBFS_CUDA(cudaMemcpyAsync(gs.data(), mj.gs_acc, sizeof(double) * M, cudaMemcpyDeviceToHost, st));
        LBFS_CUDA(cudaMemcpyAsync(kb.data(), mj.kb_acc, sizeof(double) * M, cudaMemcpyDeviceToHost, st));
    }
    LBFS_CUDA(cudaStreamSynchronize(st));
    double sigma = 0.0, gsum = 0.0, ksum = 0.0;
    for (int c = 0; c < nc; c++) sigma += sig[c];
    for (int m = 0; m < M; m++) { gsum += gs[m]; ksum += kb[m]; }
    grad[0] = gsum;
    grad[1] = ksum;
    grad[2] = sigma;
    if (times_ms) {
        float f = 0, r = 0;
        cudaEventElapsedTime(&f, e0, e1);
        cudaEventElapsedTime(&r, e1, e2);
        times_ms[0] = f;
        times_ms[1] = r;
    }
    cudaEventDestroy(e0); cudaEventDestroy(e1); cudaEventDestroy(e2);
    return LBFS_OK;
}

// ---- lossless checkpoint / restart -----------------------------------------
//
// Everything a step reads that a step or the set-up wrote: soln_t1, the
// primitive state with its ghosts, the viscosity field, the residual sums, the
// status word, the step counter; per membrane the node positions, velocities
// and forces, the scalars (V0, A0, MAD0, MAD, V, A, bounds) and every
// per-spring array.  Gradients and fluxes are not saved: each step forms them
// before reading them.  The blob starts with a header that a load checks
// against the handle (sizes, precision).

namespace {

struct CkHeader {
    char magic[8];
    int32_t version, precision, nc, nb, nf, n_membranes, total_nodes, total_springs;
    int64_t t;
    uint32_t flags, pad;
};

struct CkPart {
    void *dev;
    size_t bytes;
};

std::vector<CkPart> ck_parts(lbfs_solver *s) {
    const size_t nc = s->nc, nt = (size_t)s->nc + s->nb, N = s->total_nodes, S = s->total_springs;
    const size_t r = s->fp32 ? sizeof(float) : sizeof(double);
    void *state = s->fp32 ? (void *)s->f32.state : (void *)s->f64.state;
    void *visc = s->fp32 ? (void *)s->f32.visc_factor : (void *)s->f64.visc_factor;
    void *t1 = s->fp32 ? (void *)s->f32.t1 : (void *)s->f64.t1;
    void *rsum = s->fp32 ? (void *)s->f32.residual_sums : (void *)s->f64.residual_sums;
    std::vector<CkPart> p = {{t1, sizeof(double4) * nc}, {state, 4 * r * nt}, {visc, r * nc}, {rsum, 4 * sizeof(double)}};
    if (s->n_membranes > 0) {
        const MembraneArgs &m = s->ma;
        for (double *a : {m.x, m.y, m.z, m.vx, m.vy, m.vz, m.fx, m.fy, m.fz}) p.push_back({a, sizeof(double) * N});
        p.push_back({m.ms, sizeof(MembraneScalars) * s->n_membranes});
        for (double *a : {m.contour, m.kspring, m.curv, m.curv0, m.angle0}) p.push_back({a, sizeof(double) * S});
        for (double *a : {m.area0, m.area}) p.push_back({a, sizeof(double) * 2 * S});
    }
    return p;
}

}  // namespace

extern "C" int lbfs_checkpoint_size(lbfs_solver *s, uint64_t *bytes) {
    if (!s || !bytes) return set_error(LBFS_ERR_ARG, "null argument");
    size_t b = sizeof(CkHeader);
    for (const CkPart &p : ck_parts(s)) b += p.bytes;
    *bytes = b;
    return LBFS_OK;
}

extern "C" int lbfs_checkpoint_save(lbfs_solver *s, void *buf, uint64_t bytes) {
    uint64_t need = 0;
    int rc = lbfs_checkpoint_size(s, &need);
    if (rc) return rc;
    if (!buf || bytes < need) return set_error(LBFS_ERR_ARG, "checkpoint buffer too small (lbfs_checkpoint_size)");
    LBFS_CUDA(cudaSetDevice(s->device));
    LBFS_CUDA(cudaStreamSynchronize(s->stream));
    const unsigned int *flags = s->fp32 ? s->f32.flags : s->f64.flags;
    CkHeader h{};
    std::memcpy(h.magic, "LBFSCK01", 8);
    h.version = 1;
    h.precision = s->params.precision;
    h.nc = s->nc; h.nb = s->nb; h.nf = s->nf;
    h.n_membranes = s->n_membranes; h.total_nodes = s->total_nodes; h.total_springs = s->total_springs;
    h.t = s->t;
    LBFS_CUDA(cudaMemcpy(&h.flags, flags, sizeof(unsigned int), cudaMemcpyDeviceToHost));
    char *o = (char *)buf;
    std::memcpy(o, &h, sizeof(h));
    o += sizeof(h);
    for (const CkPart &p : ck_parts(s)) {
        LBFS_CUDA(cudaMemcpy(o, p.dev, p.bytes, cudaMemcpyDeviceToHost));
        o += p.bytes;
    }
    return LBFS_OK;
}

extern "C" int lbfs_checkpoint_load(lbfs_solver *s, const void *buf, uint64_t bytes) {
    uint64_t need = 0;
    int rc = lbfs_checkpoint_size(s, &need);
    if (rc) return rc;
    if (!buf || bytes < need) return set_error(LBFS_ERR_ARG, "checkpoint shorter than this handle's state");
    CkHeader h;
    std::memcpy(&h, buf, sizeof(h));
    if (std::memcmp(h.magic, "LBFSCK01", 8) != 0 || h.version != 1)
        return set_error(LBFS_ERR_ARG, "not an lbfs_b200 checkpoint");
    if (h.precision != s->params.precision || h.nc != s->nc || h.nb != s->nb || h.nf != s->nf ||
        h.n_membranes != s->n_membranes || h.total_nodes != s->total_nodes || h.total_springs != s->total_springs)
        return set_error(LBFS_ERR_ARG, "checkpoint of a different mesh, membrane set or precision");
    LBFS_CUDA(cudaSetDevice(s->device));
    LBFS_CUDA(cudaStreamSynchronize(s->stream));
    const char *o = (const char *)buf + sizeof(h);
    for (const CkPart &p : ck_parts(s)) {
        LBFS_CUDA(cudaMemcpy(p.dev, o, p.bytes, cudaMemcpyHostToDevice));
        o += p.bytes;
    }
    unsigned int *flags = s->fp32 ? s->f32.flags : s->f64.flags;
    LBFS_CUDA(cudaMemcpy(flags, &h.flags, sizeof(unsigned int), cudaMemcpyHostToDevice));
    s->t = h.t;
    return LBFS_OK;
}

// ---- step-level autotuner ---------------------------------------------------

namespace {

// Coordinate descent over the launch shape, each candidate timed as whole
// steps (graph replays, CUDA events on the handle's stream) from the same
// saved state: the kernels run with the contention of a real step (the
// membrane chain beside the fluid kernels), which isolated kernel timings
// miss.  The state (the checkpoint parts, the counter and the status word)
// is put back afterwards.
int autotune_steps(lbfs_solver *s, int reps, lbfs_launch_shape *out, bool fp32) {
    LBFS_CUDA(cudaStreamSynchronize(s->stream));
    const std::vector<CkPart> parts = ck_parts(s);
    size_t total = 0;
    for (const CkPart &p : parts) total += p.bytes;
    DevBuf snap;
    LBFS_CUDA(cudaMalloc(&snap.p, total + sizeof(unsigned int)));
    unsigned int *flags = fp32 ? s->f32.flags : s->f64.flags;
    auto copy_all = [&](bool save) -> int {
        char *o = (char *)snap.p;
        for (const CkPart &p : parts) {
            LBFS_CUDA(cudaMemcpyAsync(save ? (void *)o : p.dev, save ? p.dev : (void *)o, p.bytes,
                                      cudaMemcpyDeviceToDevice, s->stream));
            o += p.bytes;
        }
        LBFS_CUDA(cudaMemcpyAsync(save ? (void *)o : (void *)flags, save ? (void *)flags : (void *)o,
                                  sizeof(unsigned int), cudaMemcpyDeviceToDevice, s->stream));
        return LBFS_OK;
    };
    int rc = copy_all(true);
    if (rc) return rc;
    const long long t0 = s->t;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    LBFS_CUDA(cudaEventCreate(&e0));
    LBFS_CUDA(cudaEventCreate(&e1));
    auto measure = [&](double *us) -> int {
        int r = copy_all(false);
        if (r) return r;
        s->t = t0;
        drop_graph(s);
        if ((r = lbfs_step_graph(s, 2))) return r;  // capture + warm
        LBFS_CUDA(cudaEventRecord(e0, s->stream));
        if ((r = lbfs_step_graph(s, reps))) return r;
        LBFS_CUDA(cudaEventRecord(e1, s->stream));
        LBFS_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        LBFS_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        *us = 1000.0 * ms / reps;
        return LBFS_OK;
    };
    auto apply = [&](const lbfs_launch_shape &sh) {
        if (fp32) shape_to_args<float>(s, sh);
        else shape_to_args<double>(s, sh);
    };
    struct Knob {
        int32_t lbfs_launch_shape::*field;
        std::vector<int> values;
    };
    const bool membranes = s->n_membranes > 0;
    const std::vector<Knob> knobs = {
        {&lbfs_launch_shape::gradient_threads, {128, 256, 512}},
        {&lbfs_launch_shape::flux_threads, {64, 128, 256}},
        {&lbfs_launch_shape::general_flux_threads, {64, 128, 256}},
        {&lbfs_launch_shape::update_threads, {128, 256, 512}},
        {&lbfs_launch_shape::update_blocks, {148 * 2, 148 * 4, 148 * 8, 148 * 16}},
        {&lbfs_launch_shape::spread_blocks,
         membranes ? std::vector<int>{148, 296, 592, 1184, 2368} : std::vector<int>{}},
        {&lbfs_launch_shape::flux_chunks, s->chunkable ? std::vector<int>{1, 2, 4, 8} : std::vector<int>{}},
    };
    lbfs_launch_shape cur = fp32 ? args_to_shape<float>(s) : args_to_shape<double>(s);
    double best = 0;
    rc = measure(&best);
    for (size_t q = 0; !rc && q < knobs.size(); q++) {
        const Knob &k = knobs[q];
        for (size_t v = 0; !rc && v < k.values.size(); v++) {
            if (cur.*(k.field) == k.values[v]) continue;
            lbfs_launch_shape trial = cur;
            trial.*(k.field) = k.values[v];
            apply(trial);
            double t = 0;
            rc = measure(&t);
            if (!rc && t < 0.99 * best) {  // keep only a clear gain
                best = t;
                cur = trial;
            }
        }
        apply(cur);
    }
    // the membrane chain's form and where it starts, jointly: the cluster step behind the gradient
    // launch can win where neither change wins alone (64^3 FP64: about 5 % per step)
    if (!rc && membranes) {
        const std::vector<int> clusters =
            membrane_cluster_fits(s->ma.max_nodes) ? std::vector<int>{0, 8, 16} : std::vector<int>{0};
        const lbfs_launch_shape base = cur;
        for (int cl : clusters) {
            for (int after = 0; !rc && after < 2; after++) {
                if (cl == base.membrane_cluster && after == base.membrane_after_k1) continue;
                lbfs_launch_shape trial = base;
                trial.membrane_cluster = cl;
                trial.membrane_after_k1 = after;
                apply(trial);
                double t = 0;
                rc = measure(&t);
                if (!rc && t < 0.99 * best) {
                    best = t;
                    cur = trial;
                }
            }
        }
        apply(cur);
    }
    apply(cur);
    const int r2 = copy_all(false);
    if (!rc) rc = r2;
    s->t = t0;
    drop_graph(s);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    const cudaError_t e = cudaStreamSynchronize(s->stream);
    if (rc) return rc;
    if (e != cudaSuccess) return set_error(LBFS_ERR_CUDA, std::string("autotune: ") + cudaGetErrorString(e));
    if (out) {
        *out = cur;
        for (int q = 0; q < 5; q++) out->time_us[q] = 0.0;
        out->time_us[0] = best;
    }
    return LBFS_OK;
}

}  // namespace
