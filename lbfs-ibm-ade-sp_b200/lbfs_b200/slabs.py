"""Slab decomposition of one uniform hex mesh over several handles (one per GPU).

The reference steps one mesh on one device (Solver_gpu.cu:749-1021).  Here the
cells of a generated uniform mesh (x fastest, then y, then z) are cut into slabs
of z planes, one per rank.  Each rank's handle holds its slab and HALO planes of
each neighbour's cells.  A step of the decomposed mesh is every handle's own step
followed by a halo exchange: each rank sends its first and last HALO owned planes
(state records and FP64 accumulators) to its neighbours, which overwrite their
halo planes with them.  Two planes suffice: the gradients of the first halo plane
read the second, and the face fluxes of the owned cells read the first plane's
state and gradients, so every owned cell takes the single-mesh step bit for bit.
The halo planes' own updates (their outer neighbours are the cut's ghost cells)
are overwritten by the exchange.

Membranes stay on the rank whose window (its owned planes less HALO planes at
each cut) holds their IBM patch.  The handle checks this on the device every step
(lbfs_set_ibm_window): a patch that leaves the window spreads nothing and raises
LBFS_FLAG_IBM_RANGE.  So the IBM touches owned cells only, and the
interior-viscosity marking never reaches a halo plane.

Rejected at set-up: z-periodic boundaries, time stepping other than constant
(the minimum step would need a reduction inside the step), periodic objects,
and slab origins that are not exact in binary (the slab's vertices must be the
mesh's own, bit for bit).

The exchange runs over torch.distributed (NCCL on GPUs, point-to-point on the
handle's stream, which is set to torch's current stream; gloo through host
copies) or, for several slabs in one process, as device copies (LocalExchange).
"""
import numpy as np

from . import _abi
from .mesh import build_uniform_mesh
from .solver import GpuSolver

__all__ = ["HALO", "slab_bounds", "SlabMesh", "build_slab_mesh", "assign_membranes", "SlabSolver", "LocalExchange",
           "TorchExchange", "step_local"]

HALO = 2
_CUT_BC = (2, 2, 1.0, 0.0, 0.0, 0.0)  # the cut planes' ghosts: only the outer halo plane reads them


def slab_bounds(nz, world, planes=None):
    """(z0, z1) owned planes of each rank: `planes` (one count per rank) or nz split as evenly as possible,
    the first nz % world ranks one plane more.  Every slab needs at least HALO planes."""
    if planes is None:
        base, extra = divmod(nz, world)
        planes = [base + (1 if r < extra else 0) for r in range(world)]
    planes = [int(p) for p in planes]
    if len(planes) != world or sum(planes) != nz:
        raise ValueError("planes must give one count per rank, summing to the mesh's z planes")
    if min(planes) < HALO:
        raise ValueError(f"every slab needs at least {HALO} planes")
    out, z = [], 0
    for p in planes:
        out.append((z, z + p))
        z += p
    return out


class SlabMesh:
    """One rank's piece: its local mesh (owned planes plus halos) and the index ranges."""

    def __init__(self, mesh, nz, z0, z1, lo, hi):
        self.mesh = mesh
        self.nz, self.z0, self.z1, self.lo, self.hi = nz, z0, z1, lo, hi
        self.plane_cells = mesh.n_cells // (hi - lo)
        self.first_owned = (z0 - lo) * self.plane_cells
        self.n_owned = (z1 - z0) * self.plane_cells
        # IBM window in the local grid's z cells: the owned planes less HALO planes at each cut
        self.window = (z0 - lo + (HALO if z0 > 0 else 0), z1 - lo - (HALO if z1 < nz else 0))

    @property
    def owned(self):
        return slice(self.first_owned, self.first_owned + self.n_owned)

    def sends(self):
        """(peer offset, first local cell, cells) of the owned planes the neighbours need."""
        out = []
        if self.z0 > 0:
            out.append((-1, self.first_owned, HALO * self.plane_cells))
        if self.z1 < self.nz:
            out.append((+1, self.first_owned + self.n_owned - HALO * self.plane_cells, HALO * self.plane_cells))
        return out

    def recvs(self):
        """(peer offset, first local cell, cells) of the halo planes."""
        out = []
        if self.z0 > 0:
            out.append((-1, 0, (self.z0 - self.lo) * self.plane_cells))
        if self.z1 < self.nz:
            out.append((+1, self.first_owned + self.n_owned, (self.hi - self.z1) * self.plane_cells))
        return out


def _axis(origin, step, n):
    # the generator's uniform vertices, origin + i * step (unstructured_mesh.cpp:290-378)
    return origin + np.arange(n + 1, dtype=np.float64) * step


def build_slab_mesh(X, Y, Z, dt, bounds, rank, origin=(0.0, 0.0, 0.0), bcs=None, periodic_translation=None,
                    device=None, **mesh_kw):
    """The local mesh of `rank` for the uniform mesh (X, Y, Z, dt, origin): planes [z0 - HALO, z1 + HALO)
    clipped to the mesh, with the mesh's boundary conditions on its own patches and a zero-gradient
    condition on the cut planes.  Raises ValueError when the slab's vertices would not be the mesh's."""
    counts = np.zeros(8, np.int32)
    _abi.check(_abi.lib().lbfs_mesh_uniform_counts(X, Y, Z, dt, _abi.iptr(counts)))
    nz = int(np.ceil(Z / dt * 0.5))
    dz = Z / nz
    z0, z1 = bounds[rank]
    lo, hi = max(0, z0 - HALO), min(nz, z1 + HALO)
    Zl = (hi - lo) * dz
    oz = origin[2] + lo * dz
    if int(np.ceil(Zl / dt * 0.5)) != hi - lo or Zl / (hi - lo) != dz or \
            not np.array_equal(_axis(oz, Zl / (hi - lo), hi - lo), _axis(origin[2], dz, nz)[lo:hi + 1]):
        raise ValueError("the slab's z vertices are not exact in binary; choose a spacing and origin that are")
    if mesh_kw.get("jitter", 0.0) or mesh_kw.get("mesh_type", 6) != 6:
        raise ValueError("slabs are cut from the uniform mesh (mesh_type 6, no jitter)")
    mesh = build_uniform_mesh(X, Y, Zl, dt, origin=(origin[0], origin[1], oz), device=device, **mesh_kw)
    if bcs is not None:
        for name in ("back", "front"):
            if bcs[name][0] == 3 or bcs[name][1] == 3:
                raise ValueError("z-periodic boundaries cross the cuts; slabs are cut along z")
        spec = dict(bcs)
        if lo > 0:
            spec["back"] = _CUT_BC
        if hi < nz:
            spec["front"] = _CUT_BC
        mesh.set_boundaries(spec, periodic_translation)
    return SlabMesh(mesh, nz, z0, z1, lo, hi)


def _patch_planes(membrane, origin_z, dz, stencil):
    # z cells a membrane's IBM stencils can reach at its current nodes, with one cell of margin
    z = np.asarray(membrane.xyz_initial, np.float64).reshape(-1, 3)[:, 2]
    half = 1 if stencil == _abi.LBFS_IBM_HAT2 else 2
    return (int(np.floor((z.min() - origin_z) / dz)) - half - 1, int(np.floor((z.max() - origin_z) / dz)) + half + 2)


def assign_membranes(membranes, bounds, nz, origin_z, dz, stencil):
    """Rank of each membrane: the one whose window holds the z cells its IBM stencils reach."""
    ranks = []
    for m in membranes:
        if getattr(m, "periodic", 0):
            raise ValueError("periodic objects wrap across the cuts; not supported on slabs")
        a, b = _patch_planes(m, origin_z, dz, stencil)
        owner = None
        for r, (z0, z1) in enumerate(bounds):
            w0, w1 = z0 + (HALO if z0 > 0 else 0), z1 - (HALO if z1 < nz else 0)
            if w0 <= a and b <= w1:
                owner = r
                break
        if owner is None:
            raise ValueError("a membrane's IBM patch crosses a slab window; move the cuts")
        ranks.append(owner)
    return ranks


class SlabSolver:
    """One rank's handle on its slab, with the pack and unpack of its halo planes; an exchange
    (TorchExchange, LocalExchange) moves the planes between slabs after every step."""

    def __init__(self, slab, params, membranes=(), device=0):
        if params.time_stepping not in (0, _abi.LBFS_DT_CONSTANT):
            raise ValueError("slabs need constant time stepping (the minimum step is a reduction inside the step)")
        self.slab = slab
        self.solver = GpuSolver(slab.mesh, params, membranes, device)
        self.membranes = list(membranes)
        if self.membranes:
            self.solver.set_ibm_window(*slab.window)
        self._bufs = {}

    def set_state(self, rho, u, v, w):
        """The local cells' state from the whole mesh's arrays (owned and halo planes)."""
        s = self.slab
        sel = slice(s.lo * s.plane_cells, s.hi * s.plane_cells)
        self.solver.set_state(rho[sel], u[sel], v[sel], w[sel])

    def owned_state(self):
        return tuple(a[self.slab.owned] for a in self.solver.state())

    def buffer(self, key, n_cells, device):
        import torch
        if key not in self._bufs:
            self._bufs[key] = torch.empty(self.solver.halo_bytes(n_cells), dtype=torch.uint8, device=device)
        return self._bufs[key]

    def pack(self, device):
        """Device buffers of the owned planes the neighbours need, by peer offset."""
        out = {}
        for peer, first, n in self.slab.sends():
            b = self.buffer(("send", peer), n, device)
            self.solver.halo_pack(first, n, b.data_ptr())
            out[peer] = b
        return out

    def recv_buffers(self, device):
        return {peer: self.buffer(("recv", peer), n, device) for peer, _, n in self.slab.recvs()}

    def unpack(self, bufs):
        for peer, first, n in self.slab.recvs():
            self.solver.halo_unpack(first, n, bufs[peer].data_ptr())

    def owned_residual_squares(self):
        """Sums over the owned cells of the squared residuals (rho, u, v, w) of the last step
        (needs keep_residuals); the decomposed mesh's sums are the sum over ranks."""
        r = self.solver.field(_abi.LBFS_FIELD_RESIDUAL).reshape(-1, 4)[self.slab.owned]
        return (r * r).sum(axis=0)


class LocalExchange:
    """Halo exchange between slabs of one process: device copies, each pack ordered before the unpack."""

    def __init__(self, slabs, device):
        self.slabs, self.device = slabs, device

    def __call__(self):
        import torch
        sent = []
        for s in self.slabs:
            sent.append(s.pack(self.device))
            s.solver.synchronize()
        for r, s in enumerate(self.slabs):
            bufs = s.recv_buffers(self.device)
            for peer in bufs:
                bufs[peer].copy_(sent[r + peer][-peer])
            torch.cuda.synchronize(self.device)
            s.unpack(bufs)
            s.solver.synchronize()


def step_local(slabs, n, device, graph=True):
    """n steps of slabs held in one process: each slab's step, then the exchange."""
    ex = LocalExchange(slabs, device)
    for _ in range(n):
        for s in slabs:
            s.solver.step(1, graph=graph)
        ex()


class TorchExchange:
    """Halo exchange over torch.distributed: one process per slab, rank r's neighbours r - 1 and r + 1.
    NCCL moves the device buffers on the handle's stream (set to torch's current stream); gloo moves
    host copies."""

    def __init__(self, slab_solver, device):
        import torch
        import torch.distributed as dist
        self.s, self.device, self.dist, self.torch = slab_solver, torch.device(device), dist, torch
        self.rank = dist.get_rank()
        self.nccl = dist.get_backend() == "nccl"
        self.cuda = self.device.type == "cuda"
        # a stream of its own (graphs cannot be captured on the legacy default stream), shared by the
        # handle's step, the pack and unpack copies and the point-to-point transfers
        self.stream = torch.cuda.Stream(self.device) if self.cuda else None
        if self.cuda:
            slab_solver.solver.set_stream(self.stream.cuda_stream)

    def __call__(self):
        if not self.cuda:
            return self._exchange()
        with self.torch.cuda.stream(self.stream):
            return self._exchange()

    def _exchange(self):
        dist, torch = self.dist, self.torch
        send = self.s.pack(self.device)
        recv = self.s.recv_buffers(self.device)
        if self.nccl:
            sbuf, rbuf = send, recv
        else:
            if self.cuda:
                self.stream.synchronize()
            sbuf = {p: b.cpu() for p, b in send.items()}
            rbuf = {p: torch.empty(b.shape, dtype=b.dtype) for p, b in recv.items()}
        ops = []
        for p in sorted(sbuf):
            ops.append(dist.P2POp(dist.isend, sbuf[p], self.rank + p))
        for p in sorted(rbuf):
            ops.append(dist.P2POp(dist.irecv, rbuf[p], self.rank + p))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        if not self.nccl:
            for p in recv:
                recv[p].copy_(rbuf[p])
        self.s.unpack(recv)

    def step(self, n, graph=True):
        for _ in range(n):
            self.s.solver.step(1, graph=graph)
            self()
