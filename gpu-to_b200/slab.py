"""x-slab partitioned MGCG: one grid split along x over several GPUs.

The reference solves on one device (Cantilever/TOP3D125MGCGCUDA/mgcg1.cu:203,
cudaSetDevice(0)).  Beyond one GPU's memory the grid is cut into contiguous
slabs of element planes, one per rank.  x is the slowest index of the node
numbering (n = (nz+1)(ny+1) i + (ny+1) k + j), so a slab's node planes are a
contiguous range of the global vector.

* Ownership: rank r owns node planes [x0_r, x1_r) (the last rank also plane
  nelx).  Each rank keeps a solver (gputo.Solver) on its slab extended by
  `halo` element planes on each side (clipped at the grid's ends); the planes
  at a cut end of the extended slab are held (artificial Dirichlet dofs).
* Operator: K u on the owned planes is the extended solver's apply of u with
  the halo planes filled from the neighbours: one exchange of halo planes
  per apply, no reduction, since every element next to an owned node lies
  in the extended slab.
* Preconditioner: additive Schwarz.  The residual is extended by the
  neighbours' halo planes, zeroed on the held planes and passed through the
  extended solver's V-cycle (mgcg1.cu:468-651); the results of the slabs
  are summed where they overlap (the transpose of the halo exchange).  The
  outer iteration is flexible PCG (Polak-Ribiere beta) in FP64, as for the
  mixed-precision solver; its convergence test is the reference's
  relres = |r| / |F| (mgcg1.cu:254-275).
* Per PCG iteration: three halo exchanges (u for the apply, r into the
  V-cycles, the overlap sums out of them) and two all-reductions of FP64
  scalars (p'q; r'r, r'z, r'z_old).

Communication goes through a Comm object: DistComm runs one part per process
over torch.distributed (NCCL send/recv into local buffers on GPUs, gloo on
CPUs); LocalComm runs several parts in one process (the exchanges are
copies), which serves one-GPU runs and tests.  The local solves are a
backend object with apply(u_ext) and vcycle(r_ext) on extended-slab vectors;
GpuSlabBackend wraps gputo.Solver (there is no CPU backend in the product).
"""
from __future__ import annotations

import numpy as np


class SlabPart:
    """The geometry of one rank's slab."""

    def __init__(self, nelx, nely, nelz, nl, nparts, rank, halo=None):
        m = 1 << (nl - 1)
        if nelx % m or nely % m or nelz % m:
            raise ValueError("nelx, nely, nelz must be divisible by 2^(nl-1)")
        units = nelx // m
        if units < nparts:
            raise ValueError("fewer 2^(nl-1)-element units along x than parts")
        h = m if halo is None else int(halo)
        if h < 1 or h % m:
            raise ValueError("the halo must be a positive multiple of 2^(nl-1) element planes")
        # element slabs of whole units, as even as possible
        cuts = [m * ((units * r) // nparts) for r in range(nparts + 1)]
        self.nelx, self.nely, self.nelz, self.nl = nelx, nely, nelz, nl
        self.nparts, self.rank, self.halo = nparts, rank, h
        self.x0, self.x1 = cuts[rank], cuts[rank + 1]
        self.sizes = [cuts[r + 1] - cuts[r] for r in range(nparts)]
        if nparts > 1 and min(self.sizes) < h + 1:
            raise ValueError("every slab must be at least halo + 1 element planes thick")
        self.e0, self.e1 = max(0, self.x0 - h), min(nelx, self.x1 + h)   # extended element planes
        self.o0 = self.x0
        self.o1 = self.x1 if rank < nparts - 1 else nelx + 1              # owned node planes [o0, o1)
        self.plane = 3 * (nely + 1) * (nelz + 1)                          # dofs per node plane

    @property
    def ext_nelx(self):
        return self.e1 - self.e0

    @property
    def n_own(self):
        return (self.o1 - self.o0) * self.plane

    @property
    def n_ext(self):
        return (self.e1 - self.e0 + 1) * self.plane

    def own_slice(self):
        """The owned planes inside an extended-slab vector."""
        a = (self.o0 - self.e0) * self.plane
        return slice(a, a + self.n_own)

    def global_own_slice(self):
        return slice(self.o0 * self.plane, self.o1 * self.plane)

    def held_planes(self):
        """Extended-slab node planes held as artificial Dirichlet planes."""
        out = []
        if self.e0 > 0:
            out.append(0)
        if self.e1 < self.nelx:
            out.append(self.e1 - self.e0)
        return out

    def local_fixed(self, fixed1b):
        """1-based fixed dofs of the extended slab: the global ones inside it
        plus every dof of a held plane."""
        f = np.asarray(fixed1b, dtype=np.int64) - 1
        lo, hi = self.e0 * self.plane, (self.e1 + 1) * self.plane
        f = f[(f >= lo) & (f < hi)] - lo
        held = [np.arange(p * self.plane, (p + 1) * self.plane) for p in self.held_planes()]
        allf = np.unique(np.concatenate([f] + held)) if held else np.unique(f)
        return (allf + 1).astype(np.float64)

    def local_cx(self, CX):
        """Element scales of the extended slab (element order: x slowest)."""
        per = self.nely * self.nelz
        return np.ascontiguousarray(np.asarray(CX)[self.e0 * per:self.e1 * per])


class LocalComm:
    """Several parts in one process: exchanges are copies, reductions sums."""

    def __init__(self, parts):
        self.parts = parts

    def halo(self, own, ext):
        """own[i]: part i's owned planes; ext[i] (out): its extended vector."""
        for i, p in enumerate(self.parts):
            ext[i].zero_()
            ext[i][p.own_slice()] = own[i]
            if i > 0:   # left halo: planes [e0, o0) from part i-1's last owned planes
                q = self.parts[i - 1]
                n = (p.o0 - p.e0) * p.plane
                ext[i][:n] = own[i - 1][q.n_own - n:]
            if i + 1 < len(self.parts):   # right halo: planes [o1, e1] from part i+1's first ones
                n = (p.e1 + 1 - p.o1) * p.plane
                ext[i][p.n_ext - n:] = own[i + 1][:n]

    def halo_add(self, ext, own):
        """own[i] (out) = part i's owned planes of ext[i] plus the neighbours'
        extended-slab values on those planes (the transpose of halo)."""
        for i, p in enumerate(self.parts):
            own[i].copy_(ext[i][p.own_slice()])
            if i > 0:   # part i-1's right halo lies on my first planes
                q = self.parts[i - 1]
                n = (q.e1 + 1 - q.o1) * q.plane
                own[i][:n] += ext[i - 1][q.n_ext - n:]
            if i + 1 < len(self.parts):   # part i+1's left halo lies on my last planes
                q = self.parts[i + 1]
                n = (q.o0 - q.e0) * q.plane
                own[i][p.n_own - n:] += ext[i + 1][:n]

    def allreduce(self, partials):
        """partials[i]: part i's vector of partial sums; returns the global sums."""
        return sum(partials)


class DistComm:
    """One part per process over torch.distributed (rank order = slab order)."""

    def __init__(self, part, group=None):
        import torch.distributed as dist
        self.dist, self.part, self.group = dist, part, group
        self.parts = [part]

    def halo(self, own, ext):
        dist, p = self.dist, self.part
        o, e = own[0], ext[0]
        e.zero_()
        e[p.own_slice()] = o
        ops = []
        nl_ = (p.o0 - p.e0) * p.plane            # my left halo
        nr_ = (p.e1 + 1 - p.o1) * p.plane        # my right halo
        left, right = p.rank - 1, p.rank + 1
        recv_l = recv_r = None
        if p.rank > 0:
            recv_l = e[:nl_]
            ops.append(dist.P2POp(dist.irecv, recv_l, left, self.group))
            # the left neighbour's right halo is my first planes
            q_e1 = min(p.nelx, p.x0 + p.halo)
            ops.append(dist.P2POp(dist.isend, o[:(q_e1 + 1 - p.o0) * p.plane].contiguous(), left, self.group))
        if p.rank + 1 < p.nparts:
            recv_r = e[p.n_ext - nr_:]
            ops.append(dist.P2POp(dist.irecv, recv_r, right, self.group))
            ops.append(dist.P2POp(dist.isend, o[p.n_own - p.halo * p.plane:].contiguous(), right, self.group))
        if ops:
            for r in dist.batch_isend_irecv(ops):
                r.wait()

    def halo_add(self, ext, own):
        dist, p = self.dist, self.part
        e, o = ext[0], own[0]
        o.copy_(e[p.own_slice()])
        ops, bufs = [], []
        if p.rank > 0:   # my left halo goes to the left neighbour's last planes
            n = (p.o0 - p.e0) * p.plane
            ops.append(dist.P2POp(dist.isend, e[:n].contiguous(), p.rank - 1, self.group))
            q_e1 = min(p.nelx, p.x0 + p.halo)   # the left neighbour's right halo lies on my first planes
            b = e.new_zeros((q_e1 + 1 - p.o0) * p.plane)
            ops.append(dist.P2POp(dist.irecv, b, p.rank - 1, self.group))
            bufs.append((0, b))
        if p.rank + 1 < p.nparts:   # my right halo goes to the right neighbour's first planes
            n = (p.e1 + 1 - p.o1) * p.plane
            ops.append(dist.P2POp(dist.isend, e[p.n_ext - n:].contiguous(), p.rank + 1, self.group))
            b = e.new_zeros(p.halo * p.plane)
            ops.append(dist.P2POp(dist.irecv, b, p.rank + 1, self.group))
            bufs.append((p.n_own - p.halo * p.plane, b))
        if ops:
            for r in dist.batch_isend_irecv(ops):
                r.wait()
        for at, b in bufs:
            o[at:at + b.numel()] += b

    def allreduce(self, partials):
        t = partials[0].clone()
        self.dist.all_reduce(t, group=self.group)
        return t


class GpuSlabBackend:
    """The extended slab's gputo.Solver: apply and V-cycle on device vectors."""

    def __init__(self, part, Ke0, fixed1b, CX, options=None):
        import torch

        import gputo
        self.part = part
        self.solver = gputo.Solver(part.ext_nelx, part.nely, part.nelz, part.nl, options)
        self.solver.set_problem(Ke0, part.local_fixed(fixed1b))
        self.solver.setup(torch.as_tensor(part.local_cx(CX), dtype=torch.float64, device="cuda"))

    def apply(self, u, out):
        self.solver.apply(u, out)

    def vcycle(self, r, out):
        self.solver.vcycle(r, out)


def slab_pcg(parts, backends, comm, F_own, tol, maxit):
    """Flexible PCG over the parts this process holds (lists in part order).
    F_own[i]: part i's owned planes of F.  Returns (U_own list, relres, nit)
    with nit the reference's 0-based break index (maxit if not converged)."""
    import torch
    dev = F_own[0].device
    f64 = dict(dtype=torch.float64, device=dev)
    ext_u = [torch.zeros(p.n_ext, **f64) for p in parts]
    ext_o = [torch.zeros(p.n_ext, **f64) for p in parts]
    held = [[slice(q * p.plane, (q + 1) * p.plane) for q in p.held_planes()] for p in parts]

    def apply(P):
        comm.halo(P, ext_u)
        out = []
        for i, p in enumerate(parts):
            backends[i].apply(ext_u[i], ext_o[i])
            out.append(ext_o[i][p.own_slice()].clone())
        return out

    def precond(R):
        comm.halo(R, ext_u)
        for i, p in enumerate(parts):
            for s in held[i]:
                ext_u[i][s] = 0.0
            backends[i].vcycle(ext_u[i], ext_o[i])
        out = [torch.zeros_like(r) for r in R]
        comm.halo_add(ext_o, out)   # additive Schwarz: the overlaps' contributions summed
        return out

    def dots(pairs):
        part = [torch.stack([torch.dot(a[i], b[i]) for a, b in pairs]) for i in range(len(parts))]
        return comm.allreduce(part)

    U = [torch.zeros_like(f) for f in F_own]
    R = [f.clone() for f in F_own]
    res0 = float(torch.sqrt(dots([(R, R)])[0]))
    if not res0 > 0:
        return U, 0.0, 0
    Z = precond(R)
    rho = float(dots([(R, Z)])[0])
    P = [z.clone() for z in Z]
    Zo = [z.clone() for z in Z]
    relres, nit = 1.0, maxit
    for it in range(maxit):
        Q = apply(P)
        pq = float(dots([(P, Q)])[0])
        if not pq > 0:
            raise RuntimeError(f"slab PCG breakdown at iteration {it}: p'q = {pq}")
        alpha = rho / pq
        for i in range(len(parts)):
            U[i].add_(P[i], alpha=alpha)
            R[i].add_(Q[i], alpha=-alpha)
        Z = precond(R)
        rr, rz, rzo = (float(v) for v in dots([(R, R), (R, Z), (R, Zo)]))
        relres = np.sqrt(rr) / res0
        if relres < tol:
            nit = it
            break
        beta = (rz - rzo) / rho
        rho = rz
        for i in range(len(parts)):
            P[i].mul_(beta).add_(Z[i])
            Zo[i].copy_(Z[i])
    return U, relres, nit
