"""The x-slab partitioned MGCG (gpu-to_b200/slab.py) on the CPU.

The partition, the halo exchanges and the distributed flexible PCG are
checked against the single-rank oracle; the per-slab solves are the oracle's
apply and V-cycle on each extended slab (a test backend: the product's
backend is the CUDA solver, see test_gpu_slab.py).

 * geometry: slabs of whole 2^(nl-1) units, owned node planes cover the grid
   once, held planes only at cut ends;
 * the distributed operator (one halo exchange, no reduction) equals the
   global K u on every owned plane to 1e-13;
 * solves with 2 (gloo, two processes) and 3 (one process) parts reach the
   single-rank oracle's solution to 1e-7 at tol 1e-10.
"""
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest

from conftest import ROOT


def _slab():
    import sys
    sys.path.insert(0, os.path.join(ROOT, "gpu-to_b200"))
    import slab
    return slab


class OracleBackend:
    """apply / V-cycle of an extended slab by the oracle (test only)."""

    def __init__(self, O, part, Ke0, fixed1b, CX):
        import torch
        self.torch, self.O, self.part = torch, O, part
        self.fixed = (part.local_fixed(fixed1b) - 1).astype(np.int64)
        self.p = O.Problem(part.ext_nelx, part.nely, part.nelz, np.zeros(part.n_ext), part.local_fixed(fixed1b),
                           Ke0)
        self.CX = part.local_cx(CX)

    def apply(self, u, out):
        r = self.O.apply_fine(self.p, self.CX, u.numpy())
        r[self.fixed] = 0.0
        out.copy_(self.torch.from_numpy(r))

    def vcycle(self, r, out):
        out.copy_(self.torch.from_numpy(self.O.vcycle(self.p, self.CX, self.part.nl, r.numpy())))


def _case(O, nelx=32, nely=8, nelz=8, seed=3):
    p = O.cantilever(nelx, nely, nelz)
    CX = O.simp(O.random_density(nelx, nely, nelz, seed=seed))[0]
    return p, CX


def _solver_frame(U):
    V = U.copy()
    V[1::3] *= -1   # the oracle's mgcg1 returns the MEX frame (y negated, mgcg1.cu:282-283)
    return V


def test_partition_geometry():
    slab = _slab()
    nelx, nely, nelz, nl = 48, 8, 8, 3
    for n in (1, 2, 3, 4):
        parts = [slab.SlabPart(nelx, nely, nelz, nl, n, r) for r in range(n)]
        planes = np.concatenate([np.arange(p.o0, p.o1) for p in parts])
        assert np.array_equal(planes, np.arange(nelx + 1))   # every node plane owned once
        for p in parts:
            assert p.ext_nelx % (1 << (nl - 1)) == 0
            assert (p.e0 > 0) + (p.e1 < nelx) == len(p.held_planes())
    with pytest.raises(ValueError):
        slab.SlabPart(8, 8, 8, 3, 3, 0)   # two 4-element units cannot make three slabs


def test_distributed_apply_equals_the_global_operator(oracle):
    import torch
    slab = _slab()
    p, CX = _case(oracle, 48, 8, 8)
    nl = 3
    parts = [slab.SlabPart(p.nelx, p.nely, p.nelz, nl, 3, r) for r in range(3)]
    be = [OracleBackend(oracle, q, p.Ke0, p.fixed, CX) for q in parts]
    comm = slab.LocalComm(parts)
    u = np.random.default_rng(5).standard_normal(p.ndof)
    ref = oracle.apply_fine(p, CX, u)
    ref[p.fixed.astype(np.int64) - 1] = 0.0
    own = [torch.from_numpy(u[q.global_own_slice()].copy()) for q in parts]
    ext = [torch.zeros(q.n_ext, dtype=torch.float64) for q in parts]
    comm.halo(own, ext)
    for q, e, b in zip(parts, ext, be):
        out = torch.zeros_like(e)
        b.apply(e, out)
        got = out[q.own_slice()].numpy()
        want = ref[q.global_own_slice()]
        assert np.abs(got - want).max() <= 1e-13 * np.abs(ref).max()


def test_three_slabs_in_one_process_reach_the_single_rank_solution(oracle):
    import torch
    slab = _slab()
    p, CX = _case(oracle, 48, 8, 8, seed=7)
    nl = 3
    Uo, _, _ = oracle.mgcg1(p, CX, nl, 1e-12, 500)
    Uo = _solver_frame(Uo)
    parts = [slab.SlabPart(p.nelx, p.nely, p.nelz, nl, 3, r) for r in range(3)]
    be = [OracleBackend(oracle, q, p.Ke0, p.fixed, CX) for q in parts]
    F = [torch.from_numpy(p.F[q.global_own_slice()].copy()) for q in parts]
    U, rr, nit = slab.slab_pcg(parts, be, slab.LocalComm(parts), F, 1e-10, 500)
    assert rr < 1e-10 and 0 < nit < 500
    got = np.concatenate([u.numpy() for u in U])
    assert np.linalg.norm(got - Uo) <= 1e-7 * np.linalg.norm(Uo)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, ws, port, q):
    import sys
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws))
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    sys.path.insert(0, os.path.join(ROOT, "gpu-to_b200"))
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import datetime

    import torch
    import torch.distributed as dist

    import oracle as O
    import slab
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=120))
    p, CX = _case(O)
    part = slab.SlabPart(p.nelx, p.nely, p.nelz, 3, ws, rank)
    be = OracleBackend(O, part, p.Ke0, p.fixed, CX)
    F = torch.from_numpy(p.F[part.global_own_slice()].copy())
    U, rr, nit = slab.slab_pcg([part], [be], slab.DistComm(part), [F], 1e-10, 500)
    q.put((rank, part.o0, part.o1, U[0].numpy(), rr, nit))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_reach_the_single_rank_solution(oracle):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for pr in procs:
        pr.start()
    out = sorted((q.get(timeout=300) for _ in procs), key=lambda t: t[0])
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    assert out[0][4] == out[1][4] and out[0][5] == out[1][5]   # both ranks saw the same scalars
    p, CX = _case(oracle)
    Uo, _, _ = oracle.mgcg1(p, CX, 3, 1e-12, 500)
    Uo = _solver_frame(Uo)
    got = np.concatenate([o[3] for o in out])
    assert out[0][2] == out[1][1] and out[1][2] == p.nelx + 1
    assert out[0][4] < 1e-10
    assert np.linalg.norm(got - Uo) <= 1e-7 * np.linalg.norm(Uo)
