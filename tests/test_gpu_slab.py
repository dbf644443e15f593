"""The x-slab partitioned MGCG with the product's backend (one gputo.Solver
per extended slab) on one GPU: the parts run one after another in one
process (slab.LocalComm), which exercises the same partition, halo and PCG
code as one process per GPU (slab.DistComm, tested with gloo ranks in
test_slab.py) without ranks whose kernels wait on one another."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as T
    assert T.cuda.is_available(), "GPU tests need a CUDA device"
    return T


@pytest.mark.parametrize("nparts,prec", [(2, "fp64"), (3, "fp64"), (2, "mixed")])
def test_slabs_on_the_gpu_reach_the_single_solver_solution(oracle, gputo, torch, nparts, prec):
    import slab
    nelx, nely, nelz, nl = 96, 32, 32, 4
    p = oracle.cantilever(nelx, nely, nelz)
    CX = oracle.simp(oracle.random_density(nelx, nely, nelz, seed=2))[0]
    opts = gputo.default_options(precision=gputo.PREC_MIXED if prec == "mixed" else gputo.PREC_FP64)
    f64 = dict(dtype=torch.float64, device="cuda")
    s = gputo.Solver(nelx, nely, nelz, nl, opts)
    s.set_problem(p.Ke0, p.fixed)
    s.setup(torch.as_tensor(CX, **f64))
    Fd = torch.as_tensor(p.F, **f64)
    U1 = torch.zeros_like(Fd)
    rr1, nit1 = s.solve(Fd, U1, 1e-10, 1000)
    parts = [slab.SlabPart(nelx, nely, nelz, nl, nparts, r) for r in range(nparts)]
    be = [slab.GpuSlabBackend(q, p.Ke0, p.fixed, CX, opts) for q in parts]
    comm = slab.LocalComm(parts)
    # the distributed operator equals the single solver's apply
    u = torch.as_tensor(np.random.default_rng(3).standard_normal(p.ndof), **f64)
    ref = torch.zeros_like(u)
    s.apply(u, ref)
    ext = [torch.zeros(q.n_ext, **f64) for q in parts]
    out = [torch.zeros(q.n_ext, **f64) for q in parts]
    comm.halo([u[q.global_own_slice()].clone() for q in parts], ext)
    for q, e, o, b in zip(parts, ext, out, be):
        b.apply(e, o)
        d = (o[q.own_slice()] - ref[q.global_own_slice()]).abs().max()
        assert float(d) <= 1e-12 * float(ref.abs().max())
    F = [Fd[q.global_own_slice()].clone() for q in parts]
    U, rr, nit = slab.slab_pcg(parts, be, comm, F, 1e-10, 1000)
    assert rr < 1e-10 and nit < 1000
    got = torch.cat(U)
    assert float(torch.linalg.norm(got - U1)) <= 1e-7 * float(torch.linalg.norm(U1))
