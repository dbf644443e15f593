"""The bridge workload: supports on the two bottom corner strips and a uniform
top-face load (ArchBridge/1/top3D125modCudaBridge1.m:79-99), at parity sizes
against the oracle and at 512x256x256 (101.6M dofs, beyond the reference's
int workspace counter) through size-independent checks."""
import numpy as np
import pytest


@pytest.mark.parametrize("shape", [(8, 4, 4), (16, 8, 8), (12, 6, 10)])
def test_bridge_load_and_supports_match_oracle(oracle, gputo, shape):
    F, fixed = gputo.bridge(*shape)
    p = oracle.bridge(*shape)
    assert np.array_equal(fixed, p.fixed)
    assert np.abs(F - p.F).max() <= 1e-15
    # unit total load, downward only, none on a fixed dof
    assert abs(F.sum() + 1.0) <= 1e-12
    assert not F[0::3].any() and not F[1::3].any()
    assert not F[fixed.astype(np.int64) - 1].any()


@pytest.fixture(scope="module")
def torch():
    import torch as T
    assert T.cuda.is_available(), "GPU tests need a CUDA device"
    return T


@pytest.mark.gpu
def test_bridge_solve_matches_oracle(oracle, gputo):
    p = oracle.bridge(32, 16, 16)
    CX = oracle.simp(oracle.random_density(32, 16, 16, seed=5))[0]
    Uo, rro, nito = oracle.mgcg1(p, CX, 4, 1e-8, 300)
    U = np.zeros(p.ndof)
    rr, nit = gputo.mgcg1(p.Ke0, p.F, U, CX, p.fixed, len(p.fixed), 32, 16, 16, 4, 1e-8, 300,
                          printLev=0)
    assert nit == nito and rr < 1e-8
    assert np.linalg.norm(U - Uo) <= 1e-9 * np.linalg.norm(Uo)
    # mixed precision to 1e-8 against the same FP64 solution
    Um = np.zeros(p.ndof)
    rr, nit = gputo.mgcg1(p.Ke0, p.F, Um, CX, p.fixed, len(p.fixed), 32, 16, 16, 4, 1e-8, 300,
                          printLev=0, options=gputo.default_options(precision=gputo.PREC_MIXED))
    assert rr < 1e-8
    assert np.linalg.norm(Um - Uo) <= 1e-6 * np.linalg.norm(Uo)


@pytest.mark.gpu
def test_bridge_512x256x256_mixed(gputo, torch):
    """101.6M dofs on one device, mixed precision to 1e-6.  Checks that hold
    at any size: the true residual of the returned U (an independent FP64
    apply), and the mirror symmetries of the problem in x and y."""
    nelx, nely, nelz, nl = 512, 256, 256, 7
    F, fixed = gputo.bridge(nelx, nely, nelz)
    f64 = dict(dtype=torch.float64, device="cuda")
    Fd = torch.as_tensor(F, **f64)
    CX = torch.full((nelx * nely * nelz,), 1e-9 + 0.15 ** 3 * (1 - 1e-9), **f64)
    s = gputo.Solver(nelx, nely, nelz, nl, gputo.default_options(precision=gputo.PREC_MIXED))
    s.set_problem(gputo.hex8_stiffness(0.3), fixed)
    s.setup(CX)
    U = torch.zeros_like(Fd)
    rr, nit = s.solve(Fd, U, 1e-6, 500)
    assert 0 < nit < 500 and rr < 1e-6
    KU = torch.zeros_like(Fd)
    s.apply(U, KU)   # fixed rows come back zero, as F's do
    true_rr = float(torch.linalg.norm(Fd - KU) / torch.linalg.norm(Fd))
    assert true_rr < 2e-6
    c = float(Fd @ U)
    assert c > 0
    del KU, s
    u = U.view(nelx + 1, nelz + 1, nely + 1, 3)   # node (i, k, j), y fastest
    mx = torch.flip(u, dims=[0]) * torch.tensor([-1.0, 1.0, 1.0], **f64)
    my = torch.flip(u, dims=[2]) * torch.tensor([1.0, -1.0, 1.0], **f64)
    un = float(torch.linalg.norm(u))
    assert float(torch.linalg.norm(u - mx)) <= 1e-3 * un
    assert float(torch.linalg.norm(u - my)) <= 1e-3 * un
