"""The periodic homogenization solve (gputo_homog_*) on the GPU against the
oracle (oracle/homog.py, a direct sparse solve) and the closed forms it is
pinned to.  Six load cases per launch, FP32 V-cycle, flexible FP64 PCG.

Tolerances: solves to relres 1e-10 give C_eff within 1e-8 (relative to its
largest entry) of the oracle and fluctuations within 1e-6; the laminate and
uniform cells match their closed forms to 1e-8."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as T
    assert T.cuda.is_available(), "GPU tests need a CUDA device"
    return T


@pytest.fixture(scope="module")
def H(oracle):
    import homog
    return homog


def _dev(torch, a):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")


@pytest.mark.parametrize("shape,nl", [((8, 8, 8), 2), ((12, 8, 4), 2), ((8, 12, 16), 3)])
def test_random_cell_matches_oracle(oracle, gputo, torch, H, shape, nl):
    nx, ny, nz = shape
    x = gputo.random_field_density(nx, ny, nz, seed=4, corr_len=3.0, lo=0.1, hi=1.0)
    CX = oracle.simp(x)[0]   # moduli from 1e-3 to 1
    Ke = oracle.hex8_stiffness(0.3)
    Co, chio = H.homogenize(nx, ny, nz, CX, Ke)
    h = gputo.Homog(nx, ny, nz, nl)
    chi = torch.zeros(18 * nx * ny * nz, dtype=torch.float64, device="cuda")
    C, rr, nit = h.solve(Ke, _dev(torch, CX), tol=1e-10, maxit=2000, chi=chi)
    assert (rr < 1e-10).all() and (nit > 0).all() and (nit < 2000).all()
    assert np.abs(C - Co).max() <= 1e-8 * np.abs(Co).max()
    got = chi.cpu().numpy().reshape(-1, 6)
    assert np.abs(got - chio).max() <= 1e-6 * max(np.abs(chio).max(), 1.0)


def test_laminate_and_uniform_cells_match_the_closed_forms(oracle, gputo, torch, H):
    Ke = oracle.hex8_stiffness(0.3)
    nx, ny, nz = 16, 8, 8
    i = np.arange(nx)[:, None, None] * np.ones((1, nz, ny))
    CX = np.where((i % 4) < 2, 1.0, 0.05).reshape(-1)
    h = gputo.Homog(nx, ny, nz, 3)
    C, rr, nit = h.solve(Ke, _dev(torch, CX), tol=1e-10, maxit=2000)
    Cl = H.laminate([1.0, 0.05], [0.5, 0.5])
    assert np.abs(C - Cl).max() <= 1e-8 * np.abs(Cl).max()
    C, rr, nit = h.solve(Ke, _dev(torch, np.full(nx * ny * nz, 0.3)), tol=1e-10, maxit=2000)
    assert np.abs(C - 0.3 * H.isotropic_D(0.3)).max() <= 1e-10


def test_random_field_cell_at_32_cubed_is_within_the_bounds(oracle, gputo, torch, H):
    """32^3 seeded Gaussian random field (correlation length 8 voxels) through
    a sigmoid to [1e-3, 1], SIMP moduli: every load case converges to 1e-6,
    C_eff is symmetric and lies between the Reuss and Voigt bounds, and a
    second solve gives the same tensor bit for bit (the graph replay is
    deterministic)."""
    n = 32
    x = gputo.random_field_density(n, n, n, seed=11, corr_len=8.0)
    CX = oracle.simp(x)[0]
    Ke = oracle.hex8_stiffness(0.3)
    h = gputo.Homog(n, n, n, 4)
    C, rr, nit = h.solve(Ke, _dev(torch, CX), tol=1e-6, maxit=2000)
    assert (rr < 1e-6).all(), (rr, nit)
    V, R = H.voigt_reuss(CX)
    assert np.abs(C - C.T).max() <= 1e-12 * np.abs(C).max()
    assert np.linalg.eigvalsh(V - C).min() >= 0
    assert np.linalg.eigvalsh(C - R).min() >= -1e-9 * np.abs(C).max()
    C2, rr2, nit2 = h.solve(Ke, _dev(torch, CX), tol=1e-6, maxit=2000)
    assert np.array_equal(C, C2) and np.array_equal(nit, nit2)
