"""The periodic homogenization oracle (oracle/homog.py) against known answers.

The reference has no homogenization of a unit cell (its Homogenization
directory is a self-weight problem, Homogenization/QNC/QNC_V1_mod1m.m:180-199),
so the oracle is pinned by closed forms instead of golden vectors:
 * a uniform cell: C_eff = CX D, with the fluctuations zero;
 * a laminate of layers normal to x (each layer whole elements thick): the
   closed-form laminate tensor, which the hex8 space reproduces exactly;
 * any cell: symmetric, between the Reuss and Voigt bounds.
"""
import numpy as np
import pytest


@pytest.fixture(scope="module")
def H(oracle):
    import homog
    return homog


def test_uniform_cell_gives_the_scaled_isotropic_tensor(oracle, H):
    Ke = oracle.hex8_stiffness(0.3)
    C, chi = H.homogenize(4, 6, 4, np.full(96, 0.7), Ke)
    assert np.abs(C - 0.7 * H.isotropic_D(0.3)).max() <= 1e-13
    assert np.abs(chi).max() <= 1e-12


@pytest.mark.parametrize("layers", [(2, 2), (1, 3), (3, 1)])
def test_laminate_matches_the_closed_form(oracle, H, layers):
    Ke = oracle.hex8_stiffness(0.3)
    a, b = layers
    nx, ny, nz = 2 * (a + b), 4, 2
    i = np.arange(nx)[:, None, None] * np.ones((1, nz, ny))
    CX = np.where((i % (a + b)) < a, 1.0, 0.05).reshape(-1)
    C, _ = H.homogenize(nx, ny, nz, CX, Ke)
    Cl = H.laminate([1.0, 0.05], [a / (a + b), b / (a + b)])
    assert np.abs(C - Cl).max() <= 1e-12 * np.abs(Cl).max()


def test_random_cell_is_symmetric_and_within_the_bounds(oracle, H):
    Ke = oracle.hex8_stiffness(0.3)
    x = np.random.default_rng(3).uniform(1e-3, 1.0, 6 * 6 * 6)
    CX = oracle.simp(x)[0]
    C, _ = H.homogenize(6, 6, 6, CX, Ke)
    V, R = H.voigt_reuss(CX)
    assert np.abs(C - C.T).max() <= 1e-14
    assert np.linalg.eigvalsh(V - C).min() >= 0
    assert np.linalg.eigvalsh(C - R).min() >= 0


def test_periodic_operator_has_only_the_translations_as_null_space(oracle, H):
    Ke = oracle.hex8_stiffness(0.3)
    K = H.assemble(3, 2, 2, np.random.default_rng(1).uniform(0.2, 1.0, 12), Ke).toarray()
    w = np.linalg.eigvalsh(K)
    assert np.sum(np.abs(w) < 1e-10 * w.max()) == 3
