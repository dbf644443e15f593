"""Host-side check of the fine sweeps' Hadamard-basis operator (no GPU):
Ke = T' S T / 64 with S in the 45-entry pattern of eight constants, for every
isotropic cube element; anything else is refused (and then runs on the dense
element-row sweeps)."""
import numpy as np
import pytest

import gputo

_LX = [0, 1, 1, 0, 0, 1, 1, 0]
_LY = [0, 0, 1, 1, 0, 0, 1, 1]
_LZ = [0, 0, 0, 0, 1, 1, 1, 1]


def _T():
    T8 = np.array([[(-1) ** (((m >> 2) & 1) * _LX[b] + ((m >> 1) & 1) * _LY[b] + (m & 1) * _LZ[b])
                    for b in range(8)] for m in range(8)], float)
    return np.kron(T8, np.eye(3))


def _S_from(c):
    a, b, cc, d, e, f, g, h = c
    r = lambda m, k: 3 * m + k
    S = np.zeros((24, 24))
    for grp in ([(1, 0), (4, 2)], [(1, 1), (2, 2)], [(2, 0), (4, 1)]):
        for x in grp:
            for y in grp:
                S[r(*x), r(*y)] = a
    for grp, dg, off in (([(1, 2), (2, 1), (4, 0)], b, cc), ([(3, 0), (5, 1), (6, 2)], d, e)):
        for x in grp:
            for y in grp:
                S[r(*x), r(*y)] = dg if x == y else off
    for grp in ([(3, 1), (5, 0)], [(3, 2), (6, 0)], [(5, 2), (6, 1)]):
        for x in grp:
            for y in grp:
                S[r(*x), r(*y)] = f if x == y else g
    for k in range(3):
        S[r(7, k), r(7, k)] = h
    return S


@pytest.mark.parametrize("nu,h", [(0.3, 1.0), (0.25, 1.0), (0.45, 1.0), (0.3, 2.0), (0.0, 0.5)])
def test_cube_elements_have_the_pattern(nu, h):
    Ke = gputo.hex8_stiffness(nu, h)
    c = gputo.fine_op_constants(Ke)
    assert c is not None
    T = _T()
    back = T.T @ _S_from(c) @ T / 64.0
    assert np.abs(back - Ke).max() <= 1e-13 * np.abs(Ke).max()


def test_other_matrices_are_refused():
    Ke = gputo.hex8_stiffness(0.3)
    rng = np.random.default_rng(0)
    P = rng.standard_normal((24, 24)) * 1e-6
    assert gputo.fine_op_constants(Ke + P + P.T) is None
    # anisotropic scaling of the y displacement breaks the cubic symmetry
    D = np.diag(np.tile([1.0, 1.5, 1.0], 8))
    assert gputo.fine_op_constants(D @ Ke @ D) is None
    assert gputo.fine_op_constants(np.zeros((24, 24))) is None


def test_options_default_and_validation():
    o = gputo.default_options()
    assert o.fine_op == 0
