"""Element contraction on the tensor cores (tcgen05) against the FP64 path.

gputo_compliance_sens_tc_dev computes ce_e = u_e^T Ke u_e (the sensitivity
line of top3D125modCuda.m:139) as BF16-split tensor-core MMAs with FP32
accumulation.  Its accuracy is FP32's: every ce within 1e-6 of the largest,
compliance within 1e-6 relative, the tolerance the mixed-precision solve
is held to.
"""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

RTOL = 1e-6


def _dev(a):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")


def _compare(gputo, Ke0, U, x, shape):
    import torch
    nel = shape[0] * shape[1] * shape[2]
    CX = 1e-9 + x ** 3 * (1 - 1e-9)
    dsK = -3 * (1 - 1e-9) * x ** 2
    Ud, CXd, dsKd = _dev(U), _dev(CX), _dev(dsK)
    ce_ref, dc_ref = torch.empty(nel, dtype=torch.float64, device="cuda"), torch.empty_like(CXd)
    c_ref = gputo.compliance_sens_dev(Ke0, Ud, CXd, dsKd, *shape, ce_ref, dc_ref)
    ce = torch.full((nel,), float("nan"), dtype=torch.float64, device="cuda")
    dc = torch.full_like(ce, float("nan"))
    c = gputo.compliance_sens_tc_dev(Ke0, Ud, CXd, dsKd, *shape, ce, dc)
    ce, dc, ce_ref, dc_ref = (t.cpu().numpy() for t in (ce, dc, ce_ref, dc_ref))
    assert np.isfinite(ce).all() and np.isfinite(dc).all()
    assert np.abs(ce - ce_ref).max() <= RTOL * np.abs(ce_ref).max()
    assert np.abs(dc - dc_ref).max() <= RTOL * np.abs(dc_ref).max()
    assert abs(c - c_ref) <= RTOL * abs(c_ref)
    return ce, ce_ref


def test_tc_energy_on_a_solved_field(oracle, gputo):
    d = load_golden("solve_32x16x16_unif_nl4")
    U = d["U"].copy()
    U[1::3] *= -1   # solver frame
    x = np.random.default_rng(11).uniform(0.05, 1.0, 32 * 16 * 16)
    _compare(gputo, gputo.hex8_stiffness(), U, x, (32, 16, 16))


@pytest.mark.parametrize("shape", [(7, 5, 3), (48, 24, 20), (13, 11, 9)])
def test_tc_energy_ragged_tiles(gputo, shape):
    """Element counts that leave the last 128-element tile partly empty."""
    rng = np.random.default_rng(sum(shape))
    ndof = 3 * (shape[0] + 1) * (shape[1] + 1) * (shape[2] + 1)
    nel = shape[0] * shape[1] * shape[2]
    _compare(gputo, gputo.hex8_stiffness(), rng.standard_normal(ndof), rng.uniform(0.05, 1, nel), shape)


def test_tc_energy_other_poisson_ratio(gputo):
    """Ke is an argument: a different element matrix must flow through."""
    shape = (16, 8, 8)
    rng = np.random.default_rng(3)
    Ke = gputo.hex8_stiffness(nu=0.2)
    ndof = 3 * 17 * 9 * 9
    _compare(gputo, Ke, rng.standard_normal(ndof), rng.uniform(0.05, 1, 16 * 8 * 8), shape)
