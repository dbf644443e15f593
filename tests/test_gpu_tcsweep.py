"""Tensor-core fine-level smoother of the mixed-precision V-cycle.

The FP32 fine operator r = K u computed with tcgen05 MMAs (u and Ke split
into 1 or 2 BF16 parts, FP32 accumulation) is compared with the FP64 operator
(itself checked against the CPU oracle in test_gpu_solver.py), and mixed
solves that use the tensor-core smoother are compared with the FP64 oracle
solution at the tolerance every mixed-precision result is held to.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# relative L2 error of K u against FP64: one BF16 part per operand carries
# 8 significand bits (2^-9 rounding), two parts about 16
OP_TOL = {0: 1e-5, 1: 1e-2, 2: 1e-4}


def _dev(a):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")


@pytest.mark.parametrize("shape,nl", [((32, 16, 16), 3), ((64, 40, 24), 3), ((48, 24, 20), 3)])
def test_tc_operator_matches_fp64(oracle, gputo, shape, nl):
    """Ragged tiles in y (16, 40, 24 of 32) and z (20 of 8), several x chunks."""
    import torch
    p = oracle.cantilever(*shape)
    rng = np.random.default_rng(sum(shape))
    x = rng.uniform(0.05, 1.0, p.nel)
    CX, _ = oracle.simp(x)
    s = gputo.Solver(*shape, nl, gputo.default_options(precision=gputo.PREC_MIXED, tc_xchunk=7))
    s.set_problem(p.Ke0, p.fixed)
    s.setup(_dev(CX))
    u = _dev(rng.standard_normal(p.ndof))
    r64 = torch.empty_like(u)
    s.apply(u, r64)
    ref = r64.cpu().numpy()
    for parts, tol in OP_TOL.items():
        r = torch.full_like(u, float("nan"))
        s.apply_fp32(u, r, tc_parts=parts)
        got = r.cpu().numpy()
        assert np.isfinite(got).all(), parts
        err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
        assert err <= tol, (parts, err)
    s.close()


@pytest.mark.parametrize("parts", [1, 2])
def test_tc_smoother_solve_matches_oracle(oracle, gputo, parts):
    """Mixed solve with the tensor-core smoother, tol 1e-8: compliance and
    displacement within 1e-6 of the FP64 oracle solved to 1e-10."""
    p = oracle.cantilever(32, 16, 16)
    CX = oracle.simp(oracle.random_density(32, 16, 16, seed=9))[0]
    Uo, _, _ = oracle.mgcg1(p, CX, 4, 1e-10, 400)
    U = np.zeros(p.ndof)
    opts = gputo.default_options(precision=gputo.PREC_MIXED, tc_parts=parts)
    rr, nit = gputo.mgcg1(p.Ke0, p.F, U, CX, p.fixed, len(p.fixed), 32, 16, 16, 4, 1e-8, 400,
                          printLev=0, options=opts)
    assert rr < 1e-8 and nit > 0
    assert abs(p.F @ U - p.F @ Uo) <= 1e-6 * abs(p.F @ Uo)
    assert np.linalg.norm(U - Uo) <= 1e-6 * np.linalg.norm(Uo)


def test_tc_smoother_solve_larger_grid(oracle, gputo):
    """64x32x32 with a random SIMP design: TC-smoothed mixed solve against the
    FP64 GPU solve (several x chunks and z tiles)."""
    import torch
    shape, nl = (64, 32, 32), 4
    p = oracle.cantilever(*shape)
    x = np.random.default_rng(7).uniform(0.05, 1.0, p.nel)
    CX, _ = oracle.simp(x)
    res = {}
    for name, opts in [("fp64", gputo.default_options()),
                       ("tc2", gputo.default_options(precision=gputo.PREC_MIXED, tc_parts=2)),
                       ("tc1", gputo.default_options(precision=gputo.PREC_MIXED, tc_parts=1))]:
        U = np.zeros(p.ndof)
        rr, nit = gputo.mgcg1(p.Ke0, p.F, U, CX, p.fixed, len(p.fixed), *shape, nl, 1e-9, 300,
                              printLev=0, options=opts)
        assert rr < 1e-9, (name, rr, nit)
        res[name] = (U, nit)
    Uf = res["fp64"][0]
    for name in ("tc2", "tc1"):
        U = res[name][0]
        assert np.linalg.norm(U - Uf) <= 1e-6 * np.linalg.norm(Uf), name
        assert abs(p.F @ U - p.F @ Uf) <= 1e-6 * abs(p.F @ Uf), name
