"""Failure paths of the solver, provoked from the host, through the C ABI.

Nothing here faults, traps or hangs the GPU.  Each case makes one check of
the solver report an error and then shows that the same solver (and the
CUDA context) still gives correct results:

 * a non-finite right-hand side: the PCG start sees ||F|| = NaN and ends with
   GPUTO_ERR_BREAKDOWN; the MEX call returns cgiters = -1, the value the
   drivers test to stop their loop (top3D125modCuda.m:135).  The reference
   (mgcg1.cu:235-275) would iterate on NaNs up to cgmax;
 * a NaN element stiffness: it reaches the coarsest matrix through the
   Galerkin levels, and the coarsest Cholesky factor reports a non-positive
   pivot (GPUTO_ERR_NOT_SPD); the reference's choldc1 (mgcg1.cu:2099-2125)
   would exit the process;
 * a bounded wait that runs out: the test hook leaves one ring stage of the
   fine sweep armed with no copy in flight, so its mbarrier phase never
   completes; every wait gives up after 200 us, the sweep ends early and the
   apply reports GPUTO_ERR_TIMEOUT.  The reference has no bounded waits.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as T
    assert T.cuda.is_available(), "GPU tests need a CUDA device"
    return T


def _case(oracle, shape=(16, 8, 8), seed=3):
    p = oracle.cantilever(*shape)
    CX = oracle.simp(oracle.random_density(*shape, seed=seed))[0]
    return p, CX


@pytest.mark.parametrize("bad", [np.nan, np.inf])
def test_nonfinite_rhs_is_a_breakdown_and_the_solver_stays_usable(oracle, gputo, bad):
    p, CX = _case(oracle)
    Uo, _, nito = oracle.mgcg1(p, CX, 3, 1e-8, 200)
    for prec in (gputo.PREC_FP64, gputo.PREC_MIXED):
        opts = gputo.default_options(precision=prec)
        Fbad = p.F.copy()
        Fbad[-1] = bad
        U = np.zeros(p.ndof)
        rr, nit = gputo.mgcg1(p.Ke0, Fbad, U, CX, p.fixed, len(p.fixed), 16, 8, 8, 3, 1e-8, 200,
                              printLev=0, options=opts)
        assert nit == -1
        assert b"non-finite" in gputo.lib().gputo_last_error()
        # the same cached solver, the next call
        U2 = np.zeros(p.ndof)
        rr2, nit2 = gputo.mgcg1(p.Ke0, p.F, U2, CX, p.fixed, len(p.fixed), 16, 8, 8, 3, 1e-8, 200,
                                printLev=0, options=opts)
        assert rr2 < 1e-8 and nit2 > 0
        assert np.linalg.norm(U2 - Uo) <= 1e-6 * np.linalg.norm(Uo)


def test_nonfinite_rhs_through_mexfunction_gives_cgiters_minus_one(oracle, gputo):
    from test_capi import _load_mex, call_mex
    mex, _ = _load_mex()
    p, CX = _case(oracle)
    Fbad = p.F.copy()
    Fbad[-1] = np.nan
    U = np.zeros(p.ndof)
    res, it = call_mex(mex, [p.Ke0.reshape(-1).copy(), Fbad, U, CX, p.fixed, len(p.fixed), 16, 8, 8, 3,
                             1e-8, 200, 0])
    assert it == -1
    U2 = np.zeros(p.ndof)
    res2, it2 = call_mex(mex, [p.Ke0.reshape(-1).copy(), p.F, U2, CX, p.fixed, len(p.fixed), 16, 8, 8, 3,
                               1e-8, 200, 0])
    assert it2 > 0 and res2 < 1e-8


def test_solver_api_reports_breakdown_status(oracle, gputo, torch):
    p, CX = _case(oracle)
    f64 = dict(dtype=torch.float64, device="cuda")
    s = gputo.Solver(16, 8, 8, 3, gputo.default_options())
    s.set_problem(p.Ke0, p.fixed)
    s.setup(torch.as_tensor(CX, **f64))
    F = torch.as_tensor(p.F, **f64)
    F[-1] = float("nan")
    U = torch.zeros_like(F)
    with pytest.raises(gputo.GputoError) as e:
        s.solve(F, U, 1e-8, 200)
    assert e.value.status == gputo.GPUTO_ERR_BREAKDOWN
    F[-1] = float(p.F[-1])
    rr, nit = s.solve(F, U, 1e-8, 200)
    assert rr < 1e-8 and nit > 0


def test_nan_stiffness_is_caught_by_the_coarsest_factor(oracle, gputo):
    p, CX = _case(oracle)
    CXbad = CX.copy()
    CXbad[len(CX) // 2] = np.nan
    U = np.zeros(p.ndof)
    with pytest.raises(gputo.GputoError) as e:
        gputo.mgcg1(p.Ke0, p.F, U, CXbad, p.fixed, len(p.fixed), 16, 8, 8, 3, 1e-8, 200, printLev=0)
    assert e.value.status == gputo.GPUTO_ERR_NOT_SPD
    Uo, _, nito = oracle.mgcg1(p, CX, 3, 1e-8, 200)
    U2 = np.zeros(p.ndof)
    rr, nit = gputo.mgcg1(p.Ke0, p.F, U2, CX, p.fixed, len(p.fixed), 16, 8, 8, 3, 1e-8, 200, printLev=0)
    assert nit == nito and np.linalg.norm(U2 - Uo) <= 1e-9 * np.linalg.norm(Uo)


@pytest.mark.parametrize("prec,pairs", [("fp64", 0), ("fp32", 0), ("fp32", 1)])
def test_bounded_wait_runs_out_and_the_context_stays_usable(oracle, gputo, torch, prec, pairs):
    """pairs: the FP32 sweep variant (one or two element columns per lane)."""
    p, CX = _case(oracle, (32, 16, 16), seed=5)
    f64 = dict(dtype=torch.float64, device="cuda")
    mixed = prec == "fp32"
    s = gputo.Solver(32, 16, 16, 4, gputo.default_options(
        precision=gputo.PREC_MIXED if mixed else gputo.PREC_FP64, sweep_pairs=pairs))
    s.set_problem(p.Ke0, p.fixed)
    s.setup(torch.as_tensor(CX, **f64))
    u = torch.as_tensor(np.random.default_rng(6).standard_normal(p.ndof), **f64)
    apply = s.apply_fp32 if mixed else s.apply
    ok = torch.zeros_like(u)
    apply(u, ok)
    Fd = torch.as_tensor(p.F, **f64)
    U0 = torch.zeros_like(Fd)
    rr0, nit0 = s.solve(Fd, U0, 1e-8, 300)
    gputo.debug_set_sweep_fault(skip_stage=2, wait_us=200)
    try:
        r = torch.zeros_like(u)
        with pytest.raises(gputo.GputoError) as e:
            apply(u, r)
        assert e.value.status == gputo.GPUTO_ERR_TIMEOUT
    finally:
        gputo.debug_set_sweep_fault(-1, 0)
    again = torch.zeros_like(u)
    apply(u, again)
    assert torch.equal(again, ok)
    U = torch.zeros_like(Fd)
    rr, nit = s.solve(Fd, U, 1e-8, 300)
    assert rr0 < 1e-8 and (rr, nit) == (rr0, nit0)
    assert torch.equal(U, U0)   # the solver is deterministic: the same solve, bit for bit
