"""Parity of the CUDA solver path with the oracle and the reference's golden
solves, through the C ABI.  Needs a B200.

Tolerances: FP64 operator / preconditioner applies agree with the oracle to
1e-12 relative (only summation order differs); FP64 solves at the same
tolerance agree to 1e-9 relative in U with the same iteration count;
mixed-precision solves agree with an FP64 solve to 1e-10 within 1e-6 in
compliance and relative displacement L2, at tol 1e-8 on a small grid and at
tol 1e-6 (the benchmark's tolerance) on the 256x128x128 benchmark workload.
"""
import numpy as np
import pytest
from conftest import load_golden

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as T
    assert T.cuda.is_available(), "GPU tests need a CUDA device"
    return T


def _problem(O, d):
    return O.Problem(int(d["nelx"]), int(d["nely"]), int(d["nelz"]), d["F"], d["fixed"])


def _dev(torch, a):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")


def _solver(gputo, p, nl, CX_dev, **opt):
    s = gputo.Solver(p.nelx, p.nely, p.nelz, nl, gputo.default_options(**opt))
    s.set_problem(p.Ke0, p.fixed)
    s.setup(CX_dev)
    return s


@pytest.mark.parametrize("shape,nl", [((16, 8, 8), 3), ((34, 18, 10), 2), ((64, 32, 32), 4),
                                      ((8, 40, 6), 2)])
def test_apply_matches_oracle(oracle, gputo, torch, shape, nl):
    p = oracle.cantilever(*shape)
    rng = np.random.default_rng(1)
    CX = oracle.simp(rng.uniform(0.01, 1.0, p.nel))[0]
    u = rng.standard_normal(p.ndof)
    s = _solver(gputo, p, nl, _dev(torch, CX))
    r = torch.zeros(p.ndof, dtype=torch.float64, device="cuda")
    s.apply(_dev(torch, u), r)
    ref = oracle.apply_fine(p, CX, u)
    ref[p.fixed.astype(np.int64) - 1] = 0.0
    got = r.cpu().numpy()
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()


@pytest.mark.parametrize("shape,nl", [((16, 8, 8), 3), ((32, 16, 16), 4), ((24, 8, 16), 4)])
def test_vcycle_matches_oracle(oracle, gputo, torch, shape, nl):
    p = oracle.cantilever(*shape)
    rng = np.random.default_rng(2)
    CX = oracle.simp(oracle.random_density(*shape, seed=4))[0]
    r = rng.standard_normal(p.ndof)
    r[p.fixed.astype(np.int64) - 1] = 0.0
    s = _solver(gputo, p, nl, _dev(torch, CX))
    z = torch.zeros(p.ndof, dtype=torch.float64, device="cuda")
    s.vcycle(_dev(torch, r), z)
    ref = oracle.vcycle(p, CX, nl, r)
    got = z.cpu().numpy()
    assert np.abs(got - ref).max() <= 1e-10 * np.abs(ref).max()


@pytest.mark.parametrize("name", ["solve_16x8x8_rand_nl3", "solve_32x16x16_unif_nl4",
                                  "solve_16x8x8_maxit3_nl2", "solve_16x8x8_bridge_nl3"])
def test_mex_entry_matches_reference_golden(oracle, gputo, name):
    """gputo.mgcg1 (the MEX call layout, host buffers) vs the compiled reference."""
    d = load_golden(name)
    p = _problem(oracle, d)
    U = np.full(p.ndof, 7.0)  # input values must be ignored
    rr, nit = gputo.mgcg1(p.Ke0, p.F, U, d["CX"], p.fixed, len(p.fixed), p.nelx, p.nely, p.nelz,
                          int(d["nl"]), float(d["tol"]), int(d["maxit"]), printLev=0)
    assert nit == int(d["nit"])
    assert abs(rr - float(d["relres"])) <= 1e-6 * float(d["relres"])
    assert np.linalg.norm(U - d["U"]) <= 1e-9 * np.linalg.norm(d["U"])


def test_corner_supports_converged_solution(oracle, gputo):
    d = load_golden("solve_16x8x8_corner_nl3")
    p = _problem(oracle, d)
    U = np.zeros(p.ndof)
    rr, nit = gputo.mgcg1(p.Ke0, p.F, U, d["CX"], p.fixed, len(p.fixed), 16, 8, 8, 3, 1e-8, 200,
                          printLev=0)
    Uo, rro, nito = oracle.mgcg1(p, d["CX"], 3, 1e-8, 200)
    assert nit == nito and rr < 1e-8
    assert np.linalg.norm(U - Uo) <= 1e-9 * np.linalg.norm(Uo)
    assert np.linalg.norm(U - d["U"]) <= 1e-6 * np.linalg.norm(d["U"])


def test_cantilever_64x32x32_first_solve(oracle, gputo):
    d = load_golden("solve_c1_first")
    p = oracle.cantilever(64, 32, 32)
    CX = oracle.simp(np.full(p.nel, 0.12))[0]
    U = np.zeros(p.ndof)
    rr, nit = gputo.mgcg1(p.Ke0, p.F, U, CX, p.fixed, len(p.fixed), 64, 32, 32, 4, 1e-8, 200,
                          printLev=0)
    assert nit == int(d["nit"])
    assert abs(p.F @ U - float(d["compliance"])) <= 1e-9 * float(d["compliance"])
    s = d["sample"]
    assert np.linalg.norm(U[s] - d["U_sample"]) <= 1e-9 * np.linalg.norm(d["U_sample"])


def test_mex_gateway_through_mexfunction(oracle, gputo):
    from test_capi import _load_mex, call_mex
    mex, _ = _load_mex()
    d = load_golden("solve_16x8x8_rand_nl3")
    p = _problem(oracle, d)
    U = np.zeros(p.ndof)
    # 12-argument cantilever form (printLev absent)
    res, it = call_mex(mex, [p.Ke0.reshape(-1).copy(), p.F, U, d["CX"], p.fixed, len(p.fixed),
                             16, 8, 8, 3, 1e-8, 200])
    assert it == int(d["nit"])
    assert np.linalg.norm(U - d["U"]) <= 1e-9 * np.linalg.norm(d["U"])
    # 13-argument form, printLev = 0
    U2 = np.zeros(p.ndof)
    res2, it2 = call_mex(mex, [p.Ke0.reshape(-1).copy(), p.F, U2, d["CX"], p.fixed, len(p.fixed),
                               16, 8, 8, 3, 1e-8, 200, 0])
    assert it2 == it and np.array_equal(U, U2)


def test_repeated_calls_are_deterministic(oracle, gputo):
    d = load_golden("solve_32x16x16_unif_nl4")
    p = _problem(oracle, d)
    outs = []
    for _ in range(3):
        U = np.zeros(p.ndof)
        gputo.mgcg1(p.Ke0, p.F, U, d["CX"], p.fixed, len(p.fixed), 32, 16, 16, 4, 1e-8, 200,
                    printLev=0)
        outs.append(U)
    assert np.array_equal(outs[0], outs[1]) and np.array_equal(outs[1], outs[2])


def test_graph_and_eager_agree(oracle, gputo):
    d = load_golden("solve_16x8x8_rand_nl3")
    p = _problem(oracle, d)
    res = []
    for g in (0, 1):
        U = np.zeros(p.ndof)
        rr, nit = gputo.mgcg1(p.Ke0, p.F, U, d["CX"], p.fixed, len(p.fixed), 16, 8, 8, 3, 1e-8, 200,
                              printLev=0, options=gputo.default_options(use_graph=g, check_every=3))
        res.append((U, nit))
    assert res[0][1] == res[1][1] == int(d["nit"])
    assert np.array_equal(res[0][0], res[1][0])


def test_mixed_precision_matches_fp64_oracle(oracle, gputo):
    """FP32 V-cycle + flexible FP64 outer PCG, tol 1e-8 on a 32x16x16 random
    design: compliance and displacement within 1e-6 of the FP64 oracle solved
    to 1e-10."""
    p = oracle.cantilever(32, 16, 16)
    CX = oracle.simp(oracle.random_density(32, 16, 16, seed=9))[0]
    Uo, _, _ = oracle.mgcg1(p, CX, 4, 1e-10, 400)
    U = np.zeros(p.ndof)
    rr, nit = gputo.mgcg1(p.Ke0, p.F, U, CX, p.fixed, len(p.fixed), 32, 16, 16, 4, 1e-8, 400,
                          printLev=0, options=gputo.default_options(precision=gputo.PREC_MIXED))
    assert rr < 1e-8 and nit > 0
    assert abs(p.F @ U - p.F @ Uo) <= 1e-6 * abs(p.F @ Uo)
    assert np.linalg.norm(U - Uo) <= 1e-6 * np.linalg.norm(Uo)


def test_compliance_sensitivity_matches_oracle(oracle, gputo):
    d = load_golden("solve_32x16x16_unif_nl4")
    p = _problem(oracle, d)
    U = d["U"]  # MATLAB frame, as the MEX returns it
    xphys = np.random.default_rng(4).uniform(0.05, 1.0, p.nel)
    CX, dsK = oracle.simp(xphys)
    ce, dc, c = gputo.compliance_sens(p.Ke0, U, CX, dsK, 32, 16, 16)
    Uc = U.copy()
    Uc[1::3] *= -1  # back to the solver frame
    ce_ref = oracle.element_energy(p, Uc)
    assert np.abs(ce - ce_ref).max() <= 1e-12 * np.abs(ce_ref).max()
    assert np.abs(dc - dsK * ce_ref).max() <= 1e-12 * np.abs(dsK * ce_ref).max()
    assert abs(c - CX @ ce_ref) <= 1e-12 * abs(CX @ ce_ref)


@pytest.mark.parametrize("ke", ["cube", "perturbed"])
def test_element_energy_both_element_paths(oracle, gputo, torch, ke):
    """The cube element's Ke runs the energy pass in its Hadamard basis; a Ke
    without that pattern (a symmetric perturbation) runs the dense 24x24
    product.  Both against the oracle with the same Ke, on a grid with
    several CTAs per x plane and ragged ends."""
    nelx, nely, nelz = 20, 37, 11
    p = oracle.cantilever(nelx, nely, nelz)
    rng = np.random.default_rng(31)
    if ke == "perturbed":
        E = rng.standard_normal((24, 24)) * 1e-3
        p.Ke0 = p.Ke0 + E + E.T
    U = rng.standard_normal(p.ndof)
    CX, dsK = oracle.simp(rng.uniform(0.05, 1.0, p.nel))
    ce, dc = torch.empty(p.nel, dtype=torch.float64, device="cuda"), \
        torch.empty(p.nel, dtype=torch.float64, device="cuda")
    c = gputo.compliance_sens_dev(p.Ke0, _dev(torch, U), _dev(torch, CX), _dev(torch, dsK), nelx, nely, nelz,
                                  ce, dc)
    ce_ref = oracle.element_energy(p, U)
    ce, dc = ce.cpu().numpy(), dc.cpu().numpy()
    assert np.abs(ce - ce_ref).max() <= 1e-12 * np.abs(ce_ref).max()
    assert np.abs(dc - dsK * ce_ref).max() <= 1e-12 * np.abs(dsK * ce_ref).max()
    assert abs(c - CX @ ce_ref) <= 1e-12 * abs(CX @ ce_ref)


@pytest.mark.parametrize("rmin", [3 ** 0.5, 2 * 3 ** 0.5, 1.2, 2.5, 4.5, 0.9])
@pytest.mark.parametrize("shape", [(20, 12, 10), (70, 40, 19), (5, 33, 9)])
def test_density_filter_matches_oracle(oracle, gputo, rmin, shape):
    """The shared-memory tiled filter (plane-decomposed for stencil radius
    1-3, direct above) against the oracle's imfilter restatement: radii 1
    (rmin sqrt 3), 2, 3 (rmin 2 sqrt 3, the drivers' value), 0 and 4; grids
    with one tile, several y / z tiles and x chunks, and fewer x planes than
    the stencil is wide (the API needs more elements than the radius in each
    direction)."""
    nelx, nely, nelz = shape
    rng = np.random.default_rng(5)
    x = rng.random(nelx * nely * nelz)
    dv = rng.uniform(0.5, 2.0, x.size)
    out, hs = oracle.filter3d(x, nelx, nely, nelz, rmin)
    got = gputo.density_filter(x, nelx, nely, nelz, rmin, normalize=True)
    tol = 1e-14 if rmin < 2 else 1e-13   # sums of up to 9^3 terms in another order
    assert np.abs(got - out / hs).max() <= tol
    out2, _ = oracle.filter3d(x / dv, nelx, nely, nelz, rmin)
    got2 = gputo.density_filter(x, nelx, nely, nelz, rmin, divisor=dv, normalize=False)
    assert np.abs(got2 - out2).max() <= 1e-13 * np.abs(out2).max()


def test_bad_arguments_return_status(oracle, gputo):
    p = oracle.cantilever(16, 8, 8)
    CX = np.ones(p.nel)
    U = np.zeros(p.ndof)
    with pytest.raises(gputo.GputoError) as e:  # nl does not divide the grid
        gputo.mgcg1(p.Ke0, p.F, U, CX, p.fixed, len(p.fixed), 16, 8, 8, 5, 1e-8, 10, printLev=0)
    assert e.value.status == gputo.GPUTO_ERR_ARG
    bad = p.fixed.copy()
    bad[3] = p.ndof + 1.0  # out-of-range fixed dof
    with pytest.raises(gputo.GputoError) as e:
        gputo.mgcg1(p.Ke0, p.F, U, CX, bad, len(bad), 16, 8, 8, 3, 1e-8, 10, printLev=0)
    assert e.value.status == gputo.GPUTO_ERR_ARG
    # the context stays usable after errors
    rr, nit = gputo.mgcg1(p.Ke0, p.F, U, CX, p.fixed, len(p.fixed), 16, 8, 8, 3, 1e-8, 200, printLev=0)
    assert rr < 1e-8


def test_nonpositive_coarse_matrix_reports_not_spd(oracle, gputo):
    p = oracle.cantilever(8, 4, 4)
    CX = -np.ones(p.nel)  # negative stiffness: the coarsest Cholesky must refuse it
    U = np.zeros(p.ndof)
    with pytest.raises(gputo.GputoError) as e:
        gputo.mgcg1(p.Ke0, p.F, U, CX, p.fixed, len(p.fixed), 8, 4, 4, 2, 1e-8, 10, printLev=0)
    assert e.value.status == gputo.GPUTO_ERR_NOT_SPD


def test_zero_load_returns_zero(oracle, gputo):
    p = oracle.cantilever(8, 4, 4)
    U = np.ones(p.ndof)
    rr, nit = gputo.mgcg1(p.Ke0, np.zeros(p.ndof), U, np.ones(p.nel), p.fixed, len(p.fixed), 8, 4,
                          4, 2, 1e-8, 10, printLev=0)
    assert nit == 0 and np.all(U == 0)


def test_log_file_written_like_the_mex(oracle, gputo, tmp_path):
    p = oracle.cantilever(8, 4, 4)
    U = np.zeros(p.ndof)
    gputo.mgcg1(p.Ke0, p.F, U, np.ones(p.nel), p.fixed, len(p.fixed), 8, 4, 4, 2, 1e-8, 50,
                printLev=1)
    text = (tmp_path / "mgcg1.log").read_text()
    assert "MGCG Initial residual" in text and "Final residual" in text


def test_simp_and_oc_match_oracle(oracle, gputo, torch):
    rng = np.random.default_rng(8)
    n = 50000
    x = rng.uniform(0.0, 1.0, n)
    CX, dsK = oracle.simp(x)
    xd = _dev(torch, x)
    cxd, dsd = torch.empty_like(xd), torch.empty_like(xd)
    gputo.simp_dev(xd, cxd, dsd)
    assert np.abs(cxd.cpu().numpy() - CX).max() <= 1e-15
    assert np.abs(dsd.cpu().numpy() - dsK).max() <= 1e-14
    xo = rng.uniform(0.01, 0.4, n)
    dc = -rng.uniform(1e-3, 3.0, n)
    dv = np.full(n, 1.0 / n / 0.12)
    xn_ref, lm_ref = oracle.oc_update(xo, dc, dv, 0.12, 0.2)
    xn, lm = gputo.oc_update(xo, dc, dv, 0.12, 0.2)
    assert abs(lm - lm_ref) <= 1e-12 * lm_ref
    assert np.abs(xn - xn_ref).max() <= 1e-12


def test_design_loop_64x32x32_matches_golden(oracle, gputo, torch):
    """50 OC iterations of the 64x32x32 cantilever entirely on the GPU (FP64
    MGCG at tol 1e-8, device filter / sensitivity / OC) against the golden
    history produced with the reference's own solver: design within 1e-4
    max-abs, compliance history within 1e-6."""
    d = load_golden("design_c1")
    F, fixed = gputo.cantilever(64, 32, 32)
    dl = gputo.DesignLoop(64, 32, 32, 4, F, fixed, gputo.hex8_stiffness(), volfrac=0.12, rmin=3 ** 0.5,
                          tol=1e-8, maxit=200)
    cs, nits = [], []
    for _ in range(50):
        info = dl.step()
        cs.append(info["c"])
        nits.append(info["nit"])
    xphys = dl.xPhys.cpu().numpy()
    assert np.abs(xphys - d["xPhys"].astype(np.float64)).max() <= 1e-4
    np.testing.assert_allclose(cs, d["c"], rtol=1e-6)
    assert max(abs(a - b) for a, b in zip(nits, d["nit"])) <= 1


def test_host_calls_reuse_their_workspace(oracle, gputo):
    """The host-array entry points keep device buffers and pinned staging
    between calls: a large call, a smaller one, then the large one again
    (sizes above one 8 MB staging chunk, so several chunks are in flight)
    each match the oracle."""
    rng = np.random.default_rng(11)
    for shape in [(128, 64, 64), (16, 8, 8), (128, 64, 64)]:
        nelx, nely, nelz = shape
        nel = nelx * nely * nelz
        x = rng.uniform(0.05, 1.0, nel)
        out = gputo.density_filter(x, nelx, nely, nelz, 3 ** 0.5)
        ref, hs = oracle.filter3d(x, nelx, nely, nelz, 3 ** 0.5)
        assert np.abs(out - ref / hs).max() <= 1e-12
        p = oracle.cantilever(*shape)
        U = rng.standard_normal(p.ndof)
        CX, dsK = oracle.simp(x)
        ce, dc, c = gputo.compliance_sens(p.Ke0, U, CX, dsK, nelx, nely, nelz)
        Uc = U.copy()
        Uc[1::3] *= -1
        ce_ref = oracle.element_energy(p, Uc)
        assert np.abs(ce - ce_ref).max() <= 1e-12 * np.abs(ce_ref).max()
        assert abs(c - CX @ ce_ref) <= 1e-12 * abs(CX @ ce_ref)
        dv = np.full(nel, 1.0 / nel)
        xn, lm = gputo.oc_update(x, -np.abs(dc), dv, 0.3, 0.2)
        xr, lr = oracle.oc_update(x, -np.abs(dc), dv, 0.3, 0.2)
        assert abs(lm - lr) <= 1e-12 * abs(lr) and np.abs(xn - xr).max() <= 1e-12


def test_host_calls_write_into_caller_arrays(oracle, gputo):
    """out= (arrays a design loop allocates once): the same values as the
    allocating forms, bit for bit, also when the output is the input array
    (inputs reach the device before any output is written)."""
    rng = np.random.default_rng(13)
    nelx, nely, nelz = 64, 32, 32
    nel = nelx * nely * nelz
    p = oracle.cantilever(nelx, nely, nelz)
    x = rng.uniform(0.05, 1.0, nel)
    U = rng.standard_normal(p.ndof)
    outs = {k: np.full(nel, np.nan) for k in ("f", "CX", "dsK", "ce", "dc", "xn")}
    f = gputo.density_filter(x, nelx, nely, nelz, 3 ** 0.5)
    assert gputo.density_filter(x, nelx, nely, nelz, 3 ** 0.5, out=outs["f"]) is outs["f"]
    assert np.array_equal(outs["f"], f)
    CX, dsK = gputo.simp(f, 3.0, 1.0, 1e-9)
    gputo.simp(f, 3.0, 1.0, 1e-9, out=(outs["CX"], outs["dsK"]))
    assert np.array_equal(outs["CX"], CX) and np.array_equal(outs["dsK"], dsK)
    ce, dc, c = gputo.compliance_sens(p.Ke0, U, CX, dsK, nelx, nely, nelz)
    _, _, c2 = gputo.compliance_sens(p.Ke0, U, CX, dsK, nelx, nely, nelz, out=(outs["ce"], outs["dc"]))
    assert np.array_equal(outs["ce"], ce) and np.array_equal(outs["dc"], dc) and c2 == c
    dv = np.full(nel, 1.0 / nel)
    xn, lm = gputo.oc_update(x, -np.abs(dc), dv, 0.3, 0.2)
    _, lm2 = gputo.oc_update(x, -np.abs(dc), dv, 0.3, 0.2, out=outs["xn"])
    assert np.array_equal(outs["xn"], xn) and lm2 == lm
    xa = x.copy()
    gputo.density_filter(xa, nelx, nely, nelz, 3 ** 0.5, out=xa)   # in place
    assert np.array_equal(xa, f)


def test_host_simp_matches_oracle(oracle, gputo):
    x = np.random.default_rng(12).uniform(0.0, 1.0, 3 * 10 ** 6 + 7)   # several staging chunks
    CX, dsK = gputo.simp(x, 3.0, 1.0, 1e-9)
    CXr, dsr = oracle.simp(x)
    assert np.abs(CX - CXr).max() <= 1e-15 and np.abs(dsK - dsr).max() <= 1e-14


def _bench_design_cx(gputo, torch, nelx, nely, nelz):
    """The benchmark's design (the 64x32x32 golden design after 50 OC
    iterations, upsampled), filtered and through SIMP, on the device."""
    d = load_golden("design_c1")
    x = d["x"].astype(np.float64).reshape(64, 32, 32)   # (x, z, y) element order
    f = nelx // 64
    xb = np.repeat(np.repeat(np.repeat(x, f, 0), f, 1), f, 2).reshape(-1)
    xd = _dev(torch, xb)
    xp = torch.empty_like(xd)
    gputo.density_filter_dev(xd, xp, nelx, nely, nelz, 3 ** 0.5)
    CX = torch.empty_like(xd)
    gputo.simp_dev(xp, CX)
    return CX


def test_mixed_precision_at_the_benchmark_configuration(gputo, torch):
    """The headline workload: 256x128x128 cantilever (12.8M dofs), 6 levels,
    the benchmark's mid-optimisation design.  The mixed-precision solve at
    the benchmark tolerance 1e-6 against an FP64 solve to 1e-10: compliance
    and relative displacement L2 within 1e-6, and the true residual of the
    mixed U (an independent FP64 apply) within 2e-6 (the solve stops on the
    recursively updated residual, mgcg1.cu:254-275)."""
    nelx, nely, nelz, nl = 256, 128, 128, 6
    CX = _bench_design_cx(gputo, torch, nelx, nely, nelz)
    F, fixed = gputo.cantilever(nelx, nely, nelz)
    Fd = _dev(torch, F)
    s64 = gputo.Solver(nelx, nely, nelz, nl, gputo.default_options())
    s64.set_problem(gputo.hex8_stiffness(), fixed)
    s64.setup(CX)
    U64 = torch.zeros_like(Fd)
    rr64, nit64 = s64.solve(Fd, U64, 1e-10, 1000)
    assert rr64 < 1e-10
    sm = gputo.Solver(nelx, nely, nelz, nl, gputo.default_options(precision=gputo.PREC_MIXED))
    sm.set_problem(gputo.hex8_stiffness(), fixed)
    sm.setup(CX)
    Um = torch.zeros_like(Fd)
    rrm, nitm = sm.solve(Fd, Um, 1e-6, 500)
    assert rrm < 1e-6 and 0 < nitm < 500
    del sm
    KU = torch.zeros_like(Fd)
    s64.apply(Um, KU)
    true_rr = float(torch.linalg.norm(Fd - KU) / torch.linalg.norm(Fd))
    c64, cm = float(Fd @ U64), float(Fd @ Um)
    u_err = float(torch.linalg.norm(Um - U64) / torch.linalg.norm(U64))
    assert abs(cm - c64) <= 1e-6 * abs(c64), (cm, c64)
    assert u_err <= 1e-6, u_err
    assert true_rr <= 2e-6, true_rr
