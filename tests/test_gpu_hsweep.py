"""The fine sweeps with Ke in its Hadamard basis (fine_op = 0, the default)
against the oracle and against the dense element-row kernel (fine_op = 1).

Grid shapes exercise the kernel's tiling: clusters of 1 to 8 CTAs along y
(nely 40, 64, 96, 256) with and without the last node column on a CTA seam,
z tiles that overlap by one element, x chunks of 32 node planes with a short
last chunk, and nely = 264, which no cluster spans (the dense kernel runs).
Tolerances: FP64 1e-12 relative to the oracle's K u, 1e-13 between the two
kernels (summation order only); FP32 1e-5 relative between the two kernels."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SHAPES = [((34, 40, 10), 2), ((68, 64, 20), 3), ((8, 96, 14), 2), ((4, 256, 6), 2), ((2, 264, 2), 2),
          ((16, 8, 8), 2)]


@pytest.fixture(scope="module")
def torch():
    import torch as T
    assert T.cuda.is_available(), "GPU tests need a CUDA device"
    return T


def _dev(torch, a):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")


def _solver(gputo, p, CX, torch, nl=2, **opt):
    s = gputo.Solver(p.nelx, p.nely, p.nelz, nl, gputo.default_options(**opt))
    s.set_problem(p.Ke0, p.fixed)
    s.setup(_dev(torch, CX))
    return s


@pytest.mark.parametrize("shape,nl", SHAPES)
def test_fp64_apply_matches_oracle_and_dense(oracle, gputo, torch, shape, nl):
    p = oracle.cantilever(*shape)
    rng = np.random.default_rng(7)
    CX = oracle.simp(rng.uniform(0.01, 1.0, p.nel))[0]
    u = rng.standard_normal(p.ndof)
    ref = oracle.apply_fine(p, CX, u)
    ref[p.fixed.astype(np.int64) - 1] = 0.0
    out = {}
    for op in (0, 1):
        s = _solver(gputo, p, CX, torch, nl=nl, fine_op=op)
        r = torch.zeros(p.ndof, dtype=torch.float64, device="cuda")
        s.apply(_dev(torch, u), r)
        out[op] = r.cpu().numpy()
        s.close()
    scale = np.abs(ref).max()
    assert np.abs(out[0] - ref).max() <= 1e-12 * scale
    assert np.abs(out[0] - out[1]).max() <= 1e-13 * scale


@pytest.mark.parametrize("shape,nl", [((68, 64, 20), 3), ((34, 40, 10), 2), ((8, 96, 14), 2)])
def test_fp32_apply_matches_dense(oracle, gputo, torch, shape, nl):
    p = oracle.cantilever(*shape)
    rng = np.random.default_rng(8)
    CX = oracle.simp(rng.uniform(0.01, 1.0, p.nel))[0]
    u = rng.standard_normal(p.ndof)
    out = {}
    for op in (0, 1):
        s = _solver(gputo, p, CX, torch, nl=nl, precision=gputo.PREC_MIXED, fine_op=op)
        r = torch.zeros(p.ndof, dtype=torch.float64, device="cuda")
        s.apply_fp32(_dev(torch, u), r)
        out[op] = r.cpu().numpy()
        s.close()
    ref = oracle.apply_fine(p, CX, u)
    ref[p.fixed.astype(np.int64) - 1] = 0.0
    scale = np.abs(ref).max()
    assert np.abs(out[0] - out[1]).max() <= 1e-5 * scale
    assert np.abs(out[0] - ref).max() <= 1e-5 * scale


@pytest.mark.parametrize("shape,nl", [((48, 24, 24), 4), ((64, 64, 32), 4)])
def test_vcycle_and_solve_match_dense(oracle, gputo, torch, shape, nl):
    """Every sweep mode (pre-relaxation, Jacobi, defect, apply with its dot
    partials) inside FP64 V-cycles and PCG solves: the same iteration count
    and U to 1e-9 relative as the dense kernel."""
    p = oracle.cantilever(*shape)
    CX = oracle.simp(oracle.random_density(*shape, seed=5))[0]
    rng = np.random.default_rng(9)
    r = rng.standard_normal(p.ndof)
    r[p.fixed.astype(np.int64) - 1] = 0.0
    res = {}
    for op in (0, 1):
        s = _solver(gputo, p, CX, torch, nl=nl, fine_op=op)
        z = torch.zeros(p.ndof, dtype=torch.float64, device="cuda")
        s.vcycle(_dev(torch, r), z)
        U = torch.zeros(p.ndof, dtype=torch.float64, device="cuda")
        rr, nit = s.solve(_dev(torch, p.F), U, 1e-8, 300)
        res[op] = (z.cpu().numpy(), U.cpu().numpy(), nit, rr)
        s.close()
    z0, U0, n0, r0 = res[0]
    z1, U1, n1, r1 = res[1]
    assert np.abs(z0 - z1).max() <= 1e-11 * np.abs(z1).max()
    assert n0 == n1 and r0 < 1e-8
    assert np.linalg.norm(U0 - U1) <= 1e-9 * np.linalg.norm(U1)


def test_mixed_solve_matches_dense(oracle, gputo, torch):
    p = oracle.cantilever(64, 32, 32)
    CX = oracle.simp(oracle.random_density(64, 32, 32, seed=6))[0]
    res = {}
    for op in (0, 1):
        s = _solver(gputo, p, CX, torch, nl=4, precision=gputo.PREC_MIXED, fine_op=op)
        U = torch.zeros(p.ndof, dtype=torch.float64, device="cuda")
        rr, nit = s.solve(_dev(torch, p.F), U, 1e-8, 300)
        res[op] = (U.cpu().numpy(), nit, rr)
        s.close()
    assert abs(res[0][1] - res[1][1]) <= 1 and res[0][2] < 1e-8
    assert np.linalg.norm(res[0][0] - res[1][0]) <= 1e-6 * np.linalg.norm(res[1][0])


@pytest.mark.parametrize("shape,nl", SHAPES + [((72, 36, 20), 3)])
def test_energy_fused_into_the_apply_matches_the_separate_pass(oracle, gputo, torch, shape, nl):
    """gputo_solver_energy_dev: ce, dc and the compliance from one FP64 apply
    of the solution (each element written by exactly one CTA, although x
    chunks overlap by one element and z tiles by one row), against the
    separate energy pass (gputo_compliance_sens_dev) to 1e-12, and its true
    residual against |F - K U| from the plain apply.  nely = 264 runs the
    dense fallback (true_relres -1)."""
    p = oracle.cantilever(*shape)
    rng = np.random.default_rng(11)
    x = rng.uniform(0.05, 1.0, p.nel)
    CX, dsK = oracle.simp(x)
    s = _solver(gputo, p, CX, torch, nl=nl)
    F = _dev(torch, p.F)
    U = torch.zeros_like(F)
    rr, nit = s.solve(F, U, 1e-8, 2000)
    assert rr < 1e-8
    dsKd = _dev(torch, dsK)
    ce = torch.full((p.nel,), float("nan"), dtype=torch.float64, device="cuda")
    dc = torch.full_like(ce, float("nan"))
    c, tr = s.energy(dsKd, ce, dc)
    ce_ref, dc_ref = torch.empty_like(ce), torch.empty_like(ce)
    c_ref = gputo.compliance_sens_dev(p.Ke0, U, _dev(torch, CX), dsKd, *shape, ce=ce_ref, dc=dc_ref)
    assert not torch.isnan(ce).any() and not torch.isnan(dc).any()
    assert float((ce - ce_ref).abs().max()) <= 1e-12 * float(ce_ref.abs().max())
    assert float((dc - dc_ref).abs().max()) <= 1e-12 * float(dc_ref.abs().max())
    assert abs(c - c_ref) <= 1e-12 * abs(c_ref)
    if p.nely > 256:
        assert tr == -1.0
        return
    KU = torch.zeros_like(F)
    s.apply(U, KU)
    tr_ref = float(torch.linalg.norm(F - KU) / torch.linalg.norm(F))
    assert abs(tr - tr_ref) <= 1e-6 * tr_ref, (tr, tr_ref)
    assert tr < 1e-7


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("shape,nl", [((68, 64, 20), 3), ((16, 8, 8), 2)])
def test_prolongation_fused_into_the_first_post_sweep_is_bit_identical(oracle, gputo, torch, prec, shape, nl):
    """fuse_prolong = 1: the finest level's first post-smoothing sweep adds
    P e_c to its own node-plane tiles; the V-cycle must equal the one with the
    separate prolongation pass bit for bit (same taps, same order)."""
    p = oracle.cantilever(*shape)
    rng = np.random.default_rng(8)
    CX = oracle.simp(oracle.random_density(*shape, seed=5))[0]
    r = rng.standard_normal(p.ndof)
    r[p.fixed.astype(np.int64) - 1] = 0.0
    precision = gputo.PREC_MIXED if prec == "mixed" else gputo.PREC_FP64
    out = []
    for fp in (0, 1):
        s = _solver(gputo, p, CX, torch, nl=nl, precision=precision, fuse_prolong=fp)
        z = torch.zeros(p.ndof, dtype=torch.float64, device="cuda")
        s.vcycle(_dev(torch, r), z)
        out.append(z)
    assert torch.equal(out[0], out[1])


@pytest.mark.parametrize("xchunk", [8, 16, 24])
def test_autotuned_x_chunk_gives_the_same_operator_and_solve(oracle, gputo, torch, xchunk):
    """sweep_xchunk (the autotuner's tile choice): the fine sweeps with x chunks
    of 8, 16 or 24 node planes agree with the default chunking to rounding, and
    a mixed solve converges to the same U."""
    p = oracle.cantilever(68, 64, 20)
    CX = oracle.simp(oracle.random_density(68, 64, 20, seed=9))[0]
    u = np.random.default_rng(10).standard_normal(p.ndof)
    res = []
    for xc in (0, xchunk):
        s = _solver(gputo, p, CX, torch, nl=3, sweep_xchunk=xc)
        r = torch.zeros(p.ndof, dtype=torch.float64, device="cuda")
        s.apply(_dev(torch, u), r)
        sm = _solver(gputo, p, CX, torch, nl=3, sweep_xchunk=xc, precision=gputo.PREC_MIXED)
        F = _dev(torch, p.F)
        U = torch.zeros_like(F)
        rr, nit = sm.solve(F, U, 1e-8, 400)
        assert rr < 1e-8
        res.append((r, U))
    assert float((res[0][0] - res[1][0]).abs().max()) <= 1e-13 * float(res[0][0].abs().max())
    assert float(torch.linalg.norm(res[0][1] - res[1][1])) <= 1e-6 * float(torch.linalg.norm(res[0][1]))


@pytest.mark.parametrize("shape,nl", SHAPES + [((36, 128, 12), 3), ((20, 100, 8), 2), ((12, 16, 28), 2)])
def test_paired_fp32_sweeps_are_bit_identical(oracle, gputo, torch, shape, nl):
    """sweep_pairs = 1 (two element columns per lane, paired FP32 arithmetic):
    the FP32 apply and the mixed V-cycle (pre-relaxation, Jacobi and defect
    sweeps) equal the one-column kernel's bit for bit, on clusters of one to
    four CTAs of 64 columns with ragged and exact last CTAs (nely 8, 16, 40,
    64, 96, 100, 128, 256; 264 runs the dense kernel both ways); a mixed solve
    (its last sweep also sums r'z and r'z_old, grouped differently) takes the
    same iterations to the same U within 1e-9."""
    p = oracle.cantilever(*shape)
    rng = np.random.default_rng(12)
    CX = oracle.simp(oracle.random_density(*shape, seed=3))[0]
    u = rng.standard_normal(p.ndof)
    r = rng.standard_normal(p.ndof)
    r[p.fixed.astype(np.int64) - 1] = 0.0
    out = []
    for pairs in (0, 1):
        s = _solver(gputo, p, CX, torch, nl=nl, precision=gputo.PREC_MIXED, sweep_pairs=pairs)
        a = torch.zeros(p.ndof, dtype=torch.float64, device="cuda")
        s.apply_fp32(_dev(torch, u), a)
        z = torch.zeros(p.ndof, dtype=torch.float64, device="cuda")
        s.vcycle(_dev(torch, r), z)
        F = _dev(torch, p.F)
        U = torch.zeros_like(F)
        rr, nit = s.solve(F, U, 1e-8, 400)
        out.append((a, z, U, nit, rr))
        s.close()
    (a0, z0, U0, n0, r0), (a1, z1, U1, n1, r1) = out
    assert torch.equal(a0, a1)
    assert torch.equal(z0, z1)
    assert n0 == n1 and r1 < 1e-8
    assert float(torch.linalg.norm(U0 - U1)) <= 1e-9 * float(torch.linalg.norm(U0))
