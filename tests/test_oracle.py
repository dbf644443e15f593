"""The oracle, pinned against the reference's own outputs (CPU only).

Golden fixtures come from the reference itself (tests/golden/make_golden.py):
the MATLAB driver's Ke0 table, the compiled reference's Kem3, and solves of
the compiled, unmodified OpenMP MEX (Cantilever/omp/mgcg1.c).
"""
import os

import numpy as np
import pytest
from conftest import GOLDEN, load_golden


def _problem(O, d):
    return O.Problem(int(d["nelx"]), int(d["nely"]), int(d["nelz"]), d["F"], d["fixed"])


def test_ke_matches_matlab_driver_table(oracle):
    K = np.load(os.path.join(GOLDEN, "ke0_matlab.npy"))
    assert np.abs(oracle.hex8_stiffness(0.3) - K).max() < 1e-15


def test_ke_matches_reference_kem3(oracle):
    z = np.load(os.path.join(GOLDEN, "kem3_ref.npz"))
    assert np.abs(oracle.hex8_stiffness(0.3, 1.0) - z["h1"]).max() < 1e-15
    assert np.abs(oracle.hex8_stiffness(0.3, 2.0) - z["h2"]).max() < 1e-15


def test_ke_known_answers(oracle):
    K = oracle.hex8_stiffness(0.3)
    assert np.abs(K - K.T).max() == 0.0
    ev = np.linalg.eigvalsh(K)
    assert np.sum(np.abs(ev) < 1e-12) == 6          # 3 translations + 3 rotations
    assert ev.min() > -1e-14 and ev[6] > 1e-3
    for d in range(3):                              # rigid translation -> zero force
        t = np.zeros(24)
        t[d::3] = 1.0
        assert np.abs(K @ t).max() < 1e-15
    Kg = oracle.hex8_gauss_parts(0.3, 2.0)
    assert np.abs(Kg.sum(0) - oracle.hex8_stiffness(0.3, 2.0)).max() < 1e-15
    for g in range(8):                              # each Gauss part has rank 6
        assert np.linalg.matrix_rank(Kg[g], tol=1e-12) == 6


def test_apply_rigid_translation_is_zero_inside(oracle):
    p = oracle.cantilever(8, 4, 4)
    CX = oracle.random_density(8, 4, 4, seed=5)
    u = np.zeros(p.ndof)
    u[2::3] = 1.0
    r = oracle.apply_fine(p, CX, u)
    assert np.abs(r).max() < 1e-13


def test_apply_matches_assembled_matrix(oracle):
    """Node-gather apply == sum_e CX_e P_e^T Ke P_e u assembled densely."""
    nelx, nely, nelz = 3, 2, 2
    p = oracle.cantilever(nelx, nely, nelz)
    CX = oracle.random_density(nelx, nely, nelz, seed=2)
    Ke = oracle.hex8_stiffness()
    n = p.ndof
    K = np.zeros((n, n))
    LX, LY, LZ = [0, 1, 1, 0, 0, 1, 1, 0], [0, 0, 1, 1, 0, 0, 1, 1], [0, 0, 0, 0, 1, 1, 1, 1]
    for i in range(nelx):
        for k in range(nelz):
            for j in range(nely):
                e = nelz * nely * i + nely * k + j
                dofs = []
                for a in range(8):
                    nd = oracle.node_id(nelx, nely, nelz, i + LX[a], j + LY[a], k + LZ[a])
                    dofs += [3 * nd, 3 * nd + 1, 3 * nd + 2]
                K[np.ix_(dofs, dofs)] += CX[e] * Ke
    u = np.random.default_rng(0).standard_normal(n)
    assert np.abs(oracle.apply_fine(p, CX, u) - K @ u).max() < 1e-13 * np.abs(K @ u).max()


@pytest.mark.parametrize("name", ["solve_16x8x8_rand_nl3", "solve_32x16x16_unif_nl4",
                                  "solve_16x8x8_maxit3_nl2", "solve_16x8x8_bridge_nl3"])
def test_oracle_solver_matches_reference_mex(oracle, name):
    d = load_golden(name)
    p = _problem(oracle, d)
    U, rr, nit = oracle.mgcg1(p, d["CX"], int(d["nl"]), float(d["tol"]), int(d["maxit"]))
    assert nit == int(d["nit"])
    assert abs(rr - float(d["relres"])) <= 1e-6 * float(d["relres"])
    assert np.linalg.norm(U - d["U"]) <= 1e-10 * np.linalg.norm(d["U"])


def test_oracle_solver_corner_supports(oracle):
    """Sparse supports: the reference's OpenMP and CUDA builds differ in two
    zeroings (after prolongation, after the coarse solve); the oracle follows
    the CUDA build, so only the converged solution is compared."""
    d = load_golden("solve_16x8x8_corner_nl3")
    p = _problem(oracle, d)
    U, rr, nit = oracle.mgcg1(p, d["CX"], 3, 1e-8, 200)
    assert rr < 1e-8 and abs(nit - int(d["nit"])) <= 2
    assert np.linalg.norm(U - d["U"]) <= 1e-6 * np.linalg.norm(d["U"])
    assert abs(p.F @ U - p.F @ d["U"]) <= 1e-6 * abs(p.F @ d["U"])


def test_oracle_first_solve_cantilever_64x32x32(oracle):
    d = load_golden("solve_c1_first")
    p = oracle.cantilever(64, 32, 32)
    CX = oracle.simp(np.full(p.nel, 0.12))[0]
    U, rr, nit = oracle.mgcg1(p, CX, 4, 1e-8, 200)
    assert nit == int(d["nit"])
    assert abs(p.F @ U - float(d["compliance"])) <= 1e-9 * float(d["compliance"])
    s = d["sample"]
    assert np.linalg.norm(U[s] - d["U_sample"]) <= 1e-9 * np.linalg.norm(d["U_sample"])


def test_filter_matches_scipy_reflect(oracle):
    from scipy import ndimage
    nelx, nely, nelz = 7, 5, 6
    x = np.random.default_rng(3).random(nelx * nely * nelz)
    for rmin in (3 ** 0.5, 2 * 3 ** 0.5, 1.5):
        out, hs = oracle.filter3d(x, nelx, nely, nelz, rmin)
        R = int(np.ceil(rmin)) - 1
        d = np.arange(-R, R + 1)
        DX, DY, DZ = np.meshgrid(d, d, d, indexing="ij")
        h = np.maximum(0.0, rmin - np.sqrt(DX ** 2 + DY ** 2 + DZ ** 2))
        # element order = (x, z, y) C-order; MATLAB 'symmetric' == scipy 'reflect'
        A = x.reshape(nelx, nelz, nely)
        ref = ndimage.correlate(A, h.transpose(0, 2, 1), mode="reflect").reshape(-1)
        assert np.abs(out - ref).max() < 1e-12
        assert abs(hs - h.sum()) < 1e-12


def test_filter_preserves_constants(oracle):
    out, hs = oracle.filter3d(np.full(4 * 3 * 5, 0.3), 4, 3, 5, 3 ** 0.5)
    assert np.abs(out / hs - 0.3).max() < 1e-15


def test_oc_update_volume_and_bounds(oracle):
    rng = np.random.default_rng(1)
    x = rng.uniform(0.05, 0.3, 1000)
    dc = -rng.uniform(0.1, 2.0, 1000)
    dv = np.full(1000, 1.0 / 1000 / 0.12)
    xn, lmid = oracle.oc_update(x, dc, dv, 0.12, 0.2)
    assert abs(xn.mean() - 0.12) < 1e-3
    assert np.all(xn <= np.minimum(x + 0.2, 1.0) + 1e-15) and np.all(xn >= np.maximum(x - 0.2, 0.0) - 1e-15)


def test_design_loop_first_iterations_match_golden(oracle):
    """Three design iterations of the 64x32x32 cantilever with the oracle
    solver against the golden history made with the compiled reference."""
    path = os.path.join(GOLDEN, "design_c1.npz")
    if not os.path.exists(path):
        pytest.skip("design golden not generated")
    d = np.load(path)
    p = oracle.cantilever(64, 32, 32)
    cfg = oracle.DesignConfig(nl=4, tol=1e-8, maxit=200, iters=3)
    h = oracle.design_loop(p, cfg)
    np.testing.assert_allclose(h["c"], d["c"][:3], rtol=1e-8)
    assert h["nit"] == list(d["nit"][:3])


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(os.path.dirname(
    os.path.abspath(__file__))), "oracle", "_ref", "libmgcg1_omp_ref.so")),
    reason="compiled reference not present")
def test_restatement_vs_live_reference_random(oracle):
    rng = np.random.default_rng(11)
    for nl, (nx, ny, nz) in ((2, (8, 4, 6)), (3, (12, 8, 4))):
        p = oracle.cantilever(nx, ny, nz)
        CX = oracle.simp(rng.uniform(0.01, 1.0, p.nel))[0]
        Ur, rr_r, n_r = oracle.ref_mgcg1(p, CX, nl, 1e-9, 100)
        Uo, rr_o, n_o = oracle.mgcg1(p, CX, nl, 1e-9, 100)
        assert n_r == n_o
        assert np.linalg.norm(Ur - Uo) <= 1e-10 * np.linalg.norm(Ur)


MGCG9_CASES = ["mgcg9_16x8x8_rand_nl3", "mgcg9_32x16x16_unif_nl4", "mgcg9_24x16x8_rand_nl3_nswp3",
               "mgcg9_16x8x8_maxit3_nl2"]


@pytest.mark.parametrize("name", MGCG9_CASES)
def test_mgcg9_restatement_matches_reference_golden(oracle, name):
    """The oracle's mgcg9 (re-discretised hierarchy) against the reference's own
    CUDA mgcg9 run on a B200 (tests/golden/make_golden_mgcg9.py)."""
    d = load_golden(name)
    p = oracle.cantilever(int(d["nelx"]), int(d["nely"]), int(d["nelz"]))
    assert np.array_equal(p.F, d["F"]) and np.array_equal(p.fixed, d["fixed"])
    U, rr, nit = oracle.mgcg9(p, d["CX"], int(d["nl"]), float(d["tol"]), int(d["maxit"]), nswp=int(d["nswp"]))
    assert nit == int(d["nit"])
    assert abs(rr - float(d["relres"])) <= 1e-6 * float(d["relres"])
    assert np.linalg.norm(U - d["U"]) <= 1e-9 * np.linalg.norm(d["U"])
