"""The mgcg9 drop-in (re-discretised hierarchy) against the reference's own
CUDA mgcg9 (golden fixtures from tests/golden/make_golden_mgcg9.py) and the
CPU oracle."""
import os

import numpy as np
import pytest

from conftest import load_golden
from test_oracle import MGCG9_CASES

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", MGCG9_CASES)
def test_mgcg9_matches_reference_golden(oracle, gputo, name):
    d = load_golden(name)
    nx, ny, nz = int(d["nelx"]), int(d["nely"]), int(d["nelz"])
    p = oracle.cantilever(nx, ny, nz)
    U = np.full(p.ndof, -3.0)   # input values must be ignored
    rr, nit = gputo.mgcg9(p.Ke0, p.F, U, d["CX"], p.fixed, len(p.fixed), nx, ny, nz, int(d["nl"]),
                          float(d["tol"]), int(d["maxit"]), int(d["nswp"]), printLev=0)
    assert nit == int(d["nit"])
    assert abs(rr - float(d["relres"])) <= 1e-6 * float(d["relres"])
    assert np.linalg.norm(U - d["U"]) <= 1e-9 * np.linalg.norm(d["U"])


def test_mgcg9_gateway_through_mexfunction_and_log(oracle, gputo):
    from test_capi import _load_mex, call_mex
    mex, _ = _load_mex("libgputo_mex9.so")
    d = load_golden("mgcg9_16x8x8_rand_nl3")
    p = oracle.cantilever(16, 8, 8)
    U = np.zeros(p.ndof)
    res, it = call_mex(mex, [p.Ke0.reshape(-1).copy(), p.F, U, d["CX"], p.fixed, len(p.fixed), 16, 8, 8, 3,
                             1e-8, 200, 2, 1, 0.3, 1.0, 1.0, 1.0])
    assert it == int(d["nit"])
    assert np.linalg.norm(U - d["U"]) <= 1e-9 * np.linalg.norm(d["U"])
    assert os.path.exists("mgcg9.log")
    assert "Nit=%d" % int(d["nit"]) in open("mgcg9.log").read()


def test_mgcg9_rejects_what_the_reference_solves_differently(oracle, gputo):
    """nl = 1 (the reference then only smooths) and coarsest grids of 20,000
    dofs or more (the reference switches to Jacobi sweeps) give cgiters = -1."""
    p = oracle.cantilever(16, 8, 8)
    CX = np.ones(p.nel)
    with pytest.raises(gputo.GputoError):
        gputo.mgcg9(p.Ke0, p.F, np.zeros(p.ndof), CX, p.fixed, len(p.fixed), 16, 8, 8, 1, 1e-8, 10, 2,
                    printLev=0)
    p = oracle.cantilever(64, 32, 32)        # nl = 2: coarsest 33x17x17 nodes = 28,611 dofs
    with pytest.raises(gputo.GputoError):
        gputo.mgcg9(p.Ke0, p.F, np.zeros(p.ndof), np.ones(p.nel), p.fixed, len(p.fixed), 64, 32, 32, 2, 1e-8,
                    10, 2, printLev=0)


def test_mixed_precision_on_the_rediscretised_hierarchy(oracle, gputo):
    """FP32 V-cycle over re-discretised levels + flexible FP64 PCG: the same
    solution as the oracle's FP64 mgcg9 to 1e-6."""
    p = oracle.cantilever(32, 16, 16)
    CX = oracle.simp(oracle.random_density(32, 16, 16, seed=9))[0]
    Uo, _, _ = oracle.mgcg9(p, CX, 4, 1e-10, 400, nswp=2)
    opts = gputo.default_options(precision=gputo.PREC_MIXED, coarse=1, nswp=2, omega=0.33, prerelax=0.7)
    U = np.zeros(p.ndof)
    rr, nit = gputo.mgcg1(p.Ke0, p.F, U, CX, p.fixed, len(p.fixed), 32, 16, 16, 4, 1e-8, 400, printLev=0,
                          options=opts)
    assert rr < 1e-8 and nit > 0
    assert abs(p.F @ U - p.F @ Uo) <= 1e-6 * abs(p.F @ Uo)
    assert np.linalg.norm(U - Uo) <= 1e-6 * np.linalg.norm(Uo)
