"""Heaviside projection (ft = 3) on the device against the numpy restatement
of top3D125modCuda.m (oracle.prj/deta/dprj and its design loop)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture
def torch():
    import torch as _torch
    return _torch


def test_heaviside_matches_oracle_newton(oracle, gputo, torch):
    rng = np.random.default_rng(3)
    xt = np.clip(rng.beta(0.6, 2.5, 20000), 0.0, 1.0)
    volfrac, beta, eta0 = 0.15, 4.0, 0.4
    eta = eta0
    f = oracle.prj(xt, eta, beta).mean() - volfrac
    while abs(f) > 1e-6:
        eta = eta - f / oracle.deta(xt, eta, beta).mean()
        f = oracle.prj(xt, eta, beta).mean() - volfrac
    dev = dict(dtype=torch.float64, device="cuda")
    X = torch.as_tensor(xt, **dev)
    P, D = torch.empty_like(X), torch.empty_like(X)
    eta_g = gputo.heaviside_dev(X, P, volfrac, beta, eta0, D)
    assert abs(eta_g - eta) <= 1e-12 * abs(eta)
    np.testing.assert_allclose(P.cpu().numpy(), oracle.prj(xt, eta, beta), rtol=0, atol=1e-13)
    np.testing.assert_allclose(D.cpu().numpy(), oracle.dprj(xt, eta, beta), rtol=1e-12, atol=1e-12)
    Z = torch.empty_like(X)
    gputo.mul_dev(P, D, Z)
    np.testing.assert_allclose(Z.cpu().numpy(), P.cpu().numpy() * D.cpu().numpy(), rtol=0, atol=0)


def test_design_loop_with_projection_matches_oracle(oracle, gputo, torch):
    """Six iterations of the 32x16x16 cantilever with ft = 3 on the GPU against
    the oracle loop with the same settings: compliance history within 1e-6,
    design within 1e-6 max-abs, the same iteration counts within 1."""
    p = oracle.cantilever(32, 16, 16)
    cfg = oracle.DesignConfig(nl=3, tol=1e-9, maxit=200, iters=6, ft=3, volfrac=0.12)
    h = oracle.design_loop(p, cfg)
    F, fixed = gputo.cantilever(32, 16, 16)
    dl = gputo.DesignLoop(32, 16, 16, 3, F, fixed, gputo.hex8_stiffness(), volfrac=0.12, tol=1e-9, maxit=200,
                          ft=3, eta=0.4, beta=2.0)
    cs, nits = [], []
    for _ in range(6):
        info = dl.step()
        cs.append(info["c"])
        nits.append(info["nit"])
    np.testing.assert_allclose(cs, h["c"], rtol=1e-6)
    assert max(abs(a - b) for a, b in zip(nits, h["nit"])) <= 1
    assert np.abs(dl.xPhys.cpu().numpy() - h["xPhys"]).max() <= 1e-6
    assert np.abs(dl.x.cpu().numpy() - h["x"]).max() <= 1e-6


def test_design_loop_resume_is_seamless(gputo, torch, tmp_path):
    """Save after three ft = 3 iterations, resume in a fresh loop, run three
    more: the design and compliance match six uninterrupted iterations
    (the drivers' warm start, CrossWalk/crosswalk.m:135)."""
    F, fixed = gputo.cantilever(32, 16, 16)
    kw = dict(volfrac=0.12, tol=1e-9, maxit=200, ft=3, eta=0.4, beta=2.0)
    a = gputo.DesignLoop(32, 16, 16, 3, F, fixed, gputo.hex8_stiffness(), **kw)
    ca = [a.step()["c"] for _ in range(6)]
    b = gputo.DesignLoop(32, 16, 16, 3, F, fixed, gputo.hex8_stiffness(), **kw)
    for _ in range(3):
        b.step()
    path = tmp_path / "it3.gds"
    b.save(path, 3)
    c = gputo.DesignLoop(32, 16, 16, 3, F, fixed, gputo.hex8_stiffness(), volfrac=0.3, tol=1e-9, maxit=200,
                         ft=3, eta=0.5, beta=2.0)
    assert c.resume(path) == 3
    assert c.volfrac == 0.12 and c.eta == b.eta
    cc = [c.step()["c"] for _ in range(3)]
    np.testing.assert_allclose(cc, ca[3:], rtol=1e-9)
    assert np.abs(c.x.cpu().numpy() - a.x.cpu().numpy()).max() <= 1e-9
