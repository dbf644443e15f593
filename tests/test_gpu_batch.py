"""Batched solves (one CUDA graph launch per CG step for several designs of
different grid sizes) and the option autotuner."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _member(gputo, shape, nl, seed, precision):
    import torch
    F, fixed = gputo.cantilever(*shape)
    rng = np.random.default_rng(seed)
    x = np.full(shape[0] * shape[1] * shape[2], rng.uniform(0.1, 0.3))
    x *= gputo.random_field_density(*shape, seed=seed, corr_len=4.0, lo=0.5, hi=1.5)
    CX = torch.as_tensor(1e-9 + x ** 3 * (1 - 1e-9), dtype=torch.float64, device="cuda")
    s = gputo.Solver(*shape, nl, gputo.default_options(precision=precision))
    s.set_problem(gputo.hex8_stiffness(), fixed)
    s.setup(CX)
    return s, torch.as_tensor(F, dtype=torch.float64, device="cuda")


@pytest.mark.parametrize("precision", [0, 1])
def test_batch_matches_individual_solves(gputo, precision):
    import torch
    specs = [((32, 16, 16), 3, 1), ((48, 24, 24), 4, 2), ((64, 32, 32), 4, 3), ((40, 24, 16), 3, 4)]
    members = [_member(gputo, sh, nl, sd, precision) for sh, nl, sd in specs]
    ref = []
    for s, F in members:
        U = torch.zeros_like(F)
        rr, nit = s.solve(F, U, 1e-8, 300)
        ref.append((U.clone(), rr, nit))
    b = gputo.Batch([s for s, _ in members])
    Us = [torch.full_like(F, 3.0) for _, F in members]
    rrs, nits = b.solve([F for _, F in members], Us, 1e-8, 300, check_every=4)
    for (U0, rr0, nit0), U, rr, nit in zip(ref, Us, rrs, nits):
        assert nit == nit0 and rr == rr0
        assert torch.equal(U, U0)          # same kernels, same order: bitwise equal
    # a second call on the same batch (graph re-captured) gives the same again
    Us2 = [torch.zeros_like(F) for _, F in members]
    rrs2, nits2 = b.solve([F for _, F in members], Us2, 1e-8, 300, check_every=7)
    assert nits2 == nits and all(torch.equal(a, c) for a, c in zip(Us, Us2))


def test_autotune_picks_a_converging_option_and_keeps_the_solution(gputo):
    import torch
    s, F = _member(gputo, (64, 32, 32), 4, 5, 1)
    U0 = torch.zeros_like(F)
    rr0, nit0 = s.solve(F, U0, 1e-8, 400)
    U = torch.zeros_like(F)
    best, ms, table = gputo.autotune(s, F, U, 1e-8, 400)
    assert ms > 0 and len(table) >= 3
    assert min(t for t, n in table if t > 0) == pytest.approx(ms)
    assert best.nswp in (2, 3, 4) and best.tc_parts in (0, 2)
    U1 = torch.zeros_like(F)
    rr1, nit1 = s.solve(F, U1, 1e-8, 400)      # the solver now runs with the chosen options
    assert rr1 < 1e-8
    c0 = float(F @ U0)
    assert abs(float(F @ U1) - c0) <= 1e-6 * abs(c0)
