"""The CPU oracle of the learned-correction network (no GPU needed).

Its analytic backward pass is checked against central finite differences in
float64, and its parameter count against the library's C ABI, which shares
the flat parameter layout.
"""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "oracle"))
import learned  # noqa: E402


def test_backward_matches_finite_differences():
    rng = np.random.default_rng(0)
    th = learned.init_params(3).astype(np.float64)
    x = rng.standard_normal((4, 4, 3, 5))
    t = rng.standard_normal((3, 4, 3, 5))
    m = (rng.random((3, 4, 3, 5)) > 0.2).astype(float)
    y, acts = learned.forward(x, th, round_weights=False, dtype=np.float64)
    _, gy = learned.loss(y, t, m)
    g = learned.backward(acts, th, gy, round_weights=False)
    worst = 0.0
    for i in rng.choice(th.size, 60, replace=False):
        e = 1e-6
        tp, tm = th.copy(), th.copy()
        tp[i] += e
        tm[i] -= e
        fp = learned.loss(learned.forward(x, tp, False, np.float64)[0], t, m)[0]
        fm = learned.loss(learned.forward(x, tm, False, np.float64)[0], t, m)[0]
        fd = (fp - fm) / (2 * e)
        worst = max(worst, abs(fd - g[i]) / max(1e-8, abs(fd) + abs(g[i])))
    assert worst < 1e-4


def test_bf16_rounding_is_round_to_nearest_even():
    v = np.array([1.0, 1.00390625, 1.01171875, -2.5e-3, 3.0e38], dtype=np.float32)
    r = learned.bf16_round(v)
    assert r[0] == 1.0 and r[1] == 1.0        # halfway to 1.0078125: ties to even
    assert r[2] == np.float32(1.015625)       # halfway, rounds up to the even neighbour
    assert abs(r[3] - v[3]) <= abs(v[3]) * 2 ** -8


def test_parameter_count_matches_library(gputo):
    assert gputo.Net.num_params() == learned.num_params() == 71155
