"""The compositing pass drops a warp's 8x8 block from an entry's list when the
least value of the splat's quadratic form q(d) = a dx^2 + 2 b dx dy + c dy^2
over the block's rectangle of pixel centres exceeds k = -2 floor (so no pixel
there can reach the alpha floor). This restates that least-value formula (the
origin when the rectangle holds it, else each edge's stationary point clamped
to the edge) and checks it against dense sampling of the rectangle on random
conics, and checks the bound the kernel's margin relies on: with a c < 10 det
the absolute terms of q sum to at most 38 q."""
from __future__ import annotations

import numpy as np


def rect_min_q(a, b, c, dx0, dx1, dy0, dy1):
    if dx0 <= 0 <= dx1 and dy0 <= 0 <= dy1:
        return 0.0
    q = lambda x, y: a * x * x + 2 * b * x * y + c * y * y
    clamp = lambda v, lo, hi: min(max(v, lo), hi)
    return min(q(dx0, clamp(-b * dx0 / c, dy0, dy1)), q(dx1, clamp(-b * dx1 / c, dy0, dy1)),
               q(clamp(-b * dy0 / a, dx0, dx1), dy0), q(clamp(-b * dy1 / a, dx0, dx1), dy1))


def random_conic(rs):
    # covariance from random axes and a rotation; the conic is its inverse
    s = np.exp(rs.uniform(np.log(0.5), np.log(40.0), 2))
    t = rs.uniform(0, np.pi)
    R = np.array([[np.cos(t), -np.sin(t)], [np.sin(t), np.cos(t)]])
    inv = np.linalg.inv(R @ np.diag(s * s) @ R.T)
    return inv[0, 0], inv[0, 1], inv[1, 1]


def test_the_least_value_over_a_rectangle_matches_dense_sampling():
    rs = np.random.default_rng(11)
    g = np.linspace(0.0, 1.0, 201)
    for _ in range(400):
        a, b, c = random_conic(rs)
        x0, y0 = rs.uniform(-60, 60, 2)
        x1, y1 = x0 + 7.0, y0 + 7.0  # a block's pixel centres span 7 px
        X, Y = np.meshgrid(x0 + (x1 - x0) * g, y0 + (y1 - y0) * g)
        sampled = float((a * X * X + 2 * b * X * Y + c * Y * Y).min())
        exact = rect_min_q(a, b, c, x0, x1, y0, y1)
        assert exact <= sampled + 1e-9 * max(1.0, sampled)  # never above any point
        assert sampled - exact <= 1e-3 * max(1.0, sampled) + 1e-6  # and attained


def test_the_absolute_terms_are_bounded_for_the_refined_conics():
    rs = np.random.default_rng(12)
    for _ in range(2000):
        a, b, c = random_conic(rs)
        if not a * c < 10 * (a * c - b * b):
            continue
        x, y = rs.normal(0, 30, 2)
        q = a * x * x + 2 * b * x * y + c * y * y
        terms = a * x * x + abs(2 * b * x * y) + c * y * y
        assert terms <= 38.0 * q * (1 + 1e-12)
