"""The oracle on the plain 1D MPDATA benchmark case at full size (2000 points,
1000 steps, opts 0, n_iters 2, FP64): mass conserved, no negative values from
the nonnegative start, and the box translated by C nt = 500 cells."""
import math

import numpy as np

from libmpdataxx_b200 import setups
from runners import run_oracle


def _centroid(u, period):
    ang = 2 * np.pi * np.arange(period) / period
    w = u[:period]
    return (math.atan2(float((w * np.sin(ang)).sum()), float((w * np.cos(ang)).sum())) / (2 * np.pi) * period) % period


def test_box_1d_full_oracle():
    s = setups.box_1d()
    psi0 = s["advectee"][0]
    out = run_oracle(s, s["opts"], n_iters=s["n_iters"])[0]
    m0, m1 = math.fsum(psi0[:-1]), math.fsum(out[:-1])
    assert abs(m1 - m0) <= 1e-12 * m0
    assert out.min() >= 0.0
    assert out[-1] == out[0]
    c0 = _centroid(np.where(psi0 > 0.5, psi0, 0.0), 1999)
    c1 = _centroid(np.maximum(out - 0.105, 0.0), 1999)
    assert abs(((c1 - c0) - 500.0 + 999.5) % 1999 - 999.5) <= 1.0, (c0, c1)
