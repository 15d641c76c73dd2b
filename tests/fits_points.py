"""Plasma-parameter points for the tests of the thermal fits at points
(ipg_thermal_coefficients, orc_thermal_coefficients).

trace_points: the (nu, Ne, Thetae, B, theta) of every step of the
reference's per-step traces (tests/golden/trace_*.npz, written by the
reference's trace output, src/io.c:352-373) with the coefficients the
reference computed there, in the column order of the fits-at-points
entries: j_I/nu^2 and a_I of get_jkinv, then jI jQ jU jV aI aQ aU aV rQ rV
of jar_calc.

grid_points: a seeded sample over the ranges the fits meet in accretion
flows and beyond (Theta_e 1e-3..1e3, B 1e-3..1e4 G, Ne 1e-2..1e9 cm^-3,
nu 1e8..1e14 Hz, every k-B angle including 0 and pi).
"""
from __future__ import annotations

import numpy as np

from tests import common

COLUMNS = ["ju", "ku", "jI", "jQ", "jU", "jV", "aI", "aQ", "aU", "aV", "rQ", "rV"]


def trace_points():
    pts, ref = [], []
    for name in common.golden_names(trace=True):
        d = np.load(common.os.path.join(common.GOLDEN, name + ".npz"))
        # step 0 is not written by the reference's trace loop (i > 0)
        pts.append(np.stack([d["nu"], d["ne"], d["thetae"], d["b"], d["b_k_angle"]], 1)[1:])
        r = np.concatenate([d["j_unpol"][1:, None], d["k_unpol"][1:, None], d["j_inv"][1:], d["alpha_inv"][1:],
                            d["rho_inv"][1:, 1:]], 1)
        ref.append(np.delete(r, 11, axis=1))  # rU (always 0) has no column
    return np.concatenate(pts), np.concatenate(ref)


def grid_points(n=20000, seed=7):
    rng = np.random.default_rng(seed)
    nu = 10 ** rng.uniform(8, 14, n)
    ne = 10 ** rng.uniform(-2, 9, n)
    th = 10 ** rng.uniform(-3, 3, n)
    b = 10 ** rng.uniform(-3, 4, n)
    ang = rng.uniform(0, np.pi, n)
    k = rng.integers(0, 20, n)
    ang[k == 0] = 0.
    ang[k == 1] = np.pi
    ang[k == 2] = np.pi / 2
    return np.stack([nu, ne, th, b, ang], 1)
