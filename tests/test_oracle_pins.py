"""The oracle is pinned to the reference itself.

* gsl_sf_bessel_Kn of the oracle shim (the only GSL routine on the thermal
  path) against mpmath / scipy.
* The full image pipeline -- the product's host driver (parameters, iharm
  loader, camera, refinement bookkeeping) with the C restatement of get_pixel
  as its tracer -- against every golden image, which the reference binary
  (oracle/_ref/ipole_nofma, built from the reference sources) produced.  The
  restatement keeps the reference's operation order, so the comparison is
  bit for bit.
"""
import ctypes as C
import os

import numpy as np
import pytest

import ipole_b200 as ip
from oracle.oracle import Oracle, build as build_oracle
from tests import common


@pytest.fixture(scope="module")
def kn():
    build_oracle()
    L = C.CDLL(os.path.join(os.path.dirname(common.HERE), "oracle", "_build", "liboracle.so"))
    f = L.gsl_sf_bessel_Kn
    f.restype = C.c_double
    f.argtypes = [C.c_int, C.c_double]
    return f


def test_bessel_kn_vs_mpmath(kn):
    mp = pytest.importorskip("mpmath")
    mp.mp.dps = 40
    worst = 0.0
    for x in np.concatenate([np.logspace(-3, np.log10(740.0), 240), [1.999999, 2.0, 2.000001]]):
        for n in (0, 1, 2):
            ref = float(mp.besselk(n, x))
            if ref > 0:
                worst = max(worst, abs(kn(n, float(x)) / ref - 1))
    assert worst < 1e-14, worst


def test_bessel_kn_vs_scipy(kn):
    sp = pytest.importorskip("scipy.special")
    xs = np.logspace(-3, np.log10(600.0), 500)
    for n in (0, 1, 2):
        mine = np.array([kn(n, float(x)) for x in xs])
        rel = np.abs(mine / sp.kn(n, xs) - 1)
        assert rel.max() < 1e-13, (n, rel.max())


def test_bessel_underflow_is_zero(kn):
    assert kn(2, 800.0) == 0.0 and kn(0, 1e4) == 0.0


# images larger than this are pinned on a seeded sample of their pixels:
# the production-size goldens (128x128, 400x400) trace every pixel, so each
# pixel of the golden is that pixel's own trace, and the whole image on the
# CPU restatement would take minutes
FULL_PIN_PIXELS = 48 * 48
SAMPLE_PIXELS = 160


@pytest.mark.parametrize("case", common.golden_names(plugins=False))
def test_oracle_pipeline_matches_reference_bitwise(case, dumps):
    meta, arrs = common.load_golden(case)
    p = common.params_for(meta, dumps.get(meta))
    m = ip.Model.load(p)
    orc = Oracle(m.grid, [m.field(q) for q in range(10)])
    nx, ny = arrs["unpol"].shape
    if nx * ny > FULL_PIN_PIXELS:
        assert not any(a.startswith(("--nx_min", "--ny_min")) for a in meta["args"])  # no refinement
        rng = np.random.default_rng(7)
        flat = rng.choice(nx * ny, SAMPLE_PIXELS, replace=False)
        ij = np.stack([flat // ny, flat % ny], 1).astype(np.int32)
        cam = ip.camera_for(p, m.grid)
        o = common.oracle_tracer(orc)(cam, ij)
        f3 = p.freqcgs ** 3
        sq = 1. if p.qu_conv else -1.
        i, j = ij[:, 0], ij[:, 1]
        assert np.array_equal(o["I_unpol"] * f3, arrs["unpol"][i, j])
        if "tau" in arrs:
            assert np.array_equal(o["tau"], arrs["tau"][i, j])
        if "pol" in arrs:
            pg = arrs["pol"][i, j]
            assert np.array_equal(o["I"] * f3, pg[:, 0])
            assert np.array_equal(sq * o["Q"] * f3, pg[:, 1])
            assert np.array_equal(sq * o["U"] * f3, pg[:, 2])
            assert np.array_equal(o["V"] * f3, pg[:, 3])
        return
    img = ip.render_with(common.oracle_tracer(orc), p, m)
    assert np.array_equal(img.unpol, arrs["unpol"])
    assert np.array_equal(img.tau, arrs["tau"])
    if "pol" in arrs:
        assert np.array_equal(img.pol, arrs["pol"])
    else:
        assert img.pol is None
