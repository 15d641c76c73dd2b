"""The oracle's thermal fits at points (orc_thermal_coefficients, the fits of
jar_calc_dist without the model lookup) against the coefficients the
reference itself wrote in its per-step traces: bit-identical."""
import numpy as np

from oracle import oracle as O
from tests import fits_points


def test_oracle_fits_equal_reference_trace_coefficients():
    pts, ref = fits_points.trace_points()
    out = O.thermal_coefficients(pts, 4)
    assert len(pts) > 5000
    assert (ref[:, 2] > 0).sum() > 5000  # radiating steps
    np.testing.assert_array_equal(out, ref)


def test_oracle_fits_zero_density_and_along_field():
    pts = np.array([[2.3e11, 0., 10., 30., 1.], [2.3e11, 1e5, 10., 30., 0.], [2.3e11, 1e5, 10., 30., np.pi]])
    for em in (1, 4):
        out = O.thermal_coefficients(pts, em)
        assert not out[0].any()
        # along the field: only rho_V (src/model_radiation.c:202-207)
        for r in out[1:]:
            assert not r[:10].any() and r[11] != 0.
