"""The on-device image driver (ipole_b200/csrc/ipg_refine.cu) against the host
driver (ipg_render_image_with, the loop of src/main.c:520-792 run on the host)
fed by the same GPU tracer: every array of the image, the interpolation map
and the traced-pixel count must agree bit for bit, for power-of-two and odd
sizes, polarized and unpolarized, linear and nearest-neighbour fill,
refinement cuts, a base-to-final ratio that is not a power of two (whose
later levels revisit pixels of earlier ones), and a spacing that does not
divide the image (edge pixels without a +spacing neighbour, traced by both
drivers where the reference would read past the image)."""
import numpy as np
import pytest

import ipole_b200 as ip
from tests import common

pytestmark = pytest.mark.gpu

CASES = {
    "refine_32": ["--nx=32", "--ny=32", "--nx_min=8", "--ny_min=8", "--refine_abs=2e-2", "--refine_rel=1e-2"],
    "refine_odd_33": ["--nx=33", "--ny=33", "--nx_min=9", "--ny_min=9"],
    "refine_unpol_48": ["--nx=48", "--ny=48", "--nx_min=12", "--ny_min=12", "--refine_rel=3e-2", "-unpol"],
    "refine_nearest_32": ["--nx=32", "--ny=32", "--nx_min=8", "--ny_min=8", "--nearest_neighbor=1",
                          "--refine_cut=1e-6"],
    "refine_rect_40x24": ["--nx=40", "--ny=24", "--nx_min=10", "--ny_min=6", "--refine_abs=1e-2"],
    "refine_npot_40": ["--nx=40", "--ny=40", "--nx_min=13", "--ny_min=13"],
    "refine_ragged_43": ["--nx=43", "--ny=43", "--nx_min=11", "--ny_min=11"],
    "no_refine_20": ["--nx=20", "--ny=20", "--nx_min=20", "--ny_min=20", "--qu_conv=1"],
}


@pytest.fixture(scope="module")
def ctx():
    c = ip.Context()
    yield c
    c.close()


@pytest.mark.parametrize("case", sorted(CASES))
def test_device_driver_matches_host_driver(case, dumps, ctx):
    meta, _ = common.load_golden("c1_refine_32")
    p = common.params_for(meta, dumps.get(meta), CASES[case])  # the case's keys override the golden run's
    m = ip.Model.load(p)
    ctx.upload(m)
    dev = ctx.render(p, m)
    host = ip.render_with(lambda cam, ij: ctx.trace(cam, ij, allow_maxnstep=True), p, m)
    assert dev.internal_shape == host.internal_shape and dev.traced == host.traced
    for k in ("unpol", "tau", "pol", "interp_flag", "oddflag", "nstep"):
        a, b = getattr(dev, k), getattr(host, k)
        if a is None or b is None:
            assert a is None and b is None, k
            continue
        assert a.dtype == b.dtype and np.array_equal(a, b, equal_nan=True), k
    if case.startswith("refine"):
        assert 0 < dev.traced < dev.internal_shape[0] * dev.internal_shape[1]
