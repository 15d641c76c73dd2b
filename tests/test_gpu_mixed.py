"""Compact step records (ipg_set_record_precision(IPG_RECORDS_MIXED)) against
the FP64 records on the same images.

The compact layout stores the transport matrices A1/A2 (Gamma K at X and at
Xhalf, which push_polar applies to N, src/ipolarray.c:253-289) and the plasma
tetrad rows (src/model_tetrads.c:35-127) in FP32 between the kernels; the
coefficients and all arithmetic stay FP64.  The errors against the FP64
records are printed per case; the bounds are the ones stated for the mixed
tier (total flux 1e-3 relative, flux-weighted EVPA 0.5 degree), with the
per-pixel and polarization-fraction bounds below.
"""
import numpy as np
import pytest

import ipole_b200 as ip
from tests import common

pytestmark = pytest.mark.gpu

CASES = ["c1_bright_32", "c1_faraday_24", "c1_thick_24", "c1_incl17_rot_24", "c2_rhigh160_incl163_24",
         "c2_rhigh1_incl17_24", "c1_unpol_24", "c1_refine_32", "analytic_m2_32", "sphere_f223_i30_32"]
# The mixed tier's end targets (total flux 1e-3, flux-weighted EVPA 0.5
# degree against the FP64 images) are far above what these forms measure,
# so the bounds here are about ten times the largest error measured on the
# ten cases, per form: a regression shows long before a target is missed.
# The compact records alone (FP32 storage of order-one values; measured
# worst: total flux 3.1e-8, EVPA 8.1e-5 deg, LP 2.0e-7, CP 1.8e-9, per pixel
# 2.1e-6, the unpolarized image unchanged):
RECORD_BOUNDS = {"Ftot": 3e-7, "Ftot_unpol": 0., "EVPA_deg": 1e-3, "LP_abs": 2e-6, "CP_abs": 2e-8,
                 "pix_I_max": 2e-5, "pix_unpol_max": 0.}
# with the FP32 step and the FP32 fit shapes (measured worst: total flux
# 6.5e-6, EVPA 1.8e-2 deg on the optically thick case, LP 5.5e-6, CP 4.1e-7,
# per pixel 2.9e-5):
BOUNDS = {"Ftot": 7e-5, "Ftot_unpol": 7e-5, "EVPA_deg": 0.2, "LP_abs": 6e-5, "CP_abs": 5e-6,
          "pix_I_max": 3e-4, "pix_unpol_max": 3e-4}


@pytest.mark.parametrize("case", CASES)
def test_mixed_records_against_fp64(case, dumps):
    meta, _ = common.load_golden(case)
    p = common.params_for(meta, dumps.get(meta))
    m = ip.Model.load(p)
    with ip.Context() as c:
        c.upload(m)
        full = c.render(p, m)
        c.set_record_precision(ip.IPG_RECORDS_MIXED)
        mixed = c.render(p, m)
        c.set_record_precision(ip.IPG_RECORDS_FP64)
        again = c.render(p, m)
    assert again.unpol.tobytes() == full.unpol.tobytes()  # the setting is undone
    if full.pol is not None:
        assert again.pol.tobytes() == full.pol.tobytes()
    ref = {"unpol": full.unpol, **({"pol": full.pol} if full.pol is not None else {})}
    e = common.image_errors(mixed, ref)
    print(case, {k: f"{v:.2e}" for k, v in e.items()})
    assert np.array_equal(mixed.nstep, full.nstep)  # the geodesics are the same
    bad = {k: v for k, v in e.items() if k in RECORD_BOUNDS and not v <= RECORD_BOUNDS[k]}
    assert not bad, bad


def test_record_precision_argument():
    with ip.Context() as c:
        with pytest.raises(ip.IpgError) as err:
            c.set_record_precision(7)
        assert err.value.code == ip.IPG_E_ARG


def test_cli_mixed_records_key(dumps, tmp_path):
    """--mixed_records=1 (and --fp32_step=1) on the command line give the
    mixed forms' images, whose differences from the default run stay within
    the bounds."""
    import subprocess

    from ipole_b200 import build, ipgc
    meta, _ = common.load_golden("c1_faraday_24")
    build.build()
    imgs = {}
    for tag, extra in (("fp64", []), ("mixed", ["--mixed_records=1"]),
                       ("mixed_fp32", ["--mixed_records=1", "--fp32_step=1"])):
        out = str(tmp_path / f"{tag}.h5")
        r = subprocess.run([build.CLI, f"--dump={dumps.get(meta)}", *meta["args"], *extra, f"--outfile={out}"],
                           capture_output=True, text=True, cwd=str(tmp_path), timeout=600)
        assert r.returncode == 0, r.stderr[-2000:]
        imgs[tag] = ipgc.read(out)
    a = imgs["fp64"]["/pol"]
    for tag in ("mixed", "mixed_fp32"):
        b = imgs[tag]["/pol"]
        assert not np.array_equal(a, b)  # the keys took effect
        e = abs(b[..., 0].sum() / a[..., 0].sum() - 1)
        print(f"CLI {tag}: total flux relative difference", e)
        assert e <= BOUNDS["Ftot"]


@pytest.mark.parametrize("case", CASES)
def test_fp32_step_against_fp64(case, dumps):
    """ipg_set_step_precision(IPG_STEP_FP32): the polarized step's Faraday
    rotation and absorption/emission in FP32 (optical-depth form, Stokes
    vector and emission scaled by a power of two per step), alone and with
    the compact records, against the FP64 step on the same image."""
    meta, _ = common.load_golden(case)
    p = common.params_for(meta, dumps.get(meta))
    m = ip.Model.load(p)
    with ip.Context() as c:
        c.upload(m)
        full = c.render(p, m)
        c.set_step_precision(ip.IPG_STEP_FP32)
        step = c.render(p, m)
        c.set_record_precision(ip.IPG_RECORDS_MIXED)
        both = c.render(p, m)
    ref = {"unpol": full.unpol, **({"pol": full.pol} if full.pol is not None else {})}
    for tag, img in (("fp32 step", step), ("fp32 step + compact records", both)):
        e = common.image_errors(img, ref)
        print(case, tag, {k: f"{v:.2e}" for k, v in e.items()})
        assert np.array_equal(img.nstep, full.nstep)
        bad = {k: v for k, v in e.items() if k in BOUNDS and not v <= BOUNDS[k]}
        assert not bad, (tag, bad)


@pytest.mark.parametrize("case", CASES)
def test_fp32_fits_against_fp64(case, dumps):
    """ipg_set_fit_precision(IPG_FITS_FP32): the thermal fits with FP32
    shapes, alone and with the FP32 step and compact records (the whole
    mixed tier), against the FP64 image and against the reference's golden
    image."""
    meta, arrs = common.load_golden(case)
    p = common.params_for(meta, dumps.get(meta))
    m = ip.Model.load(p)
    with ip.Context() as c:
        c.upload(m)
        full = c.render(p, m)
        c.set_fit_precision(ip.IPG_FITS_FP32)
        fits = c.render(p, m)
        c.set_step_precision(ip.IPG_STEP_FP32)
        c.set_record_precision(ip.IPG_RECORDS_MIXED)
        tier = c.render(p, m)
        c.set_fit_precision(ip.IPG_FITS_FP64)
        c.set_step_precision(ip.IPG_STEP_FP64)
        c.set_record_precision(ip.IPG_RECORDS_FP64)
        again = c.render(p, m)
    assert again.unpol.tobytes() == full.unpol.tobytes()
    ref = {"unpol": full.unpol, **({"pol": full.pol} if full.pol is not None else {})}
    for tag, img in (("fp32 fits", fits), ("mixed tier", tier)):
        e = common.image_errors(img, ref)
        g = common.image_errors(img, arrs)
        print(case, tag, "vs fp64:", {k: f"{v:.2e}" for k, v in e.items()})
        print(case, tag, "vs reference:", {k: f"{v:.2e}" for k, v in g.items()})
        assert np.array_equal(img.nstep, full.nstep)
        bad = {k: v for k, v in e.items() if k in BOUNDS and not v <= BOUNDS[k]}
        assert not bad, (tag, bad)
