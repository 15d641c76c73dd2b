"""Batches of image instances (GPU): ipg_render_batch against one
ipg_render_image call per instance.

A batch shares the geodesics of instances with the same camera and derives
each electron model's fields on the device; every instance's image must be
the single-image path's image bit for bit (every array of the image,
refinement decisions included).  The reference renders one image per run, so
its pin is the single-image path's own parity with the reference's golden
images, checked here again for the instance that repeats a golden case.
"""
import numpy as np
import pytest

import ipole_b200 as ip
from tests import common

pytestmark = pytest.mark.gpu

BASE = ["--phicam=0", "--MBH=6.5e9", "--dsource=16.8e6", "--fov=160", "--trat_small=1"]

# (camera, electrons) of each instance: three cameras (inclination,
# frequency, rotation, size, refinement) and several electron models each
CAMS = {
    "A": ["--thetacam=163", "--rotcam=0", "--freqcgs=230.e9", "--nx=32", "--ny=32"],
    "B": ["--thetacam=17", "--rotcam=30", "--qu_conv=1", "--freqcgs=345.e9", "--nx=32", "--ny=32", "--nx_min=8",
          "--ny_min=8", "--refine_abs=2e-2", "--refine_rel=1e-2"],
    "C": ["--thetacam=60", "--rotcam=0", "--freqcgs=86.e9", "--nx=33", "--ny=33", "--nx_min=9", "--ny_min=9"],
}
ELECTRONS = {
    "A": [("3e27", "20"), ("3e27", "160"), ("9e27", "20"), ("1e26", "1")],
    "B": [("3e27", "20"), ("3e27", "160"), ("1e27", "10")],
    "C": [("3e27", "40")],
}


def _instances(dump):
    out = []
    for cam, els in ELECTRONS.items():
        for mu, rh in els:
            out.append(ip.Params.from_args([f"--dump={dump}", *BASE, *CAMS[cam], f"--M_unit={mu}",
                                            f"--trat_large={rh}"]))
    return out


@pytest.fixture(scope="module")
def c1_dump(dumps):
    meta, _ = common.load_golden("c1_bright_32")
    return dumps.get(meta)


def _diff(a, b):
    """the arrays of two images that differ, with the number of differing
    entries and their largest relative difference"""
    out = {}
    for k in ("unpol", "tau", "pol", "interp_flag", "nstep", "oddflag"):
        x, y = getattr(a, k), getattr(b, k)
        assert x.shape == y.shape, k
        if np.ascontiguousarray(x).tobytes() != np.ascontiguousarray(y).tobytes():
            d = x != y
            rel = np.abs(x.astype(float) - y.astype(float)) / np.maximum(np.abs(y.astype(float)), 1e-300)
            out[k] = (int(d.sum()), float(rel[d].max()))
    return out


def test_batch_equals_single_images(c1_dump):
    ps = _instances(c1_dump)
    base = ip.Model.load(ps[0])
    with ip.Context() as ctx:
        ctx.upload_batch(base)
        imgs = ctx.render_batch(ps, base)
        st = ctx.stats()
        assert st["ray_steps"] > 0 and st["waves"] >= 1
        bad = {}
        for q, (p, img) in enumerate(zip(ps, imgs)):
            m = ip.Model.load(p)
            ctx.upload(m)
            ref = ctx.render(p, m)
            d = _diff(img, ref)
            if d or img.traced != ref.traced:
                bad[q] = (d, img.traced, ref.traced)
        print("instances that differ from their single image:", bad)
        assert not bad, bad


def test_batch_longest_class_beside_the_waves(c1_dump):
    """A batch that takes several waves of the trajectory pool traces its
    longest predicted class beside them (blocks that fill an SM, a pool range
    of its own, joining a later wave's coefficient and transfer passes).
    Every instance is still its single image bit for bit, and a step budget
    that runs out while that class is in flight leaves the context usable."""
    ps = [ip.Params.from_args([f"--dump={c1_dump}", *BASE, *CAMS["A"][:3], "--nx=64", "--ny=64", f"--M_unit={mu}",
                               f"--trat_large={rh}"]) for mu, rh in (("3e27", "20"), ("3e27", "160"), ("9e27", "20"))]
    base = ip.Model.load(ps[0])
    with ip.Context(pool_bytes=2 << 30) as ctx:
        ctx.upload_batch(base)
        with pytest.raises(ip.IpgError) as e:
            ctx.render_batch(ps, base, step_budget=200000)
        assert e.value.code == ip.IPG_E_TIMEOUT
        imgs = ctx.render_batch(ps, base)
        st = ctx.stats()
        print("waves", st["waves"], "longest class items", st["long_class_items"])
        assert st["waves"] >= 2 and st["long_class_items"] > 0, st
        bad = {}
        for q, (p, img) in enumerate(zip(ps, imgs)):
            m = ip.Model.load(p)
            ctx.upload(m)
            ref = ctx.render(p, m)
            d = _diff(img, ref)
            if d or img.traced != ref.traced:
                bad[q] = (d, img.traced, ref.traced)
        print("longest class beside the waves: instances that differ from their single image:", bad)
        assert not bad, bad


def test_batch_instance_matches_golden(c1_dump):
    """c1_bright_32 as one instance of a batch against the reference's image"""
    meta, arrs = common.load_golden("c1_bright_32")
    ps = [common.params_for(meta, c1_dump)]
    # a second instance on the same camera with another electron model
    ps.append(common.params_for(meta, c1_dump, ["--trat_large=160"]))
    m = ip.Model.load(ps[0])
    with ip.Context() as ctx:
        ctx.upload_batch(m)
        img = ctx.render_batch(ps, m)[0]
    e = common.image_errors(img, arrs)
    for key in ("Ftot", "Ftot_unpol", "pix_I_max", "pix_unpol_max", "totQ", "totU", "totV", "EVPA_deg"):
        assert e[key] <= common.tolerance(meta, key), (key, e[key])


def test_batch_step_budget_times_out_and_context_recovers(c1_dump):
    ps = _instances(c1_dump)[:3]
    m = ip.Model.load(ps[0])
    with ip.Context() as ctx:
        ctx.upload_batch(m)
        with pytest.raises(ip.IpgError) as e:
            ctx.render_batch(ps, m, step_budget=2000)
        assert e.value.code == ip.IPG_E_TIMEOUT
        imgs = ctx.render_batch(ps, m)
        assert all(np.isfinite(i.pol).all() and i.pol[..., 0].sum() > 0 for i in imgs)


def test_batch_rejects_mixed_emission_types(c1_dump):
    ps = _instances(c1_dump)[:2]
    ps[1].set("emission_type", 1)
    m = ip.Model.load(ps[0])
    with ip.Context() as ctx:
        ctx.upload_batch(m)
        with pytest.raises(ip.IpgError) as e:
            ctx.render_batch(ps, m)
        assert e.value.code == ip.IPG_E_ARG


def test_mixed_tier_batch_equals_single_images(c1_dump):
    """With compact step records, the FP32 step and the FP32 fit shapes set on
    the context, every instance of a batch is the single image rendered with
    the same settings, bit for bit (the shared records in the compact
    layout, the instances' coefficient blocks in FP64)."""
    ps = _instances(c1_dump)
    base = ip.Model.load(ps[0])
    with ip.Context() as ctx:
        ctx.set_record_precision(ip.IPG_RECORDS_MIXED)
        ctx.set_step_precision(ip.IPG_STEP_FP32)
        ctx.set_fit_precision(ip.IPG_FITS_FP32)
        ctx.upload_batch(base)
        imgs = ctx.render_batch(ps, base)
        bad = {}
        for q, (p, img) in enumerate(zip(ps, imgs)):
            m = ip.Model.load(p)
            ctx.upload(m)
            ref = ctx.render(p, m)
            d = _diff(img, ref)
            if d or img.traced != ref.traced:
                bad[q] = (d, img.traced, ref.traced)
        print("mixed tier: instances that differ from their single image:", bad)
        assert not bad, bad
