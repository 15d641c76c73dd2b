"""The library from C, through include/ipole_b200.h and include/ipole_host.h
only (GPU test): tests/c_api/render_c1.c is compiled and linked against
libipole_b200.so, renders the 128x64x64 dump's image with the reference's
parameters (config 1's keys at 32x32, golden case c1_thin_32) and writes it;
the image must match the reference's golden image within the parity bound.
The same program loads the dump through the reference's model interface
(init_model, get_model_*) and queries a zone centre, where the
interpolation must return the zone's own values."""
import os
import subprocess

import numpy as np
import pytest

from ipole_b200 import build, ipgc
from tests import common

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def test_c_program_renders_the_golden_image(dumps, tmp_path):
    build.build()
    exe = str(tmp_path / "render_c1")
    r = subprocess.run(["gcc", "-std=gnu99", "-O2", "-I", os.path.join(ROOT, "include"),
                        os.path.join(HERE, "c_api", "render_c1.c"), "-o", exe, "-L", build.BUILD, "-lipole_b200",
                        f"-Wl,-rpath,{build.BUILD}", "-lm"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    meta, arrs = common.load_golden("c1_thin_32")
    out = str(tmp_path / "img.ipgc")
    r = subprocess.run([exe, out, f"--dump={dumps.get(meta)}", *meta["args"]], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    img = ipgc.read(out)

    class Img:
        unpol = np.array(img["/unpol"])
        pol = np.array(img["/pol"])
    e = common.image_errors(Img, arrs)
    for key in ("Ftot", "Ftot_unpol", "pix_I_max", "totQ", "totU", "totV"):
        assert e[key] <= common.tolerance(meta, key), (key, e[key])
    vals = dict(zip(r.stdout.split()[::2], r.stdout.split()[1::2]))
    assert abs(float(vals["Ftot"]) / meta["Ftot"] - 1) <= common.tolerance(meta, "Ftot")
    assert float(vals["M_unit"]) == 1e25
    # at a zone centre the trilinear weights are 1 on that zone
    for f in ("thetae", "b") + (("ne",) if float(vals["sigma_cell"]) < 1.0 else ()):
        assert float(vals[f]) == float(vals[f + "_cell"]), f
    assert abs(float(vals["udotu"]) + 1) < 1e-12
