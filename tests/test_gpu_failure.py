"""Failure paths made on the host (GPU test): NaN in a dump.

The reference stops with exit(-1) when a pixel's Stokes vector is NaN
(src/main.c:905-908, in save_pixel).  Here the NaN is planted in the dump on
the host -- rho of a block of cells in the emitting torus -- so that the rays
through it carry NaN coefficients.  The image driver must return IPG_E_NAN
through the C-ABI and the command-line program must exit with -1 (255);
nothing on the GPU faults.
"""
import os
import subprocess

import numpy as np
import pytest

import ipole_b200 as ip
from ipole_b200 import build, ipgc, synthdump

pytestmark = pytest.mark.gpu

ARGS = ["--freqcgs=230.e9", "--thetacam=163", "--phicam=0", "--rotcam=0", "--MBH=6.5e9", "--dsource=16.8e6",
        "--fov=160", "--trat_large=20", "--trat_small=1", "--M_unit=3e27", "--nx=24", "--ny=24"]


@pytest.fixture(scope="module")
def nan_dump(tmp_path_factory):
    d = tmp_path_factory.mktemp("nan")
    e = synthdump.make_iharm_dump(128, 64, 64, seed=1)
    prims = np.array(e["/prims"])
    # rho of the torus body: radial zones around r ~ 6-15 (X1 = log r),
    # the polar zones around the mid-plane, every azimuth
    prims[30:60, 24:40, :, 0] = np.nan
    e["/prims"] = prims
    path = str(d / "dump_nan.ipgc")
    ipgc.write(path, e, strlen={"/header/version": 20, "/header/metric": 20})
    return path


def test_nan_in_dump_returns_ipg_e_nan(nan_dump):
    p = ip.Params.from_args([f"--dump={nan_dump}", *ARGS])
    m = ip.Model.load(p)
    with ip.Context() as ctx:
        ctx.upload(m)
        with pytest.raises(ip.IpgError) as ei:
            ctx.render(p, m)
        assert ei.value.code == ip.IPG_E_NAN
        # the context stays usable: the same call on a clean dump succeeds
        clean = os.path.join(os.path.dirname(nan_dump), "dump_clean.ipgc")
        synthdump.write_iharm_dump(clean, 128, 64, 64, seed=1)
        p2 = ip.Params.from_args([f"--dump={clean}", *ARGS])
        m2 = ip.Model.load(p2)
        ctx.upload(m2)
        img = ctx.render(p2, m2)
        assert np.all(np.isfinite(img.pol)) and img.pol[..., 0].sum() > 0


def test_nan_in_dump_cli_exit_code(nan_dump, tmp_path):
    build.build()
    r = subprocess.run([build.CLI, f"--dump={nan_dump}", *ARGS, f"--outfile={tmp_path}/img.ipgc"],
                       capture_output=True, text=True, cwd=str(tmp_path), timeout=600)
    assert r.returncode == 256 - 1, (r.returncode, r.stderr[-2000:])
    assert not os.path.exists(tmp_path / "img.ipgc")
