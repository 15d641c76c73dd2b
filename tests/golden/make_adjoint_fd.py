"""Finite differences of an image loss from the reference itself: the pin of
the adjoint's gradients with respect to M_unit, R_high and R_low.

The loss is the one of tests/test_gpu_adjoint.py: L2 between the polarized
image (16x16, 230 GHz, inclination 163 deg, the seeded 128x64x64 dump) and a
target rendered at M_unit x 1.3 and R_high 25, normalized by the target's
largest intensity.  Every image here comes from the reference build
oracle/_ref/ipole_nofma: the target, and the images at each parameter
moved by a relative +-eps, whose central differences are stored in
tests/golden/adjoint_fd_c1_16.npz with the target image: "fd" at eps =
1e-6, and "fd_eps" at 1e-4, 1e-5 and 1e-6.  The loss turns fast with the
Faraday rotation of this optically and Faraday-thick image, so the central
difference at 1e-4 is still 1.7% (M_unit) from its limit; at 1e-6 it has
converged to ~1e-6 while FP64 rounding stays far below.

    python tests/golden/make_adjoint_fd.py

Needs the reference builds (make -C oracle ref REF=<reference checkout>).
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from ipole_b200 import ipgc, synthdump  # noqa: E402

EPS = 1e-6
EPS_ALL = (1e-4, 1e-5, 1e-6)
DUMP = (128, 64, 64, 1)
BASE = ["--freqcgs=230.e9", "--thetacam=163", "--phicam=0", "--rotcam=0", "--MBH=6.5e9", "--dsource=16.8e6",
        "--fov=160", "--trat_small=1", "--nx=16", "--ny=16"]
PARAMS = {"M_unit": 3e27, "trat_large": 20.0, "trat_small": 1.0}
TARGET = {"M_unit": 3.9e27, "trat_large": 25.0, "trat_small": 1.0}


def render(binary, dump, td, **kw):
    v = dict(PARAMS, **kw)
    out = os.path.join(td, "img.ipgc")
    r = subprocess.run([binary, f"--dump={dump}", *BASE, f"--M_unit={v['M_unit']!r}",
                        f"--trat_large={v['trat_large']!r}", f"--trat_small={v['trat_small']!r}",
                        f"--outfile={out}"], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(r.stderr[-2000:])
    return np.array(ipgc.read(out)["/pol"])[..., :4]


def main():
    binary = os.path.join(ROOT, "oracle", "_ref", "ipole_nofma")
    if not os.path.exists(binary):
        raise SystemExit("build the reference first: make -C oracle ref REF=<reference checkout>")
    with tempfile.TemporaryDirectory() as td:
        dump = os.path.join(td, "dump.ipgc")
        h = synthdump.write_iharm_dump(dump, *DUMP[:3], seed=DUMP[3])
        target = render(binary, dump, td, **TARGET)
        scale = float(np.abs(target[..., 0]).max())

        def loss(pol):
            r = (pol - target) / scale
            return float((r * r).sum())

        L0 = loss(render(binary, dump, td))
        fd_eps = {}
        for e in EPS_ALL:
            fd_eps[repr(e)] = {}
            for key in PARAMS:
                x = PARAMS[key]
                lp = loss(render(binary, dump, td, **{key: x * (1 + e)}))
                lm = loss(render(binary, dump, td, **{key: x * (1 - e)}))
                fd_eps[repr(e)][key] = (lp - lm) / (2 * e * x)
        fd = fd_eps[repr(EPS)]
    meta = {"dump_shape_seed": DUMP, "dump_sha256": h, "args": BASE, "params": PARAMS, "target_params": TARGET,
            "eps": EPS, "loss": L0, "scale": scale, "fd": fd, "fd_eps": fd_eps,
            "generator": "oracle/_ref/ipole_nofma (reference sources, -O2 -ffp-contract=off)"}
    np.savez_compressed(os.path.join(HERE, "adjoint_fd_c1_16.npz"), meta=json.dumps(meta), target=target)
    print(json.dumps(meta, indent=1))


if __name__ == "__main__":
    main()
