"""Count the reference algorithm's operations per ray step (TEST
INFRASTRUCTURE ONLY) on the 128x128 image of the 128x64x64 dump (230 GHz,
inclination 163 deg, M_unit 1e25, R_high 20, polarized): the oracle's
restatement of the reference compiled with a counting number type
(make_counting_source.py), run over every pixel in one thread.

A step that is not in the radiating region costs the geodesic and the two
push_polar connections; a radiating step adds the coefficients (point
queries, get_jkinv, jar_calc, plasma tetrad) and the transfer arithmetic.
Transcendental functions are counted as calls and weighted TRANS_FLOPS
flops each in the totals.

    python oracle/opcount/count_ops.py   # writes oracle/opcount/counts_c1_128.json
"""
from __future__ import annotations

import ctypes as C
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import ipole_b200 as ip  # noqa: E402
from ipole_b200 import synthdump  # noqa: E402
from oracle import oracle as orc  # noqa: E402
from oracle.opcount import make_counting_source as mcs  # noqa: E402

TRANS_FLOPS = 20
OPS = ["add", "mul", "div", "sqrt", "trans", "calls"]
SCOPES = ["geodesic", "push", "coeffs", "step", "evolve", "project", "other"]
ARGS = ["--freqcgs=230.e9", "--thetacam=163", "--phicam=0", "--rotcam=0", "--MBH=6.5e9", "--dsource=16.8e6",
        "--fov=160", "--trat_large=20", "--trat_small=1", "--M_unit=1e25", "--nx=128", "--ny=128"]


def flops(d):
    return d["add"] + d["mul"] + d["div"] + d["sqrt"] + TRANS_FLOPS * d["trans"]


def main(n_side=128):
    lib = C.CDLL(mcs.build())
    lib.orc_count_pixels.argtypes = [C.POINTER(orc.OrcModel), C.POINTER(orc.OrcCamera), C.c_void_p, C.c_int,
                                     C.c_void_p, C.c_void_p]
    with tempfile.TemporaryDirectory() as td:
        dump = os.path.join(td, "dump.ipgc")
        synthdump.write_iharm_dump(dump, 128, 64, 64, seed=1)
        args = [a for a in ARGS if not a.startswith(("--nx", "--ny"))] + [f"--nx={n_side}", f"--ny={n_side}"]
        p = ip.Params.from_args([f"--dump={dump}", *args])
        m = ip.Model.load(p)
        o = orc.Oracle(m.grid, [m.field(q) for q in range(10)])
        cam = o.camera(1000., 163., 0., 0., 160., 16.8e6, n_side, n_side, 230e9)
        ij = np.array([(i, j) for i in range(n_side) for j in range(n_side)], np.int32)
        ref = o.trace(cam, ij, threads=8)
        out = np.zeros((len(ij), 9))
        cnt = np.zeros(len(SCOPES) * len(OPS) + 1, dtype=np.int64)
        lib.orc_count_pixels(C.byref(o.m), C.byref(cam), ij.ctypes.data, len(ij), out.ctypes.data, cnt.ctypes.data)
    # the counting build is the same arithmetic: the same image
    assert np.array_equal(out, ref), "counting build differs from the oracle"
    c = {s: dict(zip(OPS, (int(x) for x in cnt[k * len(OPS):(k + 1) * len(OPS)]))) for k, s in enumerate(SCOPES)}
    steps = int(cnt[-1])
    rad = c["evolve"]["calls"]
    per = {
        "geodesic_per_step": flops(c["geodesic"]) / steps,
        "push_per_step": flops(c["push"]) / steps,
        "coeffs_per_radiating_step": flops(c["coeffs"]) / rad,
        "transfer_per_radiating_step": (flops(c["step"]) + flops(c["evolve"])) / rad,
    }
    per["nonradiating_step"] = per["geodesic_per_step"] + per["push_per_step"]
    per["radiating_step"] = per["nonradiating_step"] + per["coeffs_per_radiating_step"] + \
        per["transfer_per_radiating_step"]
    res = {"workload": "128x64x64 dump seed 1, %dx%d IQUV, 230 GHz, thetacam 163, M_unit 1e25, R_high 20" % (
        n_side, n_side), "ray_steps": steps, "radiating_steps": rad, "trans_flops": TRANS_FLOPS,
        "counts": c, "flops": per,
        "flops_per_step_mean": sum(flops(v) for v in c.values()) / steps,
        "transcendentals_per_step_mean": sum(v["trans"] for v in c.values()) / steps,
        "generator": "oracle/opcount/count_ops.py"}
    return res


if __name__ == "__main__":
    n = int(sys.argv[1]) if len(sys.argv) > 1 else 128
    r = main(n)
    if n == 128:
        with open(os.path.join(HERE, "counts_c1_128.json"), "w") as f:
            json.dump(r, f, indent=1)
    print(json.dumps({k: r[k] for k in ("ray_steps", "radiating_steps", "flops", "flops_per_step_mean",
                                        "transcendentals_per_step_mean")}, indent=1))
