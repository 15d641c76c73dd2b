"""Shared helpers of the test-suite: golden fixtures, dumps, comparisons."""
from __future__ import annotations

import glob
import json
import os

import numpy as np

import ipole_b200 as ip
from ipole_b200 import synthdump

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")


PLUGIN_PREFIXES = ("analytic_", "sphere_")
CHECK_PREFIX = "check_"
TRACE_PREFIX = "trace_"
ADJOINT_PREFIX = "adjoint_"  # finite differences of a loss (tests/test_gpu_adjoint.py), not images


def golden_names(plugins=True, check=False, trace=False):
    """Golden image cases; plugins=False leaves out the known-answer models'
    cases (which the C restatement of the iharm path does not cover),
    check=True gives the check-mode cases instead (their arrays are the
    check/recheck blocks, not an image), trace=True the per-step traces."""
    names = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz")))
    names = [n for n in names if not n.startswith(ADJOINT_PREFIX)]
    if check:
        return [n for n in names if n.startswith(CHECK_PREFIX)]
    if trace:
        return [n for n in names if n.startswith(TRACE_PREFIX)]
    names = [n for n in names if not n.startswith((CHECK_PREFIX, TRACE_PREFIX))]
    return names if plugins else [n for n in names if not n.startswith(PLUGIN_PREFIXES)]


def load_golden(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    meta = json.loads(str(z["meta"]))
    arrs = {k: z[k] for k in z.files if k != "meta"}
    return meta, arrs


class DumpCache:
    def __init__(self, root):
        self.root = root
        self.paths = {}

    def get(self, meta):
        """The case's dump path, or None for a known-answer model (no dump)."""
        key = meta["dump"]
        if meta.get("dump_shape_seed") is None:
            return None
        if key not in self.paths:
            n1, n2, n3, seed = meta["dump_shape_seed"]
            path = os.path.join(self.root, f"dump_{key}.ipgc")
            h = synthdump.write_iharm_dump(path, n1, n2, n3, seed=seed)
            assert h == meta["dump_sha256"], "regenerated synthetic dump differs from the golden one"
            self.paths[key] = path
        return self.paths[key]


def params_for(meta, dump_path, extra=()):
    head = [f"--dump={dump_path}"] if dump_path else []
    return ip.Params.from_args([*head, *meta["args"], *extra])


def oracle_tracer(orc, threads=8):
    """Adapter: the CPU oracle as the tracer of ipg_render_image_with."""
    from oracle.oracle import OrcCamera

    def tracer(cam, ij):
        oc = OrcCamera()
        for k, _ in OrcCamera._fields_:
            if k in ("Econ", "Ecov", "Xcam"):
                continue
            setattr(oc, k, getattr(cam, k))
        oc.Xcam = (type(oc.Xcam))(*cam.Xcam)
        for a in range(4):
            for b in range(4):
                oc.Econ[a][b] = cam.Econ[a][b]
                oc.Ecov[a][b] = cam.Ecov[a][b]
        o = orc.trace(oc, ij, threads=threads)
        res = np.zeros(len(ij), dtype=ip.PIXEL_DTYPE)
        for q, k in enumerate(["I_unpol", "tau", "tauF", "I", "Q", "U", "V"]):
            res[k] = o[:, q]
        res["nstep"] = o[:, 7]
        res["flag"] = o[:, 8]
        return res
    return tracer


def wrap180(d):
    """|d| for an angle difference in degrees, taken modulo 180 (an EVPA and
    its opposite direction are the same polarization)"""
    return float(abs((d + 90.0) % 180.0 - 90.0))


def image_errors(img, arrs):
    """Errors of a rendered image against golden arrays (relative to totals
    of I; per-pixel where I > 1e-6 max)."""
    e = {}
    u, ug = img.unpol, arrs["unpol"]
    e["Ftot_unpol"] = abs(u.sum() / ug.sum() - 1)
    m = ug > 1e-6 * ug.max()
    e["pix_unpol_max"] = float(np.max(np.abs(u[m] / ug[m] - 1)))
    e["pix_unpol_frac_1e-6"] = float(np.mean(np.abs(u[m] / ug[m] - 1) > 1e-6))
    if "pol" in arrs:
        p, pg = img.pol, arrs["pol"]
        I = pg[..., 0]
        Itot = I.sum()
        e["Ftot"] = abs(p[..., 0].sum() / Itot - 1)
        for c, n in ((1, "Q"), (2, "U"), (3, "V")):
            e["tot" + n] = abs(p[..., c].sum() - pg[..., c].sum()) / abs(Itot)
        # the deviation of the linear-polarization vector (sum Q, sum U): the
        # same for any orientation of the camera frame (rotcam, qu_conv),
        # which only redistributes it between Q and U
        e["totQU"] = float(np.hypot(p[..., 1].sum() - pg[..., 1].sum(), p[..., 2].sum() - pg[..., 2].sum())) / abs(Itot)
        m = I > 1e-6 * I.max()
        rel = np.abs(p[..., 0][m] / I[m] - 1)
        e["pix_I_max"] = float(rel.max())
        e["pix_I_frac_1e-6"] = float(np.mean(rel > 1e-6))
        e["pix_QUV_over_I_max"] = float(np.max(np.abs(p[..., 1:4][m] - pg[..., 1:4][m]) / I[m][:, None]))
        # polarization fractions and flux-weighted EVPA of the whole image
        def fr(x):
            Q, U, V, It = x[..., 1].sum(), x[..., 2].sum(), x[..., 3].sum(), x[..., 0].sum()
            return np.hypot(Q, U) / It, V / It, 0.5 * np.arctan2(U, Q)
        lp, cp, ev = fr(p)
        lpg, cpg, evg = fr(pg)
        e["LP_ref"] = float(lpg)
        e["LP_abs"] = float(abs(lp - lpg))
        e["CP_abs"] = float(abs(cp - cpg))
        e["EVPA_deg"] = wrap180(np.degrees(ev - evg))
    return e


# Parity bound of the GPU tests: error <= max(base, FLOOR_FACTOR x the case's
# reference noise floor: the largest deviation of the reference's other legal
# builds (FMA contraction, -O2/-O3, AVX2/AVX-512, a libm one ulp away) from its
# no-FMA build).  The base tolerances are the target's: 1e-8 in total flux,
# 1e-6 per pixel where I > 1e-6 max.
BASE_TOL = dict(Ftot=1e-8, Ftot_unpol=1e-8, totQ=1e-7, totU=1e-7, totV=1e-7, pix_I_max=1e-6, pix_unpol_max=1e-6,
                pix_QUV_over_I_max=1e-6, EVPA_deg=1e-5, LP_abs=1e-7, CP_abs=1e-7)
FLOOR_FACTOR = 2.0
# The flux-weighted EVPA is compared only where the image is polarized:
# below a linear polarization fraction |sum Q + i sum U| / sum I of 1e-3 the
# angle is set by rounding (the analytic models' nearly unpolarized images).
EVPA_MIN_LP = 1e-3


def tolerance(meta, key):
    """The bound of one metric.  Q and U are the components of one vector in
    the camera's frame; which of the two a build's deviation falls into is
    a matter of that frame, so their floors are the largest deviation of the
    vector itself (totQU), and the EVPA's floor is also at least the angle
    such a vector deviation subtends at the image's linear polarization."""
    fl = meta.get("ref_noise_floor") or {}
    floor = fl.get(key, 0.0)
    if key in ("totQ", "totU") and "totQU" in fl:
        floor = max(floor, fl["totQU"])
    if key == "EVPA_deg":
        floor = wrap180(floor)  # floors recorded before the angle was wrapped
        lp = fl.get("LP_ref", 0.0)
        if "totQU" in fl and lp > 0:
            floor = max(floor, float(np.degrees(fl["totQU"] / (2. * lp))))
    return max(BASE_TOL[key], FLOOR_FACTOR * floor)
