"""Build the operation-counting variant of the oracle (TEST INFRASTRUCTURE
ONLY): oracle.c compiled as C++ with its doubles replaced by the counting
type of counting.hpp, each function body opened with the scope it is
counted under, and a driver (orc_count_pixels) appended.

The scopes follow the per-step work of the reference's get_pixel
(src/main.c:822-883):
  geodesic  trace_geodesic and everything it calls (src/model_geodesics.c,
            src/geodesics.c, src/geometry.c, src/coordinates.c)
  push      push_polar and the connection it evaluates (src/ipolarray.c:253-289)
  coeffs    the model point queries, get_jkinv / jar_calc and the plasma
            tetrad (model/iharm/model.c, src/model_radiation.c,
            src/model_tetrads.c)
  step      integrate_emission's own arithmetic, approximate_solve and the
            tensor/Stokes transforms (src/ipolarray.c:59-628)
  evolve    evolve_N (src/ipolarray.c:332-575) less the coefficients and
            tetrad it asks for; its calls count the radiating steps
  project   project_N (once per ray)

    python oracle/opcount/make_counting_source.py   # writes and builds oracle/_build/liboracle_count.so
"""
from __future__ import annotations

import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE = os.path.dirname(HERE)
OUT_DIR = os.path.join(ORACLE, "_build")
SRC = os.path.join(OUT_DIR, "oracle_count.cpp")
LIB = os.path.join(OUT_DIR, "liboracle_count.so")

SCOPES = {
    "trace_geodesic": "SC_GEO",
    "push_polar": "SC_PUSH",
    "get_model_fourv": "SC_COEF", "get_model_ne": "SC_COEF", "get_model_thetae": "SC_COEF",
    "get_model_b": "SC_COEF", "radiating_region": "SC_COEF", "get_fluid_nu": "SC_COEF",
    "get_bk_angle": "SC_COEF", "jar_calc_dist": "SC_COEF", "get_jkinv": "SC_COEF",
    "make_plasma_tetrad": "SC_COEF",
    "integrate_emission": "SC_STEP", "evolve_N": "SC_EVOLVE", "approximate_solve": "SC_STEP",
    "coord_to_tetrad2": "SC_STEP", "tetrad_to_coord2": "SC_STEP", "tensor_to_stokes": "SC_STEP",
    "stokes_to_tensor": "SC_STEP",
    "project_N": "SC_PROJ",
}

DRIVER = r'''
/* ---- counting driver ---- */
extern "C" void orc_count_pixels(const orc_model *m, const orc_camera *c, const int *ij, int n, double *out,
                                 long long *counts)
{
  memset(&g_oc, 0, sizeof(g_oc));
  long long steps = 0, rad = 0;
  for (int q = 0; q < n; q++) {
    double o[9];
    orc_count_pixel_one(m, c, ij[2 * q], ij[2 * q + 1], o);
    for (int k = 0; k < 9; k++) out[9 * q + k] = o[k];
    steps += (long long)o[7];
  }
  for (int s = 0; s < SC_N; s++) {
    for (int k = 0; k < OC_N; k++) counts[s * (OC_N + 1) + k] = g_oc.c[s][k];
    counts[s * (OC_N + 1) + OC_N] = g_oc.calls[s];
  }
  counts[SC_N * (OC_N + 1)] = steps;
}
'''


def transform(src: str) -> str:
    s = src
    s = s.replace("#include <complex.h>\n", "")
    s = s.replace('#include "gsl/gsl_sf_bessel.h"\n', '#include "gsl/gsl_sf_bessel.h"\n#include "counting.hpp"\n')
    s = s.replace("double complex", "ocplx")
    s = re.sub(r"\bdouble\b", "oreal", s)
    s = re.sub(r"\bcreal\(", "ocreal(", s)
    s = re.sub(r"\bcimag\(", "ocimag(", s)
    s = re.sub(r"\bconj\(", "oconj(", s)
    s = re.sub(r"\bI\b(?!\w)", "OC_I", s)
    # the exported API keeps plain doubles at its boundary: rename the
    # pixel entry (the driver calls it) and drop the rest
    s = s.replace("int orc_trace_pixel(const orc_model *m, const orc_camera *c, int i, int j, oreal out[9])",
                  "static int orc_count_pixel_one(const orc_model *m, const orc_camera *c, int i, int j, double out[9])")
    # what follows the per-pixel function (the threaded loop, the camera
    # set-up) is not counted: the regular oracle library serves it
    cut = s.index("static long long g_last_steps")
    s = s[:cut]
    s = re.sub(r"out\[(\d)\] = (\w+);", r"out[\1] = (double)(\2);", s)
    s = s.replace("m->f[", "(const oreal *)m->f[")
    # each scoped function opens with its scope
    for fn, sc in SCOPES.items():
        pat = re.compile(r"(\nstatic [a-z ]+\b" + fn + r"\([^{;]*\)\s*\{)", re.S)
        s, k = pat.subn(lambda mt: mt.group(1) + f"\n  ORC_SCOPE({sc});", s, count=1)
        if k != 1:
            raise SystemExit(f"scope for {fn} not placed")
    return s + DRIVER


def build():
    os.makedirs(OUT_DIR, exist_ok=True)
    src = open(os.path.join(ORACLE, "oracle.c")).read()
    open(SRC, "w").write(transform(src))
    cmd = ["g++", "-std=c++17", "-O1", "-fPIC", "-shared", "-w", "-fpermissive", "-I", HERE,
           "-I", os.path.join(ORACLE, "shim"), "-I", ORACLE, SRC, os.path.join(ORACLE, "shim", "gsl_shim.c"),
           "-o", LIB, "-lm"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise SystemExit(r.stderr[-6000:])
    return LIB


if __name__ == "__main__":
    print(build())
