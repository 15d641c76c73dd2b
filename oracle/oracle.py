"""Python access to the CPU oracle (oracle.c) -- TEST INFRASTRUCTURE ONLY.

Imported by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg
to check or time the reference algorithm; never by the product package.
The oracle takes the same ghost-padded iharm fields as the product's C-ABI
(ipg_upload_iharm) and its own camera set-up (main.c:125-168).
"""
from __future__ import annotations

import ctypes as C
import os
import shutil
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")
REF_BIN = os.path.join(HERE, "_ref", "ipole")
REF_NOFMA_BIN = os.path.join(HERE, "_ref", "ipole_nofma")


class OrcModel(C.Structure):
    _fields_ = [("n1", C.c_int), ("n2", C.c_int), ("n3", C.c_int),
                ("startx", C.c_double * 4), ("stopx", C.c_double * 4), ("dx", C.c_double * 4),
                ("cstartx", C.c_double * 4), ("cstopx", C.c_double * 4),
                ("a", C.c_double), ("hslope", C.c_double), ("poly_xt", C.c_double), ("poly_alpha", C.c_double),
                ("mks_smooth", C.c_double), ("poly_norm", C.c_double),
                ("Rh", C.c_double), ("rmin_geo", C.c_double), ("rmax_geo", C.c_double), ("th_beg", C.c_double),
                ("sigma_cut", C.c_double), ("sigma_cut_high", C.c_double), ("L_unit", C.c_double),
                ("f", C.POINTER(C.c_double) * 10)]


class OrcCamera(C.Structure):
    _fields_ = [("Xcam", C.c_double * 4), ("Econ", (C.c_double * 4) * 4), ("Ecov", (C.c_double * 4) * 4),
                ("fovx", C.c_double), ("fovy", C.c_double), ("rotcam", C.c_double), ("xoff", C.c_double),
                ("yoff", C.c_double), ("freq", C.c_double), ("eps", C.c_double),
                ("nx", C.c_int), ("ny", C.c_int), ("maxnstep", C.c_int),
                ("only_unpolarized", C.c_int), ("emission_type", C.c_int), ("stokes_floors", C.c_int),
                ("target_nturns", C.c_int), ("subring_dtheta", C.c_int), ("counterjet", C.c_int)]


def build(ref_dir: str | None = None) -> str:
    """make the restatement and, when a reference checkout is given (ref_dir,
    else the IPG_REFERENCE environment variable) and present, the reference
    binaries compiled from its sources."""
    ref_dir = ref_dir or os.environ.get("IPG_REFERENCE")
    have_ref = bool(ref_dir) and os.path.isdir(ref_dir)
    targets = ["oracle"] + (["ref", f"REF={ref_dir}"] if have_ref else [])
    r = subprocess.run(["make", "-C", HERE, *targets], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stdout + r.stderr)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        L.orc_trace_pixels.argtypes = [C.POINTER(OrcModel), C.POINTER(OrcCamera), C.c_void_p, C.c_int, C.c_void_p,
                                       C.c_int]
        L.orc_trace_pixels.restype = None
        L.orc_camera_setup.argtypes = [C.POINTER(OrcModel)] + [C.c_double] * 6 + [C.c_int, C.c_int, C.c_double,
                                                                                   C.POINTER(OrcCamera)]
        L.orc_camera_setup.restype = C.c_double
        L.orc_last_steps.restype = C.c_longlong
        L.orc_thermal_coefficients.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p]
        L.orc_thermal_coefficients.restype = None
        _lib = L
    return _lib


def thermal_coefficients(points, emission_type):
    """orc_thermal_coefficients: points (n, 5) = (nu, Ne, Thetae, B, theta)
    -> (n, 12) = (jI/nu^2, aI of pol = 0; jI jQ jU jV aI aQ aU aV rQ rV)."""
    pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 5)
    out = np.zeros((len(pts), 12))
    lib().orc_thermal_coefficients(pts.ctypes.data, len(pts), int(emission_type), out.ctypes.data)
    return out


class Oracle:
    """Oracle over a grid description and 10 ghost-padded field arrays."""

    GRID_KEYS = ["n1", "n2", "n3", "a", "hslope", "poly_xt", "poly_alpha", "mks_smooth", "poly_norm", "Rh",
                 "rmin_geo", "rmax_geo", "th_beg", "sigma_cut", "sigma_cut_high", "L_unit"]

    def __init__(self, grid, fields):
        m = OrcModel()
        for k in self.GRID_KEYS:
            setattr(m, k, getattr(grid, k))
        for k in ("startx", "stopx", "dx", "cstartx", "cstopx"):
            setattr(m, k, (C.c_double * 4)(*list(getattr(grid, k))))
        self._arrs = [np.ascontiguousarray(f, dtype=np.float64).ravel() for f in fields]
        for q in range(10):
            m.f[q] = self._arrs[q].ctypes.data_as(C.POINTER(C.c_double))
        self.m = m

    def camera(self, rcam, thetacam, phicam, rotcam_deg, fov_muas, dsource_pc, nx, ny, freqcgs, **kw):
        c = OrcCamera()
        scale = lib().orc_camera_setup(C.byref(self.m), rcam, thetacam, phicam, rotcam_deg, fov_muas, dsource_pc,
                                       nx, ny, freqcgs, C.byref(c))
        for k, v in kw.items():
            setattr(c, k, v)
        c._scale = scale
        return c

    def trace(self, cam: OrcCamera, ij, threads: int = 1) -> np.ndarray:
        """(n, 9): I_unpol, tau, tauF, I, Q, U, V, nstep, oddflag per pixel."""
        ij = np.ascontiguousarray(ij, dtype=np.int32).reshape(-1, 2)
        out = np.zeros((len(ij), 9), dtype=np.float64)
        lib().orc_trace_pixels(C.byref(self.m), C.byref(cam), ij.ctypes.data, len(ij), out.ctypes.data, int(threads))
        return out

    @staticmethod
    def last_steps() -> int:
        return int(lib().orc_last_steps())


def have_reference_binary() -> bool:
    return os.path.exists(REF_BIN) and os.path.exists(REF_NOFMA_BIN)


def run_reference(args, binary=REF_NOFMA_BIN, threads=None, cwd=None):
    """Run the reference ipole built from its sources (oracle/_ref)."""
    env = dict(os.environ)
    if threads:
        env["OMP_NUM_THREADS"] = str(threads)
    r = subprocess.run([binary, *args], capture_output=True, text=True, env=env, cwd=cwd)
    return r.returncode, r.stderr


def gcc_available() -> bool:
    return shutil.which("gcc") is not None
