"""ipole_b200: B200 (sm_100a) ray pipeline of ipole behind a C-ABI.

Python mirror of the host API (``include/ipole_b200.h``,
``include/ipole_host.h``) over ctypes.  The native library must be built
(``python -m ipole_b200.build``); every compute call goes to the CUDA kernels
and fails loudly when the library or a CUDA device is missing -- there is no
CPU fallback.

Typical use, mirroring ipole's own command line::

    p = Params.from_args(["-par", "run.par", "--nx=128"])
    m = Model.load(p)
    with Context() as ctx:
        ctx.upload(m)
        img = ctx.render(p, m)        # main.c fast-light driver, refinement included
        print(img.totals())
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import build as _build

__all__ = ["lib", "Params", "Model", "Context", "Image", "Camera", "PixelOut", "Grid", "IpgError",
           "PIXEL_DTYPE", "trace_pixels", "fp64_peak_tflops", "fp32_peak_tflops",
           "convert_container"]

IPG_OK, IPG_E_ARG, IPG_E_CUDA, IPG_E_MAXNSTEP, IPG_E_NAN, IPG_E_TIMEOUT, IPG_E_NOMEM, IPG_E_IO, IPG_E_STATE, \
    IPG_E_FORMAT = range(10)
NFIELD = 10
# field order of ipg_upload_iharm (enum IPG_F_*)
(IPG_F_U1, IPG_F_U2, IPG_F_U3, IPG_F_B1, IPG_F_B2, IPG_F_B3, IPG_F_NE, IPG_F_THETAE, IPG_F_B,
 IPG_F_SIGMA) = range(NFIELD)
STRLEN = 2048
# step-record storage precision (ipg_set_record_precision)
IPG_RECORDS_FP64, IPG_RECORDS_MIXED = 0, 1
# arithmetic of the polarized step (ipg_set_step_precision)
IPG_STEP_FP64, IPG_STEP_FP32 = 0, 1
# arithmetic of the thermal fits (ipg_set_fit_precision)
IPG_FITS_FP64, IPG_FITS_FP32 = 0, 1
# per-step trace columns (include/ipole_b200.h, IPG_TRACE_*)
TRACE_DOUBLES = 127
TRACE_COLS = {"b": (0, 1), "ne": (1, 1), "thetae": (2, 1), "nu": (3, 1), "b_k_angle": (4, 1), "sigma": (5, 1),
              "beta": (6, 1), "dl": (7, 1), "r": (8, 1), "th": (9, 1), "phi": (10, 1), "j_unpol": (11, 1),
              "k_unpol": (12, 1), "I_unpol": (13, 1), "X": (14, 4), "Kcon": (18, 4), "j_inv": (22, 4),
              "alpha_inv": (26, 4), "rho_inv": (30, 4), "stokes": (34, 4), "e2Constructed": (38, 4),
              "e2ConstructedCov": (42, 4), "e2Transported": (46, 4), "e2TransportedCov": (50, 4),
              "prims": (54, 8), "ntetrad": (62, 16), "ncoord": (78, 16), "Econ": (94, 16), "Ecov": (110, 16),
              "flag": (126, 1)}


class IpgError(RuntimeError):
    def __init__(self, code, msg=""):
        self.code = code
        super().__init__(f"ipole_b200 error {code}: {msg}")


class Grid(C.Structure):
    _fields_ = [("n1", C.c_int), ("n2", C.c_int), ("n3", C.c_int),
                ("startx", C.c_double * 4), ("stopx", C.c_double * 4), ("dx", C.c_double * 4),
                ("cstartx", C.c_double * 4), ("cstopx", C.c_double * 4),
                ("a", C.c_double), ("hslope", C.c_double),
                ("poly_xt", C.c_double), ("poly_alpha", C.c_double), ("mks_smooth", C.c_double),
                ("poly_norm", C.c_double),
                ("Rin", C.c_double), ("Rout", C.c_double), ("Rh", C.c_double),
                ("rmin_geo", C.c_double), ("rmax_geo", C.c_double), ("th_beg", C.c_double),
                ("sigma_cut", C.c_double), ("sigma_cut_high", C.c_double), ("L_unit", C.c_double),
                ("metric", C.c_int)]


class Camera(C.Structure):
    _fields_ = [("Xcam", C.c_double * 4), ("Econ", (C.c_double * 4) * 4), ("Ecov", (C.c_double * 4) * 4),
                ("fovx", C.c_double), ("fovy", C.c_double), ("rotcam", C.c_double),
                ("xoff", C.c_double), ("yoff", C.c_double), ("freq", C.c_double), ("freqcgs", C.c_double),
                ("eps", C.c_double), ("nx", C.c_int), ("ny", C.c_int), ("maxnstep", C.c_int),
                ("only_unpolarized", C.c_int), ("emission_type", C.c_int), ("stokes_floors", C.c_int),
                ("target_nturns", C.c_int), ("subring_dtheta", C.c_int), ("counterjet", C.c_int)]


class PixelOut(C.Structure):
    _fields_ = [("I_unpol", C.c_double), ("tau", C.c_double), ("tauF", C.c_double),
                ("I", C.c_double), ("Q", C.c_double), ("U", C.c_double), ("V", C.c_double),
                ("nstep", C.c_int32), ("flag", C.c_int32)]


PIXEL_DTYPE = np.dtype([("I_unpol", "<f8"), ("tau", "<f8"), ("tauF", "<f8"), ("I", "<f8"), ("Q", "<f8"),
                        ("U", "<f8"), ("V", "<f8"), ("nstep", "<i4"), ("flag", "<i4")])
assert PIXEL_DTYPE.itemsize == C.sizeof(PixelOut)


class Stats(C.Structure):
    _fields_ = [("ray_steps", C.c_uint64), ("radiating_steps", C.c_uint64), ("launches", C.c_int32),
                ("waves", C.c_int32), ("geodesic_ms", C.c_double), ("transfer_ms", C.c_double),
                ("coeffs_ms", C.c_double), ("predict_ms", C.c_double), ("wall_ms", C.c_double),
                ("geodesic_span_ms", C.c_double), ("coeffs_span_ms", C.c_double), ("transfer_span_ms", C.c_double),
                ("adjoint_ms", C.c_double), ("adj_scatter_ms", C.c_double),
                ("long_class_items", C.c_uint64), ("start_waits_timed_out", C.c_uint64)]


class _Params(C.Structure):
    _fields_ = [("rcam", C.c_double), ("thetacam", C.c_double), ("phicam", C.c_double), ("rotcam", C.c_double),
                ("dx", C.c_double), ("dy", C.c_double), ("fovx_dsource", C.c_double), ("fovy_dsource", C.c_double),
                ("nx", C.c_int), ("ny", C.c_int), ("dsource", C.c_double), ("freqcgs", C.c_double),
                ("old_centering", C.c_int), ("eps", C.c_double), ("maxnstep", C.c_int),
                ("add_ppm", C.c_int), ("qu_conv", C.c_int), ("quench_output", C.c_int),
                ("only_unpolarized", C.c_int), ("perform_check", C.c_int),
                ("emission_type", C.c_int), ("stokes_floors", C.c_int), ("isolate_counterjet", C.c_int),
                ("dump", C.c_char * STRLEN), ("outf", C.c_char * STRLEN),
                ("target_nturns", C.c_int), ("subring_dtheta", C.c_int),
                ("nx_min", C.c_int), ("ny_min", C.c_int),
                ("refine_abs", C.c_double), ("refine_rel", C.c_double), ("refine_cut", C.c_double),
                ("nearest_neighbor", C.c_int), ("xoff", C.c_double), ("yoff", C.c_double),
                ("img_cadence", C.c_double), ("restart_int", C.c_double),
                ("trace", C.c_int), ("trace_stride", C.c_int), ("trace_i", C.c_int), ("trace_j", C.c_int),
                ("trace_outf", C.c_char * STRLEN), ("histo", C.c_int), ("histo_polar", C.c_int),
                ("histo_outf", C.c_char * STRLEN),
                ("MBH_solar", C.c_double), ("M_unit", C.c_double), ("target_mdot", C.c_double),
                ("tp_over_te", C.c_double), ("trat_small", C.c_double), ("trat_large", C.c_double),
                ("sigma_cut", C.c_double), ("sigma_cut_high", C.c_double), ("beta_crit", C.c_double),
                ("cooling_dynamical_times", C.c_double), ("rmax_geo", C.c_double), ("rmin_geo", C.c_double),
                ("reverse_field", C.c_int), ("polar_cut", C.c_double),
                ("dump_min", C.c_int), ("dump_max", C.c_int), ("dump_skip", C.c_int),
                ("model_kappa", C.c_double), ("powerlaw_gamma_cut", C.c_double), ("powerlaw_gamma_min", C.c_double),
                ("powerlaw_gamma_max", C.c_double), ("powerlaw_p", C.c_double), ("powerlaw_eta", C.c_double),
                ("variable_kappa", C.c_int), ("variable_kappa_min", C.c_double),
                ("variable_kappa_interp_start", C.c_double), ("variable_kappa_max", C.c_double),
                ("bremss", C.c_int), ("bremss_type", C.c_int),
                ("plugin", C.c_char * STRLEN), ("MBH_set", C.c_int), ("analytic_model", C.c_int),
                ("rho_unit", C.c_double), ("sphere_Thetae0", C.c_double), ("sphere_R0", C.c_double),
                ("sphere_tau0", C.c_double), ("sphere_beta0", C.c_double), ("sphere_gam", C.c_double),
                ("mixed_records", C.c_int), ("fp32_step", C.c_int), ("fp32_fits", C.c_int)]


class Plugin(C.Structure):
    """ipg_plugin: a known-answer model (kind 0 = the iharm dump model)."""
    _fields_ = [("kind", C.c_int), ("model", C.c_int),
                ("A", C.c_double), ("alpha", C.c_double), ("height", C.c_double), ("l0", C.c_double),
                ("freqcgs", C.c_double), ("rho_unit", C.c_double),
                ("R0", C.c_double), ("Ne0", C.c_double), ("Thetae0", C.c_double), ("B0", C.c_double),
                ("B_unit", C.c_double), ("sigma0", C.c_double), ("beta0", C.c_double)]


class _Model(C.Structure):
    _fields_ = [("grid", Grid), ("fields", C.POINTER(C.c_double) * NFIELD),
                ("M_unit", C.c_double), ("L_unit", C.c_double), ("T_unit", C.c_double), ("RHO_unit", C.c_double),
                ("U_unit", C.c_double), ("B_unit", C.c_double), ("Te_unit", C.c_double), ("MBH", C.c_double),
                ("Mdot_dump", C.c_double), ("MdotEdd_dump", C.c_double), ("Ladv_dump", C.c_double),
                ("t", C.c_double), ("DTd", C.c_double), ("electrons", C.c_int),
                ("gam", C.c_double), ("game", C.c_double), ("gamp", C.c_double), ("fluid_header", C.c_void_p),
                ("plugin", Plugin), ("trace_fields", C.POINTER(C.c_double) * 3),
                ("bmag_code", C.POINTER(C.c_double))]


class _Image(C.Structure):
    _fields_ = [("nx", C.c_size_t), ("ny", C.c_size_t), ("image", C.POINTER(C.c_double)),
                ("imageS", C.POINTER(C.c_double)), ("taus", C.POINTER(C.c_double)),
                ("interp_flag", C.POINTER(C.c_int)), ("scale", C.c_double), ("Xcam", C.c_double * 4),
                ("fovx", C.c_double), ("fovy", C.c_double), ("cam", Camera),
                ("oddflag", C.POINTER(C.c_int32)), ("nstep", C.POINTER(C.c_int32)), ("traced", C.c_size_t)]


class Grad(C.Structure):
    """ipg_grad: per-cell gradients and those of M_unit, R_high, R_low."""
    _fields_ = [("d_ne", C.POINTER(C.c_double)), ("d_thetae", C.POINTER(C.c_double)),
                ("d_b", C.POINTER(C.c_double)), ("d_M_unit", C.c_double), ("d_R_high", C.c_double),
                ("d_R_low", C.c_double)]


TRACER_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(Camera), C.POINTER(C.c_int32), C.c_size_t,
                        C.POINTER(PixelOut))

_lib = None


def lib():
    """Load libipole_b200.so (building it in-tree if it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    # IPOLE_B200_LIB selects another build of the library (code-generation
    # variants made with build.build(defines=..., out_dir=...))
    path = os.environ.get("IPOLE_B200_LIB") or _build.LIB
    if not os.path.exists(path):
        _build.build()
    L = C.CDLL(path)
    L.ipg_create.argtypes = [C.POINTER(C.c_void_p), C.c_int, C.c_size_t]
    L.ipg_destroy.argtypes = [C.c_void_p]
    L.ipg_destroy.restype = None
    L.ipg_strerror.restype = C.c_char_p
    L.ipg_strerror.argtypes = [C.c_int]
    L.ipg_last_error.restype = C.c_char_p
    L.ipg_last_error.argtypes = [C.c_void_p]
    L.ipg_upload_iharm.argtypes = [C.c_void_p, C.POINTER(Grid), C.POINTER(C.POINTER(C.c_double))]
    L.ipg_upload_plugin.argtypes = [C.c_void_p, C.POINTER(Grid), C.POINTER(Plugin)]
    L.ipg_upload_model.argtypes = [C.c_void_p, C.POINTER(_Model)]
    L.ipg_upload_trace_fields.argtypes = [C.c_void_p, C.POINTER(C.POINTER(C.c_double))]
    L.ipg_trace_ray.argtypes = [C.c_void_p, C.POINTER(Camera), C.c_int, C.c_int, C.c_size_t, C.c_void_p,
                                C.POINTER(C.c_int32)]
    L.ipg_write_traces.argtypes = [C.c_void_p, C.POINTER(_Image), C.POINTER(_Params), C.POINTER(_Model)]
    L.ipg_trace_pixels.argtypes = [C.c_void_p, C.POINTER(Camera), C.c_void_p, C.c_size_t, C.c_void_p]
    L.ipg_trace_pixels_device.argtypes = [C.c_void_p, C.POINTER(Camera), C.c_void_p, C.c_size_t, C.c_void_p,
                                          C.c_void_p]
    L.ipg_get_stats.argtypes = [C.c_void_p, C.POINTER(Stats)]
    L.ipg_get_stream.argtypes = [C.c_void_p, C.POINTER(C.c_void_p)]
    L.ipg_set_record_precision.argtypes = [C.c_void_p, C.c_int]
    L.ipg_set_step_precision.argtypes = [C.c_void_p, C.c_int]
    L.ipg_set_fit_precision.argtypes = [C.c_void_p, C.c_int]
    L.ipg_thermal_coefficients.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_int, C.c_int, C.c_void_p]
    L.ipg_camera_setup.argtypes = [C.POINTER(Grid)] + [C.c_double] * 9 + [C.c_int, C.c_int, C.c_double, C.c_int,
                                                                          C.POINTER(Camera), C.POINTER(C.c_double),
                                                                          C.POINTER(C.c_double),
                                                                          C.POINTER(C.c_double)]
    L.ipg_measure_fp64_peak.argtypes = [C.c_int, C.c_double, C.POINTER(C.c_double)]
    L.ipg_measure_fp32_peak.argtypes = [C.c_int, C.c_double, C.POINTER(C.c_double)]
    L.ipg_params_default.argtypes = [C.POINTER(_Params)]
    L.ipg_params_default.restype = None
    L.ipg_params_set.argtypes = [C.POINTER(_Params), C.c_char_p, C.c_char_p]
    L.ipg_params_set.restype = None
    L.ipg_params_load_file.argtypes = [C.POINTER(_Params), C.c_char_p]
    L.ipg_params_from_argv.argtypes = [C.POINTER(_Params), C.c_int, C.POINTER(C.c_char_p)]
    L.ipg_iharm_load.argtypes = [C.POINTER(_Params), C.POINTER(_Model)]
    L.ipg_iharm_free.argtypes = [C.POINTER(_Model)]
    L.ipg_iharm_free.restype = None
    L.ipg_render_image.argtypes = [C.c_void_p, C.POINTER(_Params), C.POINTER(_Model), C.POINTER(_Image), C.c_void_p]
    L.ipg_render_image_with.argtypes = [TRACER_FN, C.c_void_p, C.POINTER(_Params), C.POINTER(_Model),
                                        C.POINTER(_Image), C.c_void_p]
    L.ipg_image_free.argtypes = [C.POINTER(_Image)]
    L.ipg_image_free.restype = None
    L.ipg_image_totals.argtypes = [C.POINTER(_Image), C.POINTER(_Params), C.POINTER(C.c_double)]
    L.ipg_image_totals.restype = None
    L.ipg_print_image_stats.argtypes = [C.POINTER(_Image), C.POINTER(_Params), C.c_void_p]
    L.ipg_print_image_stats.restype = None
    L.ipg_write_image.argtypes = [C.c_char_p, C.POINTER(_Image), C.POINTER(_Params), C.POINTER(_Model)]
    L.ipg_container_convert.argtypes = [C.c_char_p, C.c_char_p]
    L.ipg_upload_model_batch.argtypes = [C.c_void_p, C.POINTER(_Model)]
    L.ipg_adjoint.argtypes = [C.c_void_p, C.POINTER(Camera), C.c_void_p, C.c_size_t, C.c_void_p, C.c_int,
                              C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    L.ipg_adjoint_params.argtypes = [C.c_void_p, C.POINTER(_Params), C.POINTER(_Model), C.c_void_p, C.c_int,
                                     C.POINTER(Grad), C.c_void_p]
    L.ipg_render_batch_params.argtypes = [C.c_void_p, C.POINTER(C.POINTER(_Params)), C.c_size_t, C.POINTER(_Model),
                                          C.POINTER(_Image), C.c_uint64, C.c_void_p]
    _lib = L
    return L


def _check(rc, ctx=None):
    if rc != IPG_OK:
        L = lib()
        msg = L.ipg_strerror(rc).decode()
        if ctx:
            msg += " (" + L.ipg_last_error(ctx).decode() + ")"
        raise IpgError(rc, msg)


class Params:
    """ipole parameters (src/par.c keys, iharm and radiation keys)."""

    def __init__(self):
        self._p = _Params()
        lib().ipg_params_default(C.byref(self._p))

    @classmethod
    def from_args(cls, argv):
        self = cls.__new__(cls)
        self._p = _Params()
        args = ["ipole"] + [str(a) for a in argv]
        arr = (C.c_char_p * len(args))(*[a.encode() for a in args])
        _check(lib().ipg_params_from_argv(C.byref(self._p), len(args), arr))
        return self

    def set(self, key, value):
        lib().ipg_params_set(C.byref(self._p), str(key).encode(), str(value).encode())
        return self

    def load_file(self, path):
        _check(lib().ipg_params_load_file(C.byref(self._p), str(path).encode()))
        return self

    def __getattr__(self, k):
        if k.startswith("_"):
            raise AttributeError(k)
        v = getattr(self._p, k)
        return v.decode() if isinstance(v, bytes) else v

    def copy(self):
        o = Params.__new__(Params)
        o._p = _Params()
        C.memmove(C.byref(o._p), C.byref(self._p), C.sizeof(_Params))
        return o


class Model:
    """iharm FMKS model after init_model (host arrays, ghost-padded)."""

    def __init__(self):
        self._m = _Model()
        self._owned = False

    @classmethod
    def load(cls, params: Params):
        self = cls()
        _check(lib().ipg_iharm_load(C.byref(params._p), C.byref(self._m)))
        self._owned = True
        return self

    @property
    def grid(self) -> Grid:
        return self._m.grid

    def field(self, idx: int) -> np.ndarray:
        g = self._m.grid
        n = (g.n1 + 2) * (g.n2 + 2) * (g.n3 + 2)
        return np.ctypeslib.as_array(self._m.fields[idx], shape=(n,)).reshape(g.n1 + 2, g.n2 + 2, g.n3 + 2)

    def __getattr__(self, k):
        if k.startswith("_"):
            raise AttributeError(k)
        return getattr(self._m, k)

    def close(self):
        if self._owned:
            lib().ipg_iharm_free(C.byref(self._m))
            self._owned = False

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Image:
    """Rendered image: arrays of main.c (image, imageS, taus) at params size."""

    def __init__(self, im: _Image, params: Params):
        nx, ny = int(params.nx), int(params.ny)
        inx, iny = int(im.nx), int(im.ny)
        self.internal_shape = (inx, iny)
        self.unpol = np.ctypeslib.as_array(im.image, shape=(inx * iny,)).reshape(inx, iny)[:nx, :ny].copy()
        self.tau = np.ctypeslib.as_array(im.taus, shape=(inx * iny,)).reshape(inx, iny)[:nx, :ny].copy()
        self.pol = None
        if im.imageS:
            self.pol = np.ctypeslib.as_array(im.imageS, shape=(inx * iny * 5,)).reshape(inx, iny, 5)[:nx, :ny].copy()
        self.interp_flag = np.ctypeslib.as_array(im.interp_flag, shape=(inx * iny,)).reshape(inx, iny)[:nx, :ny].copy()
        self.oddflag = np.ctypeslib.as_array(im.oddflag, shape=(inx * iny,)).reshape(inx, iny)[:nx, :ny].copy()
        self.nstep = np.ctypeslib.as_array(im.nstep, shape=(inx * iny,)).reshape(inx, iny)[:nx, :ny].copy()
        self.scale = im.scale
        self.traced = int(im.traced)
        self.camera = Camera()
        C.memmove(C.byref(self.camera), C.byref(im.cam), C.sizeof(Camera))

    def totals(self):
        """Ftot, Ftot_unpol, Qtot, Utot, Vtot in Jy (print_image_stats sums)."""
        s = self.scale
        if self.pol is None:
            return dict(Ftot=0.0, Ftot_unpol=float(self.unpol.sum() * s), Q=0.0, U=0.0, V=0.0)
        return dict(Ftot=float((self.pol[..., 0] * s).sum()), Ftot_unpol=float((self.unpol * s).sum()),
                    Q=float((self.pol[..., 1] * s).sum()), U=float((self.pol[..., 2] * s).sum()),
                    V=float((self.pol[..., 3] * s).sum()))


def camera_for(params: Params, grid: Grid) -> Camera:
    """ipg_camera_setup with the run parameters of ``params`` (main.c:125-168)."""
    p = params._p
    cam = Camera()
    scale, DX, DY = C.c_double(), C.c_double(), C.c_double()
    _check(lib().ipg_camera_setup(C.byref(grid), p.rcam, p.thetacam, p.phicam, p.rotcam, p.fovx_dsource,
                                  p.fovy_dsource, p.dx, p.dy, p.dsource, p.nx, p.ny, p.freqcgs, p.old_centering,
                                  C.byref(cam), C.byref(scale), C.byref(DX), C.byref(DY)))
    cam.xoff, cam.yoff, cam.eps, cam.maxnstep = p.xoff, p.yoff, p.eps, p.maxnstep
    cam.only_unpolarized, cam.emission_type, cam.stokes_floors = p.only_unpolarized, p.emission_type, p.stokes_floors
    cam.target_nturns, cam.subring_dtheta, cam.counterjet = p.target_nturns, p.subring_dtheta, p.isolate_counterjet
    cam._scale = scale.value
    return cam


class Context:
    """A CUDA context of the library (one per host thread)."""

    def __init__(self, device: int = 0, pool_bytes: int = 0):
        self._h = C.c_void_p()
        _check(lib().ipg_create(C.byref(self._h), int(device), int(pool_bytes)))

    def close(self):
        if self._h:
            lib().ipg_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def upload(self, model: Model):
        """The loaded model: an iharm dump's fields, or a known-answer model
        (ipg_upload_model)."""
        _check(lib().ipg_upload_model(self._h, C.byref(model._m)), self._h)

    def upload_arrays(self, grid: Grid, fields):
        arrs = [np.ascontiguousarray(f, dtype=np.float64).ravel() for f in fields]
        ptrs = (C.POINTER(C.c_double) * NFIELD)(*[a.ctypes.data_as(C.POINTER(C.c_double)) for a in arrs])
        _check(lib().ipg_upload_iharm(self._h, C.byref(grid), ptrs), self._h)

    def trace(self, cam: Camera, ij: np.ndarray, allow_maxnstep=False) -> np.ndarray:
        """ipg_trace_pixels on host arrays; ij is (n, 2) int32."""
        ij = np.ascontiguousarray(ij, dtype=np.int32).reshape(-1, 2)
        out = np.zeros(len(ij), dtype=PIXEL_DTYPE)
        rc = lib().ipg_trace_pixels(self._h, C.byref(cam), ij.ctypes.data, len(ij), out.ctypes.data)
        if not (allow_maxnstep and rc == IPG_E_MAXNSTEP):
            _check(rc, self._h)
        return out

    def trace_ray(self, cam: Camera, i: int, j: int, model: "Model" = None, max_steps: int = 50001):
        """Per-step trace of pixel (i, j) (ipg_trace_ray): (nstep, rows), rows
        an (nstep + 1, TRACE_DOUBLES) array in the IPG_TRACE_* column
        layout.  With an iharm model, its rho, u and beta are uploaded first
        so the primitives and beta columns are filled."""
        L = lib()
        if model is not None and model._m.plugin.kind == 0 and model._m.trace_fields[0]:
            ptrs = (C.POINTER(C.c_double) * 3)(*[model._m.trace_fields[k] for k in range(3)])
            _check(L.ipg_upload_trace_fields(self._h, ptrs), self._h)
        buf = np.zeros((max_steps, TRACE_DOUBLES))
        n = C.c_int32(0)
        _check(L.ipg_trace_ray(self._h, C.byref(cam), int(i), int(j), max_steps, buf.ctypes.data, C.byref(n)),
               self._h)
        return int(n.value), buf[:n.value + 1].copy()

    def trace_device(self, cam: Camera, d_ij_ptr: int, n: int, d_out_ptr: int, stream: int = 0):
        """ipg_trace_pixels_device on device pointers (e.g. torch tensors' data_ptr())."""
        _check(lib().ipg_trace_pixels_device(self._h, C.byref(cam), C.c_void_p(d_ij_ptr), n, C.c_void_p(d_out_ptr),
                                             C.c_void_p(stream)), self._h)

    def set_record_precision(self, precision: int):
        """ipg_set_record_precision: IPG_RECORDS_FP64 (default) or
        IPG_RECORDS_MIXED (transport matrices and tetrad rows stored in
        FP32 between the kernels)."""
        _check(lib().ipg_set_record_precision(self._h, int(precision)), self._h)

    def set_step_precision(self, precision: int):
        """ipg_set_step_precision: IPG_STEP_FP64 (default) or IPG_STEP_FP32
        (the polarized step's Faraday rotation and absorption/emission in
        FP32)."""
        _check(lib().ipg_set_step_precision(self._h, int(precision)), self._h)

    def set_fit_precision(self, precision: int):
        """ipg_set_fit_precision: IPG_FITS_FP64 (default) or IPG_FITS_FP32
        (the thermal fits' shapes in FP32, prefactors and exponents in
        FP64)."""
        _check(lib().ipg_set_fit_precision(self._h, int(precision)), self._h)

    def thermal_coefficients(self, points, emission_type: int = 4, precision: int = IPG_FITS_FP64):
        """ipg_thermal_coefficients: points (n, 5) = (nu, Ne, Thetae, B,
        theta) -> (n, 12) = (jI/nu^2, aI of get_jkinv; jI jQ jU jV aI aQ aU
        aV rQ rV of jar_calc)."""
        pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 5)
        out = np.zeros((len(pts), 12))
        _check(lib().ipg_thermal_coefficients(self._h, pts.ctypes.data, len(pts), int(emission_type),
                                              int(precision), out.ctypes.data), self._h)
        return out

    def stream(self) -> int:
        """The context's cudaStream_t as an integer handle."""
        s = C.c_void_p()
        _check(lib().ipg_get_stream(self._h, C.byref(s)))
        return s.value or 0

    def stats(self) -> dict:
        s = Stats()
        _check(lib().ipg_get_stats(self._h, C.byref(s)))
        return {k: getattr(s, k) for k, _ in Stats._fields_}

    def upload_batch(self, model: Model):
        """ipg_upload_model_batch: the dump's primitives for batched
        instances (render_batch)."""
        _check(lib().ipg_upload_model_batch(self._h, C.byref(model._m)), self._h)

    def render_batch(self, params_list, model: Model, step_budget: int = 0):
        """ipg_render_batch_params: one Image per Params, rendered in one
        batch (instances with the same camera share their geodesics)."""
        return _render_batch(self._h, params_list, model, step_budget)

    def adjoint(self, cam: Camera, ij: np.ndarray, dL_dout: np.ndarray, ncell: int, ckpt: int = 16):
        """ipg_adjoint: per-cell dL/dne, dL/dTheta_e, dL/d|B| (each (ncell,))
        for dL_dout = dL/d(I, Q, U, V) of the pixels ij (get_pixel outputs),
        and the forward outputs the call traced."""
        ij = np.ascontiguousarray(ij, dtype=np.int32).reshape(-1, 2)
        dL = np.ascontiguousarray(dL_dout, dtype=np.float64).reshape(len(ij), 4)
        g = np.zeros((3, ncell))
        out = np.zeros(len(ij), dtype=PIXEL_DTYPE)
        _check(lib().ipg_adjoint(self._h, C.byref(cam), ij.ctypes.data, len(ij), dL.ctypes.data, int(ckpt),
                                 g[0].ctypes.data, g[1].ctypes.data, g[2].ctypes.data, out.ctypes.data), self._h)
        return g, out

    def adjoint_image(self, params: Params, model: Model, dL_dpol: np.ndarray, ckpt: int = 16):
        """ipg_adjoint_params: gradients of a loss of the (unrefined)
        polarized image from dL/dpol (nx, ny, 4).  Returns a dict with the
        per-cell gradients (ghost-padded (n1+2, n2+2, n3+2) arrays "ne",
        "thetae", "b"), the scalars "M_unit", "R_high", "R_low" and the image
        "pol" (nx, ny, 4) the adjoint traced."""
        p = params.copy()
        gr = model.grid
        shape = (gr.n1 + 2, gr.n2 + 2, gr.n3 + 2)
        ncell = shape[0] * shape[1] * shape[2]
        dL = np.ascontiguousarray(dL_dpol, dtype=np.float64)
        arrs = [np.empty(ncell) for _ in range(3)]  # every cell is written
        g = Grad()
        g.d_ne, g.d_thetae, g.d_b = [a.ctypes.data_as(C.POINTER(C.c_double)) for a in arrs]
        pol = np.zeros(dL.shape)
        _check(lib().ipg_adjoint_params(self._h, C.byref(p._p), C.byref(model._m), dL.ctypes.data, int(ckpt),
                                        C.byref(g), pol.ctypes.data), self._h)
        return dict(ne=arrs[0].reshape(shape), thetae=arrs[1].reshape(shape), b=arrs[2].reshape(shape),
                    M_unit=g.d_M_unit, R_high=g.d_R_high, R_low=g.d_R_low, pol=pol)

    def render(self, params: Params, model: Model, log=False) -> Image:
        """Full image with adaptive refinement (main.c fast-light driver)."""
        p = params.copy()
        im = _Image()
        L = lib()
        rc = L.ipg_render_image(self._h, C.byref(p._p), C.byref(model._m), C.byref(im), None)
        try:
            _check(rc, self._h)
            img = Image(im, params)
            img.params_after = p
        finally:
            L.ipg_image_free(C.byref(im))
        return img


def _render_batch(ctx_h, params_list, model: "Model", step_budget: int = 0):
    n = len(params_list)
    ps = [p.copy() for p in params_list]
    arr = (C.POINTER(_Params) * n)(*[C.pointer(p._p) for p in ps])
    ims = (_Image * n)()
    L = lib()
    rc = L.ipg_render_batch_params(ctx_h, arr, n, C.byref(model._m), ims, int(step_budget), None)
    try:
        _check(rc, ctx_h)
        out = []
        for k in range(n):
            img = Image(ims[k], params_list[k])
            img.params_after = ps[k]
            out.append(img)
    finally:
        for k in range(n):
            L.ipg_image_free(C.byref(ims[k]))
    return out


def render_with(tracer, params: Params, model: Model) -> Image:
    """The host image driver (ipg_render_image_with) with a Python tracer:
    ``tracer(cam, ij)`` gets the Camera and an (n, 2) int32 pixel list and
    returns an (n,) PIXEL_DTYPE array (get_pixel outputs)."""
    err = []

    def cb(user, cam_p, ij_p, n, out_p):
        try:
            ij = np.ctypeslib.as_array(ij_p, shape=(2 * n,)).reshape(n, 2).copy()
            res = np.asarray(tracer(cam_p.contents, ij), dtype=PIXEL_DTYPE)
            C.memmove(out_p, res.ctypes.data, n * PIXEL_DTYPE.itemsize)
            return IPG_E_MAXNSTEP if np.any(res["nstep"] >= cam_p.contents.maxnstep - 1) else IPG_OK
        except Exception as e:  # surfaced after the call
            err.append(e)
            return IPG_E_ARG

    fn = TRACER_FN(cb)
    p = params.copy()
    im = _Image()
    L = lib()
    rc = L.ipg_render_image_with(fn, None, C.byref(p._p), C.byref(model._m), C.byref(im), None)
    try:
        if err:
            raise err[0]
        _check(rc)
        img = Image(im, params)
        img.params_after = p
    finally:
        L.ipg_image_free(C.byref(im))
    return img


def trace_pixels(ctx: Context, cam: Camera, ij) -> np.ndarray:
    return ctx.trace(cam, ij)


def convert_container(src: str, dst: str) -> None:
    """Copy a dump or image between HDF5 and the IPGC container
    (``ipg_container_convert``): the source format is detected, the
    destination is IPGC when its name ends in ``.ipgc``, HDF5 otherwise."""
    _check(lib().ipg_container_convert(os.fsencode(src), os.fsencode(dst)))


def fp64_peak_tflops(device: int = 0, ms: float = 200.0) -> float:
    v = C.c_double()
    _check(lib().ipg_measure_fp64_peak(int(device), float(ms), C.byref(v)))
    return v.value


def fp32_peak_tflops(device: int = 0, ms: float = 200.0) -> float:
    v = C.c_double()
    _check(lib().ipg_measure_fp32_peak(int(device), float(ms), C.byref(v)))
    return v.value
