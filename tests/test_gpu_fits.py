"""The thermal fits at points on the GPU (ipg_thermal_coefficients).

FP64 (the kernels' default form): against the coefficients the reference
wrote in its per-step traces, and against the oracle's fits over a seeded
sample of plasma parameters far wider than the flows' (both emission
types).  FP32 shapes (IPG_FITS_FP32): the same points, with the error
distribution printed.

Errors are taken relative to the coefficient's own family at the point:
|d - r| / (|r| + 1e-9 s), s = the magnitude of j_I (emissivities), a_I
(absorptivities) or sqrt(rho_Q^2 + rho_V^2) (rotativities), so that a
coefficient crossing zero (rho_Q's fit changes sign) is measured against
the size of its family.
"""
import numpy as np
import pytest

import ipole_b200 as ip
from oracle import oracle as O
from tests import fits_points

pytestmark = pytest.mark.gpu

COL = fits_points.COLUMNS


def family_scale(r):
    s = np.zeros_like(r)
    s[:, 0] = np.abs(r[:, 0])
    s[:, 1] = np.abs(r[:, 1])
    for k in (2, 3, 4, 5):
        s[:, k] = np.abs(r[:, 2])
    for k in (6, 7, 8, 9):
        s[:, k] = np.abs(r[:, 6])
    s[:, 10] = s[:, 11] = np.hypot(r[:, 10], r[:, 11])
    return s


# coefficients below this are far below anything an image can register
# (j/nu^2 of the flows is ~1e-43..1e-30, a ~1e-12..1e3 per cm); where one
# side underflows to zero in an intermediate and the other keeps a value of
# this size, the two agree
TINY = 1e-250


def rel_err(d, r):
    s = family_scale(r)
    den = np.abs(r) + 1e-9 * s + TINY
    return np.abs(d - r) / den


def subnormal_k2(pts):
    """Theta_e < 1/708: K_1(1/Theta_e), K_2(1/Theta_e) are subnormal (or
    zero) in FP64, so the reference's rotativities there are ratios of
    numbers with few significant bits"""
    return pts[:, 2] < 1. / 708.


def subnormal_tolerance(pts):
    """relative tolerance of a ratio K_n/K_2 whose terms are subnormal: four
    spacings of the subnormal range (4.94e-324) over the smallest term"""
    from scipy.special import kve
    a = 1. / pts[:, 2]
    with np.errstate(all="ignore"):
        k = np.minimum(kve(1, a), kve(2, a)) * np.exp(-a)
        tol = np.where(k > 0, 4 * 4.94e-324 / np.where(k > 0, k, 1.), np.inf)
    return np.maximum(tol, 1e-10)


def summary(e):
    return {COL[k]: f"{e[:, k].max():.1e}/{np.quantile(e[:, k], 0.999):.1e}" for k in range(12)}


@pytest.fixture(scope="module")
def ctx():
    with ip.Context() as c:
        yield c


def test_fp64_fits_against_reference_trace(ctx):
    pts, ref = fits_points.trace_points()
    d = ctx.thermal_coefficients(pts, 4, ip.IPG_FITS_FP64)
    e = rel_err(d, ref)
    print("fp64 vs reference trace (max/p99.9):", summary(e))
    i = int(np.argmax(e.max(1)))
    print("  worst point", pts[i].tolist(), "column", COL[int(np.argmax(e[i]))])
    assert e.max() <= 1e-12


@pytest.mark.parametrize("em", [4, 1])
def test_fp64_fits_against_oracle_wide(ctx, em):
    pts = fits_points.grid_points()
    ref = O.thermal_coefficients(pts, em)
    d = ctx.thermal_coefficients(pts, em, ip.IPG_FITS_FP64)
    finite = np.isfinite(ref).all(1)
    odd = np.where(np.isfinite(d).all(1) != finite)[0]
    for i in odd[:6]:
        print("not finite in one of the two:", pts[i].tolist(), "\n  device", d[i].tolist(), "\n  oracle", ref[i].tolist())
    assert len(odd) == 0, len(odd)
    sub = subnormal_k2(pts)
    e = rel_err(d[finite & ~sub], ref[finite & ~sub])
    es = rel_err(d[finite & sub], ref[finite & sub])
    print(f"fp64 vs oracle, emission {em} (max/p99.9):", summary(e))
    tol = subnormal_tolerance(pts[finite & sub])[:, None]
    print(f"  Theta_e < 1/708 ({int(sub.sum())} points): max {es.max() if es.size else 0.:.2e}, "
          f"max over its bound {(es / tol).max() if es.size else 0.:.2e}")
    assert e.max() <= 1e-10
    assert es.size == 0 or (es <= tol).all()


@pytest.mark.parametrize("em", [4, 1])
def test_fp32_fits_error_distribution(ctx, em):
    pts = np.concatenate([fits_points.trace_points()[0], fits_points.grid_points()])
    ref = ctx.thermal_coefficients(pts, em, ip.IPG_FITS_FP64)
    d = ctx.thermal_coefficients(pts, em, ip.IPG_FITS_FP32)
    finite = np.isfinite(ref).all(1) & np.isfinite(d).all(1)
    print("points not finite:", int((~finite).sum()))
    sub = subnormal_k2(pts)
    es = rel_err(d[finite & sub], ref[finite & sub])
    print(f"  Theta_e < 1/708 ({int((finite & sub).sum())} points, FP64 K_n subnormal): max {es.max() if es.size else 0.:.2e}")
    finite &= ~sub
    e = rel_err(d[finite], ref[finite])
    print(f"fp32 vs fp64 fits, emission {em} (max/p99.9):", summary(e))
    w = np.argsort(e.max(1))[::-1][:5]
    for i in w:
        print("  worst", pts[finite][i].tolist(), COL[int(np.argmax(e[i]))], f"{e[i].max():.2e}")
    # the flows' own points (the traces) and the wide sample
    ntr = int(finite[:len(fits_points.trace_points()[0])].sum())
    print("  trace points max:", f"{e[:ntr].max():.2e}", " wide sample p99:", f"{np.quantile(e[ntr:], 0.99):.2e}")
    assert np.quantile(e, 0.99) <= 1e-4
    assert e[:ntr].max() <= 1e-4


def test_fits_arguments(ctx):
    with pytest.raises(ip.IpgError) as err:
        ctx.thermal_coefficients(np.ones((1, 5)), 7)
    assert err.value.code == ip.IPG_E_ARG
    with pytest.raises(ip.IpgError) as err:
        ctx.thermal_coefficients(np.ones((1, 5)), 4, 5)
    assert err.value.code == ip.IPG_E_ARG
    assert ctx.thermal_coefficients(np.zeros((0, 5))).shape == (0, 12)
