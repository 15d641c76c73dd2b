"""Seeded synthetic iharm dumps in Funky MKS (FMKS) coordinates.

The reference's sample GRMHD dumps are not distributable here, so benchmarks
and parity tests image a seeded synthetic dump that follows the iharm v1
schema read by model/iharm/model.c:848-1074 (grid header) and :1876-1949
(primitives):

    /header/{version, n1, n2, n3, n_prim=8, gam=13/9, metric="FMKS"}
    /header/geom/{startx1..3, dx1..3}
    /header/geom/mmks/{a, hslope, Rin, Rout, poly_xt, poly_alpha, mks_smooth}
    /dump_cadence, /t
    /prims[N1][N2][N3][8]   rho, u, U1..U3 (utilde^i, native FMKS), B1..B3

There is no /header/has_electrons and no /header/weights, so the reference
uses its mixed R_high/R_low electron model (ELECTRONS == 2).

Physical content (all in code units, GM = c = 1):
  * an FM-like torus: rho = [1 - ((R - r_c)/w)^2 - (z/(h R))^2]_+^(1/(gam-1)),
    u = K rho^gam, on a hot power-law atmosphere; rho and u carry seeded 5%
    lognormal noise;
  * sub-Keplerian rotation utilde^3 = 1/(r^1.5 + a) with a slow radial inflow
    utilde^1 = -0.1 r^-1.5, plus 1% seeded Gaussian noise on each component;
  * B^i = *F^{it} from a vector potential: one poloidal loop A_phi ~ (rho -
    0.05 rho_max)_+ scaled so that max(P_gas) / max(P_mag) = 10, plus a
    weak vertical background field so that |b| > 0 in every zone (the
    reference's electron model divides by b^2) and sigma > 1 in the funnel.

The construction is deterministic for a given (shape, seed) through numpy's
PCG64 generator.
"""
from __future__ import annotations

import hashlib
import math

import numpy as np

from . import ipgc

FMKS_DEFAULTS = dict(a=0.9375, hslope=0.3, poly_xt=0.82, poly_alpha=14.0,
                     mks_smooth=0.5, Rin=1.2, Rout=50.0)
GAM = 13.0 / 9.0
BETA_NORM = 10.0  # max(P_gas) / max(P_mag) of the poloidal loop


def fmks_theta(X1, X2, startx1, p):
    """theta(X1, X2) of FMKS coordinates (src/coordinates.c:75-81)."""
    hslope, xt, al, sm = p["hslope"], p["poly_xt"], p["poly_alpha"], p["mks_smooth"]
    poly_norm = 0.5 * math.pi * 1.0 / (1.0 + 1.0 / (al + 1.0) * 1.0 / xt ** al)
    thG = math.pi * X2 + ((1.0 - hslope) / 2.0) * np.sin(2.0 * math.pi * X2)
    y = 2 * X2 - 1.0
    thJ = poly_norm * y * (1.0 + (y / xt) ** al / (al + 1.0)) + 0.5 * math.pi
    return thG + np.exp(sm * (startx1 - X1)) * (thJ - thG)


def fmks_dthdx2(X1, X2, startx1, p):
    """d theta / d X2 of FMKS coordinates (src/coordinates.c:294-304)."""
    hslope, xt, al, sm = p["hslope"], p["poly_xt"], p["poly_alpha"], p["mks_smooth"]
    poly_norm = 0.5 * math.pi * 1.0 / (1.0 + 1.0 / (al + 1.0) * 1.0 / xt ** al)
    y = 2.0 * X2 - 1.0
    return (math.pi + (1.0 - hslope) * math.pi * np.cos(2.0 * math.pi * X2)
            + np.exp(sm * (startx1 - X1))
            * (-math.pi + 2.0 * poly_norm * (1.0 + (y / xt) ** al / (al + 1.0))
               + (2.0 * al * poly_norm * y * (y / xt) ** (al - 1.0)) / ((1.0 + al) * xt)
               - (1.0 - hslope) * math.pi * np.cos(2.0 * math.pi * X2)))


def make_iharm_dump(n1: int, n2: int, n3: int, seed: int = 1, **geom) -> dict:
    """Return the container entries of a synthetic FMKS iharm dump."""
    p = dict(FMKS_DEFAULTS)
    p.update(geom)
    a = p["a"]
    startx1 = math.log(p["Rin"])
    dx1 = (math.log(p["Rout"]) - startx1) / n1
    startx2, dx2 = 0.0, 1.0 / n2
    startx3, dx3 = 0.0, 2.0 * math.pi / n3

    X1 = startx1 + (np.arange(n1) + 0.5) * dx1
    X2 = startx2 + (np.arange(n2) + 0.5) * dx2
    X1g, X2g = np.meshgrid(X1, X2, indexing="ij")
    r = np.exp(X1g)
    th = fmks_theta(X1g, X2g, startx1, p)
    R = r * np.sin(th)
    z = r * np.cos(th)

    # FM-like torus on a hot atmosphere (axisymmetric part)
    rc, w, h, K = 13.0, 7.0, 0.35, 0.02
    q = 1.0 - ((R - rc) / w) ** 2 - (z / (h * np.maximum(R, 1e-3))) ** 2
    rho_t = np.where(q > 0, np.maximum(q, 0.0) ** (1.0 / (GAM - 1.0)), 0.0)
    u_t = K * rho_t ** GAM
    # hot, geometrically thick inflow from the torus to the horizon
    rho_i = 0.2 * (r / 6.0) ** -1.0 * np.exp(-np.cos(th) ** 2 / (2 * 0.3 ** 2))
    u_i = rho_i * 0.8 / r
    rho_atm = 1e-4 * r ** -1.5
    u_atm = 0.05 / r * rho_atm
    rho2 = rho_t + rho_i + rho_atm
    u2 = u_t + u_i + u_atm

    # magnetic field from A_phi: one loop + weak vertical background
    rho_max = (rho_t + rho_i).max()
    A = np.maximum(rho_t + rho_i - 0.05 * rho_max, 0.0)
    sig = r * r + a * a * np.cos(th) ** 2
    gdet = sig * np.sin(th) * r * fmks_dthdx2(X1g, X2g, startx1, p)
    dAdx1, dAdx2 = np.gradient(A, dx1, dx2)
    B1l = dAdx2 / gdet
    B2l = -dAdx1 / gdet
    Ab = 0.5 * R * R
    dbdx1, dbdx2 = np.gradient(Ab, dx1, dx2)
    B1b = dbdx2 / gdet
    B2b = -dbdx1 / gdet
    # scale the loop so that max(P_gas) / max(P_mag) = 100 over the grid (the
    # usual GRMHD normalisation), with b^2 ~ g_11 B1^2 + g_22 B2^2; the
    # background field has b^2 ~ 2e-4 (it sets sigma > 1 in the polar funnel)
    g11 = (1.0 + 2.0 * r / sig) * r * r
    g22 = sig * fmks_dthdx2(X1g, X2g, startx1, p) ** 2
    bsq_loop = g11 * B1l ** 2 + g22 * B2l ** 2
    P = (GAM - 1.0) * u2.max()
    loop_scale = math.sqrt(P / (0.5 * BETA_NORM) / max(float(bsq_loop.max()), 1e-300))
    bsq_bg = g11 * B1b ** 2 + g22 * B2b ** 2
    bg_scale = math.sqrt(2e-4 / max(float(np.median(bsq_bg)), 1e-300))
    B1 = loop_scale * B1l + bg_scale * B1b
    B2 = loop_scale * B2l + bg_scale * B2b

    # velocities
    U1 = -0.1 * r ** -1.5
    U3 = 1.0 / (r ** 1.5 + a)

    rng = np.random.default_rng(seed)
    shape3 = (n1, n2, n3)
    prims = np.empty((n1, n2, n3, 8), dtype=np.float64)
    prims[..., 0] = rho2[:, :, None] * np.exp(0.05 * rng.standard_normal(shape3))
    prims[..., 1] = u2[:, :, None] * np.exp(0.05 * rng.standard_normal(shape3))
    umag = np.sqrt(U1 ** 2 + U3 ** 2)[:, :, None]
    prims[..., 2] = U1[:, :, None] + 0.01 * umag * rng.standard_normal(shape3)
    prims[..., 3] = 0.01 * umag * rng.standard_normal(shape3)
    prims[..., 4] = U3[:, :, None] + 0.01 * umag * rng.standard_normal(shape3)
    prims[..., 5] = B1[:, :, None]
    prims[..., 6] = B2[:, :, None]
    prims[..., 7] = 0.0

    e = {
        "/header/version": "iharm-synthetic-1",
        "/header/n1": np.int32(n1), "/header/n2": np.int32(n2), "/header/n3": np.int32(n3),
        "/header/n_prim": np.int32(8),
        "/header/gam": np.float64(GAM),
        "/header/metric": "FMKS",
        "/header/geom/startx1": np.float64(startx1),
        "/header/geom/startx2": np.float64(startx2),
        "/header/geom/startx3": np.float64(startx3),
        "/header/geom/dx1": np.float64(dx1),
        "/header/geom/dx2": np.float64(dx2),
        "/header/geom/dx3": np.float64(dx3),
        "/header/geom/mmks/a": np.float64(a),
        "/header/geom/mmks/hslope": np.float64(p["hslope"]),
        "/header/geom/mmks/Rin": np.float64(p["Rin"]),
        "/header/geom/mmks/Rout": np.float64(p["Rout"]),
        "/header/geom/mmks/poly_xt": np.float64(p["poly_xt"]),
        "/header/geom/mmks/poly_alpha": np.float64(p["poly_alpha"]),
        "/header/geom/mmks/mks_smooth": np.float64(p["mks_smooth"]),
        "/dump_cadence": np.float64(5.0),
        "/t": np.float64(10000.0),
        "/prims": prims,
    }
    return e


def write_iharm_dump(path: str, n1: int, n2: int, n3: int, seed: int = 1, **geom) -> str:
    """Write a synthetic dump to ``path``; returns the sha256 of its prims."""
    e = make_iharm_dump(n1, n2, n3, seed, **geom)
    ipgc.write(path, e, strlen={"/header/version": 20, "/header/metric": 20})
    return hashlib.sha256(e["/prims"].tobytes()).hexdigest()
