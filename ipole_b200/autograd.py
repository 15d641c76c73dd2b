"""torch.autograd wrapper of the adjoint, for fitting images.

``IQUVImage`` maps the per-cell fluid fields ne, Theta_e and |B| (torch
tensors in the ghost-padded (n1+2, n2+2, n3+2) layout of the model) to the
polarized image pol (nx, ny, 4) of one camera, as the image file holds it
(I, Q, U, V times nu^3, Q and U negated for qu_conv = 0).  Its forward pass
uploads the fields and traces every pixel; its backward pass calls
ipg_adjoint, which walks each ray back to front (no refinement: the adjoint
needs every pixel).

``derived_fields`` is init_physical_quantities (model/iharm/model.c:610-717,
ELECTRONS == 2) written in torch, so that the electron model's parameters
M_unit, R_high and R_low can be fitted through it: autograd chains their
gradients through ne (proportional to M_unit), |B| (to its square root) and
Theta_e (through R_high, R_low).

    fit = IQUVImage(ctx, params, model)
    ne, th, b = derived_fields(fit.prims, M_unit, R_high, R_low)
    loss = ((fit(ne, th, b) - target) ** 2).sum()
    loss.backward()
"""
from __future__ import annotations

import numpy as np
import torch

import ipole_b200 as ip

# CGS constants of the derived fields (the reference's constants.h values)
MP, ME, CL = 1.67262171e-24, 9.1093826e-28, 2.99792458e10


class _IQUV(torch.autograd.Function):
    @staticmethod
    def forward(fctx, ne, thetae, b, fit):
        fields = fit._fields(ne, thetae, b)
        fit.ctx.upload_arrays(fit.grid, fields)
        out = fit.ctx.trace(fit.cam, fit.ij)
        fctx.fit = fit
        fctx.fields = fields
        return torch.from_numpy(fit._pol(out)).to(ne.device)

    @staticmethod
    def backward(fctx, gpol):
        fit = fctx.fit
        fit.ctx.upload_arrays(fit.grid, fctx.fields)
        g = gpol.detach().cpu().numpy().astype(np.float64).reshape(-1, 4) * fit.f3
        dL = np.stack([g[:, 0], fit.sq * g[:, 1], fit.sq * g[:, 2], g[:, 3]], axis=1)
        grads, _ = fit.ctx.adjoint(fit.cam, fit.ij, dL, fit.ncell, fit.ckpt)
        dev = gpol.device
        return (torch.from_numpy(grads[0].reshape(fit.shape)).to(dev),
                torch.from_numpy(grads[1].reshape(fit.shape)).to(dev),
                torch.from_numpy(grads[2].reshape(fit.shape)).to(dev), None)


class IQUVImage:
    """The differentiable polarized image of one camera (``params``) over the
    grid and velocity/field primitives of ``model``."""

    def __init__(self, ctx: "ip.Context", params: "ip.Params", model: "ip.Model", ckpt: int = 16):
        self.ctx, self.ckpt = ctx, ckpt
        self.grid = model.grid
        g = self.grid
        self.shape = (g.n1 + 2, g.n2 + 2, g.n3 + 2)
        self.ncell = int(np.prod(self.shape))
        self.cam = ip.camera_for(params, g)
        self.nx, self.ny = int(params.nx), int(params.ny)
        self.ij = np.array([(i, j) for i in range(self.nx) for j in range(self.ny)], np.int32)
        self.f3 = float(params.freqcgs) ** 3
        self.sq = 1.0 if params.qu_conv else -1.0
        # the fields the fit does not vary: U1..3, B1..3 and sigma
        self.fixed = [np.array(model.field(q)) for q in range(6)]
        self.sigma = np.array(model.field(9))
        m = model._m
        n = self.ncell
        self.prims = dict(
            rho=torch.from_numpy(np.ctypeslib.as_array(m.trace_fields[0], shape=(n,)).reshape(self.shape).copy()),
            u=torch.from_numpy(np.ctypeslib.as_array(m.trace_fields[1], shape=(n,)).reshape(self.shape).copy()),
            b=torch.from_numpy((model.field(8).ravel() / m.B_unit).reshape(self.shape).copy()),
            L_unit=float(m.L_unit), gam=float(m.gam), game=float(m.game), gamp=float(m.gamp))

    def _fields(self, ne, thetae, b):
        t = [x.detach().cpu().numpy().astype(np.float64).reshape(self.shape) for x in (ne, thetae, b)]
        return [*self.fixed, t[0], t[1], t[2], self.sigma]

    def _pol(self, out):
        pol = np.zeros((self.nx, self.ny, 4))
        i, j = self.ij[:, 0], self.ij[:, 1]
        pol[i, j, 0] = out["I"] * self.f3
        pol[i, j, 1] = self.sq * out["Q"] * self.f3
        pol[i, j, 2] = self.sq * out["U"] * self.f3
        pol[i, j, 3] = out["V"] * self.f3
        return pol

    def __call__(self, ne, thetae, b):
        return _IQUV.apply(ne, thetae, b, self)


def derived_fields(prims: dict, M_unit, R_high, R_low, beta_crit: float = 1.0):
    """ne, Theta_e, |B| of every cell for the electron model (M_unit, R_high,
    R_low), from rho, u and |b| in code units (init_physical_quantities,
    model/iharm/model.c:610-717; Theta_e floored at 1e-3).  The arguments may
    be tensors that require gradients."""
    M_unit, R_high, R_low = (torch.as_tensor(x, dtype=torch.float64) for x in (M_unit, R_high, R_low))
    rho, u, bc = prims["rho"], prims["u"], prims["b"]
    RHO_unit = M_unit / prims["L_unit"] ** 3
    B_unit = CL * torch.sqrt(4.0 * np.pi * RHO_unit)
    ne = rho * RHO_unit / (MP + ME)
    bsq = bc * bc
    beta = u * (prims["gam"] - 1.0) / 0.5 / bsq
    betasq = beta * beta / beta_crit / beta_crit
    trat = R_high * betasq / (1.0 + betasq) + R_low / (1.0 + betasq)
    game, gamp = prims["game"], prims["gamp"]
    th = (MP / ME) * (game - 1.0) * (gamp - 1.0) / ((gamp - 1.0) + (game - 1.0) * trat) * u / rho
    th = torch.clamp(th, min=1e-3)
    return ne, th, bc * B_unit
