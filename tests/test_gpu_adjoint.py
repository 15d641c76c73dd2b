"""The adjoint of the polarized image (GPU): gradients of an image loss
against central finite differences of the GPU images and of the reference's
images, checkpoint intervals, the torch.autograd wrapper, and the forward
image the adjoint traces.

The loss is the L2 distance between the image and a target image rendered at
perturbed parameters (M_unit x 1.3, R_high 20 -> 25), normalized by the
target's largest intensity.  Finite differences are central; the adjoint
must match them to 1e-4 relative.  The loss turns fast with the Faraday
rotation of this image: the central difference with a relative step of 1e-4
is still 1.7% from its limit for M_unit (1e-5: 0.02%, 1e-6: 2e-6, measured
on the oracle), so the checks take steps of 1e-6 (FP64 rounding of the
loss stays ~1e-9 of the difference there) and show the convergence.
"""
import json
import os

import numpy as np
import pytest

import ipole_b200 as ip
from tests import common

pytestmark = pytest.mark.gpu

EPS = 1e-6
TOL = 1e-4
BASE = ["--freqcgs=230.e9", "--thetacam=163", "--phicam=0", "--rotcam=0", "--MBH=6.5e9", "--dsource=16.8e6",
        "--fov=160", "--trat_small=1", "--nx=16", "--ny=16"]
PARAMS = {"M_unit": 3e27, "trat_large": 20.0, "trat_small": 1.0}
TARGET = {"M_unit": 3.9e27, "trat_large": 25.0, "trat_small": 1.0}


def _params(dump, **kw):
    v = dict(PARAMS, **kw)
    return ip.Params.from_args([f"--dump={dump}", *BASE, f"--M_unit={v['M_unit']!r}",
                                f"--trat_large={v['trat_large']!r}", f"--trat_small={v['trat_small']!r}"])


@pytest.fixture(scope="module")
def setup(dumps):
    meta, _ = common.load_golden("c1_bright_32")
    dump = dumps.get(meta)
    ctx = ip.Context()
    pt = _params(dump, **TARGET)
    mt = ip.Model.load(pt)
    ctx.upload(mt)
    target = ctx.render(pt, mt).pol[..., :4].copy()
    scale = float(np.abs(target[..., 0]).max())
    yield dict(dump=dump, ctx=ctx, target=target, scale=scale)
    ctx.close()


def _loss(pol, s):
    r = (pol[..., :4] - s["target"]) / s["scale"]
    return float((r * r).sum()), 2.0 * r / s["scale"]


def _loss_at(s, **kw):
    p = _params(s["dump"], **kw)
    m = ip.Model.load(p)
    s["ctx"].upload(m)
    return _loss(s["ctx"].render(p, m).pol, s)[0]


def test_adjoint_scalars_match_finite_differences(setup):
    s = setup
    p = _params(s["dump"])
    m = ip.Model.load(p)
    s["ctx"].upload(m)
    img = s["ctx"].render(p, m)
    L0, dL = _loss(img.pol, s)
    res = s["ctx"].adjoint_image(p, m, dL, ckpt=16)
    # the adjoint's own forward pass is the image's, bit for bit
    assert np.array_equal(res["pol"], img.pol[..., :4])
    bad = {}
    for key, name in (("M_unit", "M_unit"), ("trat_large", "R_high"), ("trat_small", "R_low")):
        x = PARAMS[key]
        ad = res[name]
        errs = []
        for e in (1e-4, 1e-5, EPS):
            lp = _loss_at(s, **{key: x * (1 + e)})
            lm = _loss_at(s, **{key: x * (1 - e)})
            fd = (lp - lm) / (2 * e * x)
            errs.append(abs(ad / fd - 1))
            print(f"{name}: adjoint {ad:.8e} finite difference (eps {e:g}) {fd:.8e} relative {errs[-1]:.2e}")
        if not errs[-1] <= TOL:
            bad[name] = (ad, fd)
        # the differences converge on the adjoint as the step shrinks
        assert errs[-1] <= errs[0] or errs[0] <= TOL, (name, errs)
    assert not bad, bad


def _field_loss(s, m, fields, p):
    """the loss of the image traced from the given field arrays"""
    ctx = s["ctx"]
    ctx.upload_arrays(m.grid, fields)
    cam = ip.camera_for(p, m.grid)
    ij = np.array([(i, j) for i in range(16) for j in range(16)], np.int32)
    o = ctx.trace(cam, ij)
    f3 = p.freqcgs ** 3
    pol = np.zeros((16, 16, 4))
    pol[ij[:, 0], ij[:, 1], 0] = o["I"] * f3
    pol[ij[:, 0], ij[:, 1], 1] = -o["Q"] * f3
    pol[ij[:, 0], ij[:, 1], 2] = -o["U"] * f3
    pol[ij[:, 0], ij[:, 1], 3] = o["V"] * f3
    return _loss(pol, s)[0]


def test_adjoint_field_scalings_match_finite_differences(setup):
    """Directional derivatives along each whole field: scaling every cell's
    ne (Theta_e, |B|) by 1 +- 1e-4 against sum_c dL/dx_c x_c"""
    s = setup
    p = _params(s["dump"])
    m = ip.Model.load(p)
    ctx = s["ctx"]
    ctx.upload(m)
    img = ctx.render(p, m)
    _, dL = _loss(img.pol, s)
    res = ctx.adjoint_image(p, m, dL, ckpt=16)
    fields = [np.array(m.field(q)) for q in range(ip.NFIELD)]
    bad = {}
    for name, fi in (("ne", ip.IPG_F_NE), ("thetae", ip.IPG_F_THETAE), ("b", ip.IPG_F_B)):
        fp = [f.copy() for f in fields]
        fm = [f.copy() for f in fields]
        fp[fi] = fields[fi] * (1 + EPS)
        fm[fi] = fields[fi] * (1 - EPS)
        fd = (_field_loss(s, m, fp, p) - _field_loss(s, m, fm, p)) / (2 * EPS)
        ad = float(np.sum(res[name] * fields[fi]))
        print(f"field {name}: adjoint {ad:.8e} finite difference {fd:.8e} relative {abs(ad / fd - 1):.2e}")
        if not abs(ad - fd) <= TOL * abs(fd):
            bad[name] = (ad, fd)
    ctx.upload(m)
    assert not bad, bad


def test_adjoint_cells_match_finite_differences(setup):
    s = setup
    p = _params(s["dump"])
    m = ip.Model.load(p)
    ctx = s["ctx"]
    ctx.upload(m)
    img = ctx.render(p, m)
    _, dL = _loss(img.pol, s)
    res = ctx.adjoint_image(p, m, dL, ckpt=32)
    fields = [np.array(m.field(q)) for q in range(ip.NFIELD)]
    cam = ip.camera_for(p, m.grid)
    ij = np.array([(i, j) for i in range(16) for j in range(16)], np.int32)
    f3 = p.freqcgs ** 3

    def loss_with(fs):
        ctx.upload_arrays(m.grid, fs)
        o = ctx.trace(cam, ij)
        pol = np.zeros((16, 16, 4))
        pol[ij[:, 0], ij[:, 1], 0] = o["I"] * f3
        pol[ij[:, 0], ij[:, 1], 1] = -o["Q"] * f3
        pol[ij[:, 0], ij[:, 1], 2] = -o["U"] * f3
        pol[ij[:, 0], ij[:, 1], 3] = o["V"] * f3
        return _loss(pol, s)[0]

    checked = 0
    for name, fi in (("ne", ip.IPG_F_NE), ("thetae", ip.IPG_F_THETAE), ("b", ip.IPG_F_B)):
        g = res[name]
        # the three cells with the largest relative influence dL/dx * x
        infl = np.abs(g * fields[fi])
        for c in np.argsort(infl.ravel())[::-1][:3]:
            idx = np.unravel_index(c, g.shape)
            x = fields[fi][idx]
            fp = [f.copy() for f in fields]
            fm = [f.copy() for f in fields]
            fp[fi][idx] = x * (1 + EPS)
            fm[fi][idx] = x * (1 - EPS)
            fd = (loss_with(fp) - loss_with(fm)) / (2 * EPS * x)
            assert abs(g[idx] - fd) <= TOL * abs(fd), (name, idx, g[idx], fd)
            checked += 1
    assert checked == 9


def test_checkpoint_interval_leaves_gradients_unchanged(setup):
    """The segments are recomputed with the forward's own arithmetic, so the
    interval changes memory and time; the per-point gradients are the same
    bits, and only the order of the FP64 atomic scatter-adds into a cell
    varies from run to run (a few ulps of the cell's sum)"""
    s = setup
    p = _params(s["dump"])
    m = ip.Model.load(p)
    s["ctx"].upload(m)
    img = s["ctx"].render(p, m)
    _, dL = _loss(img.pol, s)
    r16 = s["ctx"].adjoint_image(p, m, dL, ckpt=16)
    r64 = s["ctx"].adjoint_image(p, m, dL, ckpt=64)
    for k in ("ne", "thetae", "b"):
        a, b = r16[k], r64[k]
        assert np.array_equal(a != 0, b != 0), k
        assert np.max(np.abs(a - b)) <= 1e-12 * np.max(np.abs(a)), k
    for k in ("M_unit", "R_high", "R_low"):
        assert abs(r16[k] - r64[k]) <= 1e-12 * abs(r16[k]), k


def test_autograd_wrapper_chains_to_the_electron_parameters(setup):
    torch = pytest.importorskip("torch")
    from ipole_b200.autograd import IQUVImage, derived_fields
    s = setup
    p = _params(s["dump"])
    m = ip.Model.load(p)
    fit = IQUVImage(s["ctx"], p, m)
    Mu = torch.tensor(PARAMS["M_unit"], dtype=torch.float64, requires_grad=True)
    Rh = torch.tensor(PARAMS["trat_large"], dtype=torch.float64, requires_grad=True)
    Rl = torch.tensor(PARAMS["trat_small"], dtype=torch.float64, requires_grad=True)
    ne, th, b = derived_fields(fit.prims, Mu, Rh, Rl)
    pol = fit(ne, th, b)
    target = torch.from_numpy(s["target"])
    loss = (((pol - target) / s["scale"]) ** 2).sum()
    loss.backward()
    s["ctx"].upload(m)
    img = s["ctx"].render(p, m)
    L0, dL = _loss(img.pol, s)
    assert abs(loss.item() / L0 - 1) < 1e-6
    res = s["ctx"].adjoint_image(p, m, dL)
    for t, key in ((Mu, "M_unit"), (Rh, "R_high"), (Rl, "R_low")):
        assert abs(t.grad.item() / res[key] - 1) < 1e-6, (key, t.grad.item(), res[key])


def test_adjoint_rejects_what_it_does_not_differentiate(setup):
    s = setup
    p = _params(s["dump"])
    m = ip.Model.load(p)
    s["ctx"].upload(m)
    dL = np.zeros((16, 16, 4))
    with pytest.raises(ip.IpgError) as e:
        s["ctx"].adjoint_image(p, m, dL, ckpt=24)
    assert e.value.code == ip.IPG_E_ARG
    pu = ip.Params.from_args([f"--dump={s['dump']}", *BASE, "--M_unit=3e27", "--trat_large=20", "-unpol"])
    with pytest.raises(ip.IpgError) as e:
        s["ctx"].adjoint_image(pu, m, dL)
    assert e.value.code == ip.IPG_E_ARG


def test_adjoint_matches_reference_finite_differences(dumps):
    """dL/dM_unit, dL/dR_high, dL/dR_low against central differences of the
    reference's own images (tests/golden/make_adjoint_fd.py), with the loss
    taken against the reference's target image"""
    z = np.load(os.path.join(common.GOLDEN, "adjoint_fd_c1_16.npz"))
    meta = json.loads(str(z["meta"]))
    target = z["target"]
    dump = dumps.get({"dump": "c1", "dump_shape_seed": meta["dump_shape_seed"], "dump_sha256": meta["dump_sha256"]})
    v = meta["params"]
    p = ip.Params.from_args([f"--dump={dump}", *meta["args"], f"--M_unit={v['M_unit']!r}",
                             f"--trat_large={v['trat_large']!r}", f"--trat_small={v['trat_small']!r}"])
    m = ip.Model.load(p)
    with ip.Context() as ctx:
        ctx.upload(m)
        img = ctx.render(p, m)
        r = (img.pol[..., :4] - target) / meta["scale"]
        L = float((r * r).sum())
        assert abs(L / meta["loss"] - 1) < 1e-5
        res = ctx.adjoint_image(p, m, 2.0 * r / meta["scale"])
    for key, name in (("M_unit", "M_unit"), ("trat_large", "R_high"), ("trat_small", "R_low")):
        fd = meta["fd"][key]
        assert abs(res[name] - fd) <= TOL * abs(fd), (name, res[name], fd)


def test_reverse_mode_step_matches_dual_numbers():
    """The walk's transfer-step VJP (reverse mode, one sweep) against the
    forward-mode dual numbers it replaced (three passes of four directions),
    on 200 000 seeded steps spanning both branches of absorb_emit, its
    small-tau series, approximate_solve's two forms and the small-rho
    Faraday form: the twelve gradients agree to rounding."""
    import ctypes as C
    L = ip.lib()
    f = L.ipg__check_step_vjp
    f.argtypes = [C.c_int, C.c_int, C.c_ulonglong, C.c_void_p, C.c_void_p]
    err = (C.c_double * 4)()
    worst = (C.c_double * 96)()
    assert f(0, 200000, 12345, C.cast(err, C.c_void_p), C.cast(worst, C.c_void_p)) == ip.IPG_OK
    print("reverse mode vs dual numbers, largest relative difference per regime:", list(err))
    for r in range(4):
        w = list(worst)[24 * r:24 * r + 24]
        print(f"  worst case of regime {r}: gradient", int(w[0]), "reverse", repr(w[1]), "dual", repr(w[2]),
              "x", repr(w[4]), "coefficients", [repr(v) for v in w[5:13]], "S", [repr(v) for v in w[13:17]],
              "group scale", w[17], "u", [repr(v) for v in w[18:22]])
    # Where polarized absorption acts (regimes 1-3) absorb_emit subtracts
    # terms of size 1/a_P and 1/(a_I - a_P); for the worst cases of this
    # check both forms were evaluated against 60-digit arithmetic and were
    # off it by the same order (reverse 8.9e-6, 4.2e-5, 4.8e-4; dual 8.8e-6,
    # 1.1e-5, 8.5e-4 in regimes 1, 2, 3): the differences are that
    # cancellation, not the derivation.
    assert err[0] <= 1e-8
    assert max(err[1], err[2]) <= 1e-4
    assert err[3] <= 1e-2
