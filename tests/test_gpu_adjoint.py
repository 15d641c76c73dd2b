"""The adjoint of the polarized image (GPU): gradients of an image loss
against central finite differences of the GPU images and of the reference's
images, checkpoint intervals, the torch.autograd wrapper, and the forward
image the adjoint traces.

The loss is the L2 distance between the image and a target image rendered at
perturbed parameters (M_unit x 1.3, R_high 20 -> 25), normalized by the
target's largest intensity.  Finite differences are central with a relative
step of 1e-4, and the adjoint must match them to 1e-4 relative.
"""
import json
import os

import numpy as np
import pytest

import ipole_b200 as ip
from tests import common

pytestmark = pytest.mark.gpu

EPS = 1e-4
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
    for key, name in (("M_unit", "M_unit"), ("trat_large", "R_high"), ("trat_small", "R_low")):
        x = PARAMS[key]
        lp = _loss_at(s, **{key: x * (1 + EPS)})
        lm = _loss_at(s, **{key: x * (1 - EPS)})
        fd = (lp - lm) / (2 * EPS * x)
        ad = res[name]
        assert abs(ad - fd) <= TOL * abs(fd), (name, ad, fd)


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
    interval changes memory and time, not a bit of the result"""
    s = setup
    p = _params(s["dump"])
    m = ip.Model.load(p)
    s["ctx"].upload(m)
    img = s["ctx"].render(p, m)
    _, dL = _loss(img.pol, s)
    r16 = s["ctx"].adjoint_image(p, m, dL, ckpt=16)
    r64 = s["ctx"].adjoint_image(p, m, dL, ckpt=64)
    for k in ("ne", "thetae", "b"):
        assert np.array_equal(r16[k], r64[k]), k
    assert (r16["M_unit"], r16["R_high"], r16["R_low"]) == (r64["M_unit"], r64["R_high"], r64["R_low"])


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
