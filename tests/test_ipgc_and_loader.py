"""Container I/O and the host iharm loader (model/iharm/model.c:848-2090)."""
import math

import numpy as np
import pytest

import ipole_b200 as ip
from ipole_b200 import ipgc, synthdump


def test_container_roundtrip(tmp_path):
    path = str(tmp_path / "x.ipgc")
    a = np.arange(24, dtype=np.float64).reshape(2, 3, 4)
    ipgc.write(path, {"/g/a": a, "/g/n": np.int32(7), "/s": "FMKS", "/g/h/x": np.float64(1.5), "/e": None},
               strlen={"/s": 20})
    d = ipgc.read(path)
    assert np.array_equal(d["/g/a"], a) and int(d["/g/n"]) == 7 and d["/s"] == "FMKS"
    assert float(d["/g/h/x"]) == 1.5 and d["/g"] is None and d["/g/h"] is None and d["/e"] is None


@pytest.fixture(scope="module")
def small_dump(tmp_path_factory):
    path = str(tmp_path_factory.mktemp("d") / "dump.ipgc")
    synthdump.write_iharm_dump(path, 16, 12, 8, seed=3)
    return path


def test_loader_grid_and_units(small_dump):
    p = ip.Params.from_args([f"--dump={small_dump}", "--M_unit=1e26", "--MBH=6.5e9", "--trat_large=20"])
    m = ip.Model.load(p)
    g = m.grid
    assert (g.n1, g.n2, g.n3) == (16, 12, 8)
    assert g.Rh == 1 + math.sqrt(1 - 0.9375 ** 2)
    assert g.rmax_geo == 50.0 and g.rmin_geo == 1.2 and g.cstopx[2] == 1.0 and g.cstopx[3] == 2 * math.pi
    assert g.poly_norm == 0.5 * math.pi * 1. / (1. + 1. / (14. + 1.) * 1. / pow(0.82, 14.))
    L = 6.6742e-8 * 6.5e9 * 1.989e33 / (2.99792458e10 ** 2)
    assert m.L_unit == L and g.L_unit == L


def test_loader_ghost_zones(small_dump):
    """radial copy, polar flip by pi in phi, periodic phi
    (model/iharm/model.c:1314-1370)"""
    p = ip.Params.from_args([f"--dump={small_dump}", "--M_unit=1e26"])
    m = ip.Model.load(p)
    for q in range(10):
        f = m.field(q)
        n1, n2, n3 = 16, 12, 8
        assert np.array_equal(f[0, 1:n2 + 1, 1:n3 + 1], f[1, 1:n2 + 1, 1:n3 + 1])
        assert np.array_equal(f[n1 + 1, 1:n2 + 1, 1:n3 + 1], f[n1, 1:n2 + 1, 1:n3 + 1])
        k = np.arange(1, n3 + 1)
        kflip = ((k - 1) + n3 // 2) % n3 + 1
        if q not in (6, 7, 9):  # prims and b are copied; ne/thetae/sigma are derived from copied values
            assert np.array_equal(f[:, 0, 1:n3 + 1], f[:, 1, kflip])
            assert np.array_equal(f[:, n2 + 1, 1:n3 + 1], f[:, n2, kflip])
        assert np.array_equal(f[:, :, 0], f[:, :, n3]) and np.array_equal(f[:, :, n3 + 1], f[:, :, 1])


def test_loader_derived_fields(small_dump):
    """ne, Theta_e (R_high/R_low model), sigma from the primitives and |b|
    (model/iharm/model.c:610-717), checked with numpy."""
    p = ip.Params.from_args([f"--dump={small_dump}", "--M_unit=1e26", "--trat_large=20", "--trat_small=1"])
    m = ip.Model.load(p)
    d = ipgc.read(small_dump)
    prims = d["/prims"]
    rho, uu = prims[..., 0], prims[..., 1]
    ne = m.field(6)[1:-1, 1:-1, 1:-1]
    b = m.field(8)[1:-1, 1:-1, 1:-1]
    np.testing.assert_allclose(ne, rho * m.RHO_unit / (1.67262171e-24 + 9.1093826e-28), rtol=1e-15)
    bsq = (b / m.B_unit) ** 2
    beta = uu * (13. / 9. - 1.) / 0.5 / bsq
    trat = 20 * beta ** 2 / (1 + beta ** 2) + 1 / (1 + beta ** 2)
    game, gamp = 1.333333333333333, 1.666666666666667
    the = (1.67262171e-24 / 9.1093826e-28) * (game - 1) * (gamp - 1) / ((gamp - 1) + (game - 1) * trat) * uu / rho
    np.testing.assert_allclose(m.field(7)[1:-1, 1:-1, 1:-1], np.maximum(the, 1e-3), rtol=1e-13)
    np.testing.assert_allclose(m.field(9)[1:-1, 1:-1, 1:-1], np.maximum(bsq / rho, 1e-40), rtol=1e-13)
    assert np.array_equal(m.field(0)[1:-1, 1:-1, 1:-1], prims[..., 2])
    assert np.array_equal(m.field(5)[1:-1, 1:-1, 1:-1], prims[..., 7])


def test_loader_errors(tmp_path):
    with pytest.raises(ip.IpgError) as e:
        ip.Model.load(ip.Params.from_args([f"--dump={tmp_path}/missing.ipgc"]))
    assert e.value.code == ip.IPG_E_IO
    bad = str(tmp_path / "mks.ipgc")
    ent = synthdump.make_iharm_dump(4, 4, 4, seed=1)
    ent["/header/metric"] = "MKS"
    ipgc.write(bad, ent, strlen={"/header/metric": 20, "/header/version": 20})
    with pytest.raises(ip.IpgError) as e:
        ip.Model.load(ip.Params.from_args([f"--dump={bad}"]))
    assert e.value.code == ip.IPG_E_FORMAT
    del ent["/prims"]
    ent["/header/metric"] = "FMKS"
    ipgc.write(bad, ent, strlen={"/header/metric": 20, "/header/version": 20})
    with pytest.raises(ip.IpgError) as e:
        ip.Model.load(ip.Params.from_args([f"--dump={bad}"]))
    assert e.value.code == ip.IPG_E_FORMAT
