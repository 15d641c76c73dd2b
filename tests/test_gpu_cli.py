"""The command-line program end to end (GPU): ipole's keys and flags, the
image file schema of src/io.c:140-273, the stderr summary line that
scripts/ipole.py scrapes (main.c:1034), and the reference's exit codes."""
import os
import subprocess

import numpy as np
import pytest

import ipole_b200 as ip
from ipole_b200 import build, ipgc
from tests import common

pytestmark = pytest.mark.gpu


def run_cli(args, cwd):
    build.build()
    return subprocess.run([build.CLI, *args], capture_output=True, text=True, cwd=cwd, timeout=600)


def test_cli_image_and_schema(dumps, tmp_path):
    meta, arrs = common.load_golden("c1_incl17_rot_24")
    par = tmp_path / "run.par"
    par.write_text("\n".join(a[2:].replace("=", " ") for a in meta["args"]) + "\n")
    out = tmp_path / "img.ipgc"
    r = run_cli(["-par", str(par), f"--dump={dumps.get(meta)}", f"--outfile={out}"], str(tmp_path))
    assert r.returncode == 0, r.stderr[-2000:]
    line = [l for l in r.stderr.splitlines() if l.startswith("freq:")][0]
    tok = line.split()
    ftot, funpol = float(tok[3]), float(tok[5].lstrip("("))
    # the line prints %g (6 significant digits); the image file carries full precision
    assert abs(ftot / meta["Ftot"] - 1) < 1e-5 and abs(funpol / meta["Ftot_unpol"] - 1) < 1e-5
    img = ipgc.read(str(out))
    for k in ("/header/version", "/header/freqcgs", "/header/scale", "/header/dsource", "/header/evpa_0",
              "/header/camera/nx", "/header/camera/fovx", "/header/camera/x", "/header/units/M_unit",
              "/header/electrons/rhigh", "/fluid_header/metric", "/Mdot", "/Ftot", "/Ftot_unpol", "/nuLnu",
              "/nuLnu_unpol", "/unpol", "/tau", "/pol"):
        assert k in img, k
    assert img["/pol"].shape == (24, 24, 5) and img["/header/evpa_0"] == "W"
    np.testing.assert_allclose(img["/pol"][..., 0], arrs["pol"][..., 0], rtol=2e-5)
    assert abs(float(img["/Ftot"]) / meta["Ftot"] - 1) <= common.tolerance(meta, "Ftot")


def test_cli_quench_unpol_and_exit_codes(dumps, tmp_path):
    meta, _ = common.load_golden("c1_unpol_24")
    base = [f"--dump={dumps.get(meta)}", *meta["args"]]
    r = run_cli([*base, "-quench", f"--outfile={tmp_path}/q.ipgc"], str(tmp_path))
    assert r.returncode == 0 and not os.path.exists(tmp_path / "q.ipgc")
    assert " Ftot: 0 Jy (" in r.stderr  # -unpol: no polarized flux
    r = run_cli([*base, "--maxnstep=50", f"--outfile={tmp_path}/m.ipgc"], str(tmp_path))
    assert r.returncode == 256 - 10 and "MaxNStep exceeded" in r.stderr
    r = run_cli(["--dump=/nonexistent.ipgc"], str(tmp_path))
    assert r.returncode == 255
    r = run_cli(["--histo=1"], str(tmp_path))
    assert r.returncode == 42


def test_cli_hdf5_dump_and_image(dumps, tmp_path):
    """The same run from an HDF5 dump to an HDF5 image (the reference's file
    formats) gives the image of the IPGC run entry for entry, bit for bit."""
    meta, _ = common.load_golden("c1_incl17_rot_24")
    dump = dumps.get(meta)
    h5 = str(tmp_path / "dump.h5")
    ip.convert_container(dump, h5)
    a, b = str(tmp_path / "a.ipgc"), str(tmp_path / "b.h5")
    r = run_cli([f"--dump={dump}", *meta["args"], f"--outfile={a}"], str(tmp_path))
    assert r.returncode == 0, r.stderr[-2000:]
    r = run_cli([f"--dump={h5}", *meta["args"], f"--outfile={b}"], str(tmp_path))
    assert r.returncode == 0, r.stderr[-2000:]
    with open(b, "rb") as f:
        assert f.read(8) == ipgc.HDF5_MAGIC
    ia, ib = ipgc.read(a), ipgc.read(b)
    assert sorted(ia) == sorted(ib)
    for k in ia:
        if isinstance(ia[k], np.ndarray):
            assert ia[k].dtype == ib[k].dtype and np.array_equal(ia[k], ib[k]), k
        else:
            assert ia[k] == ib[k], k


@pytest.mark.parametrize("case", common.golden_names(check=True))
def test_cli_check_mode(case, dumps, tmp_path):
    """-check (src/main.c:538-575): every 10th pixel and its mirror in i,
    appended to the existing image file as the _check / _recheck blocks
    (src/io.c:193-227), against the reference's own check run."""
    meta, arrs = common.load_golden(case)
    out = str(tmp_path / "img.h5")
    base = [f"--dump={dumps.get(meta)}", *meta["args"], f"--outfile={out}"]
    r = run_cli([*base[:-1], f"--outfile={tmp_path}/none.h5", "-check"], str(tmp_path))
    assert r.returncode == 0 and "no file to check" in r.stderr and not os.path.exists(tmp_path / "none.h5")
    r = run_cli(base, str(tmp_path))
    assert r.returncode == 0, r.stderr[-2000:]
    r = run_cli([*base, "-check"], str(tmp_path))
    assert r.returncode == 0 and "Running in check mode" in r.stderr, r.stderr[-2000:]
    img = ipgc.read(out)
    assert "/unpol" in img  # the original image stays
    for blk, sfx in (("", "check"), ("_recheck", "recheck")):
        class _Img:
            unpol = img[f"/unpol_{sfx}"]
            pol = img.get(f"/pol_{sfx}")
        gold = {"unpol": arrs["unpol" + blk]}
        if "pol" + blk in arrs:
            gold["pol"] = arrs["pol" + blk]
        e = common.image_errors(_Img, gold)
        bad = {k: (e[k], common.tolerance(meta, k)) for k in e if k in common.BASE_TOL
               and not e[k] <= common.tolerance(meta, k)}
        assert not bad, (sfx, bad)
        assert img[f"/tau_{sfx}"].shape == arrs["tau" + blk].shape
