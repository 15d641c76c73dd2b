"""Per-step trace output (dump_var_along, src/io.c:279-543) on the GPU against
the reference's own trace of the same pixel (tests/golden/trace_*.npz, made by
tests/golden/make_golden.py from the reference built here), and the trace file
written by the command-line program."""
import os
import subprocess

import numpy as np
import pytest

import ipole_b200 as ip
from ipole_b200 import build, ipgc
from tests import common

pytestmark = pytest.mark.gpu
BASE_TOL = 1e-6


@pytest.fixture(scope="module")
def ctx():
    c = ip.Context()
    yield c
    c.close()


def pixel_of(meta):
    kv = dict(a[2:].split("=", 1) for a in meta["args"] if a.startswith("--") and "=" in a)
    return int(kv["trace_i"]), int(kv["trace_j"])


@pytest.mark.parametrize("case", common.golden_names(trace=True))
def test_trace_matches_reference(case, dumps, ctx):
    meta, gold = common.load_golden(case)
    p = common.params_for(meta, dumps.get(meta))
    m = ip.Model.load(p)
    ctx.upload(m)
    cam = ip.camera_for(p, m.grid)
    i, j = pixel_of(meta)
    nstep, rows = ctx.trace_ray(cam, i, j, model=m)
    assert nstep == meta["nstep"]
    bad = {}
    for name, (col, w) in ip.TRACE_COLS.items():
        if name not in gold:
            continue
        g = gold[name].reshape(nstep + 1, w)
        mine = rows[:, col:col + w]
        scale = float(np.max(np.abs(g))) or 1.0
        err = float(np.max(np.abs(mine - g))) / scale
        tol = max(BASE_TOL, common.FLOOR_FACTOR * meta["ref_noise_floor"].get(name, 0.0))
        print(f"{case} {name:18s} error {err:.2e} tolerance {tol:.2e}")
        if not err <= tol:
            bad[name] = (err, tol)
    assert not bad, bad


def run_cli(args, cwd):
    build.build()
    return subprocess.run([build.CLI, *args], capture_output=True, text=True, cwd=cwd, timeout=600)


def test_cli_trace_file(dumps, tmp_path, ctx):
    """--trace with one pixel: the file holds the header, nstep and the
    per-step datasets of that ray (rows 0..nstep; zeros after), equal to
    ipg_trace_ray's rows; with --trace_stride, every stride-th pixel."""
    case = common.golden_names(trace=True)[0]
    meta, gold = common.load_golden(case)
    tr = str(tmp_path / "trace.h5")
    r = run_cli([f"--dump={dumps.get(meta)}", *meta["args"], f"--trace_outf={tr}", "-quench"], str(tmp_path))
    assert r.returncode == 0, r.stderr[-2000:]
    t = ipgc.read(tr)
    n = int(t["/nstep"][0, 0])
    assert n == meta["nstep"] and t["/nstep"].shape == (1, 1) and "/header/camera/nx" in t
    assert t["/X"].shape == (1, 1, n + 1, 4) and t["/Econ"].shape == (1, 1, n + 1, 4, 4)
    p = common.params_for(meta, dumps.get(meta))
    m = ip.Model.load(p)
    ctx.upload(m)
    _, rows = ctx.trace_ray(ip.camera_for(p, m.grid), *pixel_of(meta), model=m)
    for name, (col, w) in ip.TRACE_COLS.items():
        if name == "flag":
            continue
        assert np.array_equal(t["/" + name].reshape(n + 1, w), rows[:, col:col + w]), name
    # stride mode: a 2x2 grid of traced pixels
    tr2 = str(tmp_path / "trace2.h5")
    args = [a for a in meta["args"] if not a.startswith(("--trace_i", "--trace_j", "--nx", "--ny"))]
    r = run_cli([f"--dump={dumps.get(meta)}", *args, "--nx=16", "--ny=16", "--trace_stride=8",
                 f"--trace_outf={tr2}", "-quench"], str(tmp_path))
    assert r.returncode == 0, r.stderr[-2000:]
    t2 = ipgc.read(tr2)
    ns = t2["/nstep"]
    assert ns.shape == (2, 2) and np.all(ns > 0)
    assert t2["/dl"].shape == (2, 2, int(ns.max()) + 1)
    for a in range(2):
        for b in range(2):
            assert np.all(t2["/dl"][a, b, ns[a, b]:] == 0)
