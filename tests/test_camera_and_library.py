"""Camera set-up against the oracle, and the C-ABI library surface."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import ipole_b200 as ip
from ipole_b200 import synthdump
from oracle.oracle import Oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def model(tmp_path_factory):
    path = str(tmp_path_factory.mktemp("c") / "dump.ipgc")
    synthdump.write_iharm_dump(path, 16, 12, 8, seed=5)
    return ip.Model.load(ip.Params.from_args([f"--dump={path}", "--M_unit=1e26"]))


@pytest.mark.parametrize("theta,phi,rot", [(163., 0., 0.), (17., 30., 45.), (90., 0., -10.), (60., 180., 0.)])
def test_camera_bitwise_vs_oracle(model, theta, phi, rot):
    p = ip.Params.from_args(["--thetacam=%g" % theta, "--phicam=%g" % phi, "--rotcam=%g" % rot, "--fov=160",
                             "--dsource=16.8e6", "--nx=40", "--ny=30", "--freqcgs=230e9"])
    cam = ip.camera_for(p, model.grid)
    orc = Oracle(model.grid, [model.field(q) for q in range(10)])
    oc = orc.camera(1000., theta, phi, rot, 160., 16.8e6, 40, 30, 230e9)
    assert list(cam.Xcam) == list(oc.Xcam)
    assert np.array_equal(np.array(cam.Econ), np.array(oc.Econ))
    assert np.array_equal(np.array(cam.Ecov), np.array(oc.Ecov))
    assert (cam.fovx, cam.fovy, cam.freq, cam.rotcam) == (oc.fovx, oc.fovy, oc.freq, oc.rotcam)
    assert cam._scale == oc._scale


def _declared(header):
    txt = open(os.path.join(ROOT, "include", header)).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(ipg_[a-z0-9_]+)\s*\(", txt)) - {"ipg_tracer_fn"})


def test_library_exports_every_declared_symbol():
    L = ip.lib()
    names = _declared("ipole_b200.h") + _declared("ipole_host.h")
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_strerror_and_errors_without_device():
    L = ip.lib()
    assert L.ipg_strerror(ip.IPG_E_MAXNSTEP) == b"MaxNStep exceeded"
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(ip.IpgError) as e:
        ip.Context()
    assert e.value.code == ip.IPG_E_CUDA


def test_fp64_probe_needs_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(ip.IpgError):
        ip.fp64_peak_tflops(0, 10)
