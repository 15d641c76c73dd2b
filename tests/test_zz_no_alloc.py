"""ipg_trace_pixels_noalloc, the entry point that allocates no device memory,
against ipg_trace_pixels_device on the same pixels (GPU test).

Some callers cannot call cudaMalloc: applications that hand the library a
fixed share of device memory through their own allocator and count any
allocation made behind their back against them, and pipelines that cannot
take the device-wide synchronisation of cudaMalloc/cudaFree.  The entry point
runs on one static scratch array per device instead.

It launches the same compiled kernels as a context's FP64 path, and a ray's
result does not depend on the wave, lane or pool slot it lands in, so every
output field must equal the context's bit for bit.  The image it gives is also
checked against the reference's golden image with the parity tests' bound.
Called twice in a row: the second call runs on scratch that still holds the
first call's contents, so it also checks that the call clears what it must.
"""
import ctypes as C

import numpy as np
import pytest

import ipole_b200 as ip
from tests import common

pytestmark = pytest.mark.gpu

CASE = "c1_bright_32"


def _noalloc_fn():
    f = ip.lib().ipg_trace_pixels_noalloc
    f.argtypes = [C.POINTER(ip.Grid), C.c_void_p, C.POINTER(ip.Camera), C.c_void_p, C.c_size_t, C.c_void_p,
                  C.c_void_p]
    f.restype = C.c_int
    return f


def _image(p, cam, ij, out):
    """save_pixel of every traced pixel (src/main.c:885-910): the pol array
    the golden image holds, I, Q, U, V times nu^3 with the qu_conv sign"""
    nx, ny = p.nx, p.ny
    nu3 = cam.freqcgs ** 3
    sgn = 1.0 if p.qu_conv else -1.0
    pol = np.zeros((nx, ny, 5))
    unpol = np.zeros((nx, ny))
    i, j = ij[:, 0], ij[:, 1]
    pol[i, j, 0] = out["I"] * nu3
    pol[i, j, 1] = sgn * out["Q"] * nu3
    pol[i, j, 2] = sgn * out["U"] * nu3
    pol[i, j, 3] = out["V"] * nu3
    pol[i, j, 4] = out["tauF"]
    unpol[i, j] = out["I_unpol"] * nu3

    class Img:
        pass
    img = Img()
    img.pol, img.unpol = pol, unpol
    return img


def test_noalloc_matches_device_entry(dumps):
    torch = pytest.importorskip("torch")
    meta, arrs = common.load_golden(CASE)
    p = common.params_for(meta, dumps.get(meta))
    m = ip.Model.load(p)
    cam = ip.camera_for(p, m.grid)
    nx, ny = p.nx, p.ny
    ij = np.array([(i, j) for i in range(nx) for j in range(ny)], np.int32)
    n = len(ij)
    d_ij = torch.from_numpy(ij).cuda()

    with ip.Context() as c:
        c.upload(m)
        d_ref = torch.zeros(n * ip.PIXEL_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
        c.trace_device(cam, d_ij.data_ptr(), n, d_ref.data_ptr())
        ref_bytes = d_ref.cpu().numpy().tobytes()

    # the model in the library's device layout: the fields of a zone contiguous
    fields = np.stack([m.field(q).ravel() for q in range(ip.NFIELD)], axis=1)
    d_fields = torch.from_numpy(np.ascontiguousarray(fields)).cuda()
    fn = _noalloc_fn()
    grid = m.grid
    for call in range(2):
        d_out = torch.full((n * ip.PIXEL_DTYPE.itemsize,), 0xA5, dtype=torch.uint8, device="cuda")
        torch.cuda.synchronize()
        rc = fn(C.byref(grid), C.c_void_p(d_fields.data_ptr()), C.byref(cam), C.c_void_p(d_ij.data_ptr()), n,
                C.c_void_p(d_out.data_ptr()), None)
        assert rc == ip.IPG_OK, (call, rc, ip.lib().ipg_strerror(rc))
        got_bytes = d_out.cpu().numpy().tobytes()
        got = np.frombuffer(got_bytes, dtype=ip.PIXEL_DTYPE)
        ref = np.frombuffer(ref_bytes, dtype=ip.PIXEL_DTYPE)
        for k in ip.PIXEL_DTYPE.names:
            assert np.ascontiguousarray(got[k]).tobytes() == np.ascontiguousarray(ref[k]).tobytes(), (call, k)
        # and the image against the reference's, within the parity bound
        e = common.image_errors(_image(p, cam, ij, got), arrs)
        for key in ("Ftot", "Ftot_unpol", "pix_I_max", "totQ", "totU", "totV"):
            assert e[key] <= common.tolerance(meta, key), (call, key, e[key])


def test_noalloc_rejects_bad_arguments(dumps):
    meta, _ = common.load_golden(CASE)
    p = common.params_for(meta, dumps.get(meta))
    m = ip.Model.load(p)
    cam = ip.camera_for(p, m.grid)
    fn = _noalloc_fn()
    grid = m.grid
    # rejected before anything touches the (dummy, never dereferenced) pointers
    dummy = C.c_void_p(16)
    assert fn(C.byref(grid), dummy, C.byref(cam), dummy, 65536 + 1, dummy, None) == ip.IPG_E_ARG
    bad = ip.Grid.from_buffer_copy(grid)
    bad.metric = 1  # MKS: not an iharm dump
    assert fn(C.byref(bad), dummy, C.byref(cam), dummy, 4, dummy, None) == ip.IPG_E_ARG
    cam.maxnstep = 51200 + 1
    assert fn(C.byref(grid), dummy, C.byref(cam), dummy, 4, dummy, None) == ip.IPG_E_ARG
