"""ipg_trace_pixels_noalloc, the entry point that allocates no device memory,
against ipg_trace_pixels_device on the same pixels (GPU test).

Called twice in a row: the second call runs on scratch that still holds the
first call's contents, so it also checks that the call clears what it must.
"""
import ctypes as C

import numpy as np
import pytest

import ipole_b200 as ip
from tests import common

pytestmark = pytest.mark.gpu

# per-ray tolerances of the parity tests: I relative, Q/U/V relative to I
TOL_I = 2e-5
TOL_QUV = 2e-4


def _noalloc_fn():
    f = ip.lib().ipg_trace_pixels_noalloc
    f.argtypes = [C.POINTER(ip.Grid), C.c_void_p, C.POINTER(ip.Camera), C.c_void_p, C.c_size_t, C.c_void_p,
                  C.c_void_p]
    f.restype = C.c_int
    return f


def _compare(got, ref):
    assert np.array_equal(got["nstep"], ref["nstep"])
    assert np.array_equal(got["flag"], ref["flag"])
    for k in ("I_unpol", "I", "tau"):
        g, r = got[k], ref[k]
        assert np.array_equal(g == 0, r == 0), k
        nz = r != 0
        assert np.all(np.abs(g[nz] / r[nz] - 1) < TOL_I), k
    I = np.abs(ref["I"])
    nz = I > 0
    for k in ("Q", "U", "V"):
        assert np.all(np.abs(got[k][nz] - ref[k][nz]) / I[nz] < TOL_QUV), k


def test_noalloc_matches_device_entry(dumps):
    torch = pytest.importorskip("torch")
    meta, _ = common.load_golden("c1_bright_32")
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
        ref = np.frombuffer(d_ref.cpu().numpy().tobytes(), dtype=ip.PIXEL_DTYPE).copy()

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
        got = np.frombuffer(d_out.cpu().numpy().tobytes(), dtype=ip.PIXEL_DTYPE)
        _compare(got, ref)


def test_noalloc_rejects_sizes_beyond_its_limit(dumps):
    meta, _ = common.load_golden("c1_bright_32")
    p = common.params_for(meta, dumps.get(meta))
    m = ip.Model.load(p)
    cam = ip.camera_for(p, m.grid)
    fn = _noalloc_fn()
    grid = m.grid
    # rejected before anything touches the (dummy, never dereferenced) pointers
    dummy = C.c_void_p(16)
    assert fn(C.byref(grid), dummy, C.byref(cam), dummy, 65536 + 1, dummy, None) == ip.IPG_E_ARG
    cam.maxnstep = 51200 + 1
    assert fn(C.byref(grid), dummy, C.byref(cam), dummy, 4, dummy, None) == ip.IPG_E_ARG
