"""The allocation-free deposit entry point, through the C ABI.

pic_deposit_points_noalloc exists for callers that cannot allocate device
memory at the moment they deposit (a host framework owning a fixed device
memory budget, or a time-critical loop where cudaMalloc/cudaFree and their
device-wide synchronisation are not allowed): its only scratch is a fixed
array inside the library.  This test checks that two calls in a row give the
same final_mesh and rho as the library's regular path (pic_import_points +
pic_charge_deposition): within the deposit tolerance of the other GPU tests
(2e-6 of max|final_mesh|) and, since the fixed-point arithmetic is the same,
bit for bit -- so the shared scratch is cleared between calls.  The test's own buffers come from
torch; the entry point itself allocates nothing.

The file name sorts last so that a run stopping at the first failure has
already run every other test.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

EPS0 = 8.854e-12


def _entry(lib):
    f = lib.pic_deposit_points_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32, ctypes.c_int32,
                  ctypes.c_double, ctypes.c_double, ctypes.c_void_p, ctypes.c_double,
                  ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    return f


def test_noalloc_deposit_matches_regular_deposit_twice():
    import torch
    import pic_b200 as P
    import pic_configs as C

    w = C.cfg1()
    w.nx, w.ny = 96, 80
    w.rects = C.wall_rects(w.nx, w.ny)
    w.species = C._species(w.nx, w.ny, 10, 1e15)
    pts = C.host_points(w, 0, seed=77, ppc=10)
    pts[::97]["pointer"] = -1                      # dead points are skipped
    nodes = (w.nx + 1) * (w.ny + 1)

    with P.Pic(C.library_config(w)) as pic:      # the regular entry point
        pic.import_points(0, pts)
        pic.zero_rho()
        pic.charge_deposition(0)
        final_ref = pic.final_mesh(0)
        rho_ref = pic.rho()

    L = P.lib()
    f = _entry(L)
    sp = P.SpeciesDesc(*w.species[0])
    dev_pts = torch.from_numpy(pts.view(np.uint8).copy()).cuda()
    final = torch.empty(nodes, dtype=torch.float64, device="cuda")
    rho = torch.empty(nodes, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    tol = 2e-6 * np.abs(final_ref).max()
    for call in range(2):
        final.fill_(123.0)                         # overwritten by the call
        rho.zero_()                                # accumulated into by the call
        st = f(dev_pts.data_ptr(), len(pts), w.nx, w.ny, w.xmax, w.ymax, ctypes.byref(sp), 0.0,
               EPS0, final.data_ptr(), rho.data_ptr(), stream)
        assert st == 0, L.pic_last_error()
        torch.cuda.synchronize()
        got_final = final.cpu().numpy()
        got_rho = rho.cpu().numpy()
        # same fixed-point arithmetic as the regular path: final_mesh and rho
        # are bit-identical (the 2e-6 deposit tolerance is the outer bound)
        assert np.abs(got_final - final_ref).max() <= tol, call
        assert np.array_equal(got_final, final_ref), call
        assert np.abs(got_rho - rho_ref).max() <= 2e-6 * np.abs(rho_ref).max(), call
        assert np.array_equal(got_rho, rho_ref), call


def test_noalloc_rejects_grids_beyond_its_scratch():
    import pic_b200 as P
    L = P.lib()
    f = _entry(L)
    sp = P.SpeciesDesc(-1.602e-19, 9.109e-31, 1.0, 1.0)
    dummy = ctypes.c_double(0.0)
    st = f(None, 0, 1024, 1024, 0.256, 0.256, ctypes.byref(sp), 0.0, EPS0,
           ctypes.addressof(dummy), None, None)
    assert st == -3                                # PIC_ERR_CAPACITY
    assert b"exceeds the fixed scratch" in L.pic_last_error()
