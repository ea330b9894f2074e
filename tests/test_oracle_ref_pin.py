"""The oracle pinned to the reference's own particle code, run on this machine.

oracle/ref_build.py compiles the bodies of the reference's SYCL particle
kernels, read unchanged from a reference checkout, into a serial host harness
(oracle/_ref/libref_pic.so):
  * modulo, deterministic_mover and the MoverKernel lambda
    (SYCL-PIC-poissonsolver/src/mover.cpp:13-22, 103-176, 304-366);
  * calculate_working_size and the kernels of interpolate()
    (src/interpolation.cpp:8-12, 39-171).
These tests run the oracle restatement (oracle/pic_oracle.c) and that library
on the same inputs:
  * push: every particle's x, y, z, vx, vy, vz bit for bit (the oracle keeps
    the reference's operand order, both are built without FMA contraction),
    the same particles deleted, the same left-exit count, the same bucket
    for every particle after the move (re-inserted ones included), walled and
    periodic in y, on grids where nx*dx is not XMAX;
  * deposit: with one work item per bucket (prob_size 1) final_mesh,
    energy_mesh and rho bit for bit; with the reference's default prob_size
    24 (partial sums per work item, added in order) within 1e-13 of the
    largest value, the difference being only the order of FP64 additions.
Skipped when the library is absent and cannot be built (no reference
checkout on this machine).
"""
import ctypes

import numpy as np
import pytest

EPS0 = 8.854e-12
QE = 1.602e-19
ME = 9.109e-31
M_AR = 6.6335e-26


@pytest.fixture(scope="module")
def ref(oracle):
    L = oracle.ref_lib()
    if L is None:
        pytest.skip("reference harness not built and no reference checkout to build it from")
    return L


def _points(O, nx, ny, dx, dy, n, vmax_cells, rng, dt):
    pts = np.zeros(n, O.POINT_DTYPE)
    pts["x"] = rng.uniform(0, nx * dx, n)
    pts["y"] = rng.uniform(0, ny * dy, n)
    pts["z"] = rng.normal(0, dx, n)
    pts["vx"] = rng.normal(0, vmax_cells * dx / dt / 3, n)
    pts["vy"] = rng.normal(0, vmax_cells * dy / dt / 3, n)
    pts["vz"] = rng.normal(0, vmax_cells * dx / dt / 3, n)
    pts["pointer"] = np.arange(n, dtype=np.int32)
    # edge cases: on cell boundaries, at the walls, leaving through each wall,
    # dead points
    k = 0
    for (x, y, vx, vy) in [(0.0, 0.0, 0, 0), (3 * dx, 5 * dy, 0, 0), (nx * dx * (1 - 1e-16), dy, 0, 0),
                           (0.1 * dx, 4.5 * dy, -0.3 * dx / dt, 0), (nx * dx - 0.05 * dx, 2.5 * dy, 0.2 * dx / dt, 0),
                           (5.5 * dx, 0.05 * dy, 0, -0.2 * dy / dt), (5.5 * dx, ny * dy - 0.02 * dy, 0, 0.1 * dy / dt),
                           (2.5 * dx, 2.5 * dy, 2.5 * dx / dt, -1.5 * dy / dt)]:
        pts[k]["x"], pts[k]["y"], pts[k]["vx"], pts[k]["vy"] = x, y, vx, vy
        k += 1
    pts["pointer"][k:k + 3] = -1
    return pts


@pytest.mark.parametrize("periodic", [0, 1])
@pytest.mark.parametrize("nx,ny,xmax,ymax", [(37, 29, 0.011, 0.0093), (64, 48, 0.016, 0.012)])
def test_push_bit_exact_against_reference_mover(oracle, ref, periodic, nx, ny, xmax, ymax):
    O = oracle
    rng = np.random.default_rng(nx * 7 + periodic)
    gp = O.ref_grid_params(nx, ny, xmax, ymax)
    g = O.Grid(nx, ny, gp.dx, gp.dy, xmax, ymax)
    GX, GY = nx + 1, ny + 1
    dt = 5e-11
    for ptype, (q, m) in enumerate([(-QE, ME), (QE, M_AR)]):
        ctom_arr = np.array([-QE / ME, QE / M_AR])
        pts = _points(O, nx, ny, gp.dx, gp.dy, 4000, 1.2, rng, dt)
        ef = rng.normal(0, 2e4, (GX * GY, 2))
        bz = rng.uniform(0.0, 0.03, GX * GY)
        phi = rng.normal(0, 10, GX * GY)
        a = pts.copy()
        b = pts.copy()
        key0 = O.bucket_keys(g, pts)
        deleted, left = O.push(g, a, ctom_arr[ptype], dt, ef, bz, periodic=bool(periodic))
        ins = np.full(len(b), -1, np.int32)
        dels = np.full(len(b), -1, np.int32)
        lx = ctypes.c_int(0)
        holes = ref.ref_mover_kernel(b.ctypes.data, len(b), ctypes.byref(gp), ctom_arr.ctypes.data,
                                     ptype, dt, ef.ctypes.data, bz.ctypes.data, phi.ctypes.data,
                                     periodic, ins.ctypes.data, dels.ctypes.data, ctypes.byref(lx))
        for f in ("x", "y", "z", "vx", "vy", "vz"):
            assert np.array_equal(a[f], b[f]), (ptype, f)
        assert np.array_equal(a["pointer"] == -1, b["pointer"] == -1)
        assert deleted == holes and left == lx.value
        assert deleted > 0 and left > 0
        live = b["pointer"] != -1
        key_ref = np.where(ins >= 0, ins, key0)[live]
        assert np.array_equal(O.bucket_keys(g, a)[live], key_ref)
        assert (ins[live] >= 0).sum() > 100   # many particles changed cell


@pytest.mark.parametrize("prob_size", [1, 24])
def test_deposit_against_reference_interpolate(oracle, ref, prob_size):
    O = oracle
    nx, ny, xmax, ymax = 45, 31, 0.0112, 0.0077
    rng = np.random.default_rng(prob_size)
    gp = O.ref_grid_params(nx, ny, xmax, ymax)
    g = O.Grid(nx, ny, gp.dx, gp.dy, xmax, ymax)
    nodes = g.nodes
    for ptype in (0, 1):
        pts = _points(O, nx, ny, gp.dx, gp.dy, 30000, 1.0, rng, 5e-11)
        pts = pts[pts["x"] < nx * gp.dx]
        ctom = np.array([-QE / ME, QE / M_AR])
        charges = np.array([-QE, QE])
        sp = O.Species(str(ptype), charges[ptype], [ME, M_AR][ptype], 2e4, 3e9)
        wgt = O.weighing_factor(sp, xmax * ymax, gp.dx, gp.dy)
        weighing = np.array([wgt, wgt])
        keys = O.bucket_keys(g, pts)
        probing = int(np.bincount(keys[keys >= 0]).max()) + 3
        rho_o = rng.normal(0, 1, nodes)
        rho_r = rho_o.copy()
        fin_o, en_o = O.deposit(g, pts, sp, wgt, EPS0, rho_o)
        fin_r, en_r = np.zeros(nodes), np.zeros(nodes)
        st = ref.ref_interpolate(pts.ctypes.data, len(pts), keys.ctypes.data, ctypes.byref(gp),
                                 probing, prob_size, ctom.ctypes.data, weighing.ctypes.data,
                                 charges.ctypes.data, EPS0, ptype, fin_r.ctypes.data,
                                 en_r.ctypes.data, rho_r.ctypes.data)
        assert st == 0
        if prob_size == 1:
            assert np.array_equal(fin_o, fin_r)
            assert np.array_equal(en_o, en_r)
            assert np.array_equal(rho_o, rho_r)
        else:
            assert np.abs(fin_o - fin_r).max() <= 1e-13 * np.abs(fin_o).max()
            assert np.abs(en_o - en_r).max() <= 1e-13 * np.abs(en_o).max()
            assert np.abs(rho_o - rho_r).max() <= 1e-13 * np.abs(rho_o).max()
        assert fin_o.sum() > 0


def test_planted_mistake_in_oracle_push_is_caught(oracle, ref):
    """A half-step E kick of the wrong size in the oracle's inputs (dt*1.001)
    must break the bit-for-bit comparison."""
    O = oracle
    nx, ny, xmax, ymax = 37, 29, 0.011, 0.0093
    gp = O.ref_grid_params(nx, ny, xmax, ymax)
    g = O.Grid(nx, ny, gp.dx, gp.dy, xmax, ymax)
    rng = np.random.default_rng(5)
    pts = _points(O, nx, ny, gp.dx, gp.dy, 500, 0.5, rng, 5e-11)
    ef = rng.normal(0, 2e4, ((nx + 1) * (ny + 1), 2))
    bz = np.full((nx + 1) * (ny + 1), 0.01)
    a, b = pts.copy(), pts.copy()
    O.push(g, a, -QE / ME, 5e-11 * 1.001, ef, bz)
    ctom = np.array([-QE / ME, QE / M_AR])
    ins = np.full(len(b), -1, np.int32)
    dels = np.full(len(b), -1, np.int32)
    lx = ctypes.c_int(0)
    ref.ref_mover_kernel(b.ctypes.data, len(b), ctypes.byref(gp), ctom.ctypes.data, 0, 5e-11,
                         ef.ctypes.data, bz.ctypes.data, bz.ctypes.data, 0, ins.ctypes.data,
                         dels.ctypes.data, ctypes.byref(lx))
    assert not np.array_equal(a["x"], b["x"])
