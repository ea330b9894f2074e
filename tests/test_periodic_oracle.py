"""CPU checks of the oracle's periodic-in-y restatement (periodicBoundary = 1:
SYCL-PIC-poissonsolver/src/poissonSolver.cpp:82-180 generateCoeffsPeriodic,
:364-382 overwritePhi, :411-430 calculateElectricFieldPeriodic;
src/mover.cpp:13-22 modulo and :317-320 the wrap in MoverKernel).

The reference has no periodic fixtures, so the restatement is pinned by
properties that hold for the reference's system whatever its
implementation: a y-independent charge gives the 1-D solution of the x
problem on every row; shifting the charge by whole rows shifts the
potential by the same rows; the operator is symmetric on the non-electrode
nodes; and the push wraps y exactly as modulo(y, H) does.
"""
import ctypes

import numpy as np
import pytest


def _setup(O, nx=16, ny=12, dx=1e-3, inner=None, left=40.0, right=-5.0):
    import pic_configs as C
    GX, GY = nx + 1, ny + 1
    el = O.Electrodes(C.periodic_rects(nx, ny, left, right, inner))
    return GX, GY, dx, el


def test_y_independent_charge_gives_the_1d_solution(oracle):
    GX, GY, dx, el = _setup(oracle)
    D = oracle.DirectPoisson(GX, GY, dx, dx, el, periodic=True)
    prof = np.random.default_rng(0).normal(size=GX) * 1e4
    rho = np.tile(prof, GY)
    phi, ef = D.step(rho.copy())
    p = phi.reshape(GY, GX)
    assert np.abs(p - p[0]).max() <= 1e-9 * np.abs(p).max()
    # the 1-D problem (2 phi_i - phi_i-1 - phi_i+1)/dx^2 = -rho_i (the
    # overwriteRho sign), phi = 40 V and -5 V at the x walls
    n = GX - 2
    A = (np.diag(np.full(n, 2.0)) - np.diag(np.ones(n - 1), 1) - np.diag(np.ones(n - 1), -1)) / dx ** 2
    b = -prof[1:-1].copy()
    b[0] += 40.0 / dx ** 2
    b[-1] += -5.0 / dx ** 2
    ref = np.linalg.solve(A, b)
    assert np.abs(p[0, 1:-1] - ref).max() <= 1e-9 * np.abs(ref).max()
    e = ef.reshape(GY, GX, 2)
    assert np.abs(e[..., 1]).max() <= 1e-6 * np.abs(e[..., 0]).max()


def test_row_shift_shifts_the_potential(oracle):
    GX, GY, dx, el = _setup(oracle, left=0.0, right=0.0)
    D = oracle.DirectPoisson(GX, GY, dx, dx, el, periodic=True)
    P = GY - 1
    rho = np.zeros((GY, GX))
    rho[:P] = np.random.default_rng(1).normal(size=(P, GX)) * 1e4
    rho[P] = rho[0]
    phi0, _ = D.step(rho.ravel().copy())
    k = 5
    sh = np.zeros((GY, GX))
    sh[:P] = np.roll(rho[:P], k, axis=0)
    sh[P] = sh[0]
    phi1, _ = D.step(sh.ravel().copy())
    a, b = phi0.reshape(GY, GX)[:P], phi1.reshape(GY, GX)[:P]
    assert np.abs(np.roll(a, k, axis=0) - b).max() <= 1e-9 * np.abs(a).max()
    # the last row repeats row 0
    assert np.array_equal(phi1.reshape(GY, GX)[P], phi1.reshape(GY, GX)[0])


def test_operator_structure(oracle):
    GX, GY, dx, el = _setup(oracle, inner=(6, 3, 9, 5, 100.0))
    mask = oracle.electrode_mask(GX, GY, el)
    A = oracle.build_csr_periodic(GX, GY, dx, 2 * dx, mask).toarray()
    n = GX * (GY - 1)
    inner = mask[:n] == 0
    Ai = A[np.ix_(inner, inner)]
    assert np.array_equal(Ai, Ai.T)
    assert np.all(np.linalg.eigvalsh(Ai) > 0)
    # row of a first-row node reaches the last row, and vice versa
    i = 3
    assert A[i, n - GX + i] == -1 / (2 * dx) ** 2 and A[i, GX + i] == -1 / (2 * dx) ** 2
    j = n - GX + 3
    assert A[j, 3] == -1 / (2 * dx) ** 2
    assert np.all(np.diag(A)[~inner] == -1)
    # an x wall that is not an electrode is refused
    bad = mask.copy()
    bad[2 * GX] = 0
    with pytest.raises(ValueError):
        oracle.build_csr_periodic(GX, GY, dx, dx, bad)


def test_periodic_efield(oracle):
    GX, GY = 9, 7
    P = GY - 1
    phi = np.random.default_rng(2).random(GX * GY)
    ef = oracle.efield(GX, GY, 0.1, 0.2, phi, periodic=True).reshape(GY, GX, 2)
    p = phi.reshape(GY, GX)
    assert np.isclose(ef[3, 0, 0], -(p[3, 1] - p[3, 0]) / 0.1)
    assert np.isclose(ef[3, GX - 1, 0], -(p[3, GX - 1] - p[3, GX - 2]) / 0.1)
    assert np.isclose(ef[3, 4, 0], -(p[3, 5] - p[3, 3]) / 0.2)
    assert np.isclose(ef[0, 4, 1], -(p[1, 4] - p[P - 1, 4]) / 0.4)
    assert np.isclose(ef[P, 4, 1], -(p[1, 4] - p[P - 1, 4]) / 0.4)
    assert np.isclose(ef[P - 1, 4, 1], -(p[0, 4] - p[P - 2, 4]) / 0.4)


def test_push_wraps_y(oracle):
    import pic_b200 as Pb
    nx = ny = 8
    dx = 1e-3
    H = ny * dx
    g = oracle.Grid(nx, ny, dx, dx)
    pts = np.zeros(6, Pb.POINT_DTYPE)
    dt = 1e-9
    pts["x"] = 4.5 * dx
    pts["y"] = [0.2 * dx, H - 0.2 * dx, 3.5 * dx, 0.1 * dx, 0.5 * dx, 7.5 * dx]
    vy = np.array([-0.5, 0.5, 0.25, -0.1 - 8.0, -0.5 - 8.0, 0.0]) * dx / dt
    pts["vy"] = vy
    pts["vx"] = [0, 0, 0, 0, 0, -5.0 * dx / dt]   # the last one leaves through x < 0
    pts["pointer"] = np.arange(6)
    ef = np.zeros((g.nodes, 2))
    bz = np.zeros(g.nodes)
    y0 = pts["y"].copy()
    d, left = oracle.push(g, pts, -1.76e11, dt, ef, bz, periodic=True)
    assert d == 1 and left == 1
    want = np.mod(y0 + vy * dt, H)
    live = pts["pointer"] != -1
    assert np.allclose(pts["y"][live], want[live], rtol=0, atol=1e-15)
    assert np.all((pts["y"][live] >= 0) & (pts["y"][live] < H))
    # the same particles without the wrap are lost through y
    q = pts.copy()
    q["y"], q["pointer"] = y0, np.arange(6)
    d2, _ = oracle.push(g, q, -1.76e11, dt, ef, bz)
    assert d2 == 5


def test_config_reader_takes_the_periodic_flag(picb, tmp_path):
    import test_capi_cpu as T
    p, _ = T._write_inputs(tmp_path, periodic=1)
    g = tmp_path / "geometry3.conf"
    g.write_text(T.GEOMETRY.replace("  5\n", "  3\n"))
    cfg = picb.Config()
    st = picb.lib().pic_config_from_files(p.encode(), str(g).encode(), ctypes.byref(cfg))
    assert st == 0, picb.lib().pic_last_error()
    assert cfg.periodic_y == 1 and cfg.num_rects == 3
    # more than three rectangles with a periodic boundary: readGeometry's exit 9
    p5, g5 = T._write_inputs(tmp_path, periodic=1)
    assert picb.lib().pic_config_from_files(p5.encode(), g5.encode(), ctypes.byref(cfg)) == -2
