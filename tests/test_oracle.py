"""CPU tests of the FP64 oracle: pinned against the reference's PARDISO golden
vectors, plus physics invariants of the restated deposit and push, and the
hashmap port checked against the semantic restatement."""
import glob
import os

import numpy as np
import pytest

from conftest import GOLDEN

FIXTURES = sorted(glob.glob(os.path.join(GOLDEN, "poisson_257_iter*.npz")))


def _golden_setup(O, d):
    GX = GY = int(d["nx"]) + 1
    dx = dy = float(d["xmax"]) / int(d["nx"])
    el = O.Electrodes.from_fractions(GX, GY, O.walls(GX, GY))
    return GX, GY, dx, dy, el


@pytest.mark.parametrize("path", FIXTURES)
def test_direct_solve_reproduces_pardiso(oracle, path):
    d = np.load(path)
    GX, GY, dx, dy, el = _golden_setup(oracle, d)
    P = oracle.DirectPoisson(GX, GY, dx, dy, el)
    rho = d["rho_input"].copy()
    phi, _ = P.step(rho)
    err = np.abs(phi - d["phi_cpp"]).max()
    assert err <= 1e-9, err  # observed 2.8e-10 V


@pytest.mark.parametrize("path", FIXTURES)
def test_golden_phi_satisfies_restated_operator(oracle, path):
    """phi_cpp solves the restated generateCoeffs system to round-off: this
    pins the stencil, the electrode rows and the overwriteRho sign."""
    d = np.load(path)
    GX, GY, dx, dy, el = _golden_setup(oracle, d)
    mask = oracle.electrode_mask(GX, GY, el)
    b = d["rho_input"].copy()
    oracle.overwrite_rho(GX, GY, el, b)
    assert oracle.reduced_relres(GX, GY, dx, dy, mask, b, d["phi_cpp"]) < 1e-13


def test_planted_mistake_is_caught(oracle):
    """A wrong mesh spacing in the oracle must break the golden check."""
    d = np.load(FIXTURES[0])
    GX, GY, dx, dy, el = _golden_setup(oracle, d)
    P = oracle.DirectPoisson(GX, GY, dx * 1.001, dy, el)
    phi, _ = P.step(d["rho_input"].copy())
    assert np.abs(phi - d["phi_cpp"]).max() > 1e-5


@pytest.mark.parametrize("path", FIXTURES[:1])
def test_cg_matches_pardiso(oracle, path):
    d = np.load(path)
    GX, GY, dx, dy, el = _golden_setup(oracle, d)
    mask = oracle.electrode_mask(GX, GY, el)
    b = d["rho_input"].copy()
    oracle.overwrite_rho(GX, GY, el, b)
    phi, it, rel = oracle.cg_solve(GX, GY, dx, dy, mask, b, tol=1e-12)
    assert rel <= 1e-12
    assert np.abs(phi - d["phi_cpp"]).max() <= 1e-9


def test_efield_boundary_copy(oracle):
    GX, GY = 9, 7
    rng = np.random.default_rng(0)
    phi = rng.random(GX * GY)
    ef = oracle.efield(GX, GY, 0.1, 0.2, phi).reshape(GY, GX, 2)
    p = phi.reshape(GY, GX)
    assert np.isclose(ef[3, 4, 0], -(p[3, 5] - p[3, 3]) / 0.2)
    assert np.isclose(ef[3, 4, 1], -(p[4, 4] - p[2, 4]) / 0.4)
    assert np.array_equal(ef[0, 0], ef[1, 1])
    assert np.array_equal(ef[GY - 1, 3], ef[GY - 2, 3])
    assert np.array_equal(ef[2, GX - 1], ef[2, GX - 2])


def _small(ppc=8, nx=24, ny=20, seed=3):
    import pic_configs as C
    w = C.cfg1()
    w.nx, w.ny = nx, ny
    w.rects = C.wall_rects(nx, ny)
    w.species = C._species(nx, ny, ppc, 1e15)
    w.plasma = [C.PlasmaSpec(ppc, 2.0), C.PlasmaSpec(ppc, 0.026)]
    return w, C.host_points(w, 0, seed, ppc)


def _grid(O, w):
    return O.Grid(w.nx, w.ny, w.dx, w.dx)


def test_deposit_conserves_charge(oracle):
    w, pts = _small()
    g = _grid(oracle, w)
    sp = oracle.Species("e", *w.species[0])
    wgt = oracle.weighing_factor(sp, w.xmax * w.ymax, w.dx, w.dx)
    final, energy = oracle.deposit(g, pts, sp, wgt, 8.854e-12)
    assert np.isclose(final.sum(), len(pts) * wgt * w.dx * w.dx, rtol=1e-12)
    # uniform plasma: interior nodes carry n0 on average
    f = final.reshape(w.ny + 1, w.nx + 1)[1:-1, 1:-1]
    assert abs(f.mean() / 1e15 - 1.0) < 0.05
    assert (energy >= 0).all()


def test_push_free_streaming(oracle):
    w, pts = _small()
    g = _grid(oracle, w)
    pts["vx"] *= 1e-3
    pts["vy"] *= 1e-3
    before = pts.copy()
    ef = np.zeros((g.nodes, 2))
    bz = np.zeros(g.nodes)
    deleted, left = oracle.push(g, pts, -1.76e11, w.dt, ef, bz)
    assert deleted == 0 and left == 0
    assert np.array_equal(pts["x"], before["x"] + w.dt * before["vx"])
    assert np.array_equal(pts["vx"], before["vx"])


def test_push_boris_rotation_keeps_speed(oracle):
    w, pts = _small()
    g = _grid(oracle, w)
    pts["vx"] *= 1e-3
    pts["vy"] *= 1e-3
    v0 = np.hypot(pts["vx"], pts["vy"])
    ef = np.zeros((g.nodes, 2))
    bz = np.full(g.nodes, 0.05)
    oracle.push(g, pts, -1.76e11, w.dt, ef, bz)
    assert np.allclose(np.hypot(pts["vx"], pts["vy"]), v0, rtol=1e-13)


def test_push_absorbs_and_counts_left_exits(oracle):
    w, pts = _small()
    g = _grid(oracle, w)
    pts = pts[:4].copy()
    pts["x"] = [1e-6, 1e-6, w.xmax - 1e-6, 0.5 * w.xmax]
    pts["y"] = 0.5 * w.ymax
    pts["vx"] = [-1e6, 1e3, 1e6, 0.0]
    pts["vy"] = 0.0
    ef = np.zeros((g.nodes, 2))
    bz = np.zeros(g.nodes)
    deleted, left = oracle.push(g, pts, -1.76e11, w.dt, ef, bz)
    assert deleted == 2 and left == 1
    assert list(pts["pointer"] == -1) == [True, False, True, False]


def test_hashmap_port_matches_semantics(oracle):
    """The reference-structure port (hashmap) bins, deposits, moves, cleans and
    compacts exactly like the semantic restatement."""
    w, pts = _small(ppc=8)
    g = _grid(oracle, w)
    sp = oracle.Species("e", *w.species[0])
    wgt = oracle.weighing_factor(sp, w.xmax * w.ymax, w.dx, w.dx)
    H = oracle.RefHashmapSpecies(g, pts.copy(), probing_length=64)
    assert np.array_equal(H.counts(), oracle.bucket_counts(g, pts))
    f1, e1 = H.deposit(sp, wgt, 8.854e-12)
    f2, e2 = oracle.deposit(g, pts, sp, wgt, 8.854e-12)
    assert np.allclose(f1, f2, rtol=1e-12, atol=0)
    assert np.allclose(e1, e2, rtol=1e-12, atol=0)
    rng = np.random.default_rng(1)
    ef = rng.normal(0, 2e3, (g.nodes, 2))
    bz = np.full(g.nodes, 0.01)
    sem = pts.copy()
    for _ in range(3):
        H.move(sp.ctom, w.dt, ef, bz)
        oracle.push(g, sem, sp.ctom, w.dt, ef, bz)
        H.cleanup()
    live_h = H.pts[: H.end][H.pts[: H.end]["pointer"] != -1]
    assert np.array_equal(H.counts(), oracle.bucket_counts(g, sem))
    H.compact()
    live_h2 = H.pts[: H.end]
    assert (live_h2["pointer"] != -1).all()
    key = lambda a: np.sort(a["vz"])
    assert np.array_equal(key(live_h), key(sem[sem["pointer"] != -1]))
    assert np.array_equal(key(live_h2), key(live_h))
    assert np.array_equal(H.counts(), oracle.bucket_counts(g, sem))
