"""GPU Poisson solve against the reference's PARDISO golden vectors and the
FP64 oracle, through the C ABI.

Tolerances: at tol = 1e-8 the true relative residual of the returned phi,
measured by the oracle in FP64, is <= 1e-8; at tol = 1e-12 max |phi -
phi_PARDISO| <= 1e-8 V on the 257x257 dumps (|phi| <= 0.77 V there).  The E
field is the same FP64 formula as the oracle's (<= 1e-12 relative).
"""
import glob
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

FIXTURES = sorted(glob.glob(os.path.join(GOLDEN, "poisson_257_iter*.npz")))
EPS0 = 8.854e-12


def golden_pic(solver, tol, warm=0):
    import pic_b200 as P
    import pic_configs as C
    rects = C.wall_rects(256, 256)
    cfg = P.make_config(256, 256, 1.0, 1.0, 1e-9, [(-1.6e-19, 9.1e-31, 1.0, 1.0)], rects,
                        solver=solver, warm=warm, tol=tol, maxit=5000)
    return P.Pic(cfg)


@pytest.mark.parametrize("path", FIXTURES)
@pytest.mark.parametrize("solver", [0, 1])
def test_poisson_matches_pardiso(oracle, path, solver):
    d = np.load(path)
    with golden_pic(solver, 1e-12) as pic:
        pic.set_rho(d["rho_input"])
        pic.poisson_solve(0)
        phi = pic.phi()
        rhs = pic.rho()           # overwritten in place, as overwriteRho does
        it, rel, ms = pic.poisson_stats()
    assert rel <= 1e-12
    assert np.abs(phi - d["phi_cpp"]).max() <= 1e-8
    GX = 257
    el = oracle.Electrodes.from_fractions(GX, GX, oracle.walls(GX, GX))
    b = d["rho_input"].copy()
    oracle.overwrite_rho(GX, GX, el, b)
    assert np.array_equal(rhs, b)


@pytest.mark.parametrize("solver", [0, 1])
def test_poisson_relres_at_1e8(oracle, solver):
    d = np.load(FIXTURES[0])
    with golden_pic(solver, 1e-8) as pic:
        pic.set_rho(d["rho_input"])
        pic.poisson_solve(0)
        phi = pic.phi()
        it, rel, ms = pic.poisson_stats()
    GX = 257
    dx = 1.0 / 256
    el = oracle.Electrodes.from_fractions(GX, GX, oracle.walls(GX, GX))
    mask = oracle.electrode_mask(GX, GX, el)
    b = d["rho_input"].copy()
    oracle.overwrite_rho(GX, GX, el, b)
    true_rel = oracle.reduced_relres(GX, GX, dx, dx, mask, b, phi)
    assert true_rel <= 1e-8 and abs(true_rel - rel) <= 1e-10
    # stated max |dphi| against PARDISO at 1e-8
    assert np.abs(phi - d["phi_cpp"]).max() <= 1e-4
    if solver == 0:
        assert it <= 20  # multigrid preconditioning


def test_mg_beats_jacobi_in_iterations():
    d = np.load(FIXTURES[1])
    its = []
    for solver in (0, 1):
        with golden_pic(solver, 1e-8) as pic:
            pic.set_rho(d["rho_input"])
            pic.poisson_solve(0)
            its.append(pic.poisson_stats()[0])
    assert its[0] * 10 < its[1], its


@pytest.mark.parametrize("n", [96, 100, 129])
def test_poisson_internal_electrode_vs_direct(oracle, n):
    """Internal electrode, uneven grid sizes (odd coarsening), unequal dx/dy."""
    import pic_b200 as P
    import pic_configs as C
    dx, dy = 2.5e-4, 3.0e-4
    c = n // 2
    rects = C.wall_rects(n, n, left=75.0) + [(c - 7, c - 5, c + 9, c + 6, 200.0)]
    rng = np.random.default_rng(n)
    GX = n + 1
    rho = rng.normal(0, 1e7, GX * GX)
    cfg = P.make_config(n, n, n * dx, n * dy, 5e-11, [(-1.6e-19, 9.1e-31, 1.0, 1.0)], rects,
                        tol=1e-11, maxit=2000)
    with P.Pic(cfg) as pic:
        pic.set_rho(rho)
        pic.poisson_solve(0)
        phi = pic.phi()
        ef = pic.efield()
    el = oracle.Electrodes(rects)
    dx, dy = (n * dx) / n, (n * dy) / n   # the library's xmax/nx
    D = oracle.DirectPoisson(GX, GX, dx, dy, el)
    phi_o, ef_o = D.step(rho.copy())
    assert np.abs(phi - phi_o).max() <= 1e-7 * np.abs(phi_o).max()
    assert np.abs(ef - ef_o).max() <= 1e-6 * np.abs(ef_o).max()
    # E is the FP64 formula applied to the library's own phi
    ef_same = oracle.efield(GX, GX, dx, dy, phi)
    assert np.allclose(ef, ef_same, rtol=1e-12, atol=1e-9)


@pytest.mark.parametrize("n,inner", [(32, False), (30, True), (60, True)])
def test_exact_coarse_solve(oracle, n, inner):
    """The multigrid's coarse-grid correction is an exact solve of the first
    small level (inverted once at set-up).  On grids of at most 1,200 nodes
    that level is the grid itself (n = 32, 30: the preconditioner is the
    exact inverse in FP32, so PCG needs a few iterations at most to 1e-12);
    on 61^2 it is the 31^2 level below one tiled level.  Both against the
    direct solve to 1e-8 of max|phi|, an inner electrode included."""
    import pic_b200 as P
    import pic_configs as C
    dx = 2.5e-4
    c = n // 2
    rects = C.wall_rects(n, n, left=40.0)
    if inner:
        rects = rects + [(c - 3, c - 2, c + 4, c + 3, 90.0)]
    GX = n + 1
    rho = np.random.default_rng(n).normal(0, 1e7, GX * GX)
    cfg = P.make_config(n, n, n * dx, n * dx, 5e-11, [(-1.6e-19, 9.1e-31, 1.0, 1.0)], rects,
                        tol=1e-12, maxit=200)
    with P.Pic(cfg) as pic:
        pic.set_rho(rho)
        pic.poisson_solve(0)
        phi = pic.phi()
        iters = pic.poisson_stats()[0]
    D = oracle.DirectPoisson(GX, GX, dx, dx, oracle.Electrodes(rects))
    phi_o, _ = D.step(rho.copy())
    assert np.abs(phi - phi_o).max() <= 1e-8 * np.abs(phi_o).max()
    if GX * GX <= 1200:
        assert iters <= 4, iters


def test_warm_start_cuts_iterations():
    d0, d1 = np.load(FIXTURES[0]), np.load(FIXTURES[1])
    with golden_pic(0, 1e-8, warm=1) as pic:
        pic.set_rho(d0["rho_input"])
        pic.poisson_solve(0)
        cold = pic.poisson_stats()[0]
        pic.set_rho(d0["rho_input"])
        pic.poisson_solve(1)          # same rho again from the previous phi
        warm = pic.poisson_stats()[0]
    assert warm < cold


def test_contexts_of_different_sizes_alive_together(oracle):
    """A context keeps solving after a smaller one is created: the coarse-level
    kernel's shared-memory size is a property of the kernel, shared by every
    context of the process, and must cover the largest of them."""
    import pic_b200 as P
    import pic_configs as C
    out = []
    with P.Pic(P.make_config(250, 250, 1.0, 1.0, 1e-9, [(-1.6e-19, 9.1e-31, 1.0, 1.0)],
                             C.wall_rects(250, 250, left=5.0))) as big:
        with P.Pic(P.make_config(40, 40, 1.0, 1.0, 1e-9, [(-1.6e-19, 9.1e-31, 1.0, 1.0)],
                                 C.wall_rects(40, 40, left=5.0))) as small:
            for pic, n in ((big, 250), (small, 40)):
                rho = np.random.default_rng(n).normal(size=(n + 1) ** 2)
                pic.set_rho(rho)
                pic.poisson_solve(0)
                it, rel, _ = pic.poisson_stats()
                GX = n + 1
                mask = oracle.electrode_mask(GX, GX, oracle.Electrodes(C.wall_rects(n, n, left=5.0)))
                out.append((rel, oracle.reduced_relres(GX, GX, 1.0 / n, 1.0 / n, mask, pic.rho(), pic.phi())))
    for rel, rel_o in out:
        assert rel <= 1e-8 and rel_o <= 1e-8
