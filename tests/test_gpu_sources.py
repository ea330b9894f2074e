"""Particle sources (pic_generate_new_particles) against the reference's
generate_new_electrons / generate_pairs (SYCL-PIC-poissonsolver/src/
utils.cpp:374-777):

* re-injection: exactly (electron exits - ion exits) through x < 0, all at
  x = 0.024 m, y uniform, Maxwellian velocities with per-component sigma
  sqrt(e Te/m) (within 3 %);
* pairs: ceil(fn) pairs with fn = YMAX dt (2/pi) (x22-x11) ionimax /
  rate_div; electron and ion of a pair share the position; x follows the
  arcsine law x = xm + asin(2u-1)(x22-x11)/pi (the recovered u is uniform:
  Kolmogorov-Smirnov distance < 0.02), y uniform;
* the new particles are state at once: the next deposit counts their charge
  exactly (fixed point) and the next push keeps them.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

QE = 1.602e-19


def make(nx=128, ny=32, dx=2.5e-4):
    import pic_b200 as P
    import pic_configs as C
    w = C.cfg1()
    w.nx, w.ny, w.dx = nx, ny, dx
    w.rects = C.wall_rects(nx, ny)
    w.species = C._species(nx, ny, 8, 1e15)
    return w, P.Pic(C.library_config(w))


def test_reinjection_and_pairs():
    import pic_b200 as P
    w, pic = make()
    with pic:
        # electrons next to the left wall flying out; ions at rest
        n_out = 20000
        e = np.zeros(n_out + 5000, P.POINT_DTYPE)
        rng = np.random.default_rng(1)
        e["x"][:n_out] = 0.1 * w.dx
        e["y"][:n_out] = rng.uniform(0, w.ymax, n_out)
        e["vx"][:n_out] = -0.5 * w.dx / w.dt
        e["x"][n_out:] = rng.uniform(0.015, 0.02, 5000)      # away from the pair band
        e["y"][n_out:] = rng.uniform(0, w.ymax, 5000)
        ions = e[n_out:].copy()
        ions["vx"] = 0.0
        pic.import_points(0, e)
        pic.import_points(1, ions)
        pic.move_particles(0)
        pic.move_particles(1)
        assert pic.count(0) == 5000
        te, ti = 2.0, 0.026
        # fn = H dt (2/pi)(x22-x11) ionimax/rate_div, scaled to ~12000 pairs
        ionimax = 12000.5 / (w.ymax * w.dt * (2 / np.pi) * 0.0075 / 1.67e6)
        ne, npairs = pic.generate_new_particles(te_ev=te, ti_ev=ti, ionimax=ionimax)
        fn = w.ymax * w.dt * (2 / np.pi) * (0.01 - 0.0025) * ionimax / 1.67e6
        assert ne == n_out
        assert npairs == int(np.ceil(fn))
        assert pic.count(0) == 5000 + ne + npairs and pic.count(1) == 5000 + npairs
        ep, ip = pic.export_points(0), pic.export_points(1)
    # re-injected electrons: the ones at x = 0.024
    at = np.isclose(ep["x"], 0.024, rtol=0, atol=1e-9)
    assert at.sum() == ne
    r = ep[at]
    sig_e = np.sqrt(QE * te / 9.109e-31)
    for k in ("vx", "vy", "vz"):
        assert abs(r[k].std() / sig_e - 1) < 0.03 and abs(r[k].mean()) < 0.03 * sig_e
    assert 0 <= r["y"].min() and r["y"].max() < w.ymax
    assert abs(r["y"].mean() / (w.ymax / 2) - 1) < 0.03
    # pairs: the band, the arcsine law, matching positions
    band = (ep["x"] >= 0.0025 - 1e-12) & (ep["x"] <= 0.01 + 1e-12)
    px = np.sort(ep["x"][band])
    ib = (ip["x"] >= 0.0025 - 1e-12) & (ip["x"] <= 0.01 + 1e-12)
    assert np.allclose(px, np.sort(ip["x"][ib]), rtol=0, atol=1e-7)
    assert len(px) == npairs
    u = (np.sin((px - 0.00625) * np.pi / 0.0075) + 1) / 2
    ks = np.abs(np.sort(u) - (np.arange(len(u)) + 0.5) / len(u)).max()
    assert ks < 0.02, ks
    sig_i = np.sqrt(QE * ti / 6.6335e-26)
    assert abs(ip["vx"][ib].std() / sig_i - 1) < 0.03


def test_new_particles_deposit_exactly_and_survive_a_push():
    import pic_b200 as P
    import pic_configs as C
    w, pic = make(nx=96, ny=48)
    with pic:
        C.load_plasma(pic, w, seed=3)
        for it in range(2):
            pic.step(it)
        n0 = [pic.count(s) for s in range(2)]
        pic.zero_rho()
        pic.charge_deposition(0)
        q0 = pic.final_mesh(0).sum()
        # a push leaves the accumulators holding the new positions; sources
        # then add their particles to them
        pic.move_particles(0)
        pic.move_particles(1)
        n1 = [pic.count(s) for s in range(2)]
        ionimax = 3000.5 / (w.ymax * w.dt * (2 / np.pi) * 0.0075 / 1.67e6)
        ne, npairs = pic.generate_new_particles(ionimax=ionimax, reinject=0)
        assert ne == 0 and npairs == 3001
        pic.zero_rho()
        pic.charge_deposition(0)
        q1 = pic.final_mesh(0).sum()
        dx = w.xmax / w.nx
        wgt = w.species[0][3] * w.xmax * w.ymax / (w.species[0][2] * dx ** 4)
        assert np.isclose(q1, (n1[0] + npairs) * wgt * dx * dx, rtol=1e-12, atol=0)
        pic.poisson_solve(3)
        for s in range(2):
            pic.move_particles(s)
        n2 = [pic.count(s) for s in range(2)]
        # the new ions stay (ions hardly move in one step); electrons may
        # leave through the walls in the (electron-only) field of this test
        assert n1[1] + npairs - 5 <= n2[1] <= n1[1] + npairs
        assert n1[0] + npairs - 0.05 * n1[0] <= n2[0] <= n1[0] + npairs
    assert q0 > 0
