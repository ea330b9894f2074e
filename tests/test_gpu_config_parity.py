"""GPU against the FP64 oracle on the full-size workloads, through the C ABI.

The 512^2 workload (left wall 100 V, 64 particles per cell and species,
2 x 16,777,216 particles) and the 1024^2 workload (200 V central electrode,
100 particles per cell and species plus the drifting Gaussian blob of up to
~1,100 particles per cell, ~2.3e8 particles) at their full sizes.  The
oracle (oracle/pic_oracle.c) is pinned bit for bit to the reference's own
mover and interpolate kernels (tests/test_oracle_ref_pin.py).

Tolerances (FP32 state and 64-bit fixed-point deposit against FP64):
  * binning: bit-exact -- per-bucket counts in the reference's key layout
    equal, and the cell-sorted state equal to the expected one as a multiset
    (order-independent 64-bit hash sums over every particle);
  * deposit: max |d final_mesh| <= 2e-6 * max|final_mesh|, same for rho;
    total charge exact to 1e-12 relative;
  * push, one step, particle by particle (tags in vz): |dx|, |dy| <= 2e-6
    cell, |dv| <= 2e-5 v_thermal + 4e-7 |v| (FP32 rounding of the drift
    velocity of the blob); every surviving particle in the oracle's cell
    unless the oracle's position lies within 1e-5 cell of a cell edge; the
    deleted sets equal except for particles within 1e-5 cell of a wall;
  * Poisson: the GPU potential's true relative residual (FP64, measured by
    the oracle) <= 1e-8 at every step, and max |phi - phi_direct| <=
    1e-5 * max|phi| against a direct solve of the GPU's own charge density
    (every tenth step of the 50-step run);
  * 50 steps of the 512^2 workload, checked at every step: the GPU's
    final_mesh equals the oracle's deposit of the GPU's own particle state
    (2e-6), and over the run the total energy (kinetic + 1/2 sum rho phi
    dA; equal at the start within 1e-5) changes by the same relative amount
    as in an FP64 oracle run from the same initial particles (within 1e-4),
    with lost counts within 0.5 % + 5.  (The workload's own length is 500
    steps; 50 keep the test within a few minutes.)
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

EPS0 = 8.854e-12
QE = 1.602e-19
TAG0 = 0x00800000   # tags are the bit patterns of normal FP32 values from 2^-126 up


def _grid(O, w):
    dx = w.xmax / w.nx
    return O.Grid(w.nx, w.ny, dx, dx, w.xmax, w.ymax)


def _species(O, w, s):
    sp = O.Species(str(s), *w.species[s])
    dx = w.xmax / w.nx
    return sp, O.weighing_factor(sp, w.xmax * w.ymax, dx, dx)


def _export_state(pic, s):
    import test_gpu_particles as T
    return T.export_state(pic, s)


def _tag(pts):
    """vz := the FP32 value whose bits are TAG0 + index (exact in FP64 and
    FP32; the push carries vz unchanged)."""
    pts["vz"] = (np.arange(len(pts), dtype=np.uint32) + np.uint32(TAG0)).view(np.float32)


def _untag(vz32):
    return vz32.view(np.uint32).astype(np.int64) - TAG0


def _mix(a):
    a = a.astype(np.uint64)
    a = (a ^ (a >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    a = (a ^ (a >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return a ^ (a >> np.uint64(31))


def _multiset_hash(cell, fx, fy, vx, vy, vz):
    """Order-independent hash of a particle multiset (two 64-bit sums)."""
    u = lambda a: a.view(np.uint32).astype(np.uint64)
    c = cell.astype(np.uint64)
    h1 = _mix((c << np.uint64(32)) | u(fx))
    h2 = _mix((u(fy) << np.uint64(32)) | u(vx))
    h3 = _mix((u(vy) << np.uint64(32)) | u(vz))
    with np.errstate(over="ignore"):
        a = int((h1 + h2 * np.uint64(3) + h3 * np.uint64(7)).sum(dtype=np.uint64))
        b = int((_mix(h1 ^ h3) + h2).sum(dtype=np.uint64))
    return a, b


def _expected_state(w, pts):
    """InsertKernel's binning of FP64 points (src/particles.cpp:230-235):
    cell ((int)(y*(1/dy)), (int)(x*(1/dx))), FP32 offset from the FP64
    remainder (clamped below 1), FP32 velocities."""
    dx = w.xmax / w.nx
    sx, sy = pts["x"] * (1.0 / dx), pts["y"] * (1.0 / dx)
    gx, gy = sx.astype(np.int64), sy.astype(np.int64)
    one_below = np.float32(np.nextafter(np.float32(1), np.float32(0)))
    fx = np.minimum((sx - gx).astype(np.float32), one_below)
    fy = np.minimum((sy - gy).astype(np.float32), one_below)
    return ((gy * w.nx + gx).astype(np.int32), fx, fy, pts["vx"].astype(np.float32),
            pts["vy"].astype(np.float32), pts["vz"].astype(np.float32))


def _check_deposit(O, w, pic, pts, s, rho_acc):
    g = _grid(O, w)
    sp, wgt = _species(O, w, s)
    fin_o, _ = O.deposit(g, pts, sp, wgt, EPS0, rho_acc)
    fin = pic.final_mesh(s)
    scale = np.abs(fin_o).max()
    err = np.abs(fin - fin_o).max()
    assert err <= 2e-6 * scale, (s, err / scale)
    dx = w.xmax / w.nx
    assert np.isclose(fin.sum(), len(pts) * wgt * dx * dx, rtol=1e-12, atol=0)
    return err / scale


def _check_poisson(O, w, pic, rho_before, phi):
    """True relative residual of the GPU potential and its distance from a
    direct solve of the same charge density."""
    dx = w.xmax / w.nx
    el = O.Electrodes(w.rects)
    mask = O.electrode_mask(w.GX, w.GY, el)
    b = rho_before.copy()
    O.overwrite_rho(w.GX, w.GY, el, b)
    rel = O.reduced_relres(w.GX, w.GY, dx, dx, mask, b, phi)
    assert rel <= 1e-8, rel
    return rel


def _check_push(O, w, s, before, got, ef, bz):
    """One push of `before` (tagged FP64 points) by the oracle against the
    GPU's exported state `got`, particle by particle."""
    g = _grid(O, w)
    dx = w.xmax / w.nx
    ctom = w.species[s][0] / w.species[s][1]
    ref = before.copy()
    O.push(g, ref, ctom, w.dt, ef, bz)
    del before
    tag = _untag(got["vz"])
    n = len(ref)
    assert tag.min() >= 0 and tag.max() < n and np.bincount(tag, minlength=n).max() == 1
    alive_o = ref["pointer"] != -1
    alive_g = np.zeros(n, bool)
    alive_g[tag] = True
    # deleted sets: equal except within round-off of a wall
    sx, sy = ref["x"] * (1.0 / dx), ref["y"] * (1.0 / dx)
    near_wall = (np.abs(sx) < 1e-5) | (np.abs(sy) < 1e-5) | (np.abs(sx - w.nx) < 1e-5) | \
        (np.abs(sy - w.ny) < 1e-5)
    differ = alive_o != alive_g
    assert not (differ & ~near_wall).any(), int((differ & ~near_wall).sum())
    # per particle, on the survivors of both
    pos = np.full(n, -1, np.int64)
    pos[tag] = np.arange(len(tag))
    both = np.flatnonzero(alive_o & alive_g)
    gi = pos[both]
    cell = got["cell"][gi].astype(np.int64)
    xg = ((cell % w.nx) + got["fx"][gi].astype(np.float64))
    yg = ((cell // w.nx) + got["fy"][gi].astype(np.float64))
    ex = np.abs(xg - sx[both]).max()
    ey = np.abs(yg - sy[both]).max()
    assert ex <= 2e-6 and ey <= 2e-6, (ex, ey)
    vth = np.sqrt(QE * w.plasma[s].temperature_ev / w.species[s][1])
    for k in ("vx", "vy"):
        dv = np.abs(got[k][gi].astype(np.float64) - ref[k][both])
        lim = 2e-5 * vth + 4e-7 * np.abs(ref[k][both])
        assert (dv <= lim).all(), (k, float((dv / lim).max()))
    # cells: the oracle's InsertKernel cell, except within 1e-5 cell of an edge
    cgx, cgy = (ref["x"][both] * (1.0 / dx)).astype(np.int64), (ref["y"][both] * (1.0 / dx)).astype(np.int64)
    cell_o = cgy * w.nx + cgx
    fx, fy = sx[both] - np.round(sx[both]), sy[both] - np.round(sy[both])
    near_edge = (np.abs(fx) < 1e-5) | (np.abs(fy) < 1e-5)
    wrong = cell_o != cell
    assert not (wrong & ~near_edge).any(), int((wrong & ~near_edge).sum())
    return ex, ey, int(differ.sum()), int(wrong.sum()), int((~alive_o).sum())


def _jitter(w, pts, rng):
    """Moves each position by up to 1e-9 cell so that it is a general FP64
    value (not an FP32 offset times dx), inside the domain."""
    dx = w.xmax / w.nx
    for k, top in (("x", w.xmax), ("y", w.ymax)):
        v = pts[k] + rng.uniform(-1e-9, 1e-9, len(pts)) * dx
        pts[k] = np.clip(v, 0.0, np.nextafter(top, 0.0))


def test_cfg2_full_size_single_step(oracle):
    """512^2, 2 x 16,777,216 particles: binning of general FP64 points,
    deposit, Poisson and one push of each species against the oracle."""
    import pic_b200 as P
    import pic_configs as C
    O = oracle
    w = C.cfg2()
    rng = np.random.default_rng(12)
    with P.Pic(C.library_config(w)) as pic:
        C.load_plasma(pic, w, seed=4321)
        pts = []
        for s in range(2):
            p = pic.export_points(s)
            _jitter(w, p, rng)
            _tag(p)
            pic.import_points(s, p)
            assert np.array_equal(pic.bin_counts(s), O.bucket_counts(_grid(O, w), p))
            st = _export_state(pic, s)
            assert _multiset_hash(st["cell"], st["fx"], st["fy"], st["vx"], st["vy"], st["vz"]) == \
                _multiset_hash(*_expected_state(w, p))
            pts.append(p)
        pic.zero_rho()
        rho_o = np.zeros(pic.nodes)
        for s in range(2):
            pic.charge_deposition(s)
            _check_deposit(O, w, pic, pts[s], s, rho_o)
        rho = pic.rho()
        assert np.abs(rho - rho_o).max() <= 2e-6 * np.abs(rho_o).max()
        pic.poisson_solve(0)
        _check_poisson(O, w, pic, rho, pic.phi())
        ef = pic.efield()
        bz = np.full(pic.nodes, w.b0)
        for s in range(2):
            pic.move_particles(s)
            got = _export_state(pic, s)
            ex, ey, dead_diff, cell_diff, dead = _check_push(O, w, s, pts[s], got, ef, bz)
            print(f"species {s}: |dx| {ex:.2e} |dy| {ey:.2e} cell; deleted {dead}, "
                  f"differing deletions {dead_diff}, differing cells {cell_diff}")


def test_cfg3_full_size_single_step(oracle):
    """1024^2 with the central electrode and the blob (~2.3e8 particles, up
    to ~1,100 per cell): binning of general FP64 points, deposit, Poisson
    and one push of each species against the oracle."""
    import pic_b200 as P
    import pic_configs as C
    O = oracle
    w = C.cfg3()
    rng = np.random.default_rng(13)
    with P.Pic(C.library_config(w)) as pic:
        C.load_plasma(pic, w, seed=99)
        pts = []
        for s in range(2):
            p = pic.export_points(s)
            _jitter(w, p, rng)
            _tag(p)
            pic.import_points(s, p)
            counts = pic.bin_counts(s)
            assert np.array_equal(counts, O.bucket_counts(_grid(O, w), p))
            assert counts.max() > 1000          # the blob's peak cells
            st = _export_state(pic, s)
            assert _multiset_hash(st["cell"], st["fx"], st["fy"], st["vx"], st["vy"], st["vz"]) == \
                _multiset_hash(*_expected_state(w, p))
            del st
            pts.append(p)
        pic.zero_rho()
        rho_o = np.zeros(pic.nodes)
        for s in range(2):
            pic.charge_deposition(s)
            _check_deposit(O, w, pic, pts[s], s, rho_o)
        rho = pic.rho()
        assert np.abs(rho - rho_o).max() <= 2e-6 * np.abs(rho_o).max()
        pic.poisson_solve(0)
        _check_poisson(O, w, pic, rho, pic.phi())
        ef = pic.efield()
        bz = np.full(pic.nodes, w.b0)
        for s in range(2):
            pic.move_particles(s)
            got = _export_state(pic, s)
            p = pts[s]
            pts[s] = None
            ex, ey, dead_diff, cell_diff, dead = _check_push(O, w, s, p, got, ef, bz)
            del got, p
            print(f"species {s}: |dx| {ex:.2e} |dy| {ey:.2e} cell; deleted {dead}, "
                  f"differing deletions {dead_diff}, differing cells {cell_diff}")


def _energy(w, pts, fins, phi):
    """Kinetic energy of the simulated plasma plus 1/2 sum_nodes rho_c phi dA
    (J per metre of depth).  Each simulated particle stands for
    actual * area / sim real ones (updateWeighingFactor)."""
    dx = w.xmax / w.nx
    ke = 0.0
    rho_c = np.zeros_like(phi)
    for s in range(2):
        q, m, sim, actual = w.species[s]
        p = pts[s]
        live = p["pointer"] != -1
        v2 = p["vx"][live] ** 2 + p["vy"][live] ** 2 + p["vz"][live] ** 2
        ke += 0.5 * m * v2.sum() * actual * w.xmax * w.ymax / sim
        rho_c += q * fins[s]
    return ke, 0.5 * float((rho_c * phi).sum()) * dx * dx


def test_cfg2_fifty_steps_checked_every_step(oracle):
    """512^2 full size, 50 steps.  At every step: the GPU's final_mesh
    against the oracle's deposit of the GPU's own particles, the GPU's
    potential against a direct solve of its own charge density.  Beside it
    an FP64 oracle run from the same initial particles; at the end the
    total-energy drift and the losses of the two runs agree."""
    import pic_b200 as P
    import pic_configs as C
    O = oracle
    w = C.cfg2()
    steps = 50
    g = _grid(O, w)
    dx = w.xmax / w.nx
    sps = [_species(O, w, s) for s in range(2)]
    ctom = [w.species[s][0] / w.species[s][1] for s in range(2)]
    D = O.DirectPoisson(w.GX, w.GY, dx, dx, O.Electrodes(w.rects))
    bz = np.full(g.nodes, w.b0)
    worst_dep = worst_phi = worst_rel = 0.0
    with P.Pic(C.library_config(w)) as pic:
        C.load_plasma(pic, w, seed=777)
        ref = [pic.export_points(s) for s in range(2)]
        n0 = [len(r) for r in ref]
        e_g, e_o = [], []
        for it in range(steps):
            cur = [pic.export_points(s) for s in range(2)]
            pic.zero_rho()
            rho_chk = np.zeros(g.nodes)
            fin_g = []
            for s in range(2):
                pic.charge_deposition(s)
                worst_dep = max(worst_dep, _check_deposit(O, w, pic, cur[s], s, rho_chk))
                fin_g.append(pic.final_mesh(s))
            rho = pic.rho()
            pic.poisson_solve(it)
            phi_g = pic.phi()
            worst_rel = max(worst_rel, _check_poisson(O, w, pic, rho, phi_g))
            if it % 10 == 0 or it == steps - 1:
                phi_d, _ = D.step(rho.copy())
                worst_phi = max(worst_phi, np.abs(phi_g - phi_d).max() / np.abs(phi_d).max())
                assert worst_phi <= 1e-5
            for s in range(2):
                pic.move_particles(s, it)
            # the FP64 oracle's own run
            rho_o = np.zeros(g.nodes)
            fin_o = [O.deposit(g, ref[s], sps[s][0], sps[s][1], EPS0, rho_o)[0] for s in range(2)]
            phi_o, ef_o = D.step(rho_o)
            if it in (0, steps - 1):
                e_g.append(sum(_energy(w, cur, fin_g, phi_g)))
                e_o.append(sum(_energy(w, ref, fin_o, phi_o)))
            for s in range(2):
                O.push(g, ref[s], ctom[s], w.dt, ef_o, bz)
        n_g = [pic.count(s) for s in range(2)]
    n_o = [int((ref[s]["pointer"] != -1).sum()) for s in range(2)]
    drift_g = (e_g[1] - e_g[0]) / e_g[0]
    drift_o = (e_o[1] - e_o[0]) / e_o[0]
    print(f"deposit {worst_dep:.2e}, phi {worst_phi:.2e}, relres {worst_rel:.2e}; energy drift "
          f"gpu {drift_g:.6e} oracle {drift_o:.6e}; lost gpu {[n0[s] - n_g[s] for s in range(2)]} "
          f"oracle {[n0[s] - n_o[s] for s in range(2)]}")
    assert abs(e_g[0] - e_o[0]) <= 1e-5 * abs(e_o[0])
    assert abs(drift_g - drift_o) <= 1e-4
    for s in range(2):
        lost_g, lost_o = n0[s] - n_g[s], n0[s] - n_o[s]
        assert abs(lost_g - lost_o) <= 0.005 * lost_o + 5, (s, lost_g, lost_o)
