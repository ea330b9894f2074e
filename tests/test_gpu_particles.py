"""GPU parity of binning, deposit and push against the FP64 oracle, through the
C ABI.  Tolerances (FP32 state vs FP64 oracle):
  * binning: bit-exact (per-cell counts and cell membership as multisets);
  * deposit: max |d final_mesh| <= 2e-6 * max|final_mesh| (FP32 offsets and
    20-bit-per-axis fixed-point weights); total charge exact to 1e-12;
    energy mesh (a diagnostic; 16-bit axis weights, 2^-22 eV energies) within
    1e-5 * max;
  * push: |dx| <= 2e-6 cell, |dv| <= 2e-5 * v_thermal after one step.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

EPS0 = 8.854e-12


def small_workload(nx=48, ny=40, ppc=12, rects=None):
    import pic_configs as C
    w = C.cfg1()
    w.nx, w.ny = nx, ny
    w.rects = rects if rects is not None else C.wall_rects(nx, ny)
    w.species = C._species(nx, ny, ppc, 1e15)
    w.plasma = [C.PlasmaSpec(ppc, 2.0), C.PlasmaSpec(ppc, 0.026)]
    return w


def make_pic(w, **kw):
    import pic_b200 as P
    import pic_configs as C
    return P.Pic(C.library_config(w, **kw))


def lib_dx(w):
    """The library's spacing: xmax/nx (readPICDAT, src/particles.cpp:360)."""
    return w.xmax / w.nx, w.ymax / w.ny


def oracle_grid(O, w):
    dx, dy = lib_dx(w)
    return O.Grid(w.nx, w.ny, dx, dy)


def oracle_species(O, w, s):
    sp = O.Species(str(s), *w.species[s])
    dx, dy = lib_dx(w)
    return sp, O.weighing_factor(sp, w.xmax * w.ymax, dx, dy)


def in_domain(w, pts):
    """Points the import keeps: live and inside [0, nx) x [0, ny) cells."""
    dx, dy = lib_dx(w)
    sx, sy = pts["x"] * (1.0 / dx), pts["y"] * (1.0 / dy)
    return (pts["pointer"] != -1) & (sx >= 0) & (sy >= 0) & (sx < w.nx) & (sy < w.ny)


def expected_state(w, pts):
    """What the import must hold: cell = (int)(x*(1/dx)) (InsertKernel), FP32
    offsets from the FP64 remainder, FP32 velocities."""
    dx, dy = lib_dx(w)
    live = in_domain(w, pts)
    sx, sy = pts["x"][live] * (1.0 / dx), pts["y"][live] * (1.0 / dy)
    gx, gy = sx.astype(np.int64), sy.astype(np.int64)
    one_below = np.float32(np.nextafter(np.float32(1), np.float32(0)))
    fx = np.minimum((sx - gx).astype(np.float32), one_below)
    fy = np.minimum((sy - gy).astype(np.float32), one_below)
    p = pts[live]
    return dict(cell=(gy * w.nx + gx).astype(np.int32), fx=fx, fy=fy,
                vx=p["vx"].astype(np.float32), vy=p["vy"].astype(np.float32),
                vz=p["vz"].astype(np.float32))


def export_state(pic, s):
    import ctypes
    import pic_b200 as P
    n = ctypes.c_int64(0)
    L = P.lib()
    L.pic_export_state.argtypes = [ctypes.c_void_p, ctypes.c_int] + [ctypes.c_void_p] * 6 + [
        ctypes.c_int64, ctypes.POINTER(ctypes.c_int64)]
    L.pic_export_state.restype = ctypes.c_int
    assert L.pic_export_state(pic.h, s, None, None, None, None, None, None, 0, ctypes.byref(n)) == 0
    m = n.value
    out = dict(cell=np.zeros(m, np.int32), fx=np.zeros(m, np.float32), fy=np.zeros(m, np.float32),
               vx=np.zeros(m, np.float32), vy=np.zeros(m, np.float32), vz=np.zeros(m, np.float32))
    st = L.pic_export_state(pic.h, s, *[out[k].ctypes.data for k in ("cell", "fx", "fy", "vx", "vy", "vz")],
                            m, ctypes.byref(n))
    assert st == 0, L.pic_last_error()
    return out


def multiset(d):
    keys = ("cell", "fx", "fy", "vx", "vy", "vz")
    rec = np.stack([d[k].view(np.int32) if d[k].dtype == np.float32 else d[k] for k in keys], axis=1)
    order = np.lexsort(rec.T[::-1])
    return rec[order]


def edge_points(w, pts):
    """Appends dead, outside and exactly-on-boundary points."""
    import pic_b200 as P
    extra = np.zeros(8, P.POINT_DTYPE)
    extra["x"] = [-1e-9, w.xmax, w.xmax - 1e-12, 0.0, 3 * w.dx, 2 * w.dx, 5 * w.dx, 1e-300]
    extra["y"] = [w.dx, w.dx, w.dx, 0.0, w.ymax, w.ymax * (1 - 1e-16), 4 * w.dx, 7 * w.dx]
    extra["vx"] = 1.0
    extra["pointer"] = [0, 0, 0, 0, 0, 0, -1, 0]
    return np.concatenate([pts, extra])


def test_import_binning_bit_exact(oracle):
    import pic_configs as C
    w = small_workload()
    pts = edge_points(w, C.host_points(w, 0, seed=11))
    rng = np.random.default_rng(2)
    pts = pts[rng.permutation(len(pts))]
    with make_pic(w) as pic:
        pic.import_points(0, pts)
        exp = expected_state(w, pts)
        assert pic.count(0) == len(exp["cell"])
        # per-bucket counts in the reference's key layout
        counts = pic.bin_counts(0)
        keep = pts[in_domain(w, pts)]
        assert len(keep) == len(pts) - 4  # dead and outside points are dropped
        assert np.array_equal(counts, oracle.bucket_counts(oracle_grid(oracle, w), keep))
        got = export_state(pic, 0)
        assert np.all(np.diff(got["cell"]) >= 0)  # cell-sorted
        assert np.array_equal(multiset(got), multiset(exp))


def test_empty_species_and_reimport():
    import pic_b200 as P
    import pic_configs as C
    w = small_workload()
    with make_pic(w) as pic:
        pic.import_points(0, np.zeros(0, P.POINT_DTYPE))
        assert pic.count(0) == 0
        pic.zero_rho()
        pic.charge_deposition(0)
        pic.move_particles(0)
        assert np.count_nonzero(pic.rho()) == 0
        pts = C.host_points(w, 0, seed=5)
        pic.import_points(0, pts)
        pic.import_points(0, pts[:100])
        assert pic.count(0) == 100


@pytest.mark.parametrize("species", [0, 1])
def test_deposit_matches_oracle(oracle, species):
    import pic_configs as C
    w = small_workload()
    pts = C.host_points(w, species, seed=21 + species)
    g = oracle_grid(oracle, w)
    sp, wgt = oracle_species(oracle, w, species)
    rho_o = np.zeros(g.nodes)
    final_o, energy_o = oracle.deposit(g, pts, sp, wgt, EPS0, rho_o)
    with make_pic(w) as pic:
        pic.import_points(species, pts)
        pic.zero_rho()
        pic.charge_deposition(species)
        final, energy, rho = pic.final_mesh(species), pic.energy_mesh(species), pic.rho()
    scale = np.abs(final_o).max()
    assert np.abs(final - final_o).max() <= 2e-6 * scale
    assert np.abs(energy - energy_o).max() <= 1e-5 * np.abs(energy_o).max()
    assert np.abs(rho - rho_o).max() <= 2e-6 * np.abs(rho_o).max()
    # fixed point: the total charge is exact
    dx, dy = lib_dx(w)
    assert np.isclose(final.sum(), len(pts) * wgt * dx * dy, rtol=1e-12, atol=0)


def test_deposit_is_deterministic():
    import pic_configs as C
    w = small_workload()
    out = []
    for _ in range(2):
        with make_pic(w) as pic:
            C.load_plasma(pic, w, seed=99)
            for it in range(3):
                pic.step(it)
            pic.zero_rho()
            for s in range(2):
                pic.charge_deposition(s)
            out.append(pic.rho())
    assert np.array_equal(out[0], out[1])


def _random_fields(w, seed=4):
    rng = np.random.default_rng(seed)
    GX, GY = w.GX, w.GY
    x = np.linspace(0, 1, GX)[None, :]
    y = np.linspace(0, 1, GY)[:, None]
    phi = 40.0 * np.sin(np.pi * x) * np.sin(2 * np.pi * y) + rng.normal(0, 0.5, (GY, GX))
    return phi.ravel()


@pytest.mark.parametrize("species,bz", [(0, 0.01), (1, 0.02), (0, 0.0)])
def test_push_matches_oracle(oracle, species, bz):
    import pic_configs as C
    w = small_workload()
    w.b0 = bz
    pts = C.host_points(w, species, seed=31 + species)
    # vz is untouched by the push (Bz only, 2D E): use it as the particle tag
    pts["vz"] = np.arange(len(pts), dtype=np.float64) + 1.0
    phi = _random_fields(w)
    g = oracle_grid(oracle, w)
    # update_fields_from_phi first imposes the electrode potentials
    # (overwritePhi), as the reference's extension does
    phi_el = phi.copy()
    oracle.overwrite_phi(w.GX, w.GY, oracle.Electrodes(w.rects), phi_el)
    ef = oracle.efield(w.GX, w.GY, *lib_dx(w), phi_el)
    bzn = np.full(g.nodes, bz)
    ctom = w.species[species][0] / w.species[species][1]
    ref = pts.copy()
    oracle.push(g, ref, ctom, w.dt, ef, bzn)
    with make_pic(w) as pic:
        pic.import_points(species, pts)
        pic.set_phi(phi)
        pic.update_fields()
        pic.move_particles(species)
        got = export_state(pic, species)
        out = pic.export_points(species)
    live = ref[ref["pointer"] != -1]
    tag = got["vz"].astype(np.int64) - 1
    assert len(np.unique(tag)) == len(tag)
    # dead sets agree except for particles within round-off of a wall
    ref_live_tags = set((live["vz"] - 1).astype(np.int64))
    diff = ref_live_tags.symmetric_difference(set(tag))
    assert len(diff) <= 2
    common = np.array(sorted(ref_live_tags & set(tag)))
    rmap = {int(t): i for i, t in enumerate((live["vz"] - 1).astype(np.int64))}
    gmap = {int(t): i for i, t in enumerate(tag)}
    ri = np.array([rmap[t] for t in common])
    gi = np.array([gmap[t] for t in common])
    xg = (got["cell"][gi] % w.nx + got["fx"][gi].astype(np.float64)) * w.dx
    yg = (got["cell"][gi] // w.nx + got["fy"][gi].astype(np.float64)) * w.dx
    assert np.abs(xg - live["x"][ri]).max() <= 2e-6 * w.dx
    assert np.abs(yg - live["y"][ri]).max() <= 2e-6 * w.dx
    vth = np.sqrt(1.602e-19 * w.plasma[species].temperature_ev / w.species[species][1])
    assert np.abs(got["vx"][gi] - live["vx"][ri]).max() <= 2e-5 * vth
    assert np.abs(got["vy"][gi] - live["vy"][ri]).max() <= 2e-5 * vth
    # the reference-layout export carries the same particles
    assert len(out) == len(tag) and np.all(out["pointer"] >= 0)
    assert np.all((out["x"] >= 0) & (out["x"] < w.xmax) & (out["y"] >= 0) & (out["y"] < w.ymax))


def test_push_then_deposit_equals_fresh_deposit(oracle):
    """The deposit fused into the push equals a fresh deposit of the moved
    particles (same fixed-point sums)."""
    import pic_configs as C
    w = small_workload()
    with make_pic(w) as pic:
        C.load_plasma(pic, w, seed=7)
        pic.set_phi(_random_fields(w))
        pic.update_fields()
        for s in range(2):
            pic.move_particles(s)
        pic.zero_rho()
        for s in range(2):
            pic.charge_deposition(s)     # converts the fused accumulators
        fused = pic.rho()
        pts = [pic.export_points(s) for s in range(2)]
    with make_pic(w) as pic2:
        for s in range(2):
            pic2.import_points(s, pts[s])
        pic2.zero_rho()
        for s in range(2):
            pic2.charge_deposition(s)
        fresh = pic2.rho()
    assert np.abs(fused - fresh).max() <= 1e-6 * np.abs(fresh).max()


def test_absorbing_walls_and_left_exits():
    import pic_b200 as P
    w = small_workload()
    pts = np.zeros(4, P.POINT_DTYPE)
    pts["x"] = [0.2 * w.dx, 0.2 * w.dx, w.xmax - 0.1 * w.dx, 10.5 * w.dx]
    pts["y"] = 10.5 * w.dx
    v = 0.5 * w.dx / w.dt
    pts["vx"] = [-v, -0.1 * v, v, 0.0]
    with make_pic(w, ) as pic:
        pic.import_points(1, pts)
        pic.move_particles(1)
        assert pic.count(1) == 2
        assert pic.left_exits(1) == 1
        assert pic.left_exits(1) == 0


def test_load_plasma_counts_and_moments():
    import pic_configs as C
    w = small_workload(nx=64, ny=64, ppc=20)
    w.plasma[0].blob_peak_ppc = 50.0
    w.plasma[0].blob_cx = w.plasma[0].blob_cy = 32.0
    w.plasma[0].blob_sigma = 6.0
    with make_pic(w) as pic:
        C.load_plasma(pic, w, seed=3)
        c0, c1 = pic.bin_counts(0), pic.bin_counts(1)
        st = export_state(pic, 1)
    cells1 = c1.reshape(65, 65)[:-1, :-1]
    assert (cells1 == 20).all()
    blob = c0.reshape(65, 65)[:-1, :-1] - 20
    assert blob.min() >= 0 and abs(blob.sum() / (50 * 2 * np.pi * 36) - 1) < 0.05
    sig = np.sqrt(1.602e-19 * 0.026 / w.species[1][1])
    for k in ("vx", "vy", "vz"):
        assert abs(st[k].std() / sig - 1) < 0.02
        assert abs(st[k].mean()) < 0.02 * sig
    assert (st["fx"] >= 0).all() and (st["fx"] < 1).all()


def test_converging_flow_overflow_and_far_jumps(oracle):
    """Movers that find their target cell full (the side list, the fix-up,
    particles carried on the list across steps, re-layout) and jumps of more
    than one cell: after two pushes in a uniform field-free flow the
    particles are those of the FP64 oracle, as a multiset."""
    import pic_b200 as P
    w = small_workload(nx=24, ny=24)
    w.b0 = 0.0
    dx, dy = lib_dx(w)
    pts = []
    rng = np.random.default_rng(9)
    # 50 particles in each of the 8 cells around (12, 12), all moving exactly
    # into the centre cell; the centre cell itself holds 50 stayers
    for sx in (-1, 0, 1):
        for sy in (-1, 0, 1):
            p = np.zeros(50, P.POINT_DTYPE)
            p["x"] = (12 + sx + rng.uniform(0.3, 0.7, 50)) * dx
            p["y"] = (12 + sy + rng.uniform(0.3, 0.7, 50)) * dy
            p["vx"] = -sx * dx / w.dt
            p["vy"] = -sy * dy / w.dt
            pts.append(p)
    # far jumps: 3 cells per step to the right
    far = np.zeros(40, P.POINT_DTYPE)
    far["x"] = (3 + rng.uniform(0.2, 0.8, 40)) * dx
    far["y"] = (5 + rng.uniform(0.2, 0.8, 40)) * dy
    far["vx"] = 3 * dx / w.dt
    pts.append(far)
    pts = np.concatenate(pts)
    pts["vz"] = np.arange(len(pts), dtype=np.float64) + 1.0   # tags
    g = oracle_grid(oracle, w)
    ef = np.zeros((g.nodes, 2))
    bz = np.zeros(g.nodes)
    ref = pts.copy()
    with make_pic(w) as pic:
        pic.import_points(0, pts)
        pic.set_phi(np.zeros(g.nodes))
        pic.update_fields()
        for k in range(2):
            pic.move_particles(0)
            oracle.push(g, ref, w.species[0][0] / w.species[0][1], w.dt, ef, bz)
            if k == 0:   # everything converged on one cell (its slots overflowed)
                assert pic.bin_counts(0).reshape(w.GY, w.GX)[12, 12] == 450
        got = export_state(pic, 0)
        counts = pic.bin_counts(0)
        # the deposit of the state equals a fresh deposit
        pic.zero_rho()
        pic.charge_deposition(0)
        fin = pic.final_mesh(0)
    live = ref[ref["pointer"] != -1]
    assert len(got["cell"]) == len(live) == len(pts)
    tag = got["vz"].astype(np.int64) - 1
    order = np.argsort(tag)
    assert np.array_equal(tag[order], np.arange(len(pts)))
    lv = live[np.argsort((live["vz"] - 1).astype(np.int64))]
    xg = (got["cell"][order] % w.nx + got["fx"][order].astype(np.float64)) * dx
    yg = (got["cell"][order] // w.nx + got["fy"][order].astype(np.float64)) * dy
    assert np.abs(xg - lv["x"]).max() <= 2e-6 * dx and np.abs(yg - lv["y"]).max() <= 2e-6 * dy
    assert np.array_equal(counts, oracle.bucket_counts(g, lv))
    sp, wgt = oracle_species(oracle, w, 0)
    fin_o, _ = oracle.deposit(g, lv, sp, wgt, EPS0)
    assert np.abs(fin - fin_o).max() <= 2e-6 * np.abs(fin_o).max()


@pytest.mark.parametrize("shape,periodic", [(1, False), (2, False), (3, False), (1, True)])
def test_tile_shapes_agree(shape, periodic):
    """Every tile shape of the particle kernels gives the same run as the
    default one: bit-identical charge density, the same particle state as a
    multiset, the same counts -- on a grid that no tile shape divides, with
    the fields of a solve and Bz, over several steps."""
    import pic_b200 as P
    import pic_configs as C
    w = small_workload(nx=300, ny=37, ppc=12)
    w.b0 = 0.01
    if periodic:
        w.rects = C.periodic_rects(w.nx, w.ny, 30.0, -5.0)
    out = []
    for sh in (0, shape):
        with P.Pic(C.library_config(w, periodic_y=periodic)) as pic:
            pic.set_tile_shape(sh)
            C.load_plasma(pic, w, seed=21)
            rho = []
            for it in range(4):
                pic.step(it)
                rho.append(pic.rho())
            out.append((rho, [multiset(export_state(pic, s)) for s in range(2)],
                        [pic.count(s) for s in range(2)], [pic.bin_counts(s) for s in range(2)]))
    (r0, m0, c0, b0), (r1, m1, c1, b1) = out
    assert c0 == c1
    for a, b in zip(r0, r1):
        assert np.array_equal(a, b)
    for s in range(2):
        assert np.array_equal(m0[s], m1[s])
        assert np.array_equal(b0[s], b1[s])


@pytest.mark.parametrize("shape", [1, 2, 3])
def test_fast_particles_every_tile_shape(shape):
    """A beam whose particles jump 2-3 cells a step (longer than the one-cell
    moves the placement is built around), with thermal electrons beside it:
    every tile shape keeps every particle and gives the default shape's
    state and charge density."""
    import pic_b200 as P
    import pic_configs as C
    w = small_workload(nx=96, ny=80, ppc=10)
    rng = np.random.default_rng(8)
    pts = C.host_points(w, 0, seed=8)
    beam = rng.random(len(pts)) < 0.4
    pts["vx"][beam] = rng.uniform(2.0, 3.0, beam.sum()) * w.dx / w.dt * rng.choice([-1, 1], beam.sum())
    pts["vy"][beam] = rng.uniform(-2.5, 2.5, beam.sum()) * w.dx / w.dt
    out = []
    for sh in (0, shape):
        with make_pic(w) as pic:
            pic.set_tile_shape(sh)
            pic.import_points(0, pts)
            rho = []
            for it in range(3):
                pic.zero_rho()
                pic.charge_deposition(0)
                rho.append(pic.rho())
                pic.move_particles(0, it)
            out.append((rho, multiset(export_state(pic, 0)), pic.count(0), pic.left_exits(0)))
    (r0, m0, c0, l0), (r1, m1, c1, l1) = out
    assert c0 == c1 and l0 == l1 and c0 > 0.5 * len(pts)
    for a, b in zip(r0, r1):
        assert np.array_equal(a, b)
    assert np.array_equal(m0, m1)
