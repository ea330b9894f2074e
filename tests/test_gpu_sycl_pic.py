"""The reference's Python driver loop (SYCL-PIC-poissonsolver/src/main.py:
43-141) through the `sycl_pic`-compatible module on the GPU library.

Checks: the rho/phi arrays are zero-copy views that the operators refresh in
place; operators return elapsed seconds; after poisson_solve the (in place
overwritten) right-hand side and phi satisfy the reduced system to 1e-8
relative residual, measured by the FP64 oracle; writes through get_phi()
reach the E field via update_fields_from_phi(); the diagnostics writers
create their files and raise on a folder they cannot create; particle
counts never grow.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_reference_driver_loop(oracle, tmp_path, monkeypatch):
    import sycl_pic as sp
    from test_capi_cpu import _write_inputs
    _write_inputs(tmp_path, nx=64, ny=32, xmax=0.016, ymax=0.008, steps=4, pint=2)
    monkeypatch.chdir(tmp_path)
    sp.init("gpu", 256, 24, "e.inp", "i.inp")
    try:
        GX, GY = sp.get_grid_x(), sp.get_grid_y()
        assert (GX, GY) == (65, 33) and sp.get_grid_size() == GX * GY
        assert sp.get_num_species() == 2 and sp.get_timesteps() == 4
        rho, phi = sp.get_rho(), sp.get_phi()
        ne0, ni0 = sp.get_particle_counts()
        assert ne0 > 0 and ni0 > 0
        mask = None
        for it in range(sp.get_timesteps()):
            sp.zero_rho()
            assert not rho.any()
            t = sum(sp.charge_deposition(s) for s in range(sp.get_num_species()))
            assert t >= 0 and rho.any()          # the same array was filled in place
            assert sp.poisson_solve(it) >= 0
            if mask is None:
                g = oracle.Electrodes.from_fractions(GX, GY, [(0, 0, 0, 1, 100.0), (1, 0, 1, 1, 0.0),
                                                              (0, 1, 1, 1, 0.0), (0, 0, 1, 0, 0.0),
                                                              (0.46875, 0.46875, 0.53125, 0.53125, 200.0)])
                mask = oracle.electrode_mask(GX, GY, g)
            dx, dy = 0.016 / 64, 0.008 / 32
            assert oracle.reduced_relres(GX, GY, dx, dy, mask, rho.copy(), phi.copy()) <= 1e-8
            for s in range(sp.get_num_species()):
                assert sp.move_particles(s, it) >= 0
                el, at, st = sp.compact_particles(s)
                assert el >= 0 and sp.cleanup_map(s) >= 0
            if it % sp.get_print_interval() == 0:
                sp.print_diagnostics(str(tmp_path / "out"), it)
        ne, ni = sp.get_particle_counts()
        assert ne <= ne0 and ni <= ni0
        # a phi written from Python reaches the device through update_fields_from_phi
        phi[:] = 0.0
        sp.update_fields_from_phi()
        # overwritePhi: a left-wall node mid-height (corners belong to the
        # bottom/top walls, applied later in geometry.conf's order)
        assert phi[(GY // 2) * GX] == 100.0 and phi[(GY // 2) * GX + 1] == 0.0
        sp.dump_rho_phi_cpp(str(tmp_path / "dump"))
        assert np.array_equal(np.fromfile(tmp_path / "dump_phi_cpp.bin"), phi)
        sp.save_meshes()
        assert any(f.startswith("Mesh") for f in os.listdir(tmp_path))
        assert os.path.isdir(tmp_path / "out")
        # where the reference prints and exits, the module raises
        (tmp_path / "a_file").write_text("x")
        with pytest.raises(RuntimeError):
            sp.print_diagnostics(str(tmp_path / "a_file" / "out"), 0)
        ne1, ni1 = sp.get_particle_counts()
        assert sp.generate_new_particles() >= 0     # band inside the 16 mm domain
        ne2, ni2 = sp.get_particle_counts()
        assert ne2 > ne1 and ni2 > ni1 and ne2 - ne1 >= ni2 - ni1
    finally:
        sp.finalize()


def test_reference_driver_loop_periodic(oracle, tmp_path, monkeypatch):
    """The same loop on input files with periodicBoundary = 1 and three
    electrodes (the x walls and a central block): the solve is the periodic
    system, the last node row repeats row 0, and update_fields_from_phi
    applies the periodic overwritePhi."""
    import sycl_pic as sp
    from test_capi_cpu import GEOMETRY, _write_inputs
    _write_inputs(tmp_path, nx=64, ny=32, xmax=0.016, ymax=0.008, steps=3, pint=10, periodic=1)
    rows = GEOMETRY.splitlines()
    keep = [r for r in rows if not (r.strip().startswith("0.     1.") or r.strip().startswith("0.     0.      1."))]
    geo = "\n".join(keep).replace("  5\n", "  3\n")
    (tmp_path / "geometry.conf").write_text(geo)
    monkeypatch.chdir(tmp_path)
    sp.init("gpu", 256, 24, "e.inp", "i.inp")
    try:
        GX, GY = sp.get_grid_x(), sp.get_grid_y()
        rho, phi = sp.get_rho(), sp.get_phi()
        g = oracle.Electrodes.from_fractions(GX, GY, [(0, 0, 0, 1, 100.0), (1, 0, 1, 1, 0.0),
                                                      (0.46875, 0.46875, 0.53125, 0.53125, 200.0)])
        mask = oracle.electrode_mask(GX, GY, g)
        dx, dy = 0.016 / 64, 0.008 / 32
        for it in range(sp.get_timesteps()):
            sp.zero_rho()
            for s in range(sp.get_num_species()):
                sp.charge_deposition(s)
            assert sp.poisson_solve(it) >= 0
            assert oracle.reduced_relres(GX, GY, dx, dy, mask, rho.copy(), phi.copy(),
                                         periodic=True) <= 1e-8
            p = phi.reshape(GY, GX)
            assert np.array_equal(p[-1], p[0])
            for s in range(sp.get_num_species()):
                assert sp.move_particles(s, it) >= 0
        ne, ni = sp.get_particle_counts()
        assert ne > 0 and ni > 0
        phi[:] = np.arange(GX * GY, dtype=np.float64)
        sp.update_fields_from_phi()
        p = phi.reshape(GY, GX)
        # row 0 copied into the last row, then the electrodes
        assert p[-1, 5] == 5.0 and p[-1, 0] == 100.0 and p[0, 0] == 100.0
    finally:
        sp.finalize()
