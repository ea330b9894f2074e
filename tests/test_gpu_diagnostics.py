"""The reference's text snapshots written by the library, read back.

pic_write_diagnostics / sycl_pic_print_diagnostics write what
printNumberDensity, printEnergy, printElectricField and printPhi
(SYCL-PIC-poissonsolver/src/utils.cpp:829-991) write: for each quantity a
file dir/<quantity>/<iteration> of GRID_Y lines, each GRID_X "%lf" values
separated by single spaces.  Checks:
  * the layout: line and value counts, single spaces, no trailing space, a
    newline after every line, six decimals;
  * the text equals C's "%lf" of the library's own grids exactly (Python's
    "%f" rounds the same, correctly);
  * the values against the FP64 oracle: densities (final_mesh times the
    scale factor) within 2e-6 of their maximum, the energy columns
    0.66667 E/(n+1) (with the reference's last electron column divided by
    E+1) within 1e-5, the potential against a direct solve of the same
    charge density within 1e-5 of max|phi|, Ex/Ey against the oracle's
    central differences of the written potential within 1e-9 relative;
    plus the rounding of "%lf" (5e-7);
  * a folder that cannot be created gives PIC_ERR_IO and no partial success.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

EPS0 = 8.854e-12


def _read(path, GX, GY):
    text = open(path).read()
    lines = text.split("\n")
    assert lines[-1] == "" and len(lines) == GY + 1, path
    rows = []
    for ln in lines[:-1]:
        tok = ln.split(" ")
        assert len(tok) == GX and all(t and "." in t and len(t.split(".")[1]) == 6 for t in tok), path
        rows.append([float(t) for t in tok])
    return text, np.array(rows).ravel()


def _fmt(v, GX, GY):
    v = v.reshape(GY, GX)
    return "".join(" ".join("%f" % x for x in row) + "\n" for row in v)


def test_diagnostic_files_against_oracle(oracle, tmp_path):
    import pic_b200 as P
    import pic_configs as C
    import test_gpu_particles as T
    O = oracle
    w = T.small_workload(nx=40, ny=30, ppc=12, rects=C.wall_rects(40, 30, left=30.0))
    GX, GY = w.GX, w.GY
    dx, dy = T.lib_dx(w)
    g = O.Grid(w.nx, w.ny, dx, dy)
    pts = [C.host_points(w, s, seed=40 + s) for s in range(2)]
    sf = 1e-15
    with T.make_pic(w) as pic:
        for s in range(2):
            pic.import_points(s, pts[s])
        pic.zero_rho()
        for s in range(2):
            pic.charge_deposition(s)
        rho = pic.rho()
        pic.poisson_solve(0)
        pic.write_diagnostics(str(tmp_path / "out"), 7, sf)
        fin = [pic.final_mesh(s) for s in range(2)]
        en = [pic.energy_mesh(s) for s in range(2)]
        phi = pic.phi()
        ef = pic.efield()
        bad = tmp_path / "a_file"
        bad.write_text("x")
        with pytest.raises(P.PicError) as e:
            pic.write_diagnostics(str(bad / "out"), 7, sf)
        assert e.value.status == -7
    files = {q: _read(tmp_path / "out" / q / "7", GX, GY)
             for q in ("electronDensity", "ionDensity", "electronenergy", "ionenergy", "Ex", "Ey",
                       "potential")}
    # the exact text of the library's own grids
    te = 0.66667 * en[0] / (fin[0] + 1.0)
    last = np.arange(GX * GY) % GX == GX - 1
    te[last] = (0.66667 * en[0] / (en[0] + 1.0))[last]
    ti = 0.66667 * en[1] / (fin[1] + 1.0)
    own = {"electronDensity": fin[0] * sf, "ionDensity": fin[1] * sf, "electronenergy": te,
           "ionenergy": ti, "Ex": ef[:, 0], "Ey": ef[:, 1], "potential": phi}
    for q, v in own.items():
        assert files[q][0] == _fmt(v, GX, GY), q
    # against the oracle
    rho_o = np.zeros(g.nodes)
    dep = []
    for s in range(2):
        sp, wgt = T.oracle_species(O, w, s)
        dep.append(O.deposit(g, pts[s], sp, wgt, EPS0, rho_o))
    for s, q in enumerate(("electronDensity", "ionDensity")):
        ref = dep[s][0] * sf
        assert np.abs(files[q][1] - ref).max() <= 2e-6 * np.abs(ref).max() + 5e-7, q
    te_o = 0.66667 * dep[0][1] / (dep[0][0] + 1.0)
    te_o[last] = (0.66667 * dep[0][1] / (dep[0][1] + 1.0))[last]
    ti_o = 0.66667 * dep[1][1] / (dep[1][0] + 1.0)
    for q, ref in (("electronenergy", te_o), ("ionenergy", ti_o)):
        assert np.abs(files[q][1] - ref).max() <= 1e-5 * np.abs(ref).max() + 5e-7, q
    D = O.DirectPoisson(GX, GY, dx, dy, O.Electrodes(w.rects))
    phi_o, _ = D.step(rho.copy())
    assert np.abs(files["potential"][1] - phi_o).max() <= 1e-5 * np.abs(phi_o).max() + 5e-7
    ef_o = O.efield(GX, GY, dx, dy, phi)
    for k, q in enumerate(("Ex", "Ey")):
        assert np.abs(files[q][1] - ef_o[:, k]).max() <= 1e-9 * np.abs(ef_o).max() + 5e-7, q
