"""Full-run statistics of the GPU step against the FP64 oracle.

The 128x128 workload (electrons + Ar+, 16 particles per cell and species,
grounded walls, Bz = 0.01 T) runs its 100 steps twice from identical initial
particles: on the GPU (FP32 state, 64-bit fixed-point deposit, MG-PCG to
1e-8) and in the oracle (FP64 restatement of interpolate/mover, SuperLU as
the PARDISO restatement).  Single particles drift apart (FP32 vs FP64 round-
off can be amplified by the plasma's dynamics), so the comparison is of
run statistics:
  * particles lost through the walls: within 0.5 % (plus 5) of the oracle's;
  * time-averaged potential over steps 50-99: max difference within 1e-4 of
    max|<phi>|;
  * time-averaged electron density, averaged over y: within 1e-4 of its
    maximum at every x;
  * relative kinetic-energy change over the run: within 1e-4 of the oracle's;
  * relative total-energy change (kinetic + 1/2 sum rho phi dA, the field
    energy on the node grid) over the run: within 1e-4 of the oracle's.
Measured on a B200: identical lost counts, 2e-7 (potential), 2e-8
(density), 1e-8 (energy change): over this run the FP32 state follows the
FP64 trajectories closely.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

EPS0 = 8.854e-12


def test_cfg1_run_statistics(oracle):
    import pic_b200 as P
    import pic_configs as C
    O = oracle
    w = C.cfg1()
    steps = w.steps
    pts = [C.host_points(w, s, seed=100 + s) for s in range(2)]
    dx = w.xmax / w.nx
    GX, GY = w.GX, w.GY
    g = O.Grid(w.nx, w.ny, dx, dx)
    sps = [O.Species(str(s), *w.species[s]) for s in range(2)]
    wgt = [O.weighing_factor(sp, w.xmax * w.ymax, dx, dx) for sp in sps]
    ctom = [w.species[s][0] / w.species[s][1] for s in range(2)]
    D = O.DirectPoisson(GX, GY, dx, dx, O.Electrodes(w.rects))
    bz = np.full(g.nodes, w.b0)
    ref = [p.copy() for p in pts]
    ke0 = [O.kinetic_energy(pts[s], ctom[s]) for s in range(2)]
    acc = dict(phi_g=0.0, phi_o=0.0, ne_g=0.0, ne_o=0.0)
    n_avg = 0
    import test_gpu_config_parity as CP
    tot_g, tot_o = [], []
    with P.Pic(C.library_config(w)) as pic:
        for s in range(2):
            pic.import_points(s, pts[s])
        for it in range(steps):
            cur = [pic.export_points(s) for s in range(2)] if it in (0, steps - 1) else None
            pic.step(it)
            rho = np.zeros(g.nodes)
            fin_o = [O.deposit(g, ref[s], sps[s], wgt[s], EPS0, rho)[0] for s in range(2)]
            phi_o, ef_o = D.step(rho)
            if cur is not None:
                # state, density and potential of the same step on both sides
                tot_g.append(sum(CP._energy(w, cur, [pic.final_mesh(s) for s in range(2)], pic.phi())))
                tot_o.append(sum(CP._energy(w, ref, fin_o, phi_o)))
            for s in range(2):
                O.push(g, ref[s], ctom[s], w.dt, ef_o, bz)
            if it >= steps // 2:
                acc["phi_g"] = acc["phi_g"] + pic.phi()
                acc["phi_o"] = acc["phi_o"] + phi_o
                acc["ne_g"] = acc["ne_g"] + pic.final_mesh(0)
                acc["ne_o"] = acc["ne_o"] + fin_o[0]
                n_avg += 1
        n_g = [pic.count(s) for s in range(2)]
        out = [pic.export_points(s) for s in range(2)]
    n0 = [len(p) for p in pts]
    n_o = [int((ref[s]["pointer"] != -1).sum()) for s in range(2)]
    lost_g = [n0[s] - n_g[s] for s in range(2)]
    lost_o = [n0[s] - n_o[s] for s in range(2)]
    ke_g = [O.kinetic_energy(out[s], ctom[s]) for s in range(2)]
    ke_o = [O.kinetic_energy(ref[s], ctom[s]) for s in range(2)]
    phi_g, phi_o = acc["phi_g"] / n_avg, acc["phi_o"] / n_avg
    ne_g = (acc["ne_g"] / n_avg).reshape(GY, GX).mean(axis=0)
    ne_o = (acc["ne_o"] / n_avg).reshape(GY, GX).mean(axis=0)
    dphi = np.abs(phi_g - phi_o).max() / np.abs(phi_o).max()
    dne = np.abs(ne_g - ne_o).max() / np.abs(ne_o).max()
    dke = [abs((ke_g[s] - ke0[s]) / ke0[s] - (ke_o[s] - ke0[s]) / ke0[s]) for s in range(2)]
    print(f"lost gpu {lost_g} oracle {lost_o}; <phi> {dphi:.3e}; <n_e>(x) {dne:.3e}; "
          f"KE change gpu {[(ke_g[s] - ke0[s]) / ke0[s] for s in range(2)]} "
          f"oracle {[(ke_o[s] - ke0[s]) / ke0[s] for s in range(2)]}")
    for s in range(2):
        assert abs(lost_g[s] - lost_o[s]) <= 0.005 * lost_o[s] + 5, (lost_g, lost_o)
    assert dphi <= 1e-4
    assert dne <= 1e-4
    assert max(dke) <= 1e-4
    dtot_g = (tot_g[1] - tot_g[0]) / tot_g[0]
    dtot_o = (tot_o[1] - tot_o[0]) / tot_o[0]
    print(f"total energy change gpu {dtot_g:.6e} oracle {dtot_o:.6e}")
    assert abs(tot_g[0] - tot_o[0]) <= 1e-5 * abs(tot_o[0])
    assert abs(dtot_g - dtot_o) <= 1e-4
