"""The synthetic PIC workloads, as concrete library configurations.

cfg1  128x128 cells, dx = 2.5e-4 m, four grounded walls; electrons (Te = 2 eV)
      and Ar+ (Ti = 0.026 eV) at 1e15 m^-3, 16 particles/cell/species;
      Bz = 0.01 T, dt = 5e-11 s, 100 steps.
cfg2  512x512, left wall 100 V, other walls 0 V; 64 particles/cell/species;
      Bz = 0.01 T; 500 steps.
cfg3  1024x1024 with a 64x64-cell electrode at 200 V in the centre, walls
      0 V; 100 particles/cell/species background at 1e15 m^-3 plus a Gaussian
      electron-ion blob (sigma = 40 cells, peak 1e16 m^-3) drifting at 1e5 m/s
      in +x; Bz = 0.02 T; 1000 steps.
cfg4  cfg3 geometry; the learned warm start is trained on steps 0-2000 and
      evaluated on 2000-4000.
cfg5  64 independent instances, square grids 128^2..384^2, left electrode
      50-300 V, Bz 0-0.02 T, 32 particles/cell/species, density 5e14-2e15.

Weights follow updateWeighingFactor (SYCL-PIC-poissonsolver/src/particles.cpp:
303-305) with actual = n0 and sim = background particles/cell x cells, so a
node's final_mesh equals the local density (n0 in uniform plasma) and both
species carry equal weights.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

QE = 1.602e-19
ME = 9.109e-31
M_AR = 6.6335e-26  # 39.948 u
EPS0 = 8.854e-12


@dataclass
class PlasmaSpec:
    ppc: int
    temperature_ev: float
    blob_peak_ppc: float = 0.0
    blob_cx: float = 0.0
    blob_cy: float = 0.0
    blob_sigma: float = 0.0
    drift_vx: float = 0.0
    drift_vy: float = 0.0


@dataclass
class Workload:
    name: str
    nx: int
    ny: int
    dx: float
    dt: float
    b0: float
    steps: int
    n0: float
    ppc: int
    rects: list                     # (x1, y1, x2, y2, volts) node indices
    plasma: list                    # PlasmaSpec per species
    species: list = field(default_factory=list)  # (charge, mass, sim, actual)
    precision: str = "fp32"

    @property
    def GX(self):
        return self.nx + 1

    @property
    def GY(self):
        return self.ny + 1

    @property
    def xmax(self):
        return self.nx * self.dx

    @property
    def ymax(self):
        return self.ny * self.dx


def wall_rects(nx: int, ny: int, left=0.0, right=0.0, top=0.0, bottom=0.0) -> list:
    """The four walls as node rectangles, in geometry.conf's order
    (left, right, top, bottom; SYCL-PIC-poissonsolver/geometry.conf:6-9)."""
    return [(0, 0, 0, ny, left), (nx, 0, nx, ny, right), (0, ny, nx, ny, top), (0, 0, nx, 0, bottom)]


def periodic_rects(nx: int, ny: int, left=0.0, right=0.0, inner=None) -> list:
    """Electrodes of a run periodic in y: the two x walls over the full
    height, plus at most one more rectangle (readGeometry allows three,
    SYCL-PIC-poissonsolver/src/particles.cpp:651-654)."""
    r = [(0, 0, 0, ny, left), (nx, 0, nx, ny, right)]
    if inner is not None:
        r.append(tuple(inner))
    return r


def _species(nx, ny, ppc, n0):
    sim = float(ppc * nx * ny)
    return [(-QE, ME, sim, n0), (QE, M_AR, sim, n0)]


def cfg1() -> Workload:
    nx = ny = 128
    return Workload("cfg1", nx, ny, 2.5e-4, 5e-11, 0.01, 100, 1e15, 16, wall_rects(nx, ny),
                    [PlasmaSpec(16, 2.0), PlasmaSpec(16, 0.026)], _species(nx, ny, 16, 1e15),
                    precision="fp64-oracle")


def cfg2() -> Workload:
    nx = ny = 512
    return Workload("cfg2", nx, ny, 2.5e-4, 5e-11, 0.01, 500, 1e15, 64,
                    wall_rects(nx, ny, left=100.0),
                    [PlasmaSpec(64, 2.0), PlasmaSpec(64, 0.026)], _species(nx, ny, 64, 1e15))


def cfg3(scale: int = 1) -> Workload:
    """scale > 1 shrinks the grid by that factor (same physics per cell) for
    parity tests; scale = 1 is the full 1024^2 workload."""
    nx = ny = 1024 // scale
    c = nx // 2
    h = 32 // scale
    rects = wall_rects(nx, ny) + [(c - h, c - h, c + h, c + h, 200.0)]
    sig = 40.0 / scale
    blob = dict(blob_peak_ppc=1000.0, blob_cx=c, blob_cy=c, blob_sigma=sig, drift_vx=1e5)
    return Workload("cfg3" if scale == 1 else f"cfg3/{scale}", nx, ny, 2.5e-4, 5e-11, 0.02, 1000,
                    1e15, 100, rects,
                    [PlasmaSpec(100, 2.0, **blob), PlasmaSpec(100, 0.026, **blob)],
                    _species(nx, ny, 100, 1e15))


def cfg5_instances(n: int = 64, seed: int = 5) -> list:
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        N = int(rng.integers(128, 385))
        V = float(rng.uniform(50, 300))
        B = float(rng.uniform(0.0, 0.02))
        n0 = float(rng.uniform(5e14, 2e15))
        w = Workload(f"cfg5[{i}]", N, N, 2.5e-4, 5e-11, B, 1000, n0, 32, wall_rects(N, N, left=V),
                     [PlasmaSpec(32, 2.0), PlasmaSpec(32, 0.026)], _species(N, N, 32, n0))
        out.append(w)
    return out


def library_config(w: Workload, **kw):
    """pic_config for a workload (pic_b200.make_config)."""
    import pic_b200 as P
    return P.make_config(w.nx, w.ny, w.xmax, w.ymax, w.dt, w.species, w.rects, b0=w.b0,
                         epsilon=EPS0, **kw)


def load_plasma(pic, w: Workload, seed: int = 1234):
    for s, ps in enumerate(w.plasma):
        pic.load_plasma(s, ps.ppc, ps.temperature_ev, seed + 7919 * s, ps.blob_peak_ppc,
                        ps.blob_cx, ps.blob_cy, ps.blob_sigma, ps.drift_vx, ps.drift_vy)


def host_points(w: Workload, s: int, seed: int, ppc: int | None = None) -> np.ndarray:
    """Seeded reference-layout Points for species s: ppc uniform per cell,
    Maxwellian with per-component sigma = sqrt(e T/m) (the reference's
    v = sqrt(2|q/m|T) with z1 = sqrt(-ln u), src/particles.cpp:142-164)."""
    import pic_b200 as P
    rng = np.random.default_rng(seed)
    ppc = w.plasma[s].ppc if ppc is None else ppc
    ncell = w.nx * w.ny
    n = ncell * ppc
    cells = np.repeat(np.arange(ncell), ppc)
    gx, gy = cells % w.nx, cells // w.nx
    pts = np.zeros(n, P.POINT_DTYPE)
    pts["x"] = (gx + rng.random(n)) * w.dx
    pts["y"] = (gy + rng.random(n)) * w.dx
    m = w.species[s][1]
    sig = np.sqrt(QE * w.plasma[s].temperature_ev / m)
    pts["vx"] = rng.normal(0, sig, n)
    pts["vy"] = rng.normal(0, sig, n)
    pts["vz"] = rng.normal(0, sig, n)
    pts["pointer"] = np.arange(n, dtype=np.int32)
    return pts


WORKLOADS = {"cfg1": cfg1, "cfg2": cfg2, "cfg3": cfg3}
