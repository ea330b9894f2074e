"""FP64 CPU oracle for the 2D electrostatic PIC step of SYCL-PIC-poissonsolver.

TEST INFRASTRUCTURE ONLY.  ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` use this module as the checker.  The CUDA
library never imports it and has no path that routes through it.

The arithmetic lives in ``pic_oracle.c`` (built by the Makefile beside it).
This module adds the pieces that are easiest in NumPy/SciPy:

* the reference ``Point`` record as a NumPy structured dtype
  (SYCL-PIC-poissonsolver/include/point.hpp:11-14),
* the PARDISO restatement: the ``generateCoeffs`` CSR matrix
  (src/poissonSolver.cpp:183-241) solved by SciPy SuperLU, factored once and
  re-solved each step like PARDISO phases 11/22 then 33
  (src/poissonSolver.cpp:505-535),
* ``poisson_step``: overwriteRho -> solve -> overwritePhi -> E field
  (src/poissonSolver.cpp:459-544).

The Poisson part is pinned against the reference's own PARDISO dumps
(tests/golden/poisson_257_*.npz).  Binning, deposit and push are pinned
against the reference's own kernel bodies compiled here into a host harness
(oracle/ref_build.py, loaded by ``ref_lib``; tests/test_oracle_ref_pin.py:
bit for bit).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libpic_oracle.so")

POINT_DTYPE = np.dtype(
    [("x", "<f8"), ("y", "<f8"), ("z", "<f8"), ("vx", "<f8"), ("vy", "<f8"),
     ("vz", "<f8"), ("pointer", "<i4"), ("pad", "<i4")], align=True)
assert POINT_DTYPE.itemsize == 56

# Physical constants used by the synthetic configs.
QE = 1.602e-19
ME = 9.109e-31
M_AR = 6.6335e-26
EPS0 = 8.854e-12


class Grid(ctypes.Structure):
    """GridParams subset (include/species_ds.hpp:6-10).  width/height are
    GRID_WIDTH/GRID_HEIGHT (XMAX/YMAX as read from M_PICDAT.DAT), the bounds
    of the mover's wall test; left 0 they are nx*dx / ny*dy."""
    _fields_ = [("nx", ctypes.c_int32), ("ny", ctypes.c_int32),
                ("dx", ctypes.c_double), ("dy", ctypes.c_double),
                ("width", ctypes.c_double), ("height", ctypes.c_double)]

    @property
    def GX(self):
        return self.nx + 1

    @property
    def GY(self):
        return self.ny + 1

    @property
    def nodes(self):
        return (self.nx + 1) * (self.ny + 1)


class Geom(ctypes.Structure):
    """Geometry (include/point.hpp:21-24): inclusive node rectangle + volts."""
    _fields_ = [("x1", ctypes.c_int32), ("y1", ctypes.c_int32), ("x2", ctypes.c_int32),
                ("y2", ctypes.c_int32), ("potential", ctypes.c_double)]


_lib = None


def build() -> str:
    """Compile pic_oracle.c with the Makefile beside it; returns the .so path."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH) or (
                os.path.getmtime(_LIB_PATH) < os.path.getmtime(os.path.join(_HERE, "pic_oracle.c"))):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        P = ctypes.POINTER
        vp = ctypes.c_void_p
        i64, i32, dbl = ctypes.c_int64, ctypes.c_int32, ctypes.c_double
        sig = {
            "orc_sizeof_point": (ctypes.c_int, []),
            "orc_num_threads": (ctypes.c_int, []),
            "orc_set_threads": (None, [ctypes.c_int]),
            "orc_bucket_keys": (None, [P(Grid), vp, i64, vp]),
            "orc_bucket_sort": (i64, [vp, i64, i32, vp, vp, vp]),
            "orc_deposit": (None, [P(Grid), vp, i64, dbl, dbl, dbl, dbl, vp, vp, vp]),
            "orc_push": (i64, [P(Grid), vp, i64, dbl, dbl, vp, vp, P(i64)]),
            "orc_push_mode": (i64, [P(Grid), vp, i64, dbl, dbl, vp, vp, i32, P(i64)]),
            "orc_kinetic_energy": (dbl, [vp, i64, dbl]),
            "orc_geom_from_fractions": (None, [i32, i32, vp, i32, vp]),
            "orc_electrode_mask": (None, [i32, i32, vp, i32, vp]),
            "orc_build_csr": (i64, [i32, i32, dbl, dbl, vp, vp, vp, vp]),
            "orc_build_csr_periodic": (i64, [i32, i32, dbl, dbl, vp, vp, vp, vp]),
            "orc_overwrite_rho": (None, [i32, i32, vp, i32, vp]),
            "orc_overwrite_phi": (None, [i32, i32, vp, i32, vp]),
            "orc_overwrite_phi_periodic": (None, [i32, i32, vp, i32, vp]),
            "orc_efield": (None, [i32, i32, dbl, dbl, vp, vp]),
            "orc_efield_periodic": (None, [i32, i32, dbl, dbl, vp, vp]),
            "orc_apply_a": (None, [i32, i32, dbl, dbl, vp, vp, vp]),
            "orc_cg_solve": (ctypes.c_int, [i32, i32, dbl, dbl, vp, vp, vp, dbl, ctypes.c_int, P(dbl)]),
            "orc_hm_create": (vp, [i32, i32, dbl]),
            "orc_hm_destroy": (None, [vp]),
            "orc_ref_register": (i64, [vp, P(Grid), vp, i64]),
            "orc_hm_counts": (None, [vp, vp]),
            "orc_hm_members": (i32, [vp, i32, vp, i32]),
            "orc_ref_deposit": (None, [vp, P(Grid), vp, dbl, dbl, dbl, dbl, vp, vp, vp]),
            "orc_ref_mover": (i64, [vp, P(Grid), vp, i64, dbl, dbl, vp, vp, vp, P(i64), P(i64)]),
            "orc_ref_cleanup": (None, [vp, vp]),
            "orc_ref_compact": (i64, [vp, vp, i64, vp, i64]),
            "orc_plasma_counts": (i64, [i32, i32, i32, dbl, dbl, dbl, dbl, ctypes.c_uint64, vp]),
            "orc_plasma_fill": (None, [i32, i32, dbl, dbl, i32, dbl, dbl, dbl, ctypes.c_uint64, vp,
                                       vp, i64, vp]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        assert L.orc_sizeof_point() == 56
        _lib = L
    return _lib


def _ptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


def num_threads() -> int:
    return int(lib().orc_num_threads())


# ---------------------------------------------------------------------------
# Species / geometry description (mirrors readPICDAT's per-species table)
# ---------------------------------------------------------------------------

@dataclass
class Species:
    """One species row of M_PICDAT.DAT (src/particles.cpp:590-608)."""
    name: str
    charge: float
    mass: float
    sim: float          # simulation particle count used for the weight
    actual: float       # real particle count ("actual" column)

    @property
    def ctom(self) -> float:
        return self.charge / self.mass          # initCtoM, src/particles.cpp:298-300


def weighing_factor(sp: Species, surf_area: float, dx: float, dy: float) -> float:
    """updateWeighingFactor, src/particles.cpp:303-305."""
    return sp.actual * surf_area / (sp.sim * dx * dy * dx * dy)


@dataclass
class Electrodes:
    """Electrode rectangles as inclusive node ranges (readGeometry output)."""
    rects: list = field(default_factory=list)   # (x1, y1, x2, y2, volts) node indices

    @staticmethod
    def from_fractions(GX: int, GY: int, fracs) -> "Electrodes":
        """readGeometry, src/particles.cpp:677-681: (int)((GRID-1)*fraction)."""
        out = []
        for (fx1, fy1, fx2, fy2, v) in fracs:
            out.append((int((GX - 1) * fx1), int((GY - 1) * fy1),
                        int((GX - 1) * fx2), int((GY - 1) * fy2), float(v)))
        return Electrodes(out)

    def c_array(self):
        arr = (Geom * max(1, len(self.rects)))()
        for i, (x1, y1, x2, y2, v) in enumerate(self.rects):
            arr[i] = Geom(x1, y1, x2, y2, v)
        return arr


def walls(GX: int, GY: int, left=0.0, right=0.0, top=0.0, bottom=0.0) -> list:
    """The four domain walls in geometry.conf's fraction form
    (SYCL-PIC-poissonsolver/geometry.conf:6-9 order: left, right, top, bottom)."""
    return [(0.0, 0.0, 0.0, 1.0, left), (1.0, 0.0, 1.0, 1.0, right),
            (0.0, 1.0, 1.0, 1.0, top), (0.0, 0.0, 1.0, 0.0, bottom)]


# ---------------------------------------------------------------------------
# Particle-side wrappers
# ---------------------------------------------------------------------------

def bucket_keys(g: Grid, pts: np.ndarray) -> np.ndarray:
    keys = np.empty(len(pts), np.int32)
    lib().orc_bucket_keys(ctypes.byref(g), _ptr(pts), len(pts), _ptr(keys))
    return keys


def bucket_counts(g: Grid, pts: np.ndarray) -> np.ndarray:
    """Per node-key live-particle counts (the hashmap's key_idx semantics)."""
    keys = bucket_keys(g, pts)
    live = keys >= 0
    return np.bincount(keys[live], minlength=g.nodes).astype(np.int64)


def deposit(g: Grid, pts: np.ndarray, sp: Species, weighing: float, eps: float,
            rho: np.ndarray | None = None):
    """interpolate(): returns (final_mesh, energy_mesh); adds into rho if given."""
    final = np.zeros(g.nodes)
    energy = np.zeros(g.nodes)
    lib().orc_deposit(ctypes.byref(g), _ptr(pts), len(pts), weighing, sp.ctom, sp.charge,
                      eps, _ptr(final), _ptr(energy), _ptr(rho))
    return final, energy


def push(g: Grid, pts: np.ndarray, ctom: float, dt: float, efield: np.ndarray,
         bz: np.ndarray, periodic: bool = False):
    """MoverKernel semantics, in place (periodic: y wrapped by modulo(y, H)
    first).  Returns (deleted, left_exits)."""
    left = ctypes.c_int64(0)
    assert efield.shape == (g.nodes, 2) and efield.dtype == np.float64
    deleted = lib().orc_push_mode(ctypes.byref(g), _ptr(pts), len(pts), ctom, dt,
                                  _ptr(np.ascontiguousarray(efield)), _ptr(bz),
                                  1 if periodic else 0, ctypes.byref(left))
    return int(deleted), int(left.value)


def kinetic_energy(pts: np.ndarray, ctom: float) -> float:
    return float(lib().orc_kinetic_energy(_ptr(pts), len(pts), ctom))


# ---------------------------------------------------------------------------
# Poisson
# ---------------------------------------------------------------------------

def electrode_mask(GX: int, GY: int, el: Electrodes) -> np.ndarray:
    mask = np.zeros(GX * GY, np.uint8)
    arr = el.c_array()
    lib().orc_electrode_mask(GX, GY, ctypes.cast(arr, ctypes.c_void_p), len(el.rects), _ptr(mask))
    return mask


def build_csr(GX: int, GY: int, dx: float, dy: float, mask: np.ndarray):
    """generateCoeffs as a SciPy CSR matrix (0-based)."""
    import scipy.sparse as sps
    n = GX * GY
    row_ptr = np.zeros(n + 1, np.int64)
    col = np.zeros(5 * n, np.int64)
    val = np.zeros(5 * n)
    nnz = lib().orc_build_csr(GX, GY, dx, dy, _ptr(mask), _ptr(row_ptr), _ptr(col), _ptr(val))
    return sps.csr_matrix((val[:nnz], col[:nnz], row_ptr), shape=(n, n))


def overwrite_rho(GX: int, GY: int, el: Electrodes, rho: np.ndarray) -> None:
    arr = el.c_array()
    lib().orc_overwrite_rho(GX, GY, ctypes.cast(arr, ctypes.c_void_p), len(el.rects), _ptr(rho))


def build_csr_periodic(GX: int, GY: int, dx: float, dy: float, mask: np.ndarray):
    """generateCoeffsPeriodic as a SciPy CSR matrix over GX*(GY-1) nodes."""
    import scipy.sparse as sps
    n = GX * (GY - 1)
    row_ptr = np.zeros(n + 1, np.int64)
    col = np.zeros(5 * n, np.int64)
    val = np.zeros(5 * n)
    nnz = lib().orc_build_csr_periodic(GX, GY, dx, dy, _ptr(mask), _ptr(row_ptr), _ptr(col),
                                       _ptr(val))
    if nnz < 0:
        raise ValueError("periodic system: the first and last node columns must be electrodes")
    return sps.csr_matrix((val[:nnz], col[:nnz], row_ptr), shape=(n, n))


def overwrite_phi(GX: int, GY: int, el: Electrodes, phi: np.ndarray,
                  periodic: bool = False) -> None:
    arr = el.c_array()
    fn = lib().orc_overwrite_phi_periodic if periodic else lib().orc_overwrite_phi
    fn(GX, GY, ctypes.cast(arr, ctypes.c_void_p), len(el.rects), _ptr(phi))


def efield(GX: int, GY: int, dx: float, dy: float, phi: np.ndarray,
           periodic: bool = False) -> np.ndarray:
    ef = np.zeros((GX * GY, 2))
    fn = lib().orc_efield_periodic if periodic else lib().orc_efield
    fn(GX, GY, dx, dy, _ptr(phi), _ptr(ef))
    return ef


def apply_a(GX, GY, dx, dy, mask, x):
    y = np.empty_like(x)
    lib().orc_apply_a(GX, GY, dx, dy, _ptr(mask), _ptr(x), _ptr(y))
    return y


def reduced_relres(GX, GY, dx, dy, mask, b, phi, periodic: bool = False) -> float:
    """||b_int - A_int phi|| / ||b_int|| over the non-electrode rows, where
    b_int carries the known electrode neighbours across (the measure used for
    the 1e-8 target).  periodic: the system of rows 0..GY-2."""
    if periodic:
        n = GX * (GY - 1)
        A = build_csr_periodic(GX, GY, dx, dy, mask)
        m, bb, ph = mask[:n] == 1, b[:n], phi[:n]
        r = (bb - A @ ph)[~m]
        bi = (bb - A[:, np.flatnonzero(m)] @ ph[m])[~m]
        nb = np.linalg.norm(bi)
        return float(np.linalg.norm(r) / (nb if nb > 0 else 1.0))
    r = b - apply_a(GX, GY, dx, dy, mask, phi)
    inner = mask == 0
    cx, cy = 1.0 / dx ** 2, 1.0 / dy ** 2
    pe = np.where(mask == 1, phi, 0.0)
    bi = b.copy()
    bi[1:] += cx * pe[:-1]
    bi[:-1] += cx * pe[1:]
    bi[GX:] += cy * pe[:-GX]
    bi[:-GX] += cy * pe[GX:]
    nb = np.linalg.norm(bi[inner])
    return float(np.linalg.norm(r[inner]) / (nb if nb > 0 else 1.0))


def cg_solve(GX, GY, dx, dy, mask, b, phi0=None, tol=1e-13, maxit=100000):
    phi = np.zeros(GX * GY) if phi0 is None else phi0.copy()
    rel = ctypes.c_double(0)
    it = lib().orc_cg_solve(GX, GY, dx, dy, _ptr(mask), _ptr(b), _ptr(phi), tol, maxit,
                            ctypes.byref(rel))
    return phi, int(it), float(rel.value)


class DirectPoisson:
    """PARDISO restatement: SuperLU on the generateCoeffs matrix, factored once
    (phases 11+22) and re-solved every step (phase 33).  Single-threaded."""

    def __init__(self, GX: int, GY: int, dx: float, dy: float, el: Electrodes,
                 periodic: bool = False):
        import scipy.sparse.linalg as spla
        self.GX, self.GY, self.dx, self.dy, self.el = GX, GY, dx, dy, el
        self.periodic = periodic
        self.mask = electrode_mask(GX, GY, el)
        self.A = (build_csr_periodic if periodic else build_csr)(GX, GY, dx, dy, self.mask)
        self.n = self.A.shape[0]
        self.lu = spla.splu(self.A.tocsc())

    def solve_rhs(self, b: np.ndarray) -> np.ndarray:
        """LU solve plus two steps of iterative refinement.  PARDISO (mtype
        11 defaults: scaling and weighted matching) reaches round-off on this
        system; SuperLU on the unscaled matrix (electrode rows of order 1,
        stencil rows of order 1/dx^2) can stop near 1e-8 relative without
        the refinement."""
        x = self.lu.solve(b)
        for _ in range(2):
            x += self.lu.solve(b - self.A @ x)
        return x

    def step(self, rho: np.ndarray):
        """poissonSolver(): rho is overwritten in place (becomes the RHS);
        returns (phi, efield).  Periodic: PARDISO sees the first GX*(GY-1)
        entries of rho and writes those of phi; overwritePhi fills row GY-1."""
        overwrite_rho(self.GX, self.GY, self.el, rho)
        phi = np.zeros(self.GX * self.GY)
        phi[:self.n] = self.solve_rhs(rho[:self.n])
        overwrite_phi(self.GX, self.GY, self.el, phi, self.periodic)
        ef = efield(self.GX, self.GY, self.dx, self.dy, phi, self.periodic)
        return phi, ef


# ---------------------------------------------------------------------------
# Reference-structure port (hashmap) used as the timed CPU path
# ---------------------------------------------------------------------------

class RefHashmapSpecies:
    """One species held the reference's way: a Point AoS plus the per-node
    hashmap (include/sycl_hashmap.hpp), capacity nodes*probing*1.2."""

    def __init__(self, g: Grid, pts: np.ndarray, probing_length: int):
        self.g = g
        self.pts = pts
        self.end = len(pts)
        self.m = lib().orc_hm_create(g.nodes, probing_length, 1.2)
        self.empty = np.full(len(pts), -1, np.int32)
        self.n_empty = 0
        self.new_additions = 0
        failed = lib().orc_ref_register(self.m, ctypes.byref(g), _ptr(pts), len(pts))
        if failed:
            raise RuntimeError(f"hashmap overflow on register: {failed} particles")

    def __del__(self):
        try:
            lib().orc_hm_destroy(self.m)
        except Exception:
            pass

    def counts(self) -> np.ndarray:
        c = np.zeros(self.g.nodes, np.int32)
        lib().orc_hm_counts(self.m, _ptr(c))
        return c

    def deposit(self, sp: Species, weighing, eps, rho=None):
        final = np.zeros(self.g.nodes)
        energy = np.zeros(self.g.nodes)
        lib().orc_ref_deposit(self.m, ctypes.byref(self.g), _ptr(self.pts), weighing, sp.ctom,
                              sp.charge, eps, _ptr(final), _ptr(energy), _ptr(rho))
        return final, energy

    def move(self, ctom, dt, efield_arr, bz):
        ne = ctypes.c_int64(self.n_empty)
        na = ctypes.c_int64(self.new_additions)
        failed = lib().orc_ref_mover(self.m, ctypes.byref(self.g), _ptr(self.pts), self.end, ctom,
                                     dt, _ptr(efield_arr), _ptr(bz), _ptr(self.empty),
                                     ctypes.byref(ne), ctypes.byref(na))
        self.n_empty = int(ne.value)
        self.new_additions = int(na.value)
        if failed:
            raise RuntimeError(f"hashmap overflow in mover: {failed} particles")

    def compact(self):
        self.end = int(lib().orc_ref_compact(self.m, _ptr(self.pts), self.end, _ptr(self.empty),
                                             self.n_empty))
        self.n_empty = 0

    def cleanup(self):
        lib().orc_ref_cleanup(self.m, _ptr(self.pts))


# ---------------------------------------------------------------------------
# The reference's own particle code, compiled here (oracle/ref_build.py)
# ---------------------------------------------------------------------------

class RefGridParams(ctypes.Structure):
    """GridParams as the reference declares it (include/species_ds.hpp:6-10)."""
    _fields_ = [("NX", ctypes.c_int), ("NY", ctypes.c_int), ("GRID_X", ctypes.c_int),
                ("GRID_Y", ctypes.c_int), ("dx", ctypes.c_double), ("dy", ctypes.c_double),
                ("GRID_WIDTH", ctypes.c_double), ("GRID_HEIGHT", ctypes.c_double)]


_ref_lib = None
REF_LIB_PATH = os.path.join(_HERE, "_ref", "libref_pic.so")


def ref_lib():
    """oracle/_ref/libref_pic.so (the reference's kernel bodies in a host
    harness), built from a reference checkout when absent; None when it is
    absent and no checkout is available."""
    global _ref_lib
    if _ref_lib is None:
        if not os.path.exists(REF_LIB_PATH):
            try:
                import ref_build
                ref_build.build()
            except (FileNotFoundError, ImportError, subprocess.CalledProcessError):
                return None
        L = ctypes.CDLL(REF_LIB_PATH)
        vp, i32, dbl = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        L.ref_mover_kernel.restype = i32
        L.ref_mover_kernel.argtypes = [vp, i32, ctypes.POINTER(RefGridParams), vp, i32, dbl, vp, vp,
                                       vp, i32, vp, vp, ctypes.POINTER(i32)]
        L.ref_interpolate.restype = i32
        L.ref_interpolate.argtypes = [vp, i32, vp, ctypes.POINTER(RefGridParams), i32, i32, vp, vp,
                                      vp, dbl, i32, vp, vp, vp]
        _ref_lib = L
    return _ref_lib


def ref_grid_params(nx: int, ny: int, width: float, height: float) -> RefGridParams:
    """The reference's params1 (src/particles.cpp:357-368): dx = XMAX/NX."""
    return RefGridParams(nx, ny, nx + 1, ny + 1, width / nx, height / ny, width, height)


def generate_plasma(nx: int, ny: int, dx: float, dy: float, ppc: int, v_th: float,
                    blob_peak: float = 0.0, blob_cx: float = 0.0, blob_cy: float = 0.0,
                    blob_sigma: float = 1.0, drift_vx: float = 0.0, drift_vy: float = 0.0,
                    seed: int = 1) -> np.ndarray:
    """Seeded reference-layout Points of one species (C, OpenMP): ppc per cell
    plus floor(blob_peak exp(-r^2/(2 sigma^2)) + u) blob particles, uniform in
    the cell, Maxwellian velocities (sigma v_th per component, blob particles
    drifting), in an order random with respect to the cells."""
    L = lib()
    counts = np.zeros(nx * ny, np.int64)
    n = int(L.orc_plasma_counts(nx, ny, ppc, blob_peak, blob_cx, blob_cy, blob_sigma, seed,
                                _ptr(counts)))
    start = np.zeros(nx * ny, np.int64)
    np.cumsum(counts[:-1], out=start[1:])
    pts = np.empty(n, POINT_DTYPE)
    L.orc_plasma_fill(nx, ny, dx, dy, ppc, v_th, drift_vx, drift_vy, seed, _ptr(counts),
                      _ptr(start), n, _ptr(pts))
    return pts
