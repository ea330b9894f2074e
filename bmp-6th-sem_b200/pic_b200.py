"""ctypes binding of libpicb200.so -- the host-side mirror of the reference's
ctypes users of libsycl_pic.so (SYCL-PIC-poissonsolver/src/sycl_pic_ctypes.cpp:1-17).

Everything here is a thin wrapper over the C ABI in include/pic_capi.h; the
compute path is the CUDA library.  There is no CPU fallback: if the library
or a usable sm_100 device is missing, the calls raise.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpicb200.so")

MAX_SPECIES = 4
MAX_RECTS = 32

PIC_OK = 0
SOLVER_MG_PCG = 0
SOLVER_JACOBI_PCG = 1
WARM_ZERO = 0
WARM_PREVIOUS = 1
WARM_LEARNED = 2

POINT_DTYPE = np.dtype(
    [("x", "<f8"), ("y", "<f8"), ("z", "<f8"), ("vx", "<f8"), ("vy", "<f8"),
     ("vz", "<f8"), ("pointer", "<i4"), ("pad", "<i4")], align=True)
assert POINT_DTYPE.itemsize == 56


class SpeciesDesc(ctypes.Structure):
    _fields_ = [("charge", ctypes.c_double), ("mass", ctypes.c_double),
                ("sim_count", ctypes.c_double), ("actual_count", ctypes.c_double)]


class Rect(ctypes.Structure):
    _fields_ = [("x1", ctypes.c_int32), ("y1", ctypes.c_int32), ("x2", ctypes.c_int32),
                ("y2", ctypes.c_int32), ("potential", ctypes.c_double)]


class Config(ctypes.Structure):
    """pic_config (include/pic_capi.h)."""
    _fields_ = [
        ("nx", ctypes.c_int32), ("ny", ctypes.c_int32),
        ("xmax", ctypes.c_double), ("ymax", ctypes.c_double),
        ("dt", ctypes.c_double), ("epsilon", ctypes.c_double), ("b0", ctypes.c_double),
        ("surf_area", ctypes.c_double),
        ("num_species", ctypes.c_int32),
        ("species", SpeciesDesc * MAX_SPECIES),
        ("num_rects", ctypes.c_int32),
        ("rects", Rect * MAX_RECTS),
        ("poisson_solver", ctypes.c_int32), ("warm_start", ctypes.c_int32),
        ("poisson_tol", ctypes.c_double), ("poisson_maxit", ctypes.c_int32),
        ("deposit_energy", ctypes.c_int32), ("device", ctypes.c_int32),
        ("timesteps", ctypes.c_int32), ("print_interval", ctypes.c_int32),
        ("periodic_y", ctypes.c_int32),
    ]


class SourceDesc(ctypes.Structure):
    """pic_source_desc (include/pic_capi.h)."""
    _fields_ = [("reinject_x", ctypes.c_double), ("te_ev", ctypes.c_double), ("ti_ev", ctypes.c_double),
                ("x11", ctypes.c_double), ("x22", ctypes.c_double), ("xm", ctypes.c_double),
                ("ionimax", ctypes.c_double), ("rate_div", ctypes.c_double),
                ("reinject", ctypes.c_int32), ("pairs", ctypes.c_int32), ("seed", ctypes.c_uint64)]


class PlasmaDesc(ctypes.Structure):
    """pic_plasma_desc (include/pic_capi.h)."""
    _fields_ = [("ppc", ctypes.c_int32), ("temperature_ev", ctypes.c_double),
                ("blob_peak_ppc", ctypes.c_double), ("blob_cx", ctypes.c_double),
                ("blob_cy", ctypes.c_double), ("blob_sigma", ctypes.c_double),
                ("drift_vx", ctypes.c_double), ("drift_vy", ctypes.c_double),
                ("seed", ctypes.c_uint64)]


class PicError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"[{status}] {msg}")
        self.status = status


_lib = None


def lib():
    """Loads libpicb200.so (building it first when absent)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        import importlib.util
        spec = importlib.util.spec_from_file_location("_picb200_build", os.path.join(HERE, "build.py"))
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        mod.build()
    L = ctypes.CDLL(LIB_PATH)
    P = ctypes.POINTER
    vp, i32, i64, dbl, cint = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_double, ctypes.c_int
    sig = {
        "pic_last_error": (ctypes.c_char_p, []),
        "pic_status_string": (ctypes.c_char_p, [cint]),
        "pic_config_default": (cint, [P(Config)]),
        "pic_config_from_files": (cint, [ctypes.c_char_p, ctypes.c_char_p, P(Config)]),
        "pic_create": (cint, [P(Config), P(vp)]),
        "pic_destroy": (None, [vp]),
        "pic_set_stream": (cint, [vp, vp]),
        "pic_get_stream": (vp, [vp]),
        "pic_synchronize": (cint, [vp]),
        "pic_reserve": (cint, [vp, cint, i64]),
        "pic_import_points": (cint, [vp, cint, vp, i64]),
        "pic_export_points": (cint, [vp, cint, vp, i64, P(i64)]),
        "pic_load_plasma": (cint, [vp, cint, P(PlasmaDesc)]),
        "pic_particle_count": (cint, [vp, cint, P(i64)]),
        "pic_bin_counts": (cint, [vp, cint, vp]),
        "pic_left_exits": (cint, [vp, cint, P(i64)]),
        "pic_zero_rho": (cint, [vp]),
        "pic_charge_deposition": (cint, [vp, cint]),
        "pic_poisson_solve": (cint, [vp, cint]),
        "pic_move_particles": (cint, [vp, cint, cint]),
        "pic_compact_particles": (cint, [vp, cint]),
        "pic_cleanup_map": (cint, [vp, cint]),
        "pic_step": (cint, [vp, cint]),
        "pic_particle_phase": (cint, [vp, cint]),
        "pic_get_rho": (cint, [vp, vp]),
        "pic_get_phi": (cint, [vp, vp]),
        "pic_get_efield": (cint, [vp, vp]),
        "pic_get_final_mesh": (cint, [vp, cint, vp]),
        "pic_get_energy_mesh": (cint, [vp, cint, vp]),
        "pic_set_rho": (cint, [vp, vp]),
        "pic_set_phi": (cint, [vp, vp]),
        "pic_update_fields_from_phi": (cint, [vp]),
        "pic_set_bz": (cint, [vp, vp]),
        "pic_set_poisson": (cint, [vp, cint, cint, dbl, cint]),
        "pic_poisson_stats": (cint, [vp, P(cint), P(dbl), P(dbl)]),
        "pic_export_state": (cint, [vp, cint] + [vp] * 6 + [i64, P(i64)]),
        "pic_set_profiling": (cint, [vp, cint]),
        "pic_profile_read": (cint, [vp, vp, vp, cint]),
        "pic_launch_count": (cint, [vp, P(i64)]),
        "pic_ws_record": (cint, [vp, i64, dbl, dbl, dbl]),
        "pic_ws_pairs": (cint, [vp, P(i64)]),
        "pic_ws_train": (cint, [vp, cint, dbl, P(dbl)]),
        "pic_ws_train_cosine": (cint, [vp, cint, dbl, dbl, P(dbl)]),
        "pic_ws_num_params": (i64, []),
        "pic_ws_get_params": (cint, [vp, vp, i64]),
        "pic_ws_set_params": (cint, [vp, vp, i64, dbl, dbl, dbl]),
        "pic_ws_grid": (cint, [vp, P(cint)]),
        "pic_ws_scales": (cint, [vp, P(dbl)]),
        "pic_set_tile_shape": (cint, [vp, cint]),
        "pic_source_default": (cint, [P(SourceDesc)]),
        "pic_generate_new_particles": (cint, [vp, P(SourceDesc), P(i64), P(i64)]),
        "pic_ensemble_create": (cint, [vp, cint, P(vp)]),
        "pic_ensemble_destroy": (None, [vp]),
        "pic_ensemble_size": (cint, [vp]),
        "pic_ensemble_instance": (vp, [vp, cint]),
        "pic_ensemble_step": (cint, [vp, cint]),
        "pic_ensemble_autotune": (cint, [vp, P(cint), P(dbl)]),
        "pic_ensemble_use_graph": (cint, [vp, cint]),
        "pic_ensemble_timing": (cint, [vp, P(dbl), P(dbl), P(dbl)]),
        "pic_ensemble_info": (cint, [vp, P(cint), P(cint), P(cint)]),
        "pic_autotune": (cint, [vp, P(cint), P(dbl)]),
        "pic_ws_debug_step": (cint, [vp, vp, vp, vp, vp, P(dbl)]),
        "pic_deposit_points_noalloc": (cint, [vp, i64, i32, i32, dbl, dbl, vp, dbl, dbl, vp, vp, vp]),
        "pic_write_diagnostics": (cint, [vp, ctypes.c_char_p, cint, dbl]),
        "pic_debug_set_wait_limits": (cint, [vp, i64, i64]),
        "pic_debug_vcycle": (cint, [vp, vp, vp, cint]),
        "pic_set_poisson_graph": (cint, [vp, cint]),
        "pic_poisson_start_relres": (cint, [vp, P(dbl)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def exported_symbols() -> list:
    """Names of the pic_* and sycl_pic_* functions the library must export."""
    out = []
    root = os.path.dirname(HERE)
    for hdr in ("pic_capi.h", "sycl_pic_compat.h"):
        import re
        txt = open(os.path.join(root, "include", hdr)).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        out += re.findall(r"\b((?:pic|sycl_pic)_[a-z0-9_]+)\s*\(", txt)
    return sorted(set(out))


def _check(status: int):
    if status != PIC_OK:
        msg = lib().pic_last_error()
        raise PicError(status, msg.decode() if msg else "")


def _p(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data


def make_config(nx, ny, xmax, ymax, dt, species, rects, b0=0.0, epsilon=8.854e-12,
                surf_area=0.0, solver=SOLVER_MG_PCG, warm=WARM_PREVIOUS, tol=1e-8, maxit=500,
                deposit_energy=True, device=0, periodic_y=False) -> Config:
    """species: list of (charge, mass, sim_count, actual_count);
    rects: list of (x1, y1, x2, y2, volts) node-index rectangles;
    periodic_y: the reference's periodicBoundary = 1."""
    cfg = Config()
    _check(lib().pic_config_default(ctypes.byref(cfg)))
    cfg.nx, cfg.ny, cfg.xmax, cfg.ymax = nx, ny, xmax, ymax
    cfg.dt, cfg.epsilon, cfg.b0, cfg.surf_area = dt, epsilon, b0, surf_area
    cfg.num_species = len(species)
    for i, (q, m, sim, act) in enumerate(species):
        cfg.species[i] = SpeciesDesc(q, m, sim, act)
    cfg.num_rects = len(rects)
    for i, (x1, y1, x2, y2, v) in enumerate(rects):
        cfg.rects[i] = Rect(int(x1), int(y1), int(x2), int(y2), float(v))
    cfg.poisson_solver, cfg.warm_start = solver, warm
    cfg.poisson_tol, cfg.poisson_maxit = tol, maxit
    cfg.deposit_energy = 1 if deposit_energy else 0
    cfg.device = device
    cfg.periodic_y = 1 if periodic_y else 0
    return cfg


class Pic:
    """One simulation instance (pic_ctx)."""

    def __init__(self, cfg: Config):
        self.cfg = cfg
        self.h = ctypes.c_void_p()
        _check(lib().pic_create(ctypes.byref(cfg), ctypes.byref(self.h)))
        self.GX, self.GY = cfg.nx + 1, cfg.ny + 1
        self.nodes = self.GX * self.GY

    def close(self):
        if self.h:
            lib().pic_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ---- stream ----
    def set_stream(self, stream_handle: int | None):
        _check(lib().pic_set_stream(self.h, ctypes.c_void_p(stream_handle or 0)))

    def synchronize(self):
        _check(lib().pic_synchronize(self.h))

    # ---- particles ----
    def reserve(self, s: int, cap: int):
        _check(lib().pic_reserve(self.h, s, cap))

    def import_points(self, s: int, pts: np.ndarray):
        assert pts.dtype == POINT_DTYPE
        pts = np.ascontiguousarray(pts)
        _check(lib().pic_import_points(self.h, s, _p(pts) if len(pts) else None, len(pts)))

    def export_points(self, s: int, out: np.ndarray | None = None) -> np.ndarray:
        """Points of species s; into `out` (a POINT_DTYPE array at least as
        long as the particle count) when given, returning the filled view."""
        n = ctypes.c_int64(0)
        _check(lib().pic_export_points(self.h, s, None, 0, ctypes.byref(n)))
        if out is None:
            out = np.zeros(n.value, POINT_DTYPE)
        assert out.dtype == POINT_DTYPE and out.flags["C_CONTIGUOUS"] and len(out) >= n.value
        if n.value:
            _check(lib().pic_export_points(self.h, s, _p(out), len(out), ctypes.byref(n)))
        return out[:n.value]

    def load_plasma(self, s: int, ppc: int, temperature_ev: float, seed: int, blob_peak_ppc=0.0,
                    blob_cx=0.0, blob_cy=0.0, blob_sigma=0.0, drift_vx=0.0, drift_vy=0.0):
        d = PlasmaDesc(ppc, temperature_ev, blob_peak_ppc, blob_cx, blob_cy, blob_sigma,
                       drift_vx, drift_vy, seed)
        _check(lib().pic_load_plasma(self.h, s, ctypes.byref(d)))

    def count(self, s: int) -> int:
        n = ctypes.c_int64(0)
        _check(lib().pic_particle_count(self.h, s, ctypes.byref(n)))
        return n.value

    def bin_counts(self, s: int) -> np.ndarray:
        out = np.zeros(self.nodes, np.int32)
        _check(lib().pic_bin_counts(self.h, s, _p(out)))
        return out

    def generate_new_particles(self, **overrides):
        """Re-injection and ionisation pairs (pic_generate_new_particles);
        keyword arguments override pic_source_default's fields.  Returns
        (electrons re-injected, pairs created)."""
        d = SourceDesc()
        _check(lib().pic_source_default(ctypes.byref(d)))
        for k, v in overrides.items():
            setattr(d, k, v)
        ne, npair = ctypes.c_int64(0), ctypes.c_int64(0)
        _check(lib().pic_generate_new_particles(self.h, ctypes.byref(d), ctypes.byref(ne), ctypes.byref(npair)))
        return ne.value, npair.value

    def left_exits(self, s: int) -> int:
        n = ctypes.c_int64(0)
        _check(lib().pic_left_exits(self.h, s, ctypes.byref(n)))
        return n.value

    # ---- operators ----
    def zero_rho(self):
        _check(lib().pic_zero_rho(self.h))

    def charge_deposition(self, s: int):
        _check(lib().pic_charge_deposition(self.h, s))

    def poisson_solve(self, iteration: int = 0):
        _check(lib().pic_poisson_solve(self.h, iteration))

    def move_particles(self, s: int, iteration: int = 0):
        _check(lib().pic_move_particles(self.h, s, iteration))

    def step(self, iteration: int = 0):
        _check(lib().pic_step(self.h, iteration))

    def particle_phase(self, iteration: int = 0):
        _check(lib().pic_particle_phase(self.h, iteration))

    # ---- grids ----
    def _grid(self, fn, *args):
        out = np.zeros(self.nodes)
        _check(fn(self.h, *args, _p(out)))
        return out

    def rho(self):
        return self._grid(lib().pic_get_rho)

    def phi(self):
        return self._grid(lib().pic_get_phi)

    def final_mesh(self, s):
        return self._grid(lib().pic_get_final_mesh, s)

    def energy_mesh(self, s):
        return self._grid(lib().pic_get_energy_mesh, s)

    def efield(self):
        out = np.zeros((self.nodes, 2))
        _check(lib().pic_get_efield(self.h, _p(out)))
        return out

    def set_rho(self, rho: np.ndarray):
        rho = np.ascontiguousarray(rho, dtype=np.float64)
        _check(lib().pic_set_rho(self.h, _p(rho)))

    def set_phi(self, phi: np.ndarray):
        phi = np.ascontiguousarray(phi, dtype=np.float64)
        _check(lib().pic_set_phi(self.h, _p(phi)))

    def update_fields(self):
        _check(lib().pic_update_fields_from_phi(self.h))

    def set_bz(self, bz: np.ndarray):
        bz = np.ascontiguousarray(bz, dtype=np.float64)
        _check(lib().pic_set_bz(self.h, _p(bz)))

    def write_diagnostics(self, directory: str, iteration: int, scale_factor: float = 1.0):
        """The reference's text snapshots (pic_write_diagnostics)."""
        _check(lib().pic_write_diagnostics(self.h, directory.encode(), iteration, scale_factor))

    def set_poisson(self, solver=SOLVER_MG_PCG, warm=WARM_PREVIOUS, tol=1e-8, maxit=500):
        _check(lib().pic_set_poisson(self.h, solver, warm, tol, maxit))

    # ---- learned warm start ----
    def ws_record(self, max_pairs: int, phi_scale: float = 0.0, db_scale: float = 0.0,
                  target_scale: float = 0.0):
        _check(lib().pic_ws_record(self.h, max_pairs, phi_scale, db_scale, target_scale))

    def ws_pairs(self) -> int:
        n = ctypes.c_int64(0)
        _check(lib().pic_ws_pairs(self.h, ctypes.byref(n)))
        return n.value

    def ws_train(self, epochs: int, lr: float) -> float:
        loss = ctypes.c_double(0)
        _check(lib().pic_ws_train(self.h, epochs, lr, ctypes.byref(loss)))
        return loss.value

    def ws_train_cosine(self, epochs: int, lr_max: float, lr_min: float) -> float:
        loss = ctypes.c_double(0)
        _check(lib().pic_ws_train_cosine(self.h, epochs, lr_max, lr_min, ctypes.byref(loss)))
        return loss.value

    def ws_params(self) -> np.ndarray:
        n = lib().pic_ws_num_params()
        out = np.zeros(n, np.float32)
        _check(lib().pic_ws_get_params(self.h, _p(out), n))
        return out

    def ws_set_params(self, theta, phi_scale, db_scale, target_scale):
        theta = np.ascontiguousarray(theta, dtype=np.float32)
        _check(lib().pic_ws_set_params(self.h, _p(theta), len(theta), phi_scale, db_scale, target_scale))

    def ws_scales(self):
        out = (ctypes.c_double * 3)()
        _check(lib().pic_ws_scales(self.h, out))
        return tuple(out)

    def ws_grid(self) -> int:
        P = ctypes.c_int(0)
        _check(lib().pic_ws_grid(self.h, ctypes.byref(P)))
        return P.value

    def ws_debug_step(self, x0: np.ndarray, target: np.ndarray):
        P = self.ws_grid()
        x0 = np.ascontiguousarray(x0, dtype=np.float32)
        target = np.ascontiguousarray(target, dtype=np.float32)
        assert x0.shape == (P, P, 3) and target.size == self.nodes
        out = np.zeros((P, P), np.float32)
        grad = np.zeros(lib().pic_ws_num_params(), np.float32)
        loss = ctypes.c_double(0)
        _check(lib().pic_ws_debug_step(self.h, _p(x0), _p(target), _p(out), _p(grad), ctypes.byref(loss)))
        return out, grad, loss.value

    def autotune(self, timings: bool = False):
        """Picks the fastest particle-kernel tile shape; returns it (and the
        per-shape milliseconds when timings is set)."""
        sh = ctypes.c_int(0)
        ms = (ctypes.c_double * 4)() if timings else None
        _check(lib().pic_autotune(self.h, ctypes.byref(sh), ms))
        return (sh.value, list(ms)) if timings else sh.value

    def set_tile_shape(self, shape: int):
        _check(lib().pic_set_tile_shape(self.h, shape))

    def poisson_stats(self):
        it, rr, ms = ctypes.c_int(0), ctypes.c_double(0), ctypes.c_double(0)
        _check(lib().pic_poisson_stats(self.h, ctypes.byref(it), ctypes.byref(rr), ctypes.byref(ms)))
        return it.value, rr.value, ms.value

    def poisson_start_relres(self):
        """Relative residual of the last solve's starting guess."""
        r = ctypes.c_double(0)
        _check(lib().pic_poisson_start_relres(self.h, ctypes.byref(r)))
        return r.value


class _Instance(Pic):
    """A context owned by an Ensemble (not destroyed by itself)."""

    def __init__(self, handle, cfg: Config):
        self.cfg = cfg
        self.h = ctypes.c_void_p(handle)
        self.GX, self.GY = cfg.nx + 1, cfg.ny + 1
        self.nodes = self.GX * self.GY

    def close(self):
        self.h = ctypes.c_void_p()


class Ensemble:
    """pic_ensemble: many instances advanced together (include/pic_capi.h)."""

    def __init__(self, cfgs):
        arr = (Config * len(cfgs))(*cfgs)
        self.h = ctypes.c_void_p()
        _check(lib().pic_ensemble_create(arr, len(cfgs), ctypes.byref(self.h)))
        self.instances = [_Instance(lib().pic_ensemble_instance(self.h, i), cfgs[i])
                          for i in range(len(cfgs))]

    def __len__(self):
        return len(self.instances)

    def __getitem__(self, i) -> Pic:
        return self.instances[i]

    def step(self, iteration: int = 0):
        _check(lib().pic_ensemble_step(self.h, iteration))

    def autotune(self):
        sh = ctypes.c_int(0)
        ms = (ctypes.c_double * 4)()
        _check(lib().pic_ensemble_autotune(self.h, ctypes.byref(sh), ms))
        return sh.value, list(ms)

    def info(self):
        g, sh, b = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_int(0)
        _check(lib().pic_ensemble_info(self.h, ctypes.byref(g), ctypes.byref(sh), ctypes.byref(b)))
        return dict(graph=bool(g.value), tile_shape=sh.value, solver_blocks=b.value)

    def use_graph(self, on: bool):
        _check(lib().pic_ensemble_use_graph(self.h, 1 if on else 0))

    def timing(self):
        d, p, q = ctypes.c_double(0), ctypes.c_double(0), ctypes.c_double(0)
        _check(lib().pic_ensemble_timing(self.h, ctypes.byref(d), ctypes.byref(p), ctypes.byref(q)))
        return d.value, p.value, q.value

    def close(self):
        if self.h:
            for inst in self.instances:
                inst.close()
            lib().pic_ensemble_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
