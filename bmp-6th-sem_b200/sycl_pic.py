"""`sycl_pic`-compatible Python module over the B200 library.

The reference's CPython extension (SYCL-PIC-poissonsolver/src/
sycl_pic_module.cpp:386-410) exposes the PIC step to its Python driver
(src/main.py) as module functions with these names, arguments and return
values; this module serves the same calls from libpicb200.so through its
sycl_pic_* C ABI (include/sycl_pic_compat.h), so `import sycl_pic` in that
driver finds the same surface:

  * get_rho() / get_phi() return NumPy arrays that share memory with the
    library's host copies (zero-copy, like the reference's wrap of its
    malloc_shared arrays); the library refreshes them after every operator,
    and writes through get_phi() reach the device with
    update_fields_from_phi();
  * operators return elapsed wall seconds; compact_particles returns
    (elapsed, alloc_t, scan_t);
  * failures raise RuntimeError with the library's message where the
    reference would exit.

generate_new_particles re-injects electrons and creates ionisation pairs
with the reference's constants (pic_generate_new_particles).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

import pic_b200 as _P

_c = ctypes


def _lib():
    L = _P.lib()
    if not getattr(L, "_sycl_pic_typed", False):
        dbl, cint, cp = _c.c_double, _c.c_int, _c.c_char_p
        sig = {
            "sycl_pic_init": (cint, [cp, cint, cint, cp, cp]),
            "sycl_pic_get_grid_size": (cint, []), "sycl_pic_get_grid_x": (cint, []),
            "sycl_pic_get_grid_y": (cint, []), "sycl_pic_get_timesteps": (cint, []),
            "sycl_pic_get_print_interval": (cint, []), "sycl_pic_get_num_species": (cint, []),
            "sycl_pic_get_particle_count": (cint, [cint]),
            "sycl_pic_get_rho_ptr": (_c.POINTER(dbl), []), "sycl_pic_get_phi_ptr": (_c.POINTER(dbl), []),
            "sycl_pic_zero_rho": (None, []),
            "sycl_pic_charge_deposition": (dbl, [cint]), "sycl_pic_poisson_solve": (dbl, [cint]),
            "sycl_pic_move_particles": (dbl, [cint, cint]),
            "sycl_pic_compact_particles": (dbl, [cint, _c.POINTER(dbl), _c.POINTER(dbl)]),
            "sycl_pic_cleanup_map": (dbl, [cint]), "sycl_pic_generate_new_particles": (dbl, []),
            "sycl_pic_update_fields_from_phi": (None, []),
            "sycl_pic_print_diagnostics": (None, [cp, cint]), "sycl_pic_save_meshes": (None, []),
            "sycl_pic_last_status": (cint, []),
            "sycl_pic_finalize": (None, []),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype, f.argtypes = res, args
        L._sycl_pic_typed = True
    return L


def _err(what):
    msg = _P.lib().pic_last_error()
    raise RuntimeError(f"{what}: {msg.decode() if msg else 'failed'}")


def _checked_seconds(v, what):
    if v < 0:
        _err(what)
    return float(v)


def init(dev_type: str, wg_size: int, prob_size: int, input1: str, input2: str) -> None:
    """sycl_pic_module.cpp:53: reads ./M_PICDAT.DAT and ./geometry.conf."""
    if _lib().sycl_pic_init(dev_type.encode(), int(wg_size), int(prob_size), input1.encode(),
                            input2.encode()) != 0:
        _err("init")


def _int(name):
    v = getattr(_lib(), name)()
    if v < 0:
        _err(name)
    return int(v)


def get_grid_size() -> int:
    return _int("sycl_pic_get_grid_size")


def get_grid_x() -> int:
    return _int("sycl_pic_get_grid_x")


def get_grid_y() -> int:
    return _int("sycl_pic_get_grid_y")


def get_timesteps() -> int:
    return _int("sycl_pic_get_timesteps")


def get_print_interval() -> int:
    return _int("sycl_pic_get_print_interval")


def get_num_species() -> int:
    return _int("sycl_pic_get_num_species")


def get_particle_counts():
    """(electrons, ions) live counts (sycl_pic_module.cpp:145-149)."""
    L = _lib()
    return tuple(int(L.sycl_pic_get_particle_count(s)) for s in range(2))


def _view(ptr_fn):
    p = ptr_fn()
    if not p:
        _err("grid pointer")
    return np.ctypeslib.as_array(p, shape=(get_grid_size(),))


def get_rho() -> np.ndarray:
    """rho, GRID_X*GRID_Y doubles, sharing memory with the library (zero-copy)."""
    return _view(_lib().sycl_pic_get_rho_ptr)


def get_phi() -> np.ndarray:
    """phi, GRID_X*GRID_Y doubles, sharing memory with the library (zero-copy)."""
    return _view(_lib().sycl_pic_get_phi_ptr)


def zero_rho() -> None:
    _lib().sycl_pic_zero_rho()


def charge_deposition(species: int) -> float:
    return _checked_seconds(_lib().sycl_pic_charge_deposition(int(species)), "charge_deposition")


def poisson_solve(iteration: int) -> float:
    return _checked_seconds(_lib().sycl_pic_poisson_solve(int(iteration)), "poisson_solve")


def update_fields_from_phi() -> None:
    _lib().sycl_pic_update_fields_from_phi()


def move_particles(species: int, iteration: int) -> float:
    return _checked_seconds(_lib().sycl_pic_move_particles(int(species), int(iteration)), "move_particles")


def compact_particles(species: int):
    """(elapsed, alloc_t, scan_t) (sycl_pic_module.cpp:236-252); the sorted
    layout compacts itself, so the phases take no time."""
    a, s = _c.c_double(0), _c.c_double(0)
    t = _lib().sycl_pic_compact_particles(int(species), _c.byref(a), _c.byref(s))
    return (_checked_seconds(t, "compact_particles"), float(a.value), float(s.value))


def cleanup_map(species: int) -> float:
    return _checked_seconds(_lib().sycl_pic_cleanup_map(int(species)), "cleanup_map")


def generate_new_particles() -> float:
    return _checked_seconds(_lib().sycl_pic_generate_new_particles(), "generate_new_particles")


def _checked_status(what: str) -> None:
    if _lib().sycl_pic_last_status() != 0:
        _err(what)


def print_diagnostics(directory: str, iteration: int) -> None:
    """Text snapshots (printNumberDensity/printEnergy/printElectricField/
    printPhi); raises where the reference would print and exit."""
    _lib().sycl_pic_print_diagnostics(directory.encode(), int(iteration))
    _checked_status("print_diagnostics")


def save_meshes() -> None:
    _lib().sycl_pic_save_meshes()
    _checked_status("save_meshes")


def dump_rho_phi_cpp(prefix: str) -> None:
    """<prefix>_rho_cpp.bin / _phi_cpp.bin: the library-side arrays as raw
    doubles (sycl_pic_module.cpp:350-368)."""
    get_rho().tofile(prefix + "_rho_cpp.bin")
    get_phi().tofile(prefix + "_phi_cpp.bin")


def finalize() -> None:
    _lib().sycl_pic_finalize()


__all__ = ["init", "get_grid_size", "get_grid_x", "get_grid_y", "get_timesteps",
           "get_print_interval", "get_num_species", "get_particle_counts", "get_rho", "get_phi",
           "zero_rho", "charge_deposition", "poisson_solve", "update_fields_from_phi",
           "move_particles", "compact_particles", "cleanup_map", "generate_new_particles",
           "print_diagnostics", "save_meshes", "dump_rho_phi_cpp", "finalize"]
