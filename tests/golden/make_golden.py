"""Copies the reference's PARDISO golden vectors into small committed fixtures.

Source: SYCL-PIC-poissonsolver/validation_dumps/iter000{0-4}_{rho_input,phi_cpp}.npy
(257x257 nodes, XMAX=YMAX=1 m, NX=NY=256 from SYCL-PIC-poissonsolver/M_PICDAT.DAT:6,
four grounded walls from SYCL-PIC-poissonsolver/geometry.conf:6-9).  rho_input is
the deposited rho handed to poissonSolver() before overwriteRho; phi_cpp is the
MKL PARDISO result after overwritePhi.  All five dumped iterations are kept
(about 1 MB each, compressed).  Run once in a checkout that has the reference
tree, naming its root:

    python tests/golden/make_golden.py <reference checkout root>
"""
import argparse
import os

import numpy as np

ITERS = (0, 1, 2, 3, 4)


def main(ref_root: str) -> None:
    src = os.path.join(ref_root, "SYCL-PIC-poissonsolver", "validation_dumps")
    if not os.path.isdir(src):
        raise SystemExit(f"no validation_dumps folder under {ref_root}")
    out_dir = os.path.dirname(os.path.abspath(__file__))
    for it in ITERS:
        rho = np.load(os.path.join(src, f"iter{it:04d}_rho_input.npy"))
        phi = np.load(os.path.join(src, f"iter{it:04d}_phi_cpp.npy"))
        assert rho.shape == phi.shape == (257 * 257,)
        np.savez_compressed(os.path.join(out_dir, f"poisson_257_iter{it:04d}.npz"),
                            rho_input=rho, phi_cpp=phi, nx=256, ny=256, xmax=1.0, ymax=1.0)


if __name__ == "__main__":
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("reference_root", help="root of the vansh268p/BMP-6th-sem checkout")
    main(ap.parse_args().reference_root)
