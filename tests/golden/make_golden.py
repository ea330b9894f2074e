"""Copies the reference's PARDISO golden vectors into small committed fixtures.

Source: SYCL-PIC-poissonsolver/validation_dumps/iter000{0,4}_{rho_input,phi_cpp}.npy
(257x257 nodes, XMAX=YMAX=1 m, NX=NY=256 from SYCL-PIC-poissonsolver/M_PICDAT.DAT:6,
four grounded walls from SYCL-PIC-poissonsolver/geometry.conf:6-9).  rho_input is
the deposited rho handed to poissonSolver() before overwriteRho; phi_cpp is the
MKL PARDISO result after overwritePhi.  Only iterations 0 and 4 are kept to
keep the fixtures small.  Run once in a checkout that has the reference tree:

    python tests/golden/make_golden.py /root/reference
"""
import os
import sys

import numpy as np

ITERS = (0, 4)


def main(ref_root: str) -> None:
    src = os.path.join(ref_root, "SYCL-PIC-poissonsolver", "validation_dumps")
    out_dir = os.path.dirname(os.path.abspath(__file__))
    for it in ITERS:
        rho = np.load(os.path.join(src, f"iter{it:04d}_rho_input.npy"))
        phi = np.load(os.path.join(src, f"iter{it:04d}_phi_cpp.npy"))
        assert rho.shape == phi.shape == (257 * 257,)
        np.savez_compressed(os.path.join(out_dir, f"poisson_257_iter{it:04d}.npz"),
                            rho_input=rho, phi_cpp=phi, nx=256, ny=256, xmax=1.0, ymax=1.0)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
