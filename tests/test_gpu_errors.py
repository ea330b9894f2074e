"""Error paths of the C ABI on the GPU: each failure is reported as a status
code (the reference calls exit() in these places) and leaves the context
usable.

* more particles in one cell than the per-cell limit (43,680: a cell's slots,
  n + n/2 + 16, may not exceed 2^16, for which the fixed-point moment sums
  are sized) -> PIC_ERR_CAPACITY at import;
* a Poisson solve that reaches its iteration limit before the tolerance
  (PARDISO's error path, src/poissonSolver.cpp:459-544, has no counterpart:
  a direct solve always finishes) -> PIC_ERR_NOT_CONVERGED;
* after either, the next operation with valid inputs succeeds.
"""
import numpy as np
import pytest

from test_gpu_particles import make_pic, small_workload

pytestmark = pytest.mark.gpu


def test_cell_limit_is_an_error_and_the_context_recovers():
    import pic_b200 as P
    import pic_configs as C
    w = small_workload(nx=16, ny=16, ppc=4)
    limit = 43680
    pts = np.zeros(limit + 1, P.POINT_DTYPE)
    rng = np.random.default_rng(1)
    pts["x"] = (5 + rng.random(len(pts))) * w.dx      # all in cell (5, 7)
    pts["y"] = (7 + rng.random(len(pts))) * w.dx
    pts["pointer"] = np.arange(len(pts))
    with make_pic(w) as pic:
        with pytest.raises(P.PicError) as e:
            pic.import_points(0, pts)
        assert e.value.status == -3      # PIC_ERR_CAPACITY
        # exactly at the limit is accepted
        pic.import_points(0, pts[:limit])
        assert pic.count(0) == limit
        ok = C.host_points(w, 0, seed=3)
        pic.import_points(0, ok)
        assert pic.count(0) == len(ok)
        pic.step(0)


def test_poisson_iteration_limit_is_an_error_and_the_context_recovers(oracle):
    import pic_b200 as P
    import pic_configs as C
    w = small_workload(nx=64, ny=64)
    rng = np.random.default_rng(2)
    rho = rng.normal(size=w.GX * w.GY) * 1e7
    with make_pic(w, tol=1e-12, maxit=1) as pic:
        pic.set_rho(rho)
        with pytest.raises(P.PicError) as e:
            pic.poisson_solve(0)
        assert e.value.status == -4      # PIC_ERR_NOT_CONVERGED
        pic.set_poisson(tol=1e-8, maxit=500)
        pic.set_rho(rho)
        pic.poisson_solve(1)
        it, rel, _ = pic.poisson_stats()
        assert rel <= 1e-8 and it <= 20
        el = oracle.Electrodes(w.rects)
        mask = oracle.electrode_mask(w.GX, w.GY, el)
        dx = w.xmax / w.nx
        assert oracle.reduced_relres(w.GX, w.GY, dx, dx, mask, pic.rho(), pic.phi()) <= 1e-8
