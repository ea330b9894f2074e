"""Error paths of the C ABI on the GPU: each failure is reported as a status
code (the reference calls exit() in these places) and leaves the context
usable.

* more particles in one cell than the per-cell limit (43,680: a cell's slots,
  n + n/2 + 16, may not exceed 2^16, for which the fixed-point moment sums
  are sized) -> PIC_ERR_CAPACITY at import;
* a Poisson solve that reaches its iteration limit before the tolerance
  (PARDISO's error path, src/poissonSolver.cpp:459-544, has no counterpart:
  a direct solve always finishes) -> PIC_ERR_NOT_CONVERGED;
* after either, the next operation with valid inputs succeeds;
* the two bounded device waits (the batched solve's block barriers, the
  learned warm start's tensor-core pipeline waits), lowered through the test
  hook pic_debug_set_wait_limits, give up and return PIC_ERR_TIMEOUT; with
  the default bounds restored the same ensemble / context works.
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


def test_ensemble_barrier_timeout_is_an_error_and_the_ensemble_recovers(oracle):
    """The batched solve's block barriers give up after a bounded number of
    polls.  Lowered to one poll (pic_debug_set_wait_limits) the first block
    to arrive at a barrier gives up before the others come: the step
    returns PIC_ERR_TIMEOUT (no fault, no hang: every wait is bounded, every
    index is independent of the data).  With the default bound restored and
    fresh particles the same ensemble steps again and every instance reaches
    its tolerance (true residual measured by the oracle)."""
    import pic_b200 as P
    import pic_configs as C
    from test_gpu_ensemble import instances, load
    ws = instances()
    L = P.lib()
    with P.Ensemble([C.library_config(w) for w in ws]) as E:
        for k, w in enumerate(ws):
            load(E[k], w, k)
        E.step(0)
        assert L.pic_debug_set_wait_limits(E[0].h, 1, 0) == 0
        try:
            with pytest.raises(P.PicError) as e:
                E.step(1)
            assert e.value.status == -9      # PIC_ERR_TIMEOUT
        finally:
            assert L.pic_debug_set_wait_limits(E[0].h, 0, 0) == 0
        for k, w in enumerate(ws):
            load(E[k], w, 50 + k)
            E[k].set_phi(np.zeros(E[k].nodes))
        E.step(2)
        for k, w in enumerate(ws):
            it, rel, _ = E[k].poisson_stats()
            assert rel <= 1e-8 and it > 0
            dx = w.xmax / w.nx
            el = oracle.Electrodes(w.rects)
            mask = oracle.electrode_mask(w.GX, w.GY, el)
            assert oracle.reduced_relres(w.GX, w.GY, dx, dx, mask, E[k].rho(), E[k].phi()) <= 1e-8


def test_learned_guess_wait_timeout_is_an_error_and_recovers(oracle):
    """The learned warm start's tensor-core pipeline waits give up after a
    bounded number of SM cycles.  Lowered to one cycle, the first wait that
    is not already complete gives up: the kernel's roles leave their loops,
    the MMA warp waits (with the default bound) for the MMAs it issued
    before the tensor memory is freed, and the solve returns
    PIC_ERR_TIMEOUT.  With the default restored the same context solves
    from the network's guess to 1e-8 (true residual measured by the
    oracle)."""
    import pic_b200 as P
    import pic_configs as C
    w = C.cfg3(16)
    L = P.lib()
    with P.Pic(C.library_config(w)) as pic:
        C.load_plasma(pic, w)
        pic.ws_record(6)
        for it in range(7):
            pic.step(it)
        pic.ws_record(0)
        pic.ws_train(2, 1e-3)
        pic.zero_rho()
        for s in range(2):
            pic.charge_deposition(s)
        rho, phi_prev = pic.rho(), pic.phi()
        pic.set_poisson(P.SOLVER_MG_PCG, P.WARM_LEARNED, 1e-8, 500)
        assert L.pic_debug_set_wait_limits(pic.h, 0, 1) == 0
        try:
            with pytest.raises(P.PicError) as e:
                pic.poisson_solve(7)
            assert e.value.status == -9      # PIC_ERR_TIMEOUT
        finally:
            assert L.pic_debug_set_wait_limits(pic.h, 0, 0) == 0
        pic.set_phi(phi_prev)
        pic.set_rho(rho)
        pic.poisson_solve(7)
        it, rel, _ = pic.poisson_stats()
        assert rel <= 1e-8
        dx = w.xmax / w.nx
        mask = oracle.electrode_mask(w.GX, w.GY, oracle.Electrodes(w.rects))
        assert oracle.reduced_relres(w.GX, w.GY, dx, dx, mask, pic.rho(), pic.phi()) <= 1e-8
