"""The solver's V-cycle (each level's sweeps in one kernel over tiles held in
shared memory, halos recomputed) against the same V-cycle with one kernel
per half sweep (k_mg_init_black / k_mg_rbgs / k_mg_restrict /
k_mg_prolong_black, each node updated in place), through the test hook
pic_debug_vcycle: the two must give the same bits on walled grids of odd and
even sizes, with an inner electrode, and periodic in y (where the coarse
levels are smaller than a tile and appear in it more than once).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def vcycle_pic(nx, ny, periodic, inner):
    import pic_b200 as P
    import pic_configs as C
    if periodic:
        rects = C.periodic_rects(nx, ny, 25.0, -10.0,
                                 (nx // 2 - 3, ny // 3, nx // 2 + 3, ny // 3 + 4, 60.0) if inner else None)
    else:
        rects = C.wall_rects(nx, ny)
        if inner:
            rects = rects + [(nx // 3, ny // 3, nx // 3 + 5, ny // 3 + 7, 40.0)]
    cfg = P.make_config(nx, ny, 1.0, 1.0, 1e-9, [(-1.6e-19, 9.1e-31, 1.0, 1.0)], rects,
                        solver=0, warm=0, tol=1e-8, maxit=100, periodic_y=periodic)
    return P.Pic(cfg)


def run(pic, rhs, per_sweep):
    import pic_b200 as P
    out = np.zeros_like(rhs)
    P._check(P.lib().pic_debug_vcycle(pic.h, P._p(rhs), P._p(out), per_sweep))
    return out


@pytest.mark.parametrize("nx,ny,periodic,inner", [
    (256, 256, False, False),   # 257^2 nodes: three tiled levels
    (100, 70, False, True),     # sizes that leave partial tiles at every level
    (512, 512, False, False),   # the 513^2 workload's hierarchy
    (48, 40, True, True),       # periodic: levels of 40, 20, 10 rows
    (96, 64, True, False),
])
def test_tiled_vcycle_matches_per_sweep(nx, ny, periodic, inner):
    rng = np.random.default_rng(nx * 1000 + ny)
    with vcycle_pic(nx, ny, periodic, inner) as pic:
        rhs = rng.standard_normal(pic.nodes).astype(np.float32)
        a = run(pic, rhs, 0)
        b = run(pic, rhs, 1)
        c = run(pic, rhs, 0)
    assert np.abs(a).max() > 0
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), \
        f"{np.count_nonzero(a != b)} nodes differ, max {np.abs(a - b).max():.3e}"
    assert np.array_equal(a.view(np.uint32), c.view(np.uint32))
