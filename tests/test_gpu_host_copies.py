"""Host <-> device copies of large arrays through the C ABI.

Grids and particles cross between the caller's (pageable) memory and the
device through pinned staging chunks, the host side of each chunk split over
a pool of threads.  Every byte must arrive, whatever the length: grids of
1025^2 nodes (8,405,000 bytes, not a multiple of the pool's part size) and
particle counts just past a multiple of the parts round-trip exactly.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_large_grid_round_trip():
    import pic_b200 as P
    import pic_configs as C
    w = C.cfg3()
    rng = np.random.default_rng(3)
    with P.Pic(C.library_config(w)) as pic:
        for n in range(2):
            v = rng.normal(size=pic.nodes)
            pic.set_rho(v)
            assert np.array_equal(pic.rho(), v)
            pic.set_phi(v[::-1].copy())
            assert np.array_equal(pic.phi(), v[::-1])


@pytest.mark.parametrize("n", [16 * 65536 + 5, 3 * 1398101 + 17])
def test_particle_import_export_round_trip(n):
    """Every imported Point comes back (as the FP32 state rounds it)."""
    import pic_b200 as P
    import pic_configs as C
    import test_gpu_config_parity as CP
    w = C.cfg2()
    rng = np.random.default_rng(n)
    pts = np.zeros(n, P.POINT_DTYPE)
    pts["x"] = rng.uniform(0, w.xmax, n)
    pts["y"] = rng.uniform(0, w.ymax, n)
    pts["vx"] = rng.normal(0, 1e5, n)
    pts["vy"] = rng.normal(0, 1e5, n)
    CP._tag(pts)
    with P.Pic(C.library_config(w)) as pic:
        pic.import_points(0, pts)
        assert pic.count(0) == n
        st = CP._export_state(pic, 0)
        assert CP._multiset_hash(st["cell"], st["fx"], st["fy"], st["vx"], st["vy"], st["vz"]) == \
            CP._multiset_hash(*CP._expected_state(w, pts))
        out = pic.export_points(0)
    tag = CP._untag(out["vz"].astype(np.float32))
    assert len(out) == n and np.array_equal(np.sort(tag), np.arange(n))
