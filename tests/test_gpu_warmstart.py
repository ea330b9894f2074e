"""GPU learned warm start against the conv-network oracle, through the C ABI.

* One forward + backward pass (pic_ws_debug_step) equals oracle/convnet.py in
  its bf16 mode (activations and gradient images rounded where the kernels
  store bf16; FP32 accumulation on the GPU vs FP64 in the oracle), for the
  residual loss |rhs - kappa L(out)|^2 the network is trained on:
  output within 2e-2 of max|out|, loss within 2e-2 relative, parameter
  gradient within 5e-2 relative 2-norm overall (1e-1 per layer), cosine
  >= 0.998; the pass is bit-for-bit repeatable.
* Training on pairs the simulation records lowers the loss, and PCG started
  from the network's guess reaches the same 1e-8 relative residual as PCG
  started from phi_{n-1} on the same state: the converged potentials agree
  to 1e-6 of max|phi| (both are 1e-8-residual solutions of one system).
  The guess is strictly the better start: its starting residual
  (pic_poisson_start_relres) is below phi_{n-1}'s on every evaluation step
  and below half of it on average; it never costs iterations.
* The data gradients run on the tcgen05 row convolution (flipped,
  transposed weights, relu gate in its epilogue), the forward 32->32 layers
  too; the gradient check covers both.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def small_pic(n=60, **kw):
    import pic_b200 as P
    import pic_configs as C
    c = n // 2
    rects = C.wall_rects(n, n, left=50.0) + [(c - 6, c - 4, c + 5, c + 7, 120.0)]
    cfg = P.make_config(n, n, n * 2.5e-4, n * 2.5e-4, 5e-11, [(-1.602e-19, 9.109e-31, 1.0, 1.0)],
                        rects, **kw)
    return P.Pic(cfg), rects


def random_case(P, GX, GY, mask, seed):
    import convnet as N
    rng = np.random.default_rng(seed)
    theta = np.zeros(N.N_PARAMS, np.float32)
    o = 0
    for n, fan in [(N.IN_W, 27), (N.IN_B, 0)] + [(N.W32, 288), (N.B32, 0)] * N.N_CONV32 + \
            [(N.OUT_W, 288), (N.OUT_B, 0)]:
        theta[o:o + n] = rng.uniform(-1, 1, n) * (np.sqrt(6.0 / fan) if fan else 0.05)
        o += n
    m2 = mask.reshape(GY, GX)
    x0 = np.zeros((P, P, 3), np.float32)
    x0[:GY, :GX, 0] = rng.normal(0, 1, (GY, GX))
    x0[:GY, :GX, 1] = rng.normal(0, 1, (GY, GX)) * (1 - m2)
    x0[:GY, :GX, 2] = m2
    rhs = (rng.normal(0, 0.5, GX * GY) * (1 - mask)).astype(np.float32)
    return theta, x0, rhs


@pytest.mark.parametrize("n", [60, 71])
def test_forward_backward_match_oracle(oracle, n):
    import convnet as N
    pic, rects = small_pic(n)
    with pic:
        GX = GY = n + 1
        P = pic.ws_grid()
        assert P % 4 == 0 and P >= GX
        mask = oracle.electrode_mask(GX, GY, oracle.Electrodes(rects)).astype(np.uint8)
        theta, x0, rhs = random_case(P, GX, GY, mask, seed=n)
        pic.ws_set_params(theta, 1.0, 2.0, 1.5)      # kappa = s2/s1 = 0.75
        out, grad, loss = pic.ws_debug_step(x0, rhs)
        # the same pass again gives the same bits (deterministic reductions)
        out2, grad2, loss2 = pic.ws_debug_step(x0, rhs)
    assert np.array_equal(out, out2) and np.array_equal(grad, grad2) and loss == loss2
    loss_o, g_o, out_o = N.loss_grad(theta.astype(np.float64), x0, rhs.astype(np.float64), mask,
                                     GX, GY, 0.75, 1.0)
    assert np.abs(out - out_o).max() <= 2e-2 * np.abs(out_o).max()
    assert abs(loss - loss_o) <= 2e-2 * loss_o
    g = grad.astype(np.float64)
    rel = np.linalg.norm(g - g_o) / np.linalg.norm(g_o)
    print(f"n={n}: out {np.abs(out - out_o).max() / np.abs(out_o).max():.2e} "
          f"loss {abs(loss - loss_o) / loss_o:.2e} grad {rel:.2e}")
    assert rel <= 5e-2
    assert g @ g_o >= 0.998 * np.linalg.norm(g) * np.linalg.norm(g_o)
    offs = [0, N.IN_W + N.IN_B] + [N.IN_W + N.IN_B + (i + 1) * (N.W32 + N.B32) for i in range(N.N_CONV32)] + \
        [N.N_PARAMS]
    for a, b in zip(offs[:-1], offs[1:]):
        assert np.linalg.norm(g[a:b] - g_o[a:b]) <= 1e-1 * np.linalg.norm(g_o[a:b]), (a, b)


def test_forward_many_units_per_block(oracle):
    """A grid large enough (P = 388) that every persistent block of the
    tcgen05 convolution walks several two-row units: the ring of staged
    tiles wraps and both TMEM accumulators alternate.  The quarter-size
    level (97) is odd, so its last unit has one row outside the image.  The
    forward output matches the oracle's bf16-mode forward and repeats bit
    for bit."""
    import convnet as N
    n = 387
    pic, rects = small_pic(n)
    with pic:
        GX = GY = n + 1
        P = pic.ws_grid()
        assert P == 388
        mask = oracle.electrode_mask(GX, GY, oracle.Electrodes(rects)).astype(np.uint8)
        theta, x0, rhs = random_case(P, GX, GY, mask, seed=7)
        pic.ws_set_params(theta, 1.0, 2.0, 1.5)
        out, _, _ = pic.ws_debug_step(x0, rhs)
        out2, _, _ = pic.ws_debug_step(x0, rhs)
    assert np.array_equal(out, out2)
    out_o, _ = N.forward(theta.astype(np.float64), x0)
    err = np.abs(out.reshape(P, P) - out_o).max() / np.abs(out_o).max()
    print(f"P={P}: out {err:.2e}")
    assert err <= 2e-2


def test_scales_and_recording_controls():
    import pic_b200 as P
    import pic_configs as C
    w = C.cfg3(16)   # 64x64 cells, internal electrode, blob
    with P.Pic(C.library_config(w)) as pic:
        C.load_plasma(pic, w)
        for it in range(3):
            pic.step(it)
        with pytest.raises(P.PicError):
            pic.ws_train(1, 1e-3)            # nothing recorded yet
        pic.ws_record(4)                      # automatic scales
        for it in range(3, 10):
            pic.step(it)
        assert pic.ws_pairs() == 4            # ring buffer keeps the newest 4
        s = pic.ws_scales()
        assert all(v > 0 and np.isfinite(v) for v in s)
        pic.ws_record(0)                      # stop, keep the dataset
        pic.step(10)
        assert pic.ws_pairs() == 4
        loss = pic.ws_train(2, 1e-3)
        assert np.isfinite(loss) and loss > 0
        pic.ws_record(-1)                     # release
        assert pic.ws_pairs() == 0
        with pytest.raises(P.PicError):
            pic.ws_record(4, 1.0, -1.0, 1.0)  # scales: all positive or all zero


def test_training_and_same_state_guess(oracle):
    """Record pairs on the 128x128 version of the 1024x1024 workload (same
    per-cell physics), train, then solve each evaluation step twice from the
    same state: from the network's guess and from phi_{n-1}."""
    import pic_b200 as P
    import pic_configs as C
    w = C.cfg3(8)
    with P.Pic(C.library_config(w)) as pic:
        C.load_plasma(pic, w)
        for it in range(10):
            pic.step(it)
        pic.ws_record(48)
        for it in range(10, 59):
            pic.step(it)
        pic.ws_record(0)
        first = pic.ws_train(1, 1e-3)
        last = pic.ws_train(15, 1e-3)
        assert last < 0.5 * first, (first, last)
        GX = w.GX
        mask = oracle.electrode_mask(GX, GX, oracle.Electrodes(w.rects))
        it_l, it_p, ratio = [], [], []
        for it in range(59, 65):
            pic.zero_rho()
            for s in range(2):
                pic.charge_deposition(s)
            rho, phi_prev = pic.rho(), pic.phi()
            pic.set_poisson(P.SOLVER_MG_PCG, P.WARM_LEARNED, 1e-8, 500)
            pic.poisson_solve(it)
            nl, rl, _ = pic.poisson_stats()
            r0_l = pic.poisson_start_relres()
            phi_l, b = pic.phi(), pic.rho()
            pic.set_poisson(P.SOLVER_MG_PCG, P.WARM_PREVIOUS, 1e-8, 500)
            pic.set_phi(phi_prev)
            pic.set_rho(rho)
            pic.poisson_solve(it)
            npl, rp, _ = pic.poisson_stats()
            r0_p = pic.poisson_start_relres()
            phi_p = pic.phi()
            assert rl <= 1e-8 and rp <= 1e-8
            dxl = w.xmax / w.nx
            true_rel = oracle.reduced_relres(GX, GX, dxl, dxl, mask, b, phi_l)
            assert true_rel <= 1e-8
            assert np.abs(phi_l - phi_p).max() <= 1e-6 * np.abs(phi_p).max()
            it_l.append(nl)
            it_p.append(npl)
            ratio.append(r0_l / r0_p)
            for s in range(2):
                pic.move_particles(s, it)
    # the trained guess is a strictly better start: its starting residual is
    # below half of phi_{n-1}'s on average and below it on every step; the
    # iteration count may not move (the gain is in components the first
    # V-cycle removes), but it never grows
    assert np.mean(ratio) < 0.5 and max(ratio) < 1.0, ratio
    assert np.mean(it_l) <= np.mean(it_p), (it_l, it_p)
