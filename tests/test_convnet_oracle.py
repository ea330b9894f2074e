"""The conv-network oracle (oracle/convnet.py) against an independent FP64
implementation of the same encoder-decoder in torch (CPU autograd).

The oracle is the checker of the GPU warm-start kernels, so it is pinned here
first: in exact mode (no bfloat16 rounding) its output and its hand-written
backward pass must equal torch's to FP64 round-off; in bf16 mode (the GPU's
storage precision) they stay within bf16 error of the exact values.
"""
import numpy as np
import pytest


def torch_net(theta, x0, rhs, mask, GX, GY, kappa, beta):
    import torch
    import torch.nn.functional as F
    import convnet as N
    t = torch.tensor(np.asarray(theta, np.float64), requires_grad=True)
    o = 0

    def take(n):
        nonlocal o
        v = t[o:o + n]
        o += n
        return v

    def as_conv_weight(w, cin, cout):
        # oracle layout w[tap][ci][co], tap = ky*3 + kx -> torch [co][ci][ky][kx]
        return w.reshape(3, 3, cin, cout).permute(3, 2, 0, 1)

    w_in = as_conv_weight(take(N.IN_W), 3, N.C)
    b_in = take(N.IN_B)
    convs = [(as_conv_weight(take(N.W32), N.C, N.C), take(N.B32)) for _ in range(N.N_CONV32)]
    w_out = as_conv_weight(take(N.OUT_W), N.C, 1)
    b_out = take(N.OUT_B)
    x = torch.tensor(np.asarray(x0, np.float64)).permute(2, 0, 1)[None]
    cv = lambda v, w, b: F.conv2d(v, w, b, padding=1)
    up = lambda v: v.repeat_interleave(2, dim=2).repeat_interleave(2, dim=3)
    a1 = torch.relu(cv(x, w_in, b_in))
    a2 = torch.relu(cv(a1, *convs[0]))
    a3 = torch.relu(cv(F.avg_pool2d(a2, 2), *convs[1]))
    a4 = torch.relu(cv(a3, *convs[2]))
    a5 = torch.relu(cv(F.avg_pool2d(a4, 2), *convs[3]))
    a6 = torch.relu(cv(a5, *convs[4]))
    a7 = torch.relu(cv(up(a6) + a4, *convs[5]))
    a8 = torch.relu(cv(a7, *convs[6]))
    a9 = torch.relu(cv(up(a8) + a2, *convs[7]))
    a10 = torch.relu(cv(a9, *convs[8]))
    out = cv(a10, w_out, b_out)[0, 0]
    # residual loss, written with an explicit sparse-free stencil in torch
    free = np.asarray(N.free_nodes(mask, GX, GY))
    fr = torch.tensor(free)
    u = torch.where(fr, out[:GY, :GX], torch.zeros(()))
    up_ = F.pad(u, (1, 1, 1, 1))
    Lu = (2 + 2 * beta) * u - up_[1:-1, :-2] - up_[1:-1, 2:] - beta * (up_[:-2, 1:-1] + up_[2:, 1:-1])
    r = torch.where(fr, torch.tensor(rhs.reshape(GY, GX)) - kappa * Lu, torch.zeros(()))
    loss = (r * r).sum() / (GX * GY)
    loss.backward()
    return loss.item(), t.grad.numpy(), out.detach().numpy()


def make_case(GX, GY, P, seed):
    import convnet as N
    rng = np.random.default_rng(seed)
    theta = np.zeros(N.N_PARAMS)
    o = 0
    for n, fan in [(N.IN_W, 27), (N.IN_B, 0)] + [(N.W32, 288), (N.B32, 0)] * N.N_CONV32 + \
            [(N.OUT_W, 288), (N.OUT_B, 0)]:
        theta[o:o + n] = rng.uniform(-1, 1, n) * (np.sqrt(6.0 / fan) if fan else 0.05)
        o += n
    x0 = np.zeros((P, P, 3))
    x0[:GY, :GX, 0] = rng.normal(0, 1, (GY, GX))
    x0[:GY, :GX, 1] = rng.normal(0, 1, (GY, GX))
    mask = np.zeros(GX * GY, np.uint8)
    m2 = mask.reshape(GY, GX)
    m2[0, :] = m2[-1, :] = m2[:, 0] = m2[:, -1] = 1
    m2[GY // 3:GY // 2, GX // 3:GX // 2] = 1
    x0[:GY, :GX, 2] = m2
    x0[:GY, :GX, 1] *= 1 - m2
    rhs = rng.normal(0, 0.5, GX * GY) * (1 - mask)
    return theta, x0, rhs, mask


@pytest.mark.parametrize("GX,GY,P", [(13, 13, 16), (17, 14, 20)])
def test_exact_oracle_matches_torch_autograd(GX, GY, P):
    import convnet as N
    theta, x0, rhs, mask = make_case(GX, GY, P, seed=GX * 7 + GY)
    kappa, beta = 0.7, 1.3
    loss, g, out = N.loss_grad(theta, x0, rhs, mask, GX, GY, kappa, beta, exact=True)
    loss_t, g_t, out_t = torch_net(theta, x0, rhs, mask, GX, GY, kappa, beta)
    assert np.abs(out - out_t).max() <= 1e-12 * max(1.0, np.abs(out_t).max())
    assert abs(loss - loss_t) <= 1e-12 * loss_t
    assert np.abs(g - g_t).max() <= 1e-10 * np.abs(g_t).max()


def test_bf16_oracle_stays_near_exact():
    """Storing activations and gradient images in bf16 moves the output by
    about 1% and the gradient by about 10% (2-norm) while keeping its
    direction (cosine >= 0.98): the network trains in bf16 as in FP64."""
    import convnet as N
    theta, x0, rhs, mask = make_case(13, 13, 16, seed=3)
    loss_e, g_e, out_e = N.loss_grad(theta, x0, rhs, mask, 13, 13, 0.5, 1.0, exact=True)
    loss_b, g_b, out_b = N.loss_grad(theta, x0, rhs, mask, 13, 13, 0.5, 1.0)
    assert np.abs(out_b - out_e).max() <= 0.05 * np.abs(out_e).max()
    assert np.linalg.norm(g_b - g_e) <= 0.2 * np.linalg.norm(g_e)
    assert g_b @ g_e >= 0.98 * np.linalg.norm(g_b) * np.linalg.norm(g_e)
    assert abs(loss_b - loss_e) <= 0.05 * loss_e


def test_bf16_rounding_is_nearest_even():
    import convnet as N
    one = np.float32(1.0)
    ulp = np.float32(2.0 ** -7)
    assert N.bf16(one + ulp * np.float32(0.5)) == 1.0          # tie -> even
    assert N.bf16(one + ulp * np.float32(1.5)) == 1.0 + 2 * ulp  # tie -> even (up)
    assert N.bf16(one + ulp * np.float32(0.51)) == 1.0 + ulp
    assert N.bf16(-3.0) == -3.0
