"""FP64 NumPy restatement of the learned warm-start network (test infrastructure).

Same architecture, parameter layout and loss as
bmp-6th-sem_b200/csrc/warmstart.cu; activations and gradient images are rounded
to bfloat16 (round-to-nearest-even) exactly where the CUDA kernels store
bf16, so the GPU forward/backward can be checked against it.  Used only by
tests/ as the checker.

Parameter layout (flat float vector):
  input conv   w[tap][ci(3)][co(32)], b[32]
  9 x conv     w[tap][ci(32)][co(32)], b[32]
  output conv  w[tap][ci(32)], b[1]
tap = ky*3 + kx, offset (ky-1, kx-1).
"""
import numpy as np

C = 32
N_CONV32 = 9
IN_W, IN_B = 9 * 3 * C, C
W32, B32 = 9 * C * C, C
OUT_W, OUT_B = 9 * C, 1
N_PARAMS = IN_W + IN_B + N_CONV32 * (W32 + B32) + OUT_W + OUT_B


def bf16(x):
    """Round to bfloat16 (nearest even), returned as float64."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    bits = a.view(np.uint32).astype(np.uint64)
    r = ((bits + 0x7FFF + ((bits >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32).astype(np.float64)


def unpack(theta):
    theta = np.asarray(theta, dtype=np.float64)
    o = 0
    w_in = theta[o:o + IN_W].reshape(9, 3, C); o += IN_W
    b_in = theta[o:o + IN_B]; o += IN_B
    convs = []
    for _ in range(N_CONV32):
        w = theta[o:o + W32].reshape(9, C, C); o += W32
        b = theta[o:o + B32]; o += B32
        convs.append((w, b))
    w_out = theta[o:o + OUT_W].reshape(9, C); o += OUT_W
    b_out = theta[o:o + OUT_B]; o += OUT_B
    return w_in, b_in, convs, w_out, b_out


def _shift(x, dy, dx):
    """y[p] = x[p + (dy, dx)] with zero padding; x is [H, W, ...]."""
    H, W = x.shape[:2]
    y = np.zeros_like(x)
    ys, yd = (slice(0, H - dy), slice(dy, H)) if dy >= 0 else (slice(-dy, H), slice(0, H + dy))
    xs, xd = (slice(0, W - dx), slice(dx, W)) if dx >= 0 else (slice(-dx, W), slice(0, W + dx))
    y[ys, xs] = x[yd, xd]
    return y


def conv(x, w, b):
    """out[p][co] = b[co] + sum_tap sum_ci w[tap][ci][co] x[p + d_tap][ci]."""
    out = np.zeros(x.shape[:2] + (w.shape[-1],))
    for tap in range(9):
        out += _shift(x, tap // 3 - 1, tap % 3 - 1) @ w[tap]
    return out + b


def conv_dx(dy, w):
    """dx[q][ci] = sum_tap sum_co w[tap][ci][co] dy[q - d_tap][co]."""
    dx = np.zeros(dy.shape[:2] + (w.shape[1],))
    for tap in range(9):
        dx += _shift(dy, -(tap // 3 - 1), -(tap % 3 - 1)) @ w[tap].T
    return dx


def conv_dw(x, dy):
    """dw[tap][ci][co] = sum_p x[p + d_tap][ci] dy[p][co]; db = sum_p dy."""
    dw = np.zeros((9, x.shape[-1], dy.shape[-1]))
    for tap in range(9):
        xs = _shift(x, tap // 3 - 1, tap % 3 - 1)
        dw[tap] = np.einsum("hwi,hwo->io", xs, dy)
    return dw, dy.sum(axis=(0, 1))


def pool(x, rnd=None):
    rnd = bf16 if rnd is None else rnd
    return rnd(0.25 * (x[0::2, 0::2] + x[0::2, 1::2] + x[1::2, 0::2] + x[1::2, 1::2]))


def up(x):
    return np.repeat(np.repeat(x, 2, axis=0), 2, axis=1)


def _identity(x):
    return np.asarray(x, dtype=np.float64)


def forward(theta, x0, exact=False):
    """x0: [P, P, 3].  Returns (out [P, P], cache).  exact=True skips every
    bfloat16 rounding (plain FP64 network, for gradient checks)."""
    bf16 = _identity if exact else globals()["bf16"]
    w_in, b_in, convs, w_out, b_out = unpack(theta)
    wb = [(bf16(w), b) for (w, b) in convs]
    x0 = bf16(x0)
    a = [None] * 11
    a[1] = bf16(np.maximum(conv(x0, w_in, b_in), 0))
    a[2] = bf16(np.maximum(conv(a[1], *wb[0]), 0))
    p1 = pool(a[2], bf16)
    a[3] = bf16(np.maximum(conv(p1, *wb[1]), 0))
    a[4] = bf16(np.maximum(conv(a[3], *wb[2]), 0))
    p2 = pool(a[4], bf16)
    a[5] = bf16(np.maximum(conv(p2, *wb[3]), 0))
    a[6] = bf16(np.maximum(conv(a[5], *wb[4]), 0))
    u1 = bf16(up(a[6]) + a[4])
    a[7] = bf16(np.maximum(conv(u1, *wb[5]), 0))
    a[8] = bf16(np.maximum(conv(a[7], *wb[6]), 0))
    u0 = bf16(up(a[8]) + a[2])
    a[9] = bf16(np.maximum(conv(u0, *wb[7]), 0))
    a[10] = bf16(np.maximum(conv(a[9], *wb[8]), 0))
    out = conv(a[10], w_out[:, :, None], b_out)[..., 0]
    return out, dict(x0=x0, a=a, p1=p1, p2=p2, u0=u0, u1=u1, wb=wb, w_out=w_out)


def stencil(v, beta):
    """L(v) = (2 + 2 beta) v - (v_w + v_e) - beta (v_s + v_n), zero outside."""
    return ((2 + 2 * beta) * v - _shift(v, 0, -1) - _shift(v, 0, 1)
            - beta * (_shift(v, -1, 0) + _shift(v, 1, 0)))


def free_nodes(mask, GX, GY):
    """Non-electrode nodes off the outer ring (every wall node is an electrode)."""
    free = mask.reshape(GY, GX) == 0
    free[0, :] = free[-1, :] = free[:, 0] = free[:, -1] = False
    return free


def residual(out, rhs, mask, GX, GY, kappa, beta):
    """Scaled starting residual of PCG from the guess: r = rhs - kappa L(u) on
    free nodes, 0 elsewhere, with u = out on free nodes and 0 on electrodes."""
    free = free_nodes(mask, GX, GY)
    u = np.where(free, out[:GY, :GX], 0.0)
    return np.where(free, rhs.reshape(GY, GX) - kappa * stencil(u, beta), 0.0)


def loss_grad(theta, x0, rhs, mask, GX, GY, kappa, beta, exact=False):
    """Residual loss sum(r^2)/(GX*GY) of the guess (warmstart.cu k_resid) and
    its gradient w.r.t. theta.  Gradient images are rounded to bfloat16 where
    the CUDA kernels store them, unless exact=True.  Weight gradients are taken
    with respect to the bf16 working copies and applied to the FP32 masters
    (straight-through)."""
    bf16 = _identity if exact else globals()["bf16"]
    out, K = forward(theta, x0, exact)
    P = out.shape[0]
    n = GX * GY
    r = residual(out, rhs, mask, GX, GY, kappa, beta)
    loss = float((r * r).sum() / n)
    free = free_nodes(mask, GX, GY)
    dout = np.zeros((P, P))
    dout[:GY, :GX] = np.where(free, -2.0 * kappa / n * stencil(r, beta), 0.0)
    g = np.zeros(N_PARAMS)
    offs = [IN_W + IN_B + i * (W32 + B32) for i in range(N_CONV32)]
    o_out = IN_W + IN_B + N_CONV32 * (W32 + B32)
    a, wb = K["a"], K["wb"]

    def put(i, dw, db):
        g[offs[i]:offs[i] + W32] = dw.ravel()
        g[offs[i] + W32:offs[i] + W32 + B32] = db

    gate = lambda d, act: np.where(act > 0, d, 0.0)
    # output conv
    dwo, dbo = conv_dw(a[10], dout[..., None])
    g[o_out:o_out + OUT_W] = dwo[:, :, 0].ravel()
    g[o_out + OUT_W] = dbo[0]
    d10 = bf16(gate(conv_dx(dout[..., None], K["w_out"][:, :, None]), a[10]))
    put(8, *conv_dw(a[9], d10))
    d9 = bf16(gate(conv_dx(d10, wb[8][0]), a[9]))
    put(7, *conv_dw(K["u0"], d9))
    du0 = bf16(conv_dx(d9, wb[7][0]))
    d8 = bf16(gate(du0[0::2, 0::2] + du0[0::2, 1::2] + du0[1::2, 0::2] + du0[1::2, 1::2], a[8]))
    put(6, *conv_dw(a[7], d8))
    d7 = bf16(gate(conv_dx(d8, wb[6][0]), a[7]))
    put(5, *conv_dw(K["u1"], d7))
    du1 = bf16(conv_dx(d7, wb[5][0]))
    d6 = bf16(gate(du1[0::2, 0::2] + du1[0::2, 1::2] + du1[1::2, 0::2] + du1[1::2, 1::2], a[6]))
    put(4, *conv_dw(a[5], d6))
    d5 = bf16(gate(conv_dx(d6, wb[4][0]), a[5]))
    put(3, *conv_dw(K["p2"], d5))
    dp2 = bf16(conv_dx(d5, wb[3][0]))
    d4 = bf16(gate(du1 + 0.25 * up(dp2), a[4]))
    put(2, *conv_dw(a[3], d4))
    d3 = bf16(gate(conv_dx(d4, wb[2][0]), a[3]))
    put(1, *conv_dw(K["p1"], d3))
    dp1 = bf16(conv_dx(d3, wb[1][0]))
    d2 = bf16(gate(du0 + 0.25 * up(dp1), a[2]))
    put(0, *conv_dw(a[1], d2))
    d1 = bf16(gate(conv_dx(d2, wb[0][0]), a[1]))
    dwi, dbi = conv_dw(K["x0"], d1)
    g[:IN_W] = dwi.ravel()
    g[IN_W:IN_W + IN_B] = dbi
    return loss, g, out
