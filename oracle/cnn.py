"""ORACLE — test infrastructure only, never part of the product path.

numpy restatement of the learned-preconditioner network pieces (no reference
counterpart: the reference has no learned preconditioner), used to check the
sm_100a kernels: BF16 rounding and the 3x3 NHWC convolution in FP32 on
BF16-rounded values.
"""
import numpy as np


def to_bf16(a):
    """Round float32 values to the nearest BF16 (ties to even), returned as float32."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def bf16_ulp(a):
    """Spacing of BF16 values in the binade of each |a| (8 significant bits)."""
    m = np.maximum(np.abs(np.asarray(a, dtype=np.float64)), 1e-30)
    return 2.0 ** (np.floor(np.log2(m)) - 7)


def conv3x3(x, w, bias=None):
    """y[n,h,w,co] = sum over taps (dy,dx) and ci of x[n,h+dy,w+dx,ci] * w[tap,co,ci]
    (+ bias[co]), zero padding, tap = (dy+1)*3 + (dx+1); float64 sums, FP32 result."""
    n, h, wd, ci = x.shape
    co = w.shape[1]
    xp = np.zeros((n, h + 2, wd + 2, ci), dtype=np.float64)
    xp[:, 1:-1, 1:-1, :] = x
    y = np.zeros((n, h, wd, co), dtype=np.float64)
    for tap in range(9):
        dy, dx = tap // 3 - 1, tap % 3 - 1
        patch = xp[:, 1 + dy:1 + dy + h, 1 + dx:1 + dx + wd, :]
        y += patch @ w[tap].astype(np.float64).T
    if bias is not None:
        y += bias
    return y.astype(np.float32)


# ---------------------------------------------------------------------------
# the learned preconditioner's network (ops_b200/csrc/lmg.h)
# ---------------------------------------------------------------------------
LAYERS = [(16, 16), (16, 32), (32, 32), (32, 64), (64, 64), (64, 64), (64, 64), (64, 32), (32, 16), (16, 16)]
C0, C1A, C1B, C2A, C2B, C3A, C3B, C2U, C1U, C0U = range(10)


def unpack(p):
    """Flat FP32 parameter vector -> ([(W [9,cout,cin], b [cout])...], wout [16], bout)."""
    out, o = [], 0
    for ci, co in LAYERS:
        W = p[o:o + 9 * co * ci].reshape(9, co, ci)
        o += 9 * co * ci
        b = p[o:o + co]
        o += co
        out.append((W, b))
    wout = p[o:o + 16]
    bout = p[o + 16]
    return out, wout, bout


def features(r, Kx, Ky, rx, ry):
    """r, Kx, Ky padded (n, h+2, w+2) float64 arrays -> x0 (n, h, w, 16), z, s."""
    a = rx * Kx[:, 1:-1, 1:-1]
    b = rx * Kx[:, 1:-1, 2:]
    c = ry * Ky[:, 1:-1, 1:-1]
    d = ry * Ky[:, 2:, 1:-1]
    D = 1.0 + a + b + c + d
    ri = r[:, 1:-1, 1:-1]
    z = ri / D
    s = np.sqrt(np.mean(ri ** 2, axis=(1, 2)))
    s = np.where(s > 0, s, 1.0)
    n, h, w = z.shape
    x0 = np.zeros((n, h, w, 16), dtype=np.float64)
    x0[..., 0] = ri / s[:, None, None]
    x0[..., 1] = a / D
    x0[..., 2] = b / D
    x0[..., 3] = c / D
    x0[..., 4] = d / D
    return x0, z, s


def pool(x):
    return 0.25 * (x[:, 0::2, 0::2] + x[:, 1::2, 0::2] + x[:, 0::2, 1::2] + x[:, 1::2, 1::2])


def up(x):
    return np.repeat(np.repeat(x, 2, axis=1), 2, axis=2)


def net_forward(p, r, Kx, Ky, rx, ry, bf16=True):
    """Forward pass; with bf16 every stored activation and the weights are
    rounded to BF16 where the kernels round them (FP32 products summed
    exactly otherwise); bf16=False gives the exact FP64 network. Returns M(r)
    on the interior (n, h, w) and the activations net_loss_grad needs."""
    L, wout, bout = unpack(p)
    q = (lambda x: to_bf16(np.asarray(x, dtype=np.float32)).astype(np.float64)) if bf16 else (lambda x: x)
    Wb = [(q(W.astype(np.float64)), b.astype(np.float64)) for W, b in L]
    cv = lambda x, l: q(np.maximum(conv64(x, Wb[l][0], Wb[l][1]), 0))
    x0, z, s = features(r, Kx, Ky, rx, ry)
    A = {"x0": q(x0)}
    A["e0"] = cv(A["x0"], C0)
    A["p1"] = q(pool(A["e0"]))
    A["a1"] = cv(A["p1"], C1A)
    A["e1"] = cv(A["a1"], C1B)
    A["p2"] = q(pool(A["e1"]))
    A["a2"] = cv(A["p2"], C2A)
    A["e2"] = cv(A["a2"], C2B)
    A["p3"] = q(pool(A["e2"]))
    A["a3"] = cv(A["p3"], C3A)
    A["h3"] = cv(A["a3"], C3B)
    A["u2"] = q(up(A["h3"]) + A["e2"])
    A["h2"] = cv(A["u2"], C2U)
    A["u1"] = q(up(A["h2"]) + A["e1"])
    A["h1"] = cv(A["u1"], C1U)
    A["u0"] = q(up(A["h1"]) + A["e0"])
    A["h0"] = cv(A["u0"], C0U)
    y = A["h0"] @ wout.astype(np.float64) + float(bout)
    M = z + s[:, None, None] * y
    A["z"], A["s"], A["W"] = z, s, [W for W, _ in Wb]
    return M, A


def conv64(x, W, b):
    """conv3x3 in float64 throughout (for the exact network)."""
    n, h, wd, ci = x.shape
    xp = np.zeros((n, h + 2, wd + 2, ci))
    xp[:, 1:-1, 1:-1, :] = x
    y = np.zeros((n, h, wd, W.shape[1]))
    for tap in range(9):
        dy, dx = tap // 3 - 1, tap % 3 - 1
        y += xp[:, 1 + dy:1 + dy + h, 1 + dx:1 + dx + wd, :] @ W[tap].T
    return y + b


def conv_bwd(x, W, g):
    """Gradients of y = conv3x3(x, W) + b given g = dL/dy: (dx, dW, db)."""
    n, h, wd, ci = x.shape
    co = W.shape[1]
    xp = np.zeros((n, h + 2, wd + 2, ci))
    xp[:, 1:-1, 1:-1, :] = x
    dxp = np.zeros_like(xp)
    dW = np.zeros((9, co, ci))
    g2 = g.reshape(-1, co)
    for tap in range(9):
        dy, dx = tap // 3 - 1, tap % 3 - 1
        patch = xp[:, 1 + dy:1 + dy + h, 1 + dx:1 + dx + wd, :].reshape(-1, ci)
        dW[tap] = g2.T @ patch
        dxp[:, 1 + dy:1 + dy + h, 1 + dx:1 + dx + wd, :] += (g2 @ W[tap]).reshape(n, h, wd, ci)
    return dxp[:, 1:-1, 1:-1, :], dW, g2.sum(axis=0)


def apply_A(u, Kx, Ky, rx, ry):
    """The heat operator on interior arrays u (n, h, w), zero outside."""
    a = rx * Kx[:, 1:-1, 1:-1]
    b = rx * Kx[:, 1:-1, 2:]
    c = ry * Ky[:, 1:-1, 1:-1]
    d = ry * Ky[:, 2:, 1:-1]
    up_ = np.pad(u, ((0, 0), (1, 1), (1, 1)))
    return ((1 + a + b + c + d) * u - a * up_[:, 1:-1, :-2] - b * up_[:, 1:-1, 2:] - c * up_[:, :-2, 1:-1]
            - d * up_[:, 2:, 1:-1])


def net_loss_grad(p, r, Kx, Ky, e, rx, ry, bf16=True, anorm=False):
    """loss = mean_n ||M(r_n) - e_n||^2 / ||e_n||^2 (or, with anorm, the same
    ratio in the A-norm: d.Ad / e.Ae with d = M(r_n) - e_n) and its gradient
    (float64) with respect to the flat parameters, back-propagated through the
    stored (rounded) activations."""
    L, wout, bout = unpack(p)
    M, A = net_forward(p, r, Kx, Ky, rx, ry, bf16)
    Wb = A["W"]
    ei = e[:, 1:-1, 1:-1]
    n = r.shape[0]
    d = M - ei
    if anorm:
        Ad = apply_A(d, Kx, Ky, rx, ry)
        E = np.sum(ei * apply_A(ei, Kx, Ky, rx, ry), axis=(1, 2))
        loss = float(np.mean(np.sum(d * Ad, axis=(1, 2)) / E))
        dM = 2.0 / n * Ad / E[:, None, None]
    else:
        E = np.sum(ei ** 2, axis=(1, 2))
        loss = float(np.mean(np.sum(d ** 2, axis=(1, 2)) / E))
        dM = 2.0 / n * d / E[:, None, None]
    dy = dM * A["s"][:, None, None]
    grads = [None] * 10
    dwout = np.einsum("nhw,nhwc->c", dy, A["h0"])
    dbout = dy.sum()
    dh0 = dy[..., None] * wout.astype(np.float64)

    def layer(l, g_post, out, x):
        g = g_post * (out > 0)
        dx, dW, db = conv_bwd(x, Wb[l], g)
        grads[l] = (dW, db)
        return dx

    du0 = layer(C0U, dh0, A["h0"], A["u0"])
    dh1 = du0[:, 0::2, 0::2] + du0[:, 1::2, 0::2] + du0[:, 0::2, 1::2] + du0[:, 1::2, 1::2]
    du1 = layer(C1U, dh1, A["h1"], A["u1"])
    dh2 = du1[:, 0::2, 0::2] + du1[:, 1::2, 0::2] + du1[:, 0::2, 1::2] + du1[:, 1::2, 1::2]
    du2 = layer(C2U, dh2, A["h2"], A["u2"])
    dh3 = du2[:, 0::2, 0::2] + du2[:, 1::2, 0::2] + du2[:, 0::2, 1::2] + du2[:, 1::2, 1::2]
    da3 = layer(C3B, dh3, A["h3"], A["a3"])
    dp3 = layer(C3A, da3, A["a3"], A["p3"])
    de2 = du2 + 0.25 * up(dp3)
    da2 = layer(C2B, de2, A["e2"], A["a2"])
    dp2 = layer(C2A, da2, A["a2"], A["p2"])
    de1 = du1 + 0.25 * up(dp2)
    da1 = layer(C1B, de1, A["e1"], A["a1"])
    dp1 = layer(C1A, da1, A["a1"], A["p1"])
    de0 = du0 + 0.25 * up(dp1)
    layer(C0, de0, A["e0"], A["x0"])
    flat = []
    for dW, db in grads:
        flat += [dW.ravel(), db]
    flat += [dwout, np.array([dbout])]
    return loss, np.concatenate(flat)


def init_params(seed=5, out_scale=0.0):
    """He-normal weights, zero biases; output layer scaled by out_scale."""
    rng = np.random.default_rng(seed)
    parts = []
    for ci, co in LAYERS:
        parts += [rng.standard_normal(9 * co * ci) * np.sqrt(2.0 / (9 * ci)), np.zeros(co)]
    parts += [rng.standard_normal(16) * out_scale, np.zeros(1)]
    return np.concatenate(parts).astype(np.float32)
