"""CPU restatement of the learned closure's network and data kernels.  TEST INFRASTRUCTURE.

Only tests and bench.py's CPU legs use this module.  The closure has no
reference counterpart (the reference runs the plain method only); this file
states what ssmdlbm_b200/csrc/mlp.cu and closure.cu compute so that their
results can be checked:

- the network 12 -> 64 -> 64 -> 2 with GELU in its tanh form
  (z/2 (1 + tanh(sqrt(2/pi) (z + 0.044715 z^3))), Hendrycks & Gimpel 2016),
  in FP64 apart from the bf16 rounding of every tensor-core operand
  (standardised features, weights, hidden activations, dZ2), which is
  emulated; the kernel's tanh is the SFU's tanh.approx.f32 (absolute error
  about 2^-11), so an activation near a bf16 rounding boundary may round the
  other way there;
- its loss and gradient (the backward pass written out by hand; the weight
  and bias gradients take dZ1, dZ2 and dR rounded to bf16, the operands of
  the kernel's gradient MMAs) and Adam;
- features, 2x box filter and training targets, in FP32 arithmetic on
  [z][y][x] numpy arrays.
"""
from __future__ import annotations

import numpy as np

IN, HID, OUT, K1 = 12, 64, 2, 16
oW1 = 0
oB1 = oW1 + HID * K1
oW2 = oB1 + HID
oB2 = oW2 + HID * HID
oW3 = oB2 + HID
oB3 = oW3 + OUT * HID
PARAMS = oB3 + OUT
oMean = PARAMS
oInvStd = oMean + IN
oScale = oInvStd + IN
oOffset = oScale + OUT
NET = oOffset + OUT


def bf16(x) -> np.ndarray:
    """Round float32 values to bfloat16 (nearest, ties to even), returned as float32."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return (r & 0xFFFFFFFF).astype(np.uint32).view(np.float32).reshape(a.shape)


G0 = np.sqrt(2.0 / np.pi)
G1 = 0.044715


def gelu(z):
    return 0.5 * z * (1.0 + np.tanh(G0 * (z + G1 * z ** 3)))


def gelu_grad(z):
    t = np.tanh(G0 * (z + G1 * z ** 3))
    return 0.5 * (1.0 + t) + 0.5 * z * (1.0 - t * t) * G0 * (1.0 + 3.0 * G1 * z * z)


def unpack(net):
    net = np.asarray(net, dtype=np.float32)
    return dict(
        W1=net[oW1:oB1].reshape(HID, K1), b1=net[oB1:oW2], W2=net[oW2:oB2].reshape(HID, HID), b2=net[oB2:oW3],
        W3=net[oW3:oB3].reshape(OUT, HID), b3=net[oB3:PARAMS], mean=net[oMean:oInvStd], inv_std=net[oInvStd:oScale],
        scale=net[oScale:oOffset], offset=net[oOffset:NET])


def init_net(seed: int = 0) -> np.ndarray:
    """Fan-in scaled normal weights, zero biases, identity normalisation."""
    rng = np.random.default_rng(seed)
    net = np.zeros(NET, np.float32)
    W1 = np.zeros((HID, K1), np.float32)
    W1[:, :IN] = rng.normal(0, 1 / np.sqrt(IN), (HID, IN))
    net[oW1:oB1] = W1.reshape(-1)
    net[oW2:oB2] = rng.normal(0, 1 / np.sqrt(HID), HID * HID)
    net[oW3:oB3] = rng.normal(0, 1 / np.sqrt(HID), OUT * HID)
    net[oInvStd:oScale] = 1.0
    net[oScale:oOffset] = 1.0
    return net


def forward(net, feat, emulate_bf16: bool = True):
    """Raw output r [n, 2] and the intermediate values (for backward)."""
    P = unpack(net)
    rb = bf16 if emulate_bf16 else (lambda a: np.asarray(a, np.float32))
    x = np.zeros((feat.shape[0], K1), np.float32)
    x[:, :IN] = (np.asarray(feat, np.float32) - P["mean"]) * P["inv_std"]
    xb = rb(x).astype(np.float64)
    W1 = rb(P["W1"]).astype(np.float64)
    W2 = rb(P["W2"]).astype(np.float64)
    W3 = rb(P["W3"]).astype(np.float64)
    z1 = xb @ W1.T + P["b1"].astype(np.float64)
    h1 = rb(gelu(z1).astype(np.float32)).astype(np.float64)
    z2 = h1 @ W2.T + P["b2"].astype(np.float64)
    h2 = rb(gelu(z2).astype(np.float32)).astype(np.float64)
    r = h2 @ W3.T + P["b3"].astype(np.float64)
    return r, dict(x=xb, z1=z1, h1=h1, z2=z2, h2=h2, W2=W2, W3=W3, rb=rb)


def predict(net, feat, emulate_bf16: bool = True):
    P = unpack(net)
    r, _ = forward(net, feat, emulate_bf16)
    return P["scale"].astype(np.float64) * r + P["offset"].astype(np.float64)


def loss_and_grad(net, feat, target, weight=None, emulate_bf16: bool = True):
    """L = (1/n) sum w (r - (t - offset)/scale)^2 and dL/dparams (PARAMS values)."""
    P = unpack(net)
    n = feat.shape[0]
    r, c = forward(net, feat, emulate_bf16)
    tn = (np.asarray(target, np.float64) - P["offset"]) / P["scale"]
    w = np.ones_like(tn) if weight is None else np.asarray(weight, np.float64)
    e = r - tn
    loss = float(np.sum(w * e * e) / n)
    dr = 2.0 * w * e / n
    dh2 = dr @ P["W3"].astype(np.float64)        # CUDA cores in the kernel: fp32 W3
    dz2 = dh2 * gelu_grad(c["z2"])
    dz2b = c["rb"](dz2.astype(np.float32)).astype(np.float64)
    dh1 = dz2b @ c["W2"]                          # tensor cores: bf16 dZ2, bf16 W2
    dz1 = dh1 * gelu_grad(c["z1"])
    # the weight and bias gradients: sums over the rows of products of bf16
    # operands (tensor cores; the bias sums through a row of ones)
    dz1b = c["rb"](dz1.astype(np.float32)).astype(np.float64)
    drb = c["rb"](dr.astype(np.float32)).astype(np.float64)
    g = np.zeros(PARAMS, np.float64)
    gW1 = dz1b.T @ c["x"]
    gW1[:, IN:] = 0.0
    g[oW1:oB1] = gW1.reshape(-1)
    g[oB1:oW2] = dz1b.sum(0)
    g[oW2:oB2] = (dz2b.T @ c["h1"]).reshape(-1)
    g[oB2:oW3] = dz2b.sum(0)
    g[oW3:oB3] = (drb.T @ c["h2"]).reshape(-1)
    g[oB3:PARAMS] = drb.sum(0)
    return loss, g


def adam(net, g, m, v, t, lr, b1=0.9, b2=0.999, eps=1e-8):
    net = np.array(net, np.float64)
    m = b1 * np.asarray(m, np.float64) + (1 - b1) * g
    v = b2 * np.asarray(v, np.float64) + (1 - b2) * g * g
    mh = m / (1 - b1 ** t)
    vh = v / (1 - b2 ** t)
    net[:PARAMS] -= lr * mh / (np.sqrt(vh) + eps)
    return net, m, v


# ----------------------------------------------------------------- fields
def _shift(a, d, axis, periodic):
    """a at index i + d along axis (periodic wrap or clamp to the faces)."""
    n = a.shape[axis]
    idx = np.arange(n) + d
    idx = np.mod(idx, n) if periodic else np.clip(idx, 0, n - 1)
    return np.take(a, idx, axis=axis)


def _grad(a, per):
    """Central differences of a [z][y][x] array; per = (px, py, pz)."""
    f32 = np.float32
    gx = f32(0.5) * (_shift(a, 1, 2, per[0]) - _shift(a, -1, 2, per[0]))
    gy = f32(0.5) * (_shift(a, 1, 1, per[1]) - _shift(a, -1, 1, per[1]))
    gz = f32(0.5) * (_shift(a, 1, 0, per[2]) - _shift(a, -1, 0, per[2]))
    return gx, gy, gz


def features(rho, ux, uy, uz, phi, per, nu_w, nu_o):
    """The 12 per-cell features, [cells, 12] float32 in x-fastest cell order."""
    f32 = np.float32
    gx, gy, gz = _grad(phi, per)
    gm = np.sqrt(gx * gx + gy * gy + gz * gz)
    lap = (_shift(phi, 1, 2, per[0]) + _shift(phi, -1, 2, per[0]) + _shift(phi, 1, 1, per[1]) +
           _shift(phi, -1, 1, per[1]) + _shift(phi, 1, 0, per[2]) + _shift(phi, -1, 0, per[2]) - f32(6) * phi)
    d = [_grad(u, per) for u in (ux, uy, uz)]  # d[i][j] = d u_i / d x_j
    inv = f32(1) / (gm + f32(1e-9))
    n = (gx * inv, gy * inv, gz * inv)
    ss = np.zeros_like(phi)
    nsn = np.zeros_like(phi)
    for a in range(3):
        for b in range(3):
            s = f32(0.5) * (d[a][b] + d[b][a])
            ss += s * s
            nsn += n[a] * s * n[b]
    wx, wy, wz = d[2][1] - d[1][2], d[0][2] - d[2][0], d[1][0] - d[0][1]
    cols = [phi, f32(4) * phi * (f32(1) - phi), gm, lap, np.sqrt(f32(2) * ss), np.sqrt(wx * wx + wy * wy + wz * wz),
            nsn, np.sqrt(ux * ux + uy * uy + uz * uz), uz, rho - f32(1), d[0][0] + d[1][1] + d[2][2],
            phi * f32(nu_o - nu_w) + f32(nu_w)]
    return np.stack([c.reshape(-1) for c in cols], axis=1).astype(np.float32)


def box_filter(rho, ux, uy, uz, phi, per):
    """2x box filter (FP64 sums): coarse (rho, ux, uy, uz, phi), tau (xx, yy, zz,
    xy, xz, yz) and the mean fine |grad phi|, each [Z][Y][X]."""
    def blk(a):
        a = np.asarray(a, np.float64)
        nz, ny, nx = a.shape
        return a.reshape(nz // 2, 2, ny // 2, 2, nx // 2, 2).mean(axis=(1, 3, 5))
    gx, gy, gz = _grad(phi, per)
    area = blk(np.sqrt(gx.astype(np.float64) ** 2 + gy.astype(np.float64) ** 2 + gz.astype(np.float64) ** 2))
    m = [blk(a) for a in (rho, ux, uy, uz, phi)]
    u64 = [np.asarray(a, np.float64) for a in (ux, uy, uz)]
    pairs = [(0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2)]
    tau = [blk(u64[i] * u64[j]) - m[1 + i] * m[1 + j] for i, j in pairs]
    return ([x.astype(np.float32) for x in m], [t.astype(np.float32) for t in tau], area.astype(np.float32))


def targets(coarse, tau, area, per, nut_max):
    """Training targets and weights, [cells, 2] each."""
    f32 = np.float32
    rho, ux, uy, uz, phi = coarse
    d = [_grad(u, per) for u in (ux, uy, uz)]
    t = [[tau[0], tau[3], tau[4]], [tau[3], tau[1], tau[5]], [tau[4], tau[5], tau[2]]]
    tr = (tau[0] + tau[1] + tau[2]) * f32(1.0 / 3.0)
    num = np.zeros_like(phi)
    den = np.zeros_like(phi)
    for a in range(3):
        for b in range(3):
            s = f32(0.5) * (d[a][b] + d[b][a])
            num += (t[a][b] - (tr if a == b else f32(0))) * s
            den += s * s
    nut = np.clip(-num / (f32(2) * den + f32(1e-12)), -nut_max, nut_max)
    gx, gy, gz = _grad(phi, per)
    gm = np.sqrt(gx * gx + gy * gy + gz * gz)
    cs = np.where(gm >= f32(1e-2), np.clip(f32(2) * area / np.maximum(gm, f32(1e-30)), 0.25, 4.0), f32(1))
    tg = np.stack([nut.reshape(-1), cs.reshape(-1)], 1).astype(np.float32)
    w = np.stack([np.ones(phi.size, np.float32), (f32(4) * phi * (f32(1) - phi) + f32(0.01)).reshape(-1)], 1)
    return tg, w.astype(np.float32)
