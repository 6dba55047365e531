"""CPU oracle of the motion-proposal network (test infrastructure only).

A numpy restatement, in float64, of what riv2_b200/csrc/riv_nn.cu computes: the network input
(correlation volume, predictor prior map and predictor values of k_prop_features), the forward
pass, the head's loss and its gradient, and the backward pass.  Values are rounded to bf16 at
the same points as on the device (every stored activation and gradient operand), so the
device's f32 accumulation is the only difference; the tests compare within a tolerance.

The network has no counterpart in the reference encoder: it proposes candidate MVs for the
search the reference performs in process_block_hex (enc/motion/scalar.rs:546-636).
"""
from __future__ import annotations

import numpy as np

FEAT, WIN_OFF, NPRED = 24, 24, 7
HIN = {1: 24, 2: 12, 3: 6, 4: 6}
HOUT = {1: 12, 2: 6, 3: 6, 4: 3}
STRIDE = {1: 2, 2: 2, 3: 1, 4: 2}


ROUND = True  # False: no bf16 rounding anywhere (for the finite-difference check of the oracle itself)


def bf16(x):
    """Round to the nearest bf16 (ties to even), returned as float64."""
    if not ROUND:
        return np.asarray(x, np.float64)
    a = np.ascontiguousarray(np.asarray(x, np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def bf16_bits_to_f64(bits):
    return (np.asarray(bits, np.uint16).astype(np.uint32) << 16).view(np.float32).astype(np.float64)


# ---------------------------------------------------------------------------------------
# Network input
# ---------------------------------------------------------------------------------------

def _med3(a, b, c):
    return max(min(a, b), min(max(a, b), c))


def features(cur_y, ref_y, prev_coded=None):
    """cur_y, ref_y: (H, W) uint8; prev_coded: (nmb, 4) int8 or None.  Returns (feat (n, 24, 24, 2),
    pred16 (n, 16)) as float64 holding bf16 values."""
    H, W = cur_y.shape
    bw, bh = W // 16, H // 16
    n = bw * bh
    cur = cur_y.astype(np.int32)
    ref = ref_y.astype(np.int32)
    feat = np.zeros((n, FEAT, FEAT, 2))
    pred16 = np.zeros((n, 16))
    for mb in range(n):
        bx, by = mb % bw, mb // bw
        x0, y0 = bx * 16, by * 16
        X = x0 - WIN_OFF + 2 * np.arange(32)
        Y = y0 - WIN_OFF + 2 * np.arange(32)
        xa, xb = np.clip(X, 0, W - 1), np.clip(X + 1, 0, W - 1)
        ya, yb = np.clip(Y, 0, H - 1), np.clip(Y + 1, 0, H - 1)
        R = (ref[np.ix_(ya, xa)] + ref[np.ix_(ya, xb)] + ref[np.ix_(yb, xa)] + ref[np.ix_(yb, xb)] + 2) >> 2
        c = cur[y0:y0 + 16, x0:x0 + 16]
        Cb = (c[0::2, 0::2] + c[0::2, 1::2] + c[1::2, 0::2] + c[1::2, 1::2] + 2) >> 2
        sad = np.zeros((FEAT, FEAT), np.int64)
        for v in range(FEAT):
            for u in range(FEAT):
                sad[v, u] = np.abs(Cb - R[v:v + 8, u:u + 8]).sum()
        f0 = 1.0 - np.minimum(sad, 2048).astype(np.float32) * np.float32(1.0 / 1024.0)
        px, py = [0] * NPRED, [0] * NPRED
        if prev_coded is not None:
            def get(xx, yy):
                if xx < 0 or yy < 0 or xx >= bw or yy >= bh:
                    return 0, 0
                cc = prev_coded[yy * bw + xx].astype(np.int32)
                return 2 * cc[0] + cc[2], 2 * cc[1] + cc[3]
            for k, (xx, yy) in enumerate(((bx - 1, by), (bx, by - 1), (bx + 1, by - 1), (bx - 1, by - 1), (bx, by))):
                px[k], py[k] = get(xx, yy)
            px[6], py[6] = _med3(px[0], px[1], px[2]), _med3(py[0], py[1], py[2])
        f1 = np.zeros((FEAT, FEAT), np.float32)
        for k in range(NPRED):
            u, v = ((px[k] + 2) >> 2) + 12, ((py[k] + 2) >> 2) + 12
            if 0 <= u < FEAT and 0 <= v < FEAT:
                f1[v, u] = 1.0
        feat[mb, :, :, 0] = bf16(f0)
        feat[mb, :, :, 1] = bf16(f1)
        vals = np.zeros(16, np.float32)
        for k in range(NPRED):
            vals[2 * k] = np.float32(px[k]) * np.float32(1.0 / 64.0)
            vals[2 * k + 1] = np.float32(py[k]) * np.float32(1.0 / 64.0)
        pred16[mb] = bf16(vals)
    return feat, pred16


# ---------------------------------------------------------------------------------------
# Layers
# ---------------------------------------------------------------------------------------

def im2col(x, layer):
    """x: (n, hin, hin, c) -> (n * hout^2, 9 * c), column k = tap * c + channel."""
    n, hin, _, c = x.shape
    ho, s = HOUT[layer], STRIDE[layer]
    xp = np.zeros((n, hin + 2, hin + 2, c))
    xp[:, 1:-1, 1:-1] = x
    cols = np.zeros((n, ho, ho, 9, c))
    for t in range(9):
        ky, kx = t // 3, t % 3
        cols[:, :, :, t] = xp[:, ky:ky + s * ho:s, kx:kx + s * ho:s][:, :ho, :ho]
    return cols.reshape(n * ho * ho, 9 * c)


def col2im(dcol, n, layer, c=32):
    """Adjoint of im2col: (n * hout^2, 9 * c) -> (n, hin, hin, c)."""
    hin, ho, s = HIN[layer], HOUT[layer], STRIDE[layer]
    d = dcol.reshape(n, ho, ho, 9, c)
    xp = np.zeros((n, hin + 2, hin + 2, c))
    for t in range(9):
        ky, kx = t // 3, t % 3
        xp[:, ky:ky + s * ho:s, kx:kx + s * ho:s][:, :ho, :ho] += d[:, :, :, t]
    return xp[:, 1:-1, 1:-1]


def unpack(p, layout):
    """Split a flat f32 parameter vector into weights (bf16-rounded, real columns only) and biases."""
    out = {}
    for name, (off, r, c, fan) in layout.items():
        if c == 1:
            out[name] = np.asarray(p[off:off + r], np.float64)
        else:
            out[name] = bf16(p[off:off + r * c]).reshape(r, c)[:, :fan]
    return out


def forward(P, feat, pred16):
    """Returns (output (n, 16), saved activations)."""
    n = feat.shape[0]
    a = {0: feat}
    x = feat
    for layer in (1, 2, 3, 4):
        cols = im2col(x, layer)
        z = cols @ P[f"w{layer}"].T + P[f"b{layer}"]
        ho = HOUT[layer]
        x = bf16(np.maximum(z, 0.0)).reshape(n, ho, ho, 32)
        a[layer] = x
    x1 = np.concatenate([x.reshape(n, 288), pred16], axis=1)  # 304 real inputs
    h1 = bf16(np.maximum(x1 @ P["f1"].T + P["bf1"], 0.0))
    h2 = bf16(np.maximum(h1 @ P["f2"].T + P["bf2"], 0.0))
    o = h2 @ P["f3"].T + P["bf3"]
    a.update(x1=x1, h1=h1, h2=h2)
    return o, a


def head_loss(o, tmv, tskip):
    """Mean loss and dO (n, 16), the head of k_nn_head_loss."""
    n = o.shape[0]
    t = tmv.astype(np.float64) / 32.0
    dl = 1.0 / 32.0
    g = np.zeros((n, 16))
    total = 0.0
    for r in range(n):
        h, gx, gy = [], [], []
        for k in range(4):
            e = (o[r, 2 * k] - t[r, 0], o[r, 2 * k + 1] - t[r, 1])
            hh = [0.5 * v * v / dl if abs(v) < dl else abs(v) - 0.5 * dl for v in e]
            gg = [v / dl if abs(v) < dl else np.sign(v) for v in e]
            h.append(hh[0] + hh[1])
            gx.append(gg[0])
            gy.append(gg[1])
        best = int(np.argmin(h))
        for k in range(4):
            w = 1.0 if k == best else 0.05
            total += w * h[k]
            g[r, 2 * k] = w * gx[k] / n
            g[r, 2 * k + 1] = w * gy[k] / n
        z, y = o[r, 8], float(tskip[r])
        total += 0.5 * (max(z, 0.0) - z * y + np.log1p(np.exp(-abs(z))))
        g[r, 8] = 0.5 * (1.0 / (1.0 + np.exp(-z)) - y) / n
    return total / n, g


def backward(P, a, g_out):
    """Gradients (same keys as P, real columns only) from dO, with the device's bf16 roundings."""
    n = g_out.shape[0]
    G = {}
    dz = bf16(g_out)
    acts = (("f3", "bf3", a["h2"]), ("f2", "bf2", a["h1"]), ("f1", "bf1", a["x1"]))
    for i, (wn, bn, x) in enumerate(acts):
        G[bn] = dz.sum(axis=0)
        G[wn] = dz.T @ x
        dx = dz @ P[wn]
        if i < 2:  # through the ReLU that produced this layer's input
            dz = bf16(dx * (x > 0))
    dxc = dx[:, :288].reshape(n, 3, 3, 32)
    dz = bf16(dxc * (a[4] > 0)).reshape(-1, 32)
    for layer in (4, 3, 2, 1):
        G[f"b{layer}"] = dz.sum(axis=0)
        cols = im2col(a[layer - 1], layer)
        G[f"w{layer}"] = dz.T @ cols
        if layer == 1:
            break
        dcol = dz @ P[f"w{layer}"]
        dxi = col2im(dcol, n, layer)
        dz = bf16(dxi * (a[layer - 1] > 0)).reshape(-1, 32)
    return G
