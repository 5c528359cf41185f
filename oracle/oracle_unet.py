"""CPU restatement of the learned preconditioner's U-Net -- TEST INFRASTRUCTURE ONLY.

The network has no counterpart in the reference.  This numpy version restates
the device network of easyfsi_b200/csrc/efsi_unet.cu (the same 15 layers,
channel counts, 3x3x3 zero-padded convolutions with tap t = (di + 1) * 9 +
(dj + 1) * 3 + (dk + 1), average pooling over the existing 2 x 2 x 2
children, nearest-neighbour upsampling, concatenation order [upsampled,
skip], masked mean-square loss on output channel 0) in float64, and rounds to
BF16 where the device stores BF16: the input, the weights, every layer output
and every pre-activation gradient.  It is used only by the tests, to check the
device forward pass, loss and parameter gradients; it is itself pinned by a
central finite-difference check (tests/test_oracle_unet.py).
"""

from __future__ import annotations

import numpy as np

CH = (16, 32, 48, 64)
IN_CH = 16
OUT_CH = 16
# (level, cin, cout, relu) per layer, in the device's order
LAYERS = (
    (0, IN_CH, 16, 1), (0, 16, 16, 1),
    (1, 16, 32, 1), (1, 32, 32, 1),
    (2, 32, 48, 1), (2, 48, 48, 1),
    (3, 48, 64, 1), (3, 64, 64, 1),
    (2, 64 + 48, 48, 1), (2, 48, 48, 1),
    (1, 48 + 32, 32, 1), (1, 32, 32, 1),
    (0, 32 + 16, 16, 1), (0, 16, 16, 1),
    (0, 16, OUT_CH, 0),
)


def bf16(a: np.ndarray) -> np.ndarray:
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    a32 = np.ascontiguousarray(a, dtype=np.float32)
    u = a32.view(np.uint32).astype(np.uint64)
    rounded = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return rounded.astype(np.uint32).view(np.float32).astype(np.float64)


def param_layout():
    """(weight offset, bias offset) per layer and the total count (device packing)."""
    offs, off = [], 0
    for _, cin, cout, _ in LAYERS:
        w = off
        off += cout * 27 * cin
        offs.append((w, off))
        off += cout
    return offs, off


def unpack(params: np.ndarray):
    offs, _ = param_layout()
    ws, bs = [], []
    for (w, b), (_, cin, cout, _) in zip(offs, LAYERS):
        ws.append(params[w : w + cout * 27 * cin].reshape(cout, 27, cin).astype(np.float64))
        bs.append(params[b : b + cout].astype(np.float64))
    return ws, bs


def _shifted(x: np.ndarray, t: int) -> np.ndarray:
    """x[v + off(t)] with zeros outside the volume; x is (nx, ny, nz, c)."""
    di, dj, dk = t // 9 - 1, (t // 3) % 3 - 1, t % 3 - 1
    nx, ny, nz, _ = x.shape
    out = np.zeros_like(x)
    src = x[max(di, 0) : nx + min(di, 0), max(dj, 0) : ny + min(dj, 0), max(dk, 0) : nz + min(dk, 0)]
    out[max(-di, 0) : nx + min(-di, 0), max(-dj, 0) : ny + min(-dj, 0), max(-dk, 0) : nz + min(-dk, 0)] = src
    return out


def conv(x: np.ndarray, w: np.ndarray, b: np.ndarray | None) -> np.ndarray:
    """y[v][co] = sum_t sum_ci x[v + off(t)][ci] w[co][t][ci] + b[co]."""
    y = np.zeros(x.shape[:3] + (w.shape[0],))
    for t in range(27):
        y += _shifted(x, t) @ w[:, t, :].T
    if b is not None:
        y += b
    return y


def conv_input_grad(g: np.ndarray, w: np.ndarray) -> np.ndarray:
    """Adjoint of conv in x: dx[u] = sum_t g[u - off(t)] w[:, t, :]."""
    dx = np.zeros(g.shape[:3] + (w.shape[2],))
    for t in range(27):
        dx += _shifted(g, 26 - t) @ w[:, t, :]
    return dx


def conv_weight_grad(x: np.ndarray, g: np.ndarray) -> np.ndarray:
    """dw[co][t][ci] = sum_v g[v][co] x[v + off(t)][ci]."""
    cin, cout = x.shape[3], g.shape[3]
    dw = np.zeros((cout, 27, cin))
    g2 = g.reshape(-1, cout)
    for t in range(27):
        dw[:, t, :] = g2.T @ _shifted(x, t).reshape(-1, cin)
    return dw


def coarse_shape(s):
    return tuple((n + 1) // 2 for n in s)


def pool(x: np.ndarray) -> np.ndarray:
    nx, ny, nz, c = x.shape
    cs = coarse_shape((nx, ny, nz))
    s = np.zeros(cs + (c,))
    cnt = np.zeros(cs + (1,))
    for a in range(2):
        for b_ in range(2):
            for d in range(2):
                part = x[a::2, b_::2, d::2]
                s[: part.shape[0], : part.shape[1], : part.shape[2]] += part
                cnt[: part.shape[0], : part.shape[1], : part.shape[2]] += 1
    return s / cnt


def pool_back(gc: np.ndarray, fine_shape) -> np.ndarray:
    cs = gc.shape[:3]
    cnt = np.zeros(cs + (1,))
    for a in range(2):
        for b_ in range(2):
            for d in range(2):
                n0 = len(range(a, fine_shape[0], 2))
                n1 = len(range(b_, fine_shape[1], 2))
                n2 = len(range(d, fine_shape[2], 2))
                cnt[:n0, :n1, :n2] += 1
    return up(gc / cnt, fine_shape)


def up(xc: np.ndarray, fine_shape) -> np.ndarray:
    i = np.arange(fine_shape[0]) // 2
    j = np.arange(fine_shape[1]) // 2
    k = np.arange(fine_shape[2]) // 2
    return xc[i][:, j][:, :, k]


def up_back(g: np.ndarray, coarse) -> np.ndarray:
    out = np.zeros(tuple(coarse) + (g.shape[3],))
    for a in range(2):
        for b_ in range(2):
            for d in range(2):
                part = g[a::2, b_::2, d::2]
                out[: part.shape[0], : part.shape[1], : part.shape[2]] += part
    return out


def _layer(x, w, b, relu, rounding):
    pre = conv(x, bf16(w) if rounding else w, b)
    y = np.maximum(pre, 0.0) if relu else pre
    return (bf16(y) if rounding else y), pre


def forward(params: np.ndarray, x: np.ndarray, rounding: bool = True):
    """Forward pass; x is (nx, ny, nz, 16).  Returns (output FP32-accumulated
    channels (nx, ny, nz, 16), cache for backward)."""
    ws, bs = unpack(params)
    shapes = [x.shape[:3]]
    for _ in range(3):
        shapes.append(coarse_shape(shapes[-1]))
    acts, ins = [None] * len(LAYERS), [None] * len(LAYERS)
    h = bf16(x) if rounding else x
    enc = []
    for lv in range(4):
        if lv > 0:
            h = pool(enc[-1])
            if rounding:
                h = bf16(h)
        for l in (2 * lv, 2 * lv + 1):
            ins[l] = h
            h, _ = _layer(h, ws[l], bs[l], LAYERS[l][3], rounding)
            acts[l] = h
        enc.append(h)
    coarse = enc[3]
    for q in range(3):
        lv = 2 - q
        cat = np.concatenate([up(coarse, shapes[lv]), enc[lv]], axis=3)
        h = cat
        for l in (8 + 2 * q, 9 + 2 * q):
            ins[l] = h
            h, _ = _layer(h, ws[l], bs[l], LAYERS[l][3], rounding)
            acts[l] = h
        coarse = h
    ins[14] = coarse
    out = conv(coarse, bf16(ws[14]) if rounding else ws[14], bs[14])
    acts[14] = out
    return out, {"ins": ins, "acts": acts, "shapes": shapes, "ws": ws}


def loss_and_grad(params: np.ndarray, x: np.ndarray, target: np.ndarray, mask: np.ndarray,
                  rounding: bool = True):
    """Masked mean-square loss of output channel 0 (mean over all voxels) and
    the gradient of every parameter, packed like the device's."""
    out, c = forward(params, x, rounding)
    n = out.shape[0] * out.shape[1] * out.shape[2]
    e = mask * (out[..., 0] - target)
    loss = float((e * e).sum() / n)
    dout = np.zeros_like(out)
    dout[..., 0] = 2.0 * e / n
    return loss, backward(params, c, dout, rounding)


def backward(params: np.ndarray, c: dict, dout: np.ndarray, rounding: bool = True) -> np.ndarray:
    ws = c["ws"]
    offs, total = param_layout()
    grad = np.zeros(total)
    shapes = c["shapes"]

    def layer_back(l, gy, need_input_grad=True):
        relu = LAYERS[l][3]
        g = gy * (c["acts"][l] > 0) if relu else gy
        if rounding:
            g = bf16(g)
        w0, b0 = offs[l]
        grad[w0 : w0 + ws[l].size] += conv_weight_grad(c["ins"][l], g).ravel()
        grad[b0 : b0 + ws[l].shape[0]] += g.reshape(-1, g.shape[3]).sum(axis=0)
        if not need_input_grad:
            return None
        return conv_input_grad(g, bf16(ws[l]) if rounding else ws[l])

    gskip = [np.zeros(tuple(shapes[lv]) + (CH[lv],)) for lv in range(4)]
    g = layer_back(14, dout)
    for q in (2, 1, 0):
        lv = 2 - q
        g = layer_back(9 + 2 * q, g)
        g = layer_back(8 + 2 * q, g)
        ca = CH[lv + 1]
        gskip[lv] += g[..., ca:]
        g = up_back(g[..., :ca], shapes[lv + 1])
    for lv in (3, 2, 1, 0):
        gin = g if lv == 3 else gskip[lv]
        g1 = layer_back(2 * lv + 1, gin)
        if lv == 0:
            layer_back(0, g1, need_input_grad=False)
            break
        g2 = layer_back(2 * lv, g1)
        gskip[lv - 1] += pool_back(g2, shapes[lv - 1])
    return grad
