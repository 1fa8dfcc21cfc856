"""FP64 NumPy restatement of libairt's U-Net (TEST INFRASTRUCTURE ONLY).

The network has no counterpart in the reference; this module is the checker
for the GPU forward and backward kernels.  It follows the same architecture,
parameter packing and rounding points as the GPU implementation: the input
image, every activation and the masked output gradients are rounded to BF16,
the weights enter the products as BF16; products and sums are FP64.
"""
from __future__ import annotations

import numpy as np


EXACT = False  # True: no BF16 rounding (for finite-difference checks)


def bf16(x):
    """Round to BF16 (round to nearest even), returned as float64."""
    if EXACT:
        return np.asarray(x, np.float64)
    a = np.ascontiguousarray(np.asarray(x, np.float32)).view(np.uint32)
    r = ((a >> 16) & 1) + 0x7FFF
    return ((a + r) & 0xFFFF0000).astype(np.uint32).view(np.float32).astype(np.float64)


def layer_shapes(base, levels):
    """(cin, cout) of every 3x3 convolution in forward order."""
    shapes = []
    for l in range(levels):
        cin = 1 if l == 0 else base << (l - 1)
        shapes += [(cin, base << l), (base << l, base << l)]
    for l in range(levels - 2, -1, -1):
        cin = (base << (l + 1)) + (base << l)
        shapes += [(cin, base << l), (base << l, base << l)]
    return shapes


def unpack(params, base, levels):
    off = 0
    convs = []
    for cin, cout in layer_shapes(base, levels):
        W = params[off:off + cout * 9 * cin].reshape(cout, 9 * cin).astype(np.float64)
        off += cout * 9 * cin
        b = params[off:off + cout].astype(np.float64)
        off += cout
        convs.append((W, b))
    hw = params[off:off + base].astype(np.float64)
    hb = float(params[off + base])
    return convs, hw, hb


def im2col(X):
    """X [B,H,W,C] -> [B*H*W, 9*C] with K index (kh*3+kw)*C + ci, zero pad."""
    B, H, W, Cc = X.shape
    Xp = np.zeros((B, H + 2, W + 2, Cc))
    Xp[:, 1:-1, 1:-1, :] = X
    cols = [Xp[:, kh:kh + H, kw:kw + W, :] for kh in range(3) for kw in range(3)]
    return np.concatenate(cols, axis=3).reshape(B * H * W, 9 * Cc)


def col2im(dcol, shape):
    B, H, W, Cc = shape
    d = dcol.reshape(B, H, W, 9, Cc)
    dXp = np.zeros((B, H + 2, W + 2, Cc))
    for kh in range(3):
        for kw in range(3):
            dXp[:, kh:kh + H, kw:kw + W, :] += d[:, :, :, kh * 3 + kw, :]
    return dXp[:, 1:-1, 1:-1, :]


def pool(X):
    B, H, W, Cc = X.shape
    return X.reshape(B, H // 2, 2, W // 2, 2, Cc).max(axis=(2, 4))


def pool_back(X, dY):
    """Gradient to the first maximal element of each 2x2 window (row-major)."""
    B, H, W, Cc = X.shape
    dX = np.zeros_like(X)
    Y = pool(X)
    taken = np.zeros(Y.shape, bool)
    for i in range(2):
        for j in range(2):
            hit = (X[:, i::2, j::2, :] == Y) & ~taken
            dX[:, i::2, j::2, :] += np.where(hit, dY, 0.0)
            taken |= hit
    return dX


def up(X):
    return X.repeat(2, axis=1).repeat(2, axis=2)


def up_back(dY):
    B, H, W, Cc = dY.shape
    return dY.reshape(B, H // 2, 2, W // 2, 2, Cc).sum(axis=(2, 4))


def images_to_nhwc(imgs, H, W):
    """[B, H*W] column-major images -> [B,H,W,1] with h = row index."""
    B = imgs.shape[0]
    return imgs.reshape(B, W, H).transpose(0, 2, 1)[..., None]


def forward_backward(params, x_in, target, base, levels, H, W):
    """Loss and the flattened gradient (same packing as params)."""
    convs, hw, hb = unpack(params, base, levels)
    B = x_in.shape[0]
    X0 = bf16(images_to_nhwc(x_in, H, W))
    T = images_to_nhwc(target, H, W)[..., 0]
    acts = {}
    ci = 0
    tape = []

    def conv(X, idx):
        Wm, b = convs[idx]
        col = im2col(X)
        Y = bf16(np.maximum(col @ bf16(Wm).T + b, 0.0))
        Bn, Hh, Ww, _ = X.shape
        Y = Y.reshape(Bn, Hh, Ww, -1)
        tape.append((idx, X, Y))
        return Y

    ea, eb, pl = [None] * levels, [None] * levels, [None] * levels
    for l in range(levels):
        inp = X0 if l == 0 else pool(eb[l - 1])
        pl[l] = inp
        ea[l] = conv(inp, ci); ci += 1
        eb[l] = conv(ea[l], ci); ci += 1
    prev = eb[levels - 1]
    cats, da, db = {}, {}, {}
    for l in range(levels - 2, -1, -1):
        cats[l] = np.concatenate([up(prev), eb[l]], axis=3)
        da[l] = conv(cats[l], ci); ci += 1
        db[l] = conv(da[l], ci); ci += 1
        prev = db[l]
    out = db[0] @ hw + hb
    P = B * H * W
    diff = out - T
    loss = float(np.mean(diff * diff))
    dout = 2.0 * diff / P
    ghw = np.einsum("bhw,bhwc->c", dout, db[0])
    ghb = float(dout.sum())
    grads_W = [None] * len(convs)
    grads_b = [None] * len(convs)
    dact = {}

    def add(key, g):
        dact[key] = dact.get(key, 0.0) + g

    add(("db", 0), dout[..., None] * hw)

    def conv_back(idx, X, Y, dY, need_dx):
        Wm, _ = convs[idx]
        dYm = bf16(np.where(Y > 0, dY, 0.0)).reshape(-1, Y.shape[3])
        col = im2col(X)
        grads_W[idx] = dYm.T @ col
        grads_b[idx] = dYm.sum(axis=0)
        if not need_dx:
            return None
        dcol = dYm @ bf16(Wm)
        return col2im(dcol, X.shape)

    nconv = len(convs)
    ci = nconv - 1
    for l in range(0, levels - 1):
        dda = conv_back(ci, da[l], db[l], dact[("db", l)], True); ci -= 1
        dcat = conv_back(ci, cats[l], da[l], dda, True); ci -= 1
        C1 = (base << (l + 1))
        key = ("eb", levels - 1) if l == levels - 2 else ("db", l + 1)
        add(key, up_back(dcat[..., :C1]))
        add(("eb", l), dcat[..., C1:])
    for l in range(levels - 1, -1, -1):
        dea = conv_back(ci, ea[l], eb[l], dact[("eb", l)], True); ci -= 1
        dinp = conv_back(ci, pl[l], ea[l], dea, l > 0); ci -= 1
        if l > 0:
            add(("eb", l - 1), pool_back(eb[l - 1], dinp))
    flat = []
    for (cin, cout), gW, gb in zip(layer_shapes(base, levels), grads_W, grads_b):
        flat += [gW.ravel(), gb]
    flat += [ghw, [ghb]]
    return loss, np.concatenate([np.asarray(f, np.float64).ravel() for f in flat]), out
