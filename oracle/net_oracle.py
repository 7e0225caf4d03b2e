"""CPU restatement (float64, numpy) of the learned warm start's network: the forward pass, the masked mean-squared-error
loss and its gradient with respect to every parameter, for the same layer table and flat parameter layout as the CUDA
network (bowshock_b200/csrc/net.cu, declared in include/bowshock_b200.h).

Test infrastructure only: the GPU tests compare the tensor-core forward and backward passes with it, and its own
backward pass is pinned by central finite differences (tests/test_net_oracle.py). There is no reference counterpart (the
reference has no learned component), so this restatement is the network's oracle. It is written independently of the
CUDA path: convolutions as explicit tap sums, the input gradient scattered back tap by tap (the CUDA path uses im2col
GEMMs and a flipped-kernel convolution)."""
from __future__ import annotations

import numpy as np

NET_IN, NET_OUT, NET_OUT_PAD, NET_CELLS, SLOPE = 16, 6, 16, 2048, 0.1
H_OUT, W_OUT = 32, 64


def layers():
    """Layer table: dicts with fc, cin, cout, H, W, up, act, kin, woff, boff (offsets into the flat parameter vector)."""
    L = []

    def fc(cin, cout):
        L.append(dict(fc=1, cin=cin, cout=cout, H=1, W=1, up=0, act=1, kin=cin))

    def cv(cin, cout, H, W, up, act):
        L.append(dict(fc=0, cin=cin, cout=cout, H=H, W=W, up=up, act=act, kin=9 * cin))

    fc(NET_IN, 256)
    fc(256, 4 * 8 * 128)
    cv(128, 128, 4, 8, 0, 1)
    cv(128, 128, 4, 8, 0, 1)
    cv(128, 128, 8, 16, 1, 1)
    cv(128, 128, 8, 16, 0, 1)
    cv(128, 64, 16, 32, 1, 1)
    cv(64, 64, 16, 32, 0, 1)
    cv(64, 64, 32, 64, 1, 1)
    cv(64, 64, 32, 64, 0, 1)
    cv(64, NET_OUT_PAD, 32, 64, 0, 0)
    off = 0
    for l in L:
        l["woff"] = off
        off += l["cout"] * l["kin"]
        l["boff"] = off
        off += l["cout"]
        off = (off + 7) & ~7
    return L, off


def init_params(seed=0, L=None, n=None):
    """He-uniform weights for the leaky ReLU (gain sqrt(2 / (1 + slope^2))), zero biases; the output layer scaled down."""
    if L is None:
        L, n = layers()
    rng = np.random.default_rng(seed)
    p = np.zeros(n, dtype=np.float32)
    for k, l in enumerate(L):
        fan_in = l["kin"]
        gain = np.sqrt(2.0 / (1.0 + SLOPE ** 2)) if l["act"] else 0.1
        bound = gain * np.sqrt(3.0 / fan_in)
        p[l["woff"]:l["woff"] + l["cout"] * l["kin"]] = rng.uniform(-bound, bound, l["cout"] * l["kin"]).astype(np.float32)
    return p


def _lrelu(z):
    return np.where(z > 0.0, z, SLOPE * z)


def _up(x, up):
    return x.repeat(2, axis=1).repeat(2, axis=2) if up else x


def _conv_forward(x, w, b):
    """3x3 'same' convolution of NHWC x with w [cout, 3, 3, cin] as a sum over the nine taps."""
    B, H, W, C = x.shape
    xp = np.zeros((B, H + 2, W + 2, C))
    xp[:, 1:-1, 1:-1] = x
    y = np.zeros((B, H, W, w.shape[0])) + b
    for ky in range(3):
        for kx in range(3):
            y += xp[:, ky:ky + H, kx:kx + W, :] @ w[:, ky, kx, :].T
    return y


def forward(params, x, L=None, bf16=False):
    """x [B, 16] -> (out [B, 32, 64, 16] linear output, cache of every layer's input and output). bf16: round every
    activated layer's output to BF16, as the tensor-core path stores its activations."""
    if L is None:
        L, _ = layers()
    p = np.asarray(params, dtype=np.float64)
    h = np.asarray(x, dtype=np.float64)
    cache = []
    B = h.shape[0]
    for l in L:
        W = p[l["woff"]:l["woff"] + l["cout"] * l["kin"]].reshape(l["cout"], l["kin"])
        b = p[l["boff"]:l["boff"] + l["cout"]]
        if l["fc"]:
            xin = h.reshape(B, -1)
            z = xin @ W.T + b
        else:
            xin = h.reshape(B, l["H"] >> l["up"], l["W"] >> l["up"], l["cin"])
            z = _conv_forward(_up(xin, l["up"]), W.reshape(l["cout"], 3, 3, l["cin"]), b)
        y = _lrelu(z) if l["act"] else z
        if bf16 and l["act"]:
            y = bf16_round(y.astype(np.float32)).astype(np.float64)
        cache.append((xin, y))
        h = y
    return h.reshape(B, H_OUT, W_OUT, NET_OUT_PAD), cache


def loss_and_grad(params, x, target, mask, L=None, bf16=False):
    """Masked mean squared error over [B, 2048, 6] (mean over every entry, masked ones counting 0) and its gradient.
    bf16: the tensor-core path's roundings (BF16 activations, BF16 output gradients of every layer), the rest float64."""
    if L is None:
        L, n = layers()
    else:
        n = len(params)
    p = np.asarray(params, dtype=np.float64)
    out, cache = forward(p, x, L, bf16=bf16)
    B = out.shape[0]
    o = out.reshape(B, NET_CELLS, NET_OUT_PAD)[:, :, :NET_OUT]
    t = np.asarray(target, dtype=np.float64).reshape(B, NET_CELLS, NET_OUT)
    m = (np.asarray(mask).reshape(1, NET_CELLS, 1) != 0).astype(np.float64)
    count = B * NET_CELLS * NET_OUT
    e = (o - t) * m
    loss = float(np.sum(e * e) / count)
    g = np.zeros((B, NET_CELLS, NET_OUT_PAD))
    g[:, :, :NET_OUT] = 2.0 * e / count
    grad = np.zeros(n)
    gy = g.reshape(B, H_OUT, W_OUT, NET_OUT_PAD)
    for k in range(len(L) - 1, -1, -1):
        l = L[k]
        xin, y = cache[k]
        gz = gy * np.where(y > 0.0, 1.0, SLOPE) if l["act"] else gy
        if bf16:
            gz = bf16_round(gz.astype(np.float32)).astype(np.float64)
        W = p[l["woff"]:l["woff"] + l["cout"] * l["kin"]].reshape(l["cout"], l["kin"])
        if l["fc"]:
            gz2 = gz.reshape(B, l["cout"])
            grad[l["woff"]:l["woff"] + l["cout"] * l["kin"]] = (gz2.T @ xin).ravel()
            grad[l["boff"]:l["boff"] + l["cout"]] = gz2.sum(0)
            gx = gz2 @ W
        else:
            xu = _up(xin, l["up"])
            Bn, H, Wd, C = xu.shape
            xp = np.zeros((Bn, H + 2, Wd + 2, C))
            xp[:, 1:-1, 1:-1] = xu
            w4 = W.reshape(l["cout"], 3, 3, C)
            gw = np.zeros_like(w4)
            gxp = np.zeros_like(xp)
            for ky in range(3):
                for kx in range(3):
                    patch = xp[:, ky:ky + H, kx:kx + Wd, :].reshape(-1, C)
                    gw[:, ky, kx, :] = gz.reshape(-1, l["cout"]).T @ patch
                    gxp[:, ky:ky + H, kx:kx + Wd, :] += gz @ w4[:, ky, kx, :]
            grad[l["woff"]:l["woff"] + l["cout"] * l["kin"]] = gw.ravel()
            grad[l["boff"]:l["boff"] + l["cout"]] = gz.reshape(-1, l["cout"]).sum(0)
            gxu = gxp[:, 1:-1, 1:-1]
            gx = gxu.reshape(Bn, H // 2, 2, Wd // 2, 2, C).sum(axis=(2, 4)) if l["up"] else gxu
        gy = gx.reshape(cache[k - 1][1].shape) if k > 0 else gx
    return loss, grad


def bf16_round(a):
    """Round float32 values to the nearest BF16 (ties to even), returned as float32."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)
