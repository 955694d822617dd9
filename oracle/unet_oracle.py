"""FP64 numpy oracle of the warm-start network (test infrastructure only).

The reference (Kraken.jl) has no learned component, so there is no reference
file to follow here: this module restates, in plain numpy and FP64, the
network that `krakenn.jl_b200/csrc/kb_surrogate.cu` trains on the tensor
cores, so that the GPU forward pass and gradients can be checked against it.
It is pinned by central finite differences (`tests/test_unet_oracle.py`),
not by golden vectors.  Only tests and the bench's checks import it.

Conventions shared with the CUDA code:
  * activations NHWC; input 8 channels; head 16 channels of which 0..2 are
    the normalised (rho, ux, uy);
  * 3x3 convolutions with zero padding; weights W[cout][9*cin] with
    k = tap*cin + c and tap = (dy+1)*3 + (dx+1); bias b[cout]; the flat
    parameter array holds W then b for each layer in order;
  * ReLU after every convolution but the head, 2x2 average pooling,
    nearest-neighbour upsampling, skip concatenation [upsampled, skip];
  * loss = mean over pixels and the 3 channels of e^2 + gw ((e(x+1) - e(x))^2 +
    (e(y+1) - e(y))^2), e = pred - (t - off)*scale (gw = 0: mean-squared error).
"""
from __future__ import annotations

import numpy as np

IN_CH, OUT_CH = 8, 16
# tensor name -> (channel multiple of C, or -absolute, level)
TENSORS = {
    "in": (-IN_CH, 0), "e1a": (1, 0), "e1b": (1, 0), "p1": (1, 1), "e2a": (2, 1), "e2b": (2, 1),
    "p2": (2, 2), "e3a": (4, 2), "e3b": (4, 2), "p3": (4, 3), "ba": (8, 3), "bb": (8, 3),
    "d3a": (4, 2), "d3b": (4, 2), "d2a": (2, 1), "d2b": (2, 1), "d1a": (1, 0), "d1b": (1, 0),
    "out": (-OUT_CH, 0),
}
# (in1, in2 or None, out, relu, pooled input)
LAYERS = [
    ("in", None, "e1a", True, False), ("e1a", None, "e1b", True, False),
    ("p1", None, "e2a", True, True), ("e2a", None, "e2b", True, False),
    ("p2", None, "e3a", True, True), ("e3a", None, "e3b", True, False),
    ("p3", None, "ba", True, True), ("ba", None, "bb", True, False),
    ("bb", "e3b", "d3a", True, False), ("d3a", None, "d3b", True, False),
    ("d3b", "e2b", "d2a", True, False), ("d2a", None, "d2b", True, False),
    ("d2b", "e1b", "d1a", True, False), ("d1a", None, "d1b", True, False),
    ("d1b", None, "out", False, False),
]
POOL_OF = {"p1": "e1b", "p2": "e2b", "p3": "e3b"}


def channels(name: str, C: int) -> int:
    m = TENSORS[name][0]
    return -m if m < 0 else m * C


def layer_table(C: int):
    """Per layer (cin, cout, w_off, b_off) in the flat parameter array."""
    out, off = [], 0
    for in1, in2, o, _, _ in LAYERS:
        cin = channels(in1, C) + (channels(in2, C) if in2 else 0)
        cout = channels(o, C)
        out.append((cin, cout, off, off + cout * 9 * cin))
        off += cout * 9 * cin + cout
    return out, off


def _im2col(x):
    B, H, W, C = x.shape
    xp = np.zeros((B, H + 2, W + 2, C), dtype=x.dtype)
    xp[:, 1:-1, 1:-1] = x
    cols = [xp[:, 1 + dy:1 + dy + H, 1 + dx:1 + dx + W] for dy in (-1, 0, 1) for dx in (-1, 0, 1)]
    return np.concatenate(cols, axis=-1)


def _col2im(dcols, C):
    B, H, W, _ = dcols.shape
    dxp = np.zeros((B, H + 2, W + 2, C), dtype=dcols.dtype)
    t = 0
    for dy in (-1, 0, 1):
        for dx in (-1, 0, 1):
            dxp[:, 1 + dy:1 + dy + H, 1 + dx:1 + dx + W] += dcols[..., t * C:(t + 1) * C]
            t += 1
    return dxp[:, 1:-1, 1:-1]


def _up(x):
    return np.repeat(np.repeat(x, 2, axis=1), 2, axis=2)


def _up_grad(d):
    B, H, W, C = d.shape
    return d.reshape(B, H // 2, 2, W // 2, 2, C).sum(axis=(2, 4))


def _pool(x):
    B, H, W, C = x.shape
    return x.reshape(B, H // 2, 2, W // 2, 2, C).mean(axis=(2, 4))


def _pool_grad(d):
    return _up(d) * 0.25


def bf16(x):
    """Round to the nearest BFloat16 (ties to even) through FP32, as the GPU
    rounds its FP32 accumulators when it stores BF16 tensors."""
    a = np.ascontiguousarray(np.asarray(x, np.float64).astype(np.float32))
    b = a.view(np.uint32)
    r = ((b + np.uint32(0x7FFF) + ((b >> np.uint32(16)) & np.uint32(1))) &
         np.uint32(0xFFFF0000)).astype(np.uint32)
    return r.view(np.float32).astype(np.float64)


def _ident(x):
    return x


def _layer_input(acts, in1, in2):
    return np.concatenate([_up(acts[in1]), acts[in2]], axis=-1) if in2 else acts[in1]


def forward(params, x, C, round_bf16=False):
    """Returns (head output [B,H,W,16], activations dict).  With round_bf16
    every stored activation but the FP32 head output is rounded to BF16, at
    the points where the CUDA kernels store BF16."""
    rnd = bf16 if round_bf16 else _ident
    table, n = layer_table(C)
    assert params.size == n
    acts = {"in": np.asarray(x, np.float64)}
    for (in1, in2, o, relu, pooled), (cin, cout, wo, bo) in zip(LAYERS, table):
        if pooled:
            acts[in1] = rnd(_pool(acts[POOL_OF[in1]]))
        X = _layer_input(acts, in1, in2)
        Wm = params[wo:wo + cout * 9 * cin].reshape(cout, 9 * cin)
        y = _im2col(X) @ Wm.T + params[bo:bo + cout]
        acts[o] = rnd(np.maximum(y, 0.0)) if relu else y
    return acts["out"], acts


def normalised_target(target, scale, offset):
    """Planar [B][3][H][W] physical target -> NHWC normalised [B,H,W,3]."""
    t = np.moveaxis(np.asarray(target, np.float64), 1, -1)
    return (t - np.asarray(offset)) * np.asarray(scale)


def loss_and_grad(params, x, target, scale, offset, C, round_bf16=False, grad_weight=0.0):
    """Mean-squared error and its gradient with respect to the flat
    parameters.  With round_bf16 the activations and the activation gradients
    are rounded to BF16 where the CUDA kernels store them (the head gradient,
    each data gradient after its ReLU mask, the upsampling and skip sums);
    weight gradients stay unrounded, as the kernels keep them in FP32."""
    rnd = bf16 if round_bf16 else _ident
    table, n = layer_table(C)
    out, acts = forward(params, x, C, round_bf16)
    t = normalised_target(target, scale, offset)
    d = out[..., :3] - t
    M = d.shape[0] * d.shape[1] * d.shape[2]
    # e^2 + gw * (forward differences in x and y)^2, within each image
    dx = d[:, :, 1:] - d[:, :, :-1]
    dy = d[:, 1:, :] - d[:, :-1, :]
    loss = float((np.sum(d * d) + grad_weight * (np.sum(dx * dx) + np.sum(dy * dy))) / (3 * M))
    lap = np.zeros_like(d)                     # sum over neighbours of (e - e_neighbour)
    lap[:, :, :-1] -= dx
    lap[:, :, 1:] += dx
    lap[:, :-1, :] -= dy
    lap[:, 1:, :] += dy
    grads = np.zeros(n)
    g = {"out": np.zeros_like(out)}
    g["out"][..., :3] = rnd(2.0 * (d + grad_weight * lap) / (3 * M))
    dcat = {}
    for li in range(len(LAYERS) - 1, -1, -1):
        in1, in2, o, relu, pooled = LAYERS[li]
        cin, cout, wo, bo = table[li]
        dy = g[o]
        X = _layer_input(acts, in1, in2)
        cols = _im2col(X)
        Wm = params[wo:wo + cout * 9 * cin].reshape(cout, 9 * cin)
        grads[wo:wo + cout * 9 * cin] = (dy.reshape(-1, cout).T @ cols.reshape(-1, 9 * cin)).ravel()
        grads[bo:bo + cout] = dy.reshape(-1, cout).sum(axis=0)
        if li == 0:
            break
        dX = _col2im(dy @ Wm, cin)
        if not pooled:            # the input is a post-ReLU tensor (or a concat of two)
            dX = rnd(dX * (X > 0))
        else:
            dX = rnd(dX)
        if in2:
            c1 = channels(in1, C)
            g[in1] = rnd(_up_grad(dX[..., :c1]))
            dcat[in2] = dX[..., c1:]
        else:
            g[in1] = dX
        if pooled:
            src = POOL_OF[in1]
            g[src] = rnd(dcat[src] + _pool_grad(g[in1]) * (acts[src] > 0))
    return loss, grads


def cavity_inputs(re, H, W, n_nodes):
    """The network input of lid-driven cavities (same channels as the CUDA kernel)."""
    re = np.asarray(re, np.float64)
    x = np.zeros((len(re), H, W, IN_CH))
    h = np.arange(H)[:, None]
    w = np.arange(W)[None, :]
    x[..., 0] = ((w == 0) | (w == W - 1) | (h == 0)).astype(float)
    x[..., 1] = (np.broadcast_to(h, (H, W)) == H - 1).astype(float)
    x[..., 2] = ((np.log(re) - np.log(100.0)) / np.log(32.0))[:, None, None]
    x[..., 3] = n_nodes / 512.0
    x[..., 4] = np.broadcast_to(2.0 * (w + 0.5) / W - 1.0, (H, W))
    x[..., 5] = np.broadcast_to(2.0 * (h + 0.5) / H - 1.0, (H, W))
    return x
