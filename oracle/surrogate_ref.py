"""NumPy restatement of the surrogate's layers, forward and backward, in
FP64.  TEST INFRASTRUCTURE ONLY: the checker of the CUDA kernels of
dsmc_erlend_b200/csrc/surrogate.cu and of the network's gradients.

The surrogate has no counterpart in the reference (it predicts fields for
the warm start), so this file restates the textbook operations: a 3x3
convolution with zero padding 1 and stride 1 in NHWC with weights
[Cout][3][3][Cin], its input and weight gradients, 2x2 average pooling,
nearest 2x upsampling, ReLU and a masked mean squared error.
"""
from __future__ import annotations

import numpy as np


def conv3x3(x: np.ndarray, w: np.ndarray, b: np.ndarray | None = None) -> np.ndarray:
    """x (n, h, w, cin), w (cout, 3, 3, cin) -> (n, h, w, cout)."""
    n, h, wd, _ = x.shape
    xp = np.pad(x, ((0, 0), (1, 1), (1, 1), (0, 0)))
    y = np.zeros((n, h, wd, w.shape[0]))
    for kh in range(3):
        for kw in range(3):
            y += np.einsum("nhwc,oc->nhwo", xp[:, kh:kh + h, kw:kw + wd, :], w[:, kh, kw, :])
    if b is not None:
        y += b
    return y


def conv3x3_dgrad(dy: np.ndarray, w: np.ndarray) -> np.ndarray:
    """Input gradient of conv3x3: (n, h, w, cout) -> (n, h, w, cin)."""
    n, h, wd, _ = dy.shape
    dx = np.zeros((n, h + 2, wd + 2, w.shape[3]))
    for kh in range(3):
        for kw in range(3):
            dx[:, kh:kh + h, kw:kw + wd, :] += np.einsum("nhwo,oc->nhwc", dy, w[:, kh, kw, :])
    return dx[:, 1:-1, 1:-1, :]


def conv3x3_wgrad(dy: np.ndarray, x: np.ndarray) -> np.ndarray:
    """Weight gradient of conv3x3: (cout, 3, 3, cin)."""
    n, h, wd, _ = x.shape
    xp = np.pad(x, ((0, 0), (1, 1), (1, 1), (0, 0)))
    dw = np.zeros((dy.shape[3], 3, 3, x.shape[3]))
    for kh in range(3):
        for kw in range(3):
            dw[:, kh, kw, :] = np.einsum("nhwo,nhwc->oc", dy, xp[:, kh:kh + h, kw:kw + wd, :])
    return dw


def pool2(x: np.ndarray) -> np.ndarray:
    n, h, w, c = x.shape
    return x.reshape(n, h // 2, 2, w // 2, 2, c).mean(axis=(2, 4))


def pool2_bwd(dy: np.ndarray) -> np.ndarray:
    return np.repeat(np.repeat(dy, 2, axis=1), 2, axis=2) / 4.0


def up2(x: np.ndarray) -> np.ndarray:
    return np.repeat(np.repeat(x, 2, axis=1), 2, axis=2)


def up2_bwd(dy: np.ndarray) -> np.ndarray:
    n, h, w, c = dy.shape
    return dy.reshape(n, h // 2, 2, w // 2, 2, c).sum(axis=(2, 4))


def mse(out: np.ndarray, target: np.ndarray, mask: np.ndarray, k: int):
    """Masked MSE over the first k channels; returns (loss, d loss / d out)."""
    d = (out[..., :k] - target) * mask[..., None]
    scale = 1.0 / (k * max(mask.sum(), 1.0))
    g = np.zeros_like(out)
    g[..., :k] = 2.0 * d * scale
    return float((d * d).sum() * scale), g


def round_bf16(a) -> np.ndarray:
    """Rounds to bfloat16 (nearest, ties to even) and back to FP64."""
    u = np.asarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def network_forward(params: dict, x: np.ndarray, layers, bf16: bool = True) -> dict:
    """The encoder-decoder of dsmc_erlend_b200.surrogate in FP64: `layers`
    is its LAYERS table; returns every activation by name.  With bf16 the
    values the kernels store in bfloat16 are rounded at the same points
    (pooled inputs, activations, sums with a skip), so that only the order
    of the FP32 accumulations differs from the kernels."""
    r = round_bf16 if bf16 else (lambda v: v)
    acts = {"x": x}
    for name, src, op, cin, cout, relu, skip in layers:
        a = acts[src]
        if op == "pool":
            a = r(pool2(a))
        elif op == "up":
            a = up2(a)
        y = conv3x3(a, params[name + ".w"], params[name + ".b"])
        last = name == layers[-1][0]
        if relu:
            y = np.maximum(y, 0.0)
        acts[name + ".relu"] = r(y)
        if not last:
            y = acts[name + ".relu"]
        if skip:
            y = r(y + acts[skip])
        acts[name + ".in"] = a
        acts[name] = y
    return acts


def network_backward(params: dict, acts: dict, dout: np.ndarray, layers,
                     bf16: bool = True) -> dict:
    """Gradients of every weight and bias for the output gradient dout, the
    activation gradients rounded where the kernels store them."""
    r = round_bf16 if bf16 else (lambda v: v)
    grads = {}
    dacts = {layers[-1][0]: dout}
    for name, src, op, cin, cout, relu, skip in reversed(layers):
        dy = dacts.pop(name)
        if skip:
            dacts[skip] = r(dacts.get(skip, 0.0) + dy)
        if relu:
            dy = dy * (acts[name + ".relu"] > 0)
        grads[name + ".w"] = conv3x3_wgrad(dy, acts[name + ".in"])
        grads[name + ".b"] = dy.sum(axis=(0, 1, 2))
        if src == "x":
            continue
        da = r(conv3x3_dgrad(dy, params[name + ".w"]))
        if op == "pool":
            da = r(pool2_bwd(da))
        elif op == "up":
            da = r(up2_bwd(da))
        dacts[src] = r(dacts.get(src, 0.0) + da)
    return grads
