"""The field surrogate: a BF16 convolutional encoder-decoder that maps a case
to its sampled field, trained on DSMC ensembles, whose predictions seed the
warm start (dsmc_init_warm).  The reference has no counterpart.

Every layer runs through the C ABI of include/dsmc_surrogate.h (CUDA kernels
in csrc/surrogate.cu: implicit-GEMM 3x3 convolutions on the tensor cores,
their input and weight gradients, pooling, upsampling, the masked loss and
Adam).  torch provides device memory only.

Canvas: the domain [X1, X2] x [Y1, Y2] on RES x RES cells (x-major like the
solver's fields).  Inputs (IN_CH channels, padded to 32): box mask, x and y
of the cell centre, Mach / 8, cos and sin of the angle, log10(n) - 17, the
wall model as three indicators, the CLL coefficients, box width and height /
6.  Network: LAYERS below (about 1.47M weights).  Outputs (8 of 32 channels): n / NFree, ux / UFree, uy / UFree,
T / (TFree (1 + Ma^2 / 3)) (the stagnation temperature, gamma = 5/3) and the
components Txx, Tyy, Tzz, Txy of the temperature tensor on the same scale.
"""
from __future__ import annotations

import ctypes as C
import math
import os
from pathlib import Path

import numpy as np

RES = 128
CH = 32
# The predicted channels: n, ux, uy, T and the temperature tensor's Txx,
# Tyy, Tzz, Txy (for dsmc_init_warm_tensor).
OUT_NAMES = ("n", "ux", "uy", "t", "txx", "tyy", "tzz", "txy")
OUT_CH = len(OUT_NAMES)
IN_CH = 14

# (name, source, resampling before the conv, cin, cout, relu, skip added after)
# Four levels of 128, 64, 32 and 16 pixels with 32, 64, 128 and 128 channels:
# two 3x3 convolutions per level at 128 and 64 pixels, three at 32 and 16,
# the decoder mirroring the encoder with additive skips from the last
# convolution of each encoder level; 1.47M weights.
LAYERS = [
    ("e1a", "x", None, 32, 32, True, None),
    ("e1b", "e1a", None, 32, 32, True, None),
    ("e2a", "e1b", "pool", 32, 64, True, None),
    ("e2b", "e2a", None, 64, 64, True, None),
    ("e3a", "e2b", "pool", 64, 128, True, None),
    ("e3b", "e3a", None, 128, 128, True, None),
    ("e3c", "e3b", None, 128, 128, True, None),
    ("ba", "e3c", "pool", 128, 128, True, None),
    ("bb", "ba", None, 128, 128, True, None),
    ("bc", "bb", None, 128, 128, True, None),
    ("d3a", "bc", "up", 128, 128, True, None),
    ("d3b", "d3a", None, 128, 128, True, None),
    ("d3c", "d3b", None, 128, 128, True, "e3c"),
    ("d2a", "d3c", "up", 128, 64, True, None),
    ("d2b", "d2a", None, 64, 64, True, "e2b"),
    ("d1a", "d2b", "up", 64, 32, True, None),
    ("d1b", "d1a", None, 32, 32, True, "e1b"),
    ("out", "d1b", None, 32, 32, False, None),
]

_LIB = Path(__file__).resolve().parent / "lib" / "libdsmc_surrogate.so"
_lib = None

_P = C.c_void_p
_SIGS = {
    "dsmc_sg_conv_fwd": [_P, _P, _P, _P, _P, _P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                         C.c_int, _P],
    "dsmc_sg_conv_dgrad": [_P, _P, _P, _P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _P],
    "dsmc_sg_conv_wgrad": [_P, _P, _P, _P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _P],
    "dsmc_sg_conv_fwd_skip": [_P, _P, _P, _P, _P, _P, C.c_int, C.c_int, C.c_int, C.c_int,
                              C.c_int, C.c_int, _P],
    "dsmc_sg_rotate_layers": [_P, _P, _P, _P, _P, C.c_int, _P],
    "dsmc_sg_relu_bwd": [_P, _P, C.c_int64, _P],
    "dsmc_sg_relu_bias_bwd": [_P, _P, _P, C.c_int, _P, C.c_int64, C.c_int, _P],
    "dsmc_sg_pool_bwd_acc": [_P, _P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _P],
    "dsmc_sg_up_bwd_acc": [_P, _P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _P],
    "dsmc_sg_pool_fwd": [_P, _P, C.c_int, C.c_int, C.c_int, C.c_int, _P],
    "dsmc_sg_pool_bwd": [_P, _P, C.c_int, C.c_int, C.c_int, C.c_int, _P],
    "dsmc_sg_up_fwd": [_P, _P, C.c_int, C.c_int, C.c_int, C.c_int, _P],
    "dsmc_sg_up_bwd": [_P, _P, C.c_int, C.c_int, C.c_int, C.c_int, _P],
    "dsmc_sg_add": [_P, _P, C.c_int64, _P],
    "dsmc_sg_mse": [_P, _P, _P, _P, _P, C.c_int64, C.c_int, C.c_int, _P],
    "dsmc_sg_adam": [_P, _P, _P, _P, _P, C.c_int64, C.c_float, C.c_float, C.c_float, C.c_float,
                     C.c_int, _P],
    "dsmc_sg_adam_dev": [_P, _P, _P, _P, _P, C.c_int64, _P, C.c_float, C.c_float, C.c_float,
                         _P],
    "dsmc_sg_to_bf16": [_P, _P, C.c_int64, _P],
    "dsmc_sg_check": [_P],
}


def lib():
    """The surrogate kernel library; fails loudly when it is not built."""
    global _lib
    if _lib is None:
        if not _LIB.exists():
            raise RuntimeError(f"{_LIB} is not built: python -m dsmc_erlend_b200.build")
        _lib = C.CDLL(os.fspath(_LIB))
        for name, args in _SIGS.items():
            fn = getattr(_lib, name)
            fn.restype = C.c_int
            fn.argtypes = args
    return _lib


def _ok(status: int, what: str):
    if status != 0:
        raise RuntimeError(f"{what}: status {status}")


def ptr(t) -> int | None:
    return None if t is None else t.data_ptr()


class Surrogate:
    """Weights (FP32 masters, BF16 copies, Adam moments) and the activation
    and gradient buffers of one batch size, on the current CUDA device."""

    def __init__(self, batch: int, res: int = RES, seed: int = 0, stream=None):
        import torch

        self.torch = torch
        self.n, self.res = batch, res
        self.stream = stream
        g = torch.Generator().manual_seed(seed)
        dev = torch.device("cuda")
        # All parameters in flat buffers, per layer its weights then its bias
        # (every segment a multiple of 32 elements, so each view stays 64-byte
        # aligned): masters, bf16 copies, gradients and Adam moments share the
        # offsets, so one launch updates all of them and one fill zeroes the
        # gradients.  The per-layer tensors below are views.
        segs = []
        for name, _, _, cin, cout, _, _ in LAYERS:
            segs += [(name, "w", (cout, 3, 3, cin)), (name, "b", (cout,))]
        self.n_params = sum(math.prod(shp) for _, _, shp in segs)
        self.p32 = torch.zeros(self.n_params, device=dev)
        self.pb = torch.zeros(self.n_params, dtype=torch.bfloat16, device=dev)
        self.g_all = torch.zeros(self.n_params, device=dev)
        self.m_all = torch.zeros(self.n_params, device=dev)
        self.v_all = torch.zeros(self.n_params, device=dev)
        # The input-gradient weights (each layer's rotated bf16 copy at its
        # weights' offsets), made for all layers by one launch per backward.
        self.prot = torch.zeros(self.n_params, dtype=torch.bfloat16, device=dev)
        self.w32, self.wb, self.b32, self.m, self.v, self.gw, self.gb = {}, {}, {}, {}, {}, {}, {}
        self.wrot = {}
        rot_off, rot_cin, rot_cout = [], [], []
        off = 0
        for name, kind, shp in segs:
            k = math.prod(shp)
            views = [t[off:off + k].view(shp)
                     for t in (self.p32, self.pb, self.g_all, self.m_all, self.v_all)]
            if kind == "w":
                self.wrot[name] = self.prot[off:off + k]
                rot_off.append(off)
                rot_cout.append(shp[0])
                rot_cin.append(shp[3])
            off += k
            self.m[name + "." + kind], self.v[name + "." + kind] = views[3], views[4]
            if kind == "w":
                self.w32[name], self.wb[name], self.gw[name] = views[:3]
            else:
                self.b32[name], self.gb[name] = views[0], views[2]
        for name, _, _, cin, cout, _, _ in LAYERS:
            std = math.sqrt(2.0 / (9 * cin))  # He initialisation
            w = torch.randn(cout, 3, 3, cin, generator=g) * std
            self.w32[name].copy_(w)
            self.wb[name].copy_(w.to(torch.bfloat16))
        self.t = 0
        nl = len(rot_off)
        self._rot = ((C.c_int64 * nl)(*rot_off), (C.c_int * nl)(*rot_cin),
                     (C.c_int * nl)(*rot_cout), nl)
        self.shape = {"x": (res, CH)}
        for name, src, op, cin, cout, _, _ in LAYERS:
            r = self.shape[src][0]
            r = r // 2 if op == "pool" else (r * 2 if op == "up" else r)
            self.shape[name] = (r, cout)
        bf = torch.bfloat16

        def buf(r, c, dtype=bf):
            return torch.empty(batch, r, r, c, dtype=dtype, device=dev)

        self.a_in, self.relu_out, self.y = {}, {}, {}
        for name, src, op, cin, cout, relu, skip in LAYERS:
            r = self.shape[name][0]
            self.a_in[name] = buf(r, cin) if op else None
            self.relu_out[name] = buf(r, cout)
            self.y[name] = buf(r, cout) if skip else self.relu_out[name]
        self.out32 = buf(res, CH, torch.float32)
        self.dy = {k: buf(*self.shape[k]) for k in self.shape}
        self.da_in = {name: buf(self.shape[name][0], cin)
                      for name, _, op, cin, _, _, _ in LAYERS}
        self.loss = torch.zeros(2, device=dev)

    @property
    def _s(self):
        return None if self.stream is None else C.c_void_p(self.stream)

    def act(self, name):
        return self.y[name]

    # -- forward --------------------------------------------------------------
    def forward(self, x) -> "torch.Tensor":
        """x: (n, res, res, 32) bf16 -> (n, res, res, 32) fp32 (channels 0..3
        are the prediction)."""
        L, s, n = lib(), self._s, self.n
        acts = {"x": x}
        for name, src, op, cin, cout, relu, skip in LAYERS:
            a = acts[src]
            r = self.shape[name][0]
            if op == "pool":
                _ok(L.dsmc_sg_pool_fwd(ptr(a), ptr(self.a_in[name]), n, 2 * r, 2 * r, cin, s),
                    "pool")
                a = self.a_in[name]
            elif op == "up":
                _ok(L.dsmc_sg_up_fwd(ptr(a), ptr(self.a_in[name]), n, r // 2, r // 2, cin, s),
                    "up")
                a = self.a_in[name]
            last = name == LAYERS[-1][0]
            if skip:  # relu_out for the ReLU's gradient, y = relu_out + skip
                _ok(L.dsmc_sg_conv_fwd_skip(ptr(a), ptr(self.wb[name]), ptr(self.b32[name]),
                                            ptr(acts[skip]), ptr(self.relu_out[name]),
                                            ptr(self.y[name]), n, r, r, cin, cout, int(relu), s),
                    f"conv {name}")
            else:
                _ok(L.dsmc_sg_conv_fwd(ptr(a), ptr(self.wb[name]), ptr(self.b32[name]), None,
                                       ptr(self.relu_out[name]),
                                       ptr(self.out32) if last else None,
                                       n, r, r, cin, cout, int(relu), s), f"conv {name}")
            acts[name] = self.y[name]
        self._acts = acts
        return self.out32

    # -- backward -------------------------------------------------------------
    def backward(self, dout):
        """Weight and bias gradients (FP32, in gw / gb) for the output
        gradient dout (bf16, same shape as the output)."""
        L, s, n = lib(), self._s, self.n
        acts = self._acts
        self.g_all.zero_()
        last = LAYERS[-1][0]
        if dout.data_ptr() != self.dy[last].data_ptr():
            self.dy[last].copy_(dout)
        # A gradient buffer is written by its first contribution and added to
        # by later ones (a skip source gets the decoder's gradient first, then
        # its pooled consumer's), so no buffer is zero-filled first.
        written = {last}
        offs, cins, couts, nl = self._rot
        _ok(L.dsmc_sg_rotate_layers(ptr(self.pb), ptr(self.prot), offs, cins, couts, nl, s),
            "rotate weights")
        for name, src, op, cin, cout, relu, skip in reversed(LAYERS):
            r = self.shape[name][0]
            dy = self.dy[name]
            _ok(L.dsmc_sg_relu_bias_bwd(ptr(dy), ptr(self.relu_out[name]) if relu else None,
                                        ptr(self.dy[skip]) if skip else None,
                                        int(skip in written), ptr(self.gb[name]), n * r * r,
                                        cout, s), f"relu and bias {name}")
            if skip:
                written.add(skip)
            a = self.a_in[name] if op else acts[src]
            _ok(L.dsmc_sg_conv_wgrad(ptr(dy), ptr(a), ptr(self.gw[name]), None,
                                     n, r, r, cin, cout, s), f"wgrad {name}")
            if src == "x":
                continue
            acc = src in written
            # The input gradient goes straight into dy[src] when it is the
            # first contribution and needs no resampling.
            da = self.dy[src] if (op is None and not acc) else self.da_in[name]
            # The input gradient: the forward convolution of dy with the
            # rotated weights (Cout in, Cin out).
            _ok(L.dsmc_sg_conv_fwd(ptr(dy), ptr(self.wrot[name]), None, None, ptr(da), None,
                                   n, r, r, cout, cin, 0, s), f"dgrad {name}")
            if op == "pool":
                _ok(L.dsmc_sg_pool_bwd_acc(ptr(da), ptr(self.dy[src]), n, 2 * r, 2 * r, cin,
                                           int(acc), s), "pool bwd")
            elif op == "up":
                _ok(L.dsmc_sg_up_bwd_acc(ptr(da), ptr(self.dy[src]), n, r // 2, r // 2, cin,
                                         int(acc), s), "up bwd")
            elif acc:
                _ok(L.dsmc_sg_add(ptr(self.dy[src]), ptr(da), da.numel(), s), "grad add")
            written.add(src)

    def loss_and_grad(self, target, mask):
        """Masked MSE of the last forward against target (n, res, res, OUT_CH)
        fp32 with mask (n, res, res) fp32; returns the loss tensor [1] and
        fills the output gradient."""
        L = lib()
        dout = self.dy[LAYERS[-1][0]]
        _ok(L.dsmc_sg_mse(ptr(self.out32), ptr(target), ptr(mask), ptr(dout), ptr(self.loss),
                          self.n * self.res * self.res, CH, OUT_CH, self._s), "mse")
        return self.loss[:1], dout

    def adam_step(self, lr: float = 1e-3, beta1: float = 0.9, beta2: float = 0.999,
                  eps: float = 1e-8):
        L, s = lib(), self._s
        self.t += 1
        # All parameters in one launch (the biases' bf16 copies are unused).
        _ok(L.dsmc_sg_adam(ptr(self.p32), ptr(self.pb), ptr(self.g_all), ptr(self.m_all),
                           ptr(self.v_all), self.n_params, lr, beta1, beta2, eps, self.t, s),
            "adam")

    def train_step(self, x, target, mask, lr: float = 1e-3):
        self.forward(x)
        loss, dout = self.loss_and_grad(target, mask)
        self.backward(dout)
        self.adam_step(lr)
        return loss

    def train_step_graph(self, x, target, mask, lr: float = 1e-3, beta1: float = 0.9,
                         beta2: float = 0.999, eps: float = 1e-8):
        """train_step replayed as one CUDA graph on the network's stream
        (which must be set): captured on the first call for these x / target
        / mask buffers (refill them between steps), the learning rate and
        Adam's bias corrections written to device memory before each replay.
        Returns the loss tensor [1]."""
        torch = self.torch
        if self.stream is None:
            raise RuntimeError("graph training needs the network's own CUDA stream")
        s = torch.cuda.ExternalStream(self.stream)
        # The Adam settings are kernel arguments inside the graph: new values
        # capture a new graph.
        key = (x.data_ptr(), target.data_ptr(), mask.data_ptr(), float(beta1), float(beta2),
               float(eps))
        if getattr(self, "_graph_key", None) != key:
            self._hp = torch.zeros(3, device="cuda")
            # Pinned staging of the step's values, four in flight.
            self._hp_ring = [torch.zeros(3).pin_memory() for _ in range(4)]
            self._hp_ev = [None] * 4
            with torch.cuda.stream(s):
                # Kernel attributes, tensor maps and SM counts are set on
                # first use: run every kernel of the step once outside the
                # capture (the gradients are overwritten by the captured
                # step, the weights are not touched).
                self.forward(x)
                _, dout = self.loss_and_grad(target, mask)
                self.backward(dout)
            s.synchronize()
            g = torch.cuda.CUDAGraph()
            L = lib()
            with torch.cuda.graph(g, stream=s):
                self.forward(x)
                _, dout = self.loss_and_grad(target, mask)
                self.backward(dout)
                _ok(L.dsmc_sg_adam_dev(ptr(self.p32), ptr(self.pb), ptr(self.g_all),
                                       ptr(self.m_all), ptr(self.v_all), self.n_params,
                                       ptr(self._hp), beta1, beta2, eps, self._s), "adam")
            self._graph, self._graph_key = g, key
        self.t += 1
        # The bias corrections as dsmc_sg_adam forms them (FP32 powf).
        t32 = np.float32(self.t)
        c1 = np.float32(1.0) - np.power(np.float32(beta1), t32)
        c2 = np.float32(1.0) - np.power(np.float32(beta2), t32)
        i = self.t % 4
        if self._hp_ev[i] is not None:
            self._hp_ev[i].synchronize()  # its last copy has been read
        self._hp_ring[i].copy_(torch.tensor([lr, float(c1), float(c2)], dtype=torch.float32))
        with torch.cuda.stream(s):
            self._hp.copy_(self._hp_ring[i], non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(s)
            self._hp_ev[i] = ev
            self._graph.replay()
        return self.loss[:1]

    def flops_per_step(self) -> float:
        """Tensor-core FLOPs of one train step: forward 2 Cin Cout 9 H W per
        sample and layer, backward twice that (dgrad and wgrad; the first
        layer has no dgrad)."""
        f = 0.0
        for name, src, op, cin, cout, _, _ in LAYERS:
            r = self.shape[name][0]
            one = 2.0 * cin * cout * 9 * r * r * self.n
            f += one * (2 if src == "x" else 3)
        return f

    def state_dict(self) -> dict:
        out = {}
        for name in self.w32:
            out[name + ".w"] = self.w32[name].cpu().numpy()
            out[name + ".b"] = self.b32[name].cpu().numpy()
        return out

    def load_state_dict(self, sd: dict):
        torch = self.torch
        for name in self.w32:
            self.w32[name].copy_(torch.from_numpy(np.asarray(sd[name + ".w"], np.float32)))
            self.b32[name].copy_(torch.from_numpy(np.asarray(sd[name + ".b"], np.float32)))
            self.wb[name].copy_(self.w32[name].to(torch.bfloat16))


# -- training ---------------------------------------------------------------------

def relative_errors(pred: np.ndarray, target: np.ndarray, mask: np.ndarray) -> dict:
    """Relative L2 error per output channel over the masked canvas cells:
    ||pred - target|| / ||target|| for n and the temperatures,
    ||pred - target|| / sqrt(cells) for the velocities (already in units of
    the freestream speed) and for Txy (in units of the temperature scale)."""
    m = mask.astype(bool)
    out = {}
    for i, k in enumerate(OUT_NAMES[:min(pred.shape[-1], target.shape[-1])]):
        d = (pred[..., i] - target[..., i])[m]
        if k not in ("ux", "uy", "txy"):
            out[k] = float(np.linalg.norm(d) / max(np.linalg.norm(target[..., i][m]), 1e-30))
        else:
            out[k] = float(np.linalg.norm(d) / np.sqrt(max(m.sum(), 1)))
    return out


def train(x: np.ndarray, target: np.ndarray, mask: np.ndarray, epochs: int = 40,
          batch: int = 32, lr: float = 2e-3, seed: int = 0, log=None) -> tuple:
    """Trains a Surrogate on (N, RES, RES, CH) inputs, (N, RES, RES, OUT_CH)
    targets and (N, RES, RES) masks with Adam (cosine learning-rate decay).
    Returns the network and a history of (epoch, mean loss, step ms, TFLOP/s)."""
    import torch

    n = x.shape[0]
    # One stream for the batch gathers and the graph-replayed steps.
    st = torch.cuda.Stream()
    net = Surrogate(batch, res=x.shape[1], seed=seed, stream=st.cuda_stream)
    dx = _to_device_input(torch, x)
    dt = torch.from_numpy(target.astype(np.float32)).cuda()
    dm = torch.from_numpy(mask.astype(np.float32)).cuda()
    bx = torch.empty((batch,) + dx.shape[1:], dtype=torch.bfloat16, device="cuda")
    bt = torch.empty((batch,) + dt.shape[1:], dtype=torch.float32, device="cuda")
    bm = torch.empty((batch,) + dm.shape[1:], dtype=torch.float32, device="cuda")
    rng = np.random.default_rng(seed)
    steps_per_epoch = n // batch
    total = epochs * steps_per_epoch
    history = []
    step = 0
    for ep in range(epochs):
        order = torch.from_numpy(rng.permutation(n)).cuda()
        torch.cuda.current_stream().synchronize()
        losses = []
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for s in range(steps_per_epoch):
            cur = lr * 0.5 * (1.0 + math.cos(math.pi * step / max(total, 1)))
            with torch.cuda.stream(st):
                idx = order[s * batch:(s + 1) * batch]
                torch.index_select(dx, 0, idx, out=bx)
                torch.index_select(dt, 0, idx, out=bt)
                torch.index_select(dm, 0, idx, out=bm)
            loss = net.train_step_graph(bx, bt, bm, lr=cur)
            with torch.cuda.stream(st):
                losses.append(loss.clone())
            step += 1
        e1.record(st)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / max(steps_per_epoch, 1)
        mean = float(torch.stack(losses).mean().item()) if losses else float("nan")
        tf = net.flops_per_step() / (ms * 1e-3) / 1e12
        history.append((ep, mean, ms, tf))
        if log:
            log(f"epoch {ep} loss {mean:.4e} {ms:.2f} ms/step {tf:.1f} TFLOP/s")
    # Hand the network back on the default stream (predictions read their
    # outputs there).
    st.synchronize()
    net.stream = None
    return net, history


def _to_device_input(torch, x: np.ndarray):
    """(N, RES, RES, c) inputs, c = IN_CH (stored compactly) or CH, as the
    network's bf16 (N, RES, RES, CH) device tensor (channels past c are
    zero), copied in slices to bound the host-side conversion."""
    n, c = x.shape[0], x.shape[-1]
    out = torch.zeros((n,) + x.shape[1:-1] + (CH,), dtype=torch.bfloat16, device="cuda")
    for i in range(0, n, 256):
        part = torch.from_numpy(np.ascontiguousarray(x[i:i + 256], dtype=np.float32))
        out[i:i + 256, ..., :c] = part.to(torch.bfloat16).cuda()
    return out


def predict(net: Surrogate, x: np.ndarray) -> np.ndarray:
    """Predictions (N, RES, RES, OUT_CH) for inputs (N, RES, RES, CH) with a
    trained network (its weights copied into a network of this batch)."""
    import torch

    out = []
    b = net.n
    for i in range(0, x.shape[0], b):
        part = x[i:i + b]
        pad = b - part.shape[0]
        if pad:
            part = np.concatenate([part, np.zeros((pad,) + part.shape[1:], part.dtype)])
        y = net.forward(_to_device_input(torch, part))
        out.append(y[: b - pad, ..., :OUT_CH].cpu().numpy())
    return np.concatenate(out)
