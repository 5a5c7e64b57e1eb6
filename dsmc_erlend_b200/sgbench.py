"""Throughput of the surrogate's tensor-core convolutions and of one training
step: each layer shape of the network at a batch size, forward
(dsmc_sg_conv_fwd), input gradient (dsmc_sg_conv_dgrad) and weight gradient
(dsmc_sg_conv_wgrad), timed with CUDA events on random bf16 tensors.

    python -m dsmc_erlend_b200.sgbench [--batch 32] [--iters 20]
    python -m dsmc_erlend_b200.sgbench --shape 128x128:32:32 --profile
    python -m dsmc_erlend_b200.sgbench --batch 64 --step-profile

Prints one JSON line: per shape and op, milliseconds per call and TFLOP/s
(2 Cin Cout 9 H W N), and the training step's milliseconds and TFLOP/s,
eager and replayed as one CUDA graph.
`--profile` runs forward, input gradient and weight gradient of one shape
twice each (in that order) with no timing, for a profiler to capture the
second round.  `--step-profile` runs three eager training steps with no
timing (a profiler's launch list of the last one is the step's kernels).
"""
from __future__ import annotations

import argparse
import json

from . import surrogate as S


def _shapes(batch: int):
    net_res = {"x": S.RES}
    out = []
    for name, src, op, cin, cout, _, _ in S.LAYERS:
        r = net_res[src]
        r = r // 2 if op == "pool" else (r * 2 if op == "up" else r)
        net_res[name] = r
        if (r, cin, cout) not in [(o[1], o[3], o[4]) for o in out]:
            out.append((batch, r, r, cin, cout))
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--batch", type=int, default=32)
    ap.add_argument("--iters", type=int, default=20)
    ap.add_argument("--shape", default=None, help="HxW:Cin:Cout, e.g. 128x128:32:32")
    ap.add_argument("--profile", action="store_true")
    ap.add_argument("--step-profile", action="store_true")
    args = ap.parse_args()

    import torch

    if args.step_profile:
        net = S.Surrogate(args.batch)
        x = torch.randn(args.batch, S.RES, S.RES, S.CH, device="cuda").to(torch.bfloat16)
        tgt = torch.randn(args.batch, S.RES, S.RES, S.OUT_CH, device="cuda")
        mask = torch.ones(args.batch, S.RES, S.RES, device="cuda")
        for _ in range(3):
            net.train_step(x, tgt, mask)
        torch.cuda.synchronize()
        S._ok(S.lib().dsmc_sg_check(None), "tensor-core wait")
        print(json.dumps({"step_profile": args.batch}))
        return

    L = S.lib()
    if args.shape:
        hw, cin, cout = args.shape.split(":")
        h, w = (int(v) for v in hw.split("x"))
        shapes = [(args.batch, h, w, int(cin), int(cout))]
    else:
        shapes = _shapes(args.batch)

    def ops(n, h, w, cin, cout):
        x = torch.randn(n, h, w, cin, device="cuda").to(torch.bfloat16)
        wt = (0.05 * torch.randn(cout, 3, 3, cin, device="cuda")).to(torch.bfloat16)
        b = torch.zeros(cout, device="cuda")
        y = torch.empty(n, h, w, cout, dtype=torch.bfloat16, device="cuda")
        dy = torch.randn(n, h, w, cout, device="cuda").to(torch.bfloat16)
        dx = torch.empty_like(x)
        w_rot = torch.empty(9 * cin * cout, dtype=torch.bfloat16, device="cuda")
        dw = torch.zeros(cout, 3, 3, cin, device="cuda")
        p = S.ptr
        return {
            "fwd": lambda: L.dsmc_sg_conv_fwd(p(x), p(wt), p(b), None, p(y), None, n, h, w, cin,
                                              cout, 1, None),
            "dgrad": lambda: L.dsmc_sg_conv_dgrad(p(dy), p(wt), p(w_rot), p(dx), n, h, w, cin,
                                                  cout, None),
            "wgrad": lambda: L.dsmc_sg_conv_wgrad(p(dy), p(x), p(dw), None, n, h, w, cin, cout,
                                                  None),
        }

    if args.profile:
        f = ops(*shapes[0])
        for _ in range(2):
            for name in ("fwd", "dgrad", "wgrad"):
                S._ok(f[name](), "conv " + name)
        torch.cuda.synchronize()
        S._ok(L.dsmc_sg_check(None), "tensor-core wait")
        print(json.dumps({"profile": args.shape or "x".join(map(str, shapes[0]))}))
        return

    res = {}
    for shp in shapes:
        n, h, w, cin, cout = shp
        flop = 2.0 * n * h * w * cin * cout * 9
        f = ops(*shp)
        row = {}
        for name, fn in f.items():
            for _ in range(3):
                S._ok(fn(), name)
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(args.iters):
                fn()
            e1.record()
            e1.synchronize()
            ms = e0.elapsed_time(e1) / args.iters
            row[name] = {"ms": round(ms, 4), "tflops": round(flop / ms / 1e9, 1)}
        res[f"{h}x{w} {cin}->{cout}"] = row
    S._ok(L.dsmc_sg_check(None), "tensor-core wait")

    out = {"batch": args.batch, "conv": res}
    if not args.shape:
        net = S.Surrogate(args.batch)
        x = torch.randn(args.batch, S.RES, S.RES, S.CH, device="cuda").to(torch.bfloat16)
        tgt = torch.randn(args.batch, S.RES, S.RES, S.OUT_CH, device="cuda")
        mask = torch.ones(args.batch, S.RES, S.RES, device="cuda")
        for _ in range(3):
            net.train_step(x, tgt, mask)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.iters):
            net.train_step(x, tgt, mask)
        e1.record()
        e1.synchronize()
        ms = e0.elapsed_time(e1) / args.iters
        out["train_step"] = {"ms": round(ms, 4),
                             "tflops": round(net.flops_per_step() / ms / 1e9, 1)}
        # The same step replayed as one CUDA graph on the network's stream.
        st = torch.cuda.Stream()
        gnet = S.Surrogate(args.batch, stream=st.cuda_stream)
        for _ in range(3):
            gnet.train_step_graph(x, tgt, mask)
        torch.cuda.synchronize()
        e0.record(st)
        for _ in range(args.iters):
            gnet.train_step_graph(x, tgt, mask)
        e1.record(st)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / args.iters
        out["train_step_graph"] = {"ms": round(ms, 4),
                                   "tflops": round(gnet.flops_per_step() / ms / 1e9, 1)}
    print(json.dumps(out))


if __name__ == "__main__":
    main()
