"""Throughput of the warm-start network's GPU kernels.

    python -m ctbb_icd_b200.cnn_bench [--shape 16 256 256] [--blocks 4] [--reps 5]

Times (CUDA events around synchronous library calls) the forward pass and one
training step (forward, loss, backward, gradient accumulation) of the 3D
residual CNN on a synthetic volume, and reports the tensor-core FLOP rate of
the 32 -> 32 convolutions (2 * 27 * 32 * 32 FLOP per voxel each: 2 per block
forward; forward + backward-data + weight gradient per block in training).
One JSON line on stdout.
"""
from __future__ import annotations

import argparse
import json
import sys


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--shape", type=int, nargs=3, default=[16, 256, 256])
    ap.add_argument("--blocks", type=int, default=4)
    ap.add_argument("--reps", type=int, default=5)
    args = ap.parse_args(argv)

    import torch

    import ctbb_icd_b200 as C
    from ctbb_icd_b200 import learned as L

    torch.cuda.set_device(0)
    ctx = C.Context(0)
    net = L.WarmStartNet(ctx, args.blocks, seed=0)
    g = torch.Generator(device="cuda").manual_seed(0)
    x = (0.15 + 0.1 * torch.rand(*args.shape, device="cuda", generator=g)).contiguous()
    xc = (x + 0.002 * torch.randn(*args.shape, device="cuda", generator=g)).contiguous()
    nvox = x.numel()
    conv_flop = 2.0 * 27 * 32 * 32 * nvox

    def timed(fn, reps):
        fn()  # warm-up (workspace, weight copies)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            fn()
        b.record()
        b.synchronize()
        return a.elapsed_time(b) / reps

    fwd_ms = timed(lambda: net.forward(x), args.reps)
    train_ms = timed(lambda: net.accumulate_gradient(x, xc), args.reps)
    net.zero_gradient()
    out = {
        "metric": "warm-start network throughput", "shape": args.shape, "blocks": args.blocks,
        "forward_ms": fwd_ms, "train_step_ms": train_ms,
        "forward_voxels_per_s": nvox / (fwd_ms / 1e3),
        "forward_conv_tflops": 2 * args.blocks * conv_flop / (fwd_ms / 1e3) / 1e12,
        "train_conv_tflops": 6 * args.blocks * conv_flop / (train_ms / 1e3) / 1e12,
        "dtype": "bf16 operands, fp32 accumulation",
    }
    print(json.dumps(out), flush=True)
    net.free()
    ctx.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
