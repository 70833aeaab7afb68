"""Train the warm-start network on GPU-generated ICD pairs and evaluate it.

    python -m ctbb_icd_b200.train_warm_start [--train-seeds 100:300] [--heldout-seeds 900:920]
        [--steps 1500] [--out ctbb_icd_b200/weights/warm_start.npz] [--report report.json]

1. For each seed: synthetic scan of the training geometry (cfg2's scanner,
   flying focal spot, phantom and penalty, 256 x 256 over the 30 cm field of
   view, 32 slices of 0.6 mm; learned.TRAIN_WORKLOAD), n_early plain
   grouped-ICD iterations from the zero start (the network's input), then
   plain ICD to a relative cost change below 1e-7 per iteration (the
   target); both rotated to the fixed frame, interior slices kept. Grouped
   ICD runs with autotuned warps in flight and tile edge. One matrix serves
   every seed (same geometry).
2. Adam on random crops (8 x 128 x 128) of the training pairs.
3. Held-out seeds: loss before and after training, and time to <= 0.5 HU
   RMSE against the plain converged image for plain ICD and for the learned
   warm start on the training grid. Full-size (512 x 512 x 64) evaluation:
   python -m ctbb_icd_b200.eval_warm_start.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np


def _seeds(spec: str):
    a, b = spec.split(":")
    return list(range(int(a), int(b)))


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--train-seeds", default="100:300")
    ap.add_argument("--heldout-seeds", default="900:920")
    ap.add_argument("--steps", type=int, default=1500)
    ap.add_argument("--batch", type=int, default=4)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--blocks", type=int, default=4)
    ap.add_argument("--n-early", type=int, default=3)
    ap.add_argument("--max-iter", type=int, default=400)
    ap.add_argument("--prio-fraction", type=float, default=0.2)
    ap.add_argument("--prio-passes", type=int, default=2)
    ap.add_argument("--eval-scans", type=int, default=2)
    ap.add_argument("--pairs", default=None, help="npz cache of the generated pairs (read if present, else written)")
    ap.add_argument("--engine", choices=["tcgen05", "mma_sync"], default="mma_sync",
                    help="tensor-core path of the 32 -> 32 convolutions")
    ap.add_argument("--out", default=None)
    ap.add_argument("--report", default=None)
    args = ap.parse_args(argv)

    import torch

    import ctbb_icd_b200 as C
    from ctbb_icd_b200 import learned as L

    torch.cuda.set_device(0)
    ctx = C.Context(0)
    report = {"args": vars(args), "workload": L.TRAIN_WORKLOAD}
    log = lambda m: print(m, flush=True)  # noqa: E731
    opts, trials = L.tuned_opts(ctx, n_early=args.n_early, log=log)
    report["autotune"] = trials
    report["opts"] = {"warps_in_flight": opts.warps_in_flight, "lattice": opts.lattice}

    # The early-iterate protocol the network is trained for (and recorded
    # with its weights): the tuned tile edge and density of in-flight updates.
    net = L.WarmStartNet(ctx, args.blocks, seed=0)
    net.set_engine(C.CNN_ENGINE_TCGEN05 if args.engine == "tcgen05" else C.CNN_ENGINE_MMA_SYNC)
    nvox = int(np.prod(L.workload_shape(L.TRAIN_WORKLOAD)))
    net.n_early = args.n_early
    net.early_lattice = int(opts.lattice)
    net.early_density = float(opts.warps_in_flight) / max(1, opts.warps_per_voxel) / nvox
    t0 = time.time()
    if args.pairs and os.path.exists(args.pairs):
        z = np.load(args.pairs)
        xe, xc, he, hc, mask = z["xe"], z["xc"], z["he"], z["hc"], z["mask"]
    else:
        def early(rc):
            return net.early_opts(rc, opts)

        xe, xc, mask = L.make_pairs(ctx, _seeds(args.train_seeds), n_early=args.n_early, opts=opts,
                                    max_iter=args.max_iter, log=log, early_opts=early)
        he, hc, _ = L.make_pairs(ctx, _seeds(args.heldout_seeds), n_early=args.n_early, opts=opts,
                                 max_iter=args.max_iter, log=log, early_opts=early)
        if args.pairs:
            np.savez(args.pairs, xe=xe, xc=xc, he=he, hc=hc, mask=mask)
    report["data_seconds"] = time.time() - t0

    report["heldout_loss_init"] = L.eval_loss(net, he, hc, mask)
    t0 = time.time()
    hist = L.train(net, xe, xc, mask, steps=args.steps, batch=args.batch, lr=args.lr, log=log)
    report["train_seconds"] = time.time() - t0
    report["train_loss_first"] = float(np.mean(hist[:50]))
    report["train_loss_last"] = float(np.mean(hist[-50:]))
    report["heldout_loss"] = L.eval_loss(net, he, hc, mask)
    # A zero prediction (the early iterate as is) for scale.
    zero = L.WarmStartNet(ctx, 0)
    zero.set_params(np.zeros(zero.n_params, np.float32))
    report["heldout_loss_zero_prediction"] = L.eval_loss(zero, he, hc, mask)
    zero.free()
    log(f"held-out loss: init {report['heldout_loss_init']:.5f} trained {report['heldout_loss']:.5f} "
        f"zero-prediction {report['heldout_loss_zero_prediction']:.5f}")
    if args.out:
        net.save(args.out, train_seeds=args.train_seeds, steps=args.steps, n_early=args.n_early)

    evals = []
    ssm = None
    for s in _seeds(args.heldout_seeds)[:args.eval_scans]:
        scan = L.make_scan(ctx, L.TRAIN_WORKLOAD, s, ssm)
        ssm = scan.ssm
        L.converge(scan, opts, max_iter=args.max_iter)
        x_ref = scan.rc.volume()
        plain = L.time_to_tolerance(scan, x_ref, opts)
        learned = L.time_to_tolerance(scan, x_ref, opts, net=net, n_early=args.n_early,
                                      prio_fraction=args.prio_fraction, prio_passes=args.prio_passes)
        evals.append({"seed": s, "plain": plain, "learned": learned})
        log(f"seed {s}: plain {plain['seconds']:.2f} s / {plain['iterations']} it, learned "
            f"{learned['seconds']:.2f} s / {learned['iterations']} it "
            f"(ratio {learned['seconds'] / plain['seconds']:.3f})")
        log("  learned trace: " + ", ".join(f"{a}:{c:.2f}HU" for a, _, c in learned["trace"][:8]))
        scan.rc.free()
    report["time_to_0p5hu"] = evals
    if args.report:
        os.makedirs(os.path.dirname(os.path.abspath(args.report)), exist_ok=True)
        with open(args.report, "w") as f:
            json.dump(report, f, indent=1, default=float)
    print(json.dumps({k: v for k, v in report.items() if k != "time_to_0p5hu"}, default=float))
    return 0


if __name__ == "__main__":
    sys.exit(main())
