"""Time to a given accuracy: plain grouped ICD vs the learned warm start.

    python -m ctbb_icd_b200.eval_warm_start [--workload cfg2] [--seed 950]
        [--weights ctbb_icd_b200/weights/warm_start.npz] [--tol 0.5] [--max-iter 400]
        [--ref-iter 1200] [--autotune] [--out result.json]

Both arms start from the zero image (initialize_recon_volume's default) on the
same scan and run the same grouped-ICD settings (autotuned once with
--autotune). On a scan twice the network's training grid in-plane (cfg2,
512 x 512, for the 256 x 256 training grid) the learned arm starts on the
scan's half-size grid (learned.warm_start_coarse); its matrix build is timed
and reported apart from the reconstruction time, like the full-size matrix
both arms use. The reference image is the unique minimiser of the convex cost,
approached by the learned path followed by --ref-iter further iterations; the
run reports how far that reference still moved over its last ten
iterations. Errors are RMSE in HU inside the object support on the interior
slices (learned.Scan.error_hu); times are wall seconds of the reconstruction
calls (device-synchronous), error checks excluded. One JSON line on stdout.
"""
from __future__ import annotations

import argparse
import json
import sys
import time

import numpy as np


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--workload", default=None)
    ap.add_argument("--seed", type=int, default=950)
    ap.add_argument("--weights", default=None)
    ap.add_argument("--tol", type=float, default=0.5)
    ap.add_argument("--max-iter", type=int, default=400)
    ap.add_argument("--ref-iter", type=int, default=1200)
    ap.add_argument("--n-early", type=int, default=3)
    ap.add_argument("--prio-fraction", type=float, default=0.2)
    ap.add_argument("--prio-passes", type=int, default=2)
    ap.add_argument("--autotune", action="store_true")
    ap.add_argument("--wpv", type=int, default=1)
    ap.add_argument("--out", default=None)
    args = ap.parse_args(argv)

    import torch

    import ctbb_icd_b200 as C
    from ctbb_icd_b200 import learned as L

    torch.cuda.set_device(0)
    ctx = C.Context(0)
    name = args.workload or "cfg2"
    log = lambda m: print(m, file=sys.stderr, flush=True)  # noqa: E731
    net = L.WarmStartNet.load(ctx, args.weights or L.WEIGHTS_PATH)
    scan = L.make_scan(ctx, name, args.seed)
    coarse, coarse_setup_s = None, None
    train_nx = L.workload_shape(L.TRAIN_WORKLOAD)[2]
    if int(scan.rp.geom.nx) == 2 * train_nx:
        t0 = time.time()
        coarse = L.make_scan(ctx, L.coarse_workload(name), args.seed, raw_from=scan)
        coarse_setup_s = time.time() - t0
        log(f"half-size grid {coarse.rp.shape}: matrix and setup {coarse_setup_s:.2f} s")
    opts = C.icd_opts(mode=C.ICD_GROUPED, weights=C.SSM_FP32, warps_per_voxel=args.wpv)
    tune = None
    if args.autotune:
        scan.rc.iterate(scan.ssm, args.n_early, opts)
        opts, trials = scan.rc.autotune(scan.ssm, opts, probe_iters=2)
        tune = {"warps_per_voxel": opts.warps_per_voxel, "warps_in_flight": opts.warps_in_flight,
                "lattice": opts.lattice}
        log(f"autotune: {tune}")

    # Reference: learned start, then ref_iter iterations with FP64 refreshes.
    t0 = time.time()
    copts = C.icd_opts(mode=C.ICD_GROUPED, weights=C.SSM_FP32)
    if coarse is not None:
        L.warm_start_coarse(scan, coarse, net, args.n_early, copts)
    else:
        scan.rc.set_volume(scan.ssm, None)
        scan.rc.iterate(scan.ssm, args.n_early, net.early_opts(scan.rc, opts))
        scan.rc.warm_start(scan.ssm, net, scan.tables.tube_angles)
    done = 0
    while done < args.ref_iter:
        n = min(50, args.ref_iter - done)
        scan.rc.iterate(scan.ssm, n, opts)
        scan.rc.refresh_residual(scan.ssm)
        done += n
        if done % 200 == 0:
            log(f"reference: {done} iterations, cost {scan.rc.cost():.12e}")
    x_tail = scan.rc.volume()
    scan.rc.iterate(scan.ssm, 10, opts)
    scan.rc.refresh_residual(scan.ssm)
    x_ref = scan.rc.volume()
    ref_cost = scan.rc.cost()
    ref_motion = scan.error_hu(x_tail, x_ref)
    ref_seconds = time.time() - t0
    log(f"reference: {done + 10} iterations, last-10-iteration motion {ref_motion:.3f} HU")

    plain = L.time_to_tolerance(scan, x_ref, opts, tol_hu=args.tol, max_iter=args.max_iter)
    log(f"plain: {plain['seconds']:.2f} s, {plain['iterations']} iterations, reached {plain['reached']}")
    learned = L.time_to_tolerance(scan, x_ref, opts, tol_hu=args.tol, max_iter=args.max_iter, net=net,
                                  n_early=args.n_early, prio_fraction=args.prio_fraction,
                                  prio_passes=args.prio_passes, coarse=coarse, coarse_opts=copts)
    log(f"learned: {learned['seconds']:.2f} s, {learned['iterations']} iterations, reached {learned['reached']}")

    ladder = [1000.0, 500.0, 200.0, 100.0, 50.0, 25.0, 10.0, 5.0, 1.0, args.tol]

    def seconds_to(r, tol):
        for _, t, e in r["trace"]:
            if e <= tol:
                return t
        return None

    thresholds = []
    for tol in ladder:
        a, b = seconds_to(plain, tol), seconds_to(learned, tol)
        thresholds.append({"hu": tol, "plain_s": a, "learned_s": b,
                           "ratio": (b / a) if (a is not None and b is not None and a > 0) else None})

    def brief(r):
        tr = r["trace"]
        pick = tr[:6] + [t for t in tr[6:] if t[0].startswith("iter") and int(t[0].split()[1]) % 25 == 0] + tr[-1:]
        # (label, seconds, HU) at the start, every 25 iterations and the end
        return {"seconds": r["seconds"], "iterations": r["iterations"], "reached": r["reached"],
                "final_hu": tr[-1][2], "trace": [(a, round(s, 3), round(e, 3)) for a, s, e in pick]}

    out = {
        "metric": f"time to <= {args.tol} HU RMSE vs converged image",
        "workload": name, "seed": args.seed, "voxels": int(np.prod(scan.rp.shape)),
        "opts": {"warps_per_voxel": max(1, opts.warps_per_voxel), "warps_in_flight": opts.warps_in_flight,
                 "lattice": opts.lattice, "weights": "fp32"},
        "autotune": tune,
        "learned_start": ("half-size grid: n_early iterations + network + 2x upsampling" if coarse is not None
                          else "n_early iterations + network + priority passes"),
        "half_grid_setup_s": coarse_setup_s,
        "reference": {"iterations": done + 10 + args.n_early, "cost": ref_cost,
                      "motion_last_10_iterations_hu": ref_motion, "seconds": ref_seconds},
        "plain": brief(plain), "learned": brief(learned),
        "ratio_learned_over_plain": (learned["seconds"] / plain["seconds"]
                                     if plain["reached"] and learned["reached"] else None),
        "time_to_threshold": thresholds,
        "error_region": "object support r < 13 cm, interior slices",
    }
    line = json.dumps(out, default=float)
    print(line, flush=True)
    if args.out:
        with open(args.out, "w") as f:
            f.write(line + "\n")
    return 0


if __name__ == "__main__":
    sys.exit(main())
