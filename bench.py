#!/usr/bin/env python
"""Benchmark: voxel updates per second of grouped ICD on the full-size helical
workload (512 x 512 x 64 slices, 736 channels x 64 rows, in-plane flying
focal spot, 2304 views/turn, 4 turns, edge-preserving penalty).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A step is one ICD iteration: every voxel of the volume updated once by the
persistent grouped-ICD kernel. Inputs (raw data, stored system matrix, image,
error sinogram) are resident in HBM before timing; the e2e figure repeats the
measurement through the reference-facing one-call API (ctbb_gpu_icd) with
host buffers, so host<->device copies are inside the timed region.

With N > 1 (torchrun) every rank reconstructs its own independent scan
(replicas, weak scaling, no data-path collective); `value` is the sum of all
ranks' voxel updates over the slowest rank's time.

--impl reference times the reference program (oracle/_ref/icd_ref_O2, the
CTBB_ICD sources built unmodified) on the host cores: its ICD iterations on a
bounded sample of the same geometry (see cpu_sample()).
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = "cfg2"
WORKLOAD_TEXT = ("grouped ICD, 512x512x64 @ 0.6 mm, 30 cm FOV, 736 ch x 64 rows, in-plane FFS, "
                 "2304 views/turn, 4 turns (9216 views), edge-preserving (delta 9.6e-4, lambda 0.1)")
HBM_FALLBACK_GBS = 6650.0
HBM_NOMINAL_GBS = 8000.0  # B200 HBM3e nominal, for context beside the measured copy peak


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return HBM_FALLBACK_GBS, "fallback"


# --------------------------------------------------------------------------
# nvidia-smi clock sampling during the timed region
# --------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int, enabled: bool = True):
        self.gpu = gpu_index
        self.enabled = enabled
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        if not self.enabled:
            return
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, FileNotFoundError):
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.time(), line.strip()))

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for _, line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": mx, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# --------------------------------------------------------------------------
# Our arm
# --------------------------------------------------------------------------
def setup_workload(ctx, workdir, seed, weights, name=WORKLOAD):
    import ctbb_icd_b200 as C
    from ctbb_icd_b200 import workloads as W

    w = W.workload(name)
    w["phantom"]["seed"] = seed
    prm = w["prm"]
    prm.update(sinogram_path=os.path.join(workdir, "raw.bin"), output_dir=workdir, output_file="out.img")
    open(prm["sinogram_path"], "wb").close()
    rp = C.configure_recon_params(W.write_prm(os.path.join(workdir, "bench.prm"), prm))
    tables = C.slice_tables(rp)
    spec = W.phantom_spec(w["phantom"])
    spec.ellipsoid_z_lo = min(prm["z_start"], prm["z_end"])
    spec.ellipsoid_z_hi = max(prm["z_start"], prm["z_end"])
    # Phantom cut to the reconstructed slab: data consistent with the model.
    spec.clip_z_lo, spec.clip_z_hi = W.slab_clip(rp, tables.slice_locations)
    rc = C.Recon(rp, tables.slice_indices, ctx)
    C.check(C.lib().ctbb_gpu_synth_raw(ctx.handle, ctypes.byref(rp.geom), ctypes.byref(spec),
                                       ctypes.c_void_p(rc.raw_device_ptr())))
    ssm = C.Ssm.generate(rp, ctx, weights)
    rc.set_volume(ssm, None)
    return rp, tables, rc, ssm


def run_ours(args, rank, world, dist):
    import torch

    import ctbb_icd_b200 as C

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    torch_stream = torch.cuda.Stream(device=local)
    if args.own_stream:
        ctx = C.Context(local)
        torch_stream = torch.cuda.ExternalStream(ctx.stream, device=local)
    else:
        ctx = C.Context(local, ctypes.c_void_p(torch_stream.cuda_stream))
    weights_fmt = C.SSM_FP16 if args.weights == "fp16" else C.SSM_FP32
    workdir = tempfile.mkdtemp(prefix="ctbb_bench_")
    t0 = time.time()
    rp, tables, rc, ssm = setup_workload(ctx, workdir, seed=rank, weights=C.SSM_BOTH if args.e2e else weights_fmt,
                                         name=args.workload)
    setup_s = time.time() - t0
    info = ssm.info()
    opts = C.icd_opts(mode=C.ICD_GROUPED, weights=weights_fmt, warps_in_flight=args.warps, lattice=args.lattice,
                      warps_per_voxel=args.wpv, entries_per_lane=args.epl, stage_column=max(0, args.stage_column),
                      entry_pairs=args.entry_pairs, stack_align=args.stack_align, l2_hints=args.l2_hints)
    nvox = int(np.prod(rp.shape))
    tune = None
    if args.autotune:
        # Probe from an early iterate, as a user would before a long run.
        rc.iterate(ssm, 3, opts)
        opts, trials = rc.autotune(ssm, opts, probe_iters=2)
        tune = {"chosen": {"warps_per_voxel": opts.warps_per_voxel, "warps_in_flight": opts.warps_in_flight,
                           "entries_per_lane": opts.entries_per_lane, "lattice": opts.lattice,
                           "stage_column": opts.stage_column, "entry_pairs": opts.entry_pairs},
                "trials": [[t["warps_per_voxel"], t["warps_in_flight"], t["entries_per_lane"], t["lattice"],
                            t["stage_column"], t["entry_pairs"], round(t["device_ms"], 1), round(t["score"], 1)]
                           for t in trials],
                "trial_fields": ["warps_per_voxel", "warps_in_flight", "entries_per_lane", "lattice",
                                 "stage_column", "entry_pairs", "ms_2_iterations", "cost_decrease_per_ms"]}
        rc.set_volume(ssm, None)

    rc.iterate(ssm, args.warmup, opts)
    st = rc.iterate(ssm, 1, opts)
    entries = rc.entries(ssm)
    w_bytes = 2 if weights_fmt == C.SSM_FP16 else 4
    # The iterate the timed region starts from, for the e2e leg (same range).
    x_start = rc.volume() if args.e2e else None

    clocks = ClockSampler(local, enabled=args.clocks)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(torch_stream):
        start.record(torch_stream)
        st = rc.iterate(ssm, args.steps, opts)
        end.record(torch_stream)
    end.synchronize()
    torch.cuda.synchronize()
    elapsed_ms = start.elapsed_time(end)
    clocks.stop()
    kernel_ms_per_launch = st.device_ms / max(1, st.iterations)
    # Algorithmic bytes per iteration (one launch), from what the timed
    # launches did: e read once per in-range entry gathered (4 B) and written
    # once per entry of the updates that changed their voxel (4 B; an update
    # with du == 0, e.g. an air voxel held at 0 by the positivity clamp,
    # scatters nothing), the matrix read once (index + weight), image r+w.
    gathered = st.entries / max(1, st.iterations)
    scattered = st.entries_scattered / max(1, st.iterations)
    # The matrix in the form the kernel reads: entry pairs (8 B per pair of
    # rows) when the iteration used them, else index + weight per entry.
    n_pairs = int(ssm.info().n_pairs)
    uses_pairs = (n_pairs > 0 and weights_fmt == C.SSM_FP16
                  and (opts.stage_column >= 4 or (opts.entry_pairs == 0
                                                  and (opts.warps_per_voxel > 1 or opts.stage_column == 0))))
    ssm_read = 8.0 * n_pairs if uses_pairs else (4 + w_bytes) * float(info.nnz)
    b_iter = 4.0 * gathered + 4.0 * scattered + ssm_read + 8.0 * nvox

    e2e = None
    if args.e2e:
        e2e = run_e2e(C, ctx, rp, tables, ssm, rc, opts, args, x_start)

    from ctbb_icd_b200.replicas import max_over_ranks

    t_max = max_over_ranks(elapsed_ms, dist, device="cuda")
    if e2e and dist:
        e2e["seconds"] = max_over_ranks(e2e["seconds"], dist, device="cuda")
        e2e["value"] = world * e2e["updates"] / e2e["seconds"]
    out = None
    if rank == 0:
        peak, peak_kind = measured_peak()
        achieved = b_iter / (kernel_ms_per_launch / 1e3) / 1e9
        value = world * nvox * args.steps / (t_max / 1e3)
        kernel = ("icd_bulk_pipe_kernel" if opts.stage_column == 6 else
                  "icd_bulk_kernel" if opts.stage_column >= 4 else
                  ("icd_lockstep_kernel" if opts.stage_column == 3 else
                   "icd_staged_kernel" if opts.stage_column else
                   "icd_grouped_pairs_kernel" if uses_pairs else "icd_grouped_kernel")
                  if opts.warps_per_voxel <= 1 else ("icd_cta_pairs_kernel" if uses_pairs else "icd_cta_kernel"))
        traffic = read_traffic(kernel)
        out = {
            "metric": "voxel-updates/s",
            "value": value,
            "unit": "voxel-updates/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": t_max / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic (seeded phantom: water + 6 inserts + 40 ellipsoids, Poisson noise, GPU projector)",
            "config": {
                "workload": WORKLOAD_TEXT if args.workload == WORKLOAD else args.workload,
                "weights": args.weights, "error_sinogram": "fp32", "voxels": nvox,
                "ssm_nnz": int(info.nnz), "ssm_bytes": int(info.bytes_device),
                "ssm_build_ms": round(info.build_ms, 2), "inrange_entries_per_iter": entries,
                "scattered_entries_per_iter": scattered, "stage_column": int(opts.stage_column),
                "l2_hints": int(opts.l2_hints),
                "matrix_read_as": (f"{n_pairs} entry pairs (8 B each)" if uses_pairs
                                   else f"entries ({4 + w_bytes} B each)"),
                "warps_in_flight": opts.warps_in_flight or "auto", "warps_per_voxel": max(1, opts.warps_per_voxel),
                "entries_per_lane": opts.entries_per_lane or 8,
                "lattice": opts.lattice or "auto", "autotune": tune,
                "l2": "inputs larger than L2 (e 1.74 GB, SSM > 20 GB)",
                "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
                "setup_s": round(setup_s, 1),
            },
            "roofline": {
                "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic,
                "kernel": kernel,
                "algorithmic_bytes_per_launch": b_iter,
                "kernel_ms_per_launch": kernel_ms_per_launch, "peak_source": peak_kind,
                "frac_of_nominal": achieved / HBM_NOMINAL_GBS, "nominal_peak": HBM_NOMINAL_GBS,
                "traffic_gbs": None if traffic is None else traffic / (kernel_ms_per_launch / 1e3) / 1e9,
            },
            "gpu_launches": int(args.steps),
            "clocks": clocks.summary(),
        }
        if e2e:
            out["e2e"] = {"value": e2e["value"], "unit": "voxel-updates/s",
                          "h2d_bytes_per_step": e2e["h2d"], "d2h_bytes_per_step": e2e["d2h"]}
            out["gpu_launches"] += e2e["launches"]
        if args.cpu_baseline and world == 1:
            cb = cpu_sample(iterations=3)
            out["cpu_baseline"] = {k: cb.get(k) for k in ("value", "unit", "cores", "kind", "sample")}
    rc.free()
    ssm.free()
    if out is not None and args.ttt and world == 1:
        out["time_to_tolerance"] = time_to_tolerance_sample(ctx, opts)
    ctx.close()
    return out


def _geometry(workdir, name):
    """The workload's recon params and slice tables (no raw data)."""
    import ctbb_icd_b200 as C
    from ctbb_icd_b200 import workloads as W

    prm = W.workload(name)["prm"]
    prm.update(sinogram_path=os.path.join(workdir, "raw.bin"), output_dir=workdir, output_file="out.img")
    open(prm["sinogram_path"], "wb").close()
    rp = C.configure_recon_params(W.write_prm(os.path.join(workdir, "stage.prm"), prm))
    return rp, C.slice_tables(rp)


def run_stage(args):
    """--stage ssm | rotate: the other two subsystems of the path on their own.

    ssm: generate_system_matrix_ffs on the GPU (cell-count pass, column scan,
    fill pass), FP16 weights, timed per build; algorithmic bytes = the matrix
    written (index + weight per entry, per-view offsets, column pointers).
    rotate: rotate_slices_rotating2fixed of the workload's volume, device to
    device; algorithmic bytes = the volume read once and written once."""
    import torch

    import ctbb_icd_b200 as C

    torch.cuda.set_device(0)
    ctx = C.Context(0)
    workdir = tempfile.mkdtemp(prefix="ctbb_stage_")
    peak, peak_kind = measured_peak()
    clocks = ClockSampler(0, enabled=args.clocks)
    if args.stage in ("cnn", "batch"):
        line = (_stage_cnn if args.stage == "cnn" else _stage_batch)(args, C, ctx, torch, clocks)
        line.update({"n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
                     "data": "synthetic", "clocks": clocks.summary()})
        ctx.close()
        return line
    rp, tables = _geometry(workdir, args.workload)
    if args.stage == "ssm":
        for _ in range(args.warmup):
            C.Ssm.generate(rp, ctx, C.SSM_FP16).free()
        clocks.start()
        ms, info = [], None
        for _ in range(args.steps):
            s = C.Ssm.generate(rp, ctx, C.SSM_FP16)
            info = s.info()
            ms.append(info.build_ms)
            s.free()
        clocks.stop()
        ncol, nvsm = int(info.n_columns), int(info.n_views)
        out_bytes = 6.0 * info.nnz + 4.0 * ncol * (nvsm + 1) + 8.0 * (ncol + 1)
        t = float(np.median(ms))
        line = {"metric": "ssm-entries/s", "value": info.nnz / (t / 1e3), "unit": "entries/s",
                "ms_per_step": t, "config": {"workload": args.workload, "stage": "generate_system_matrix",
                                             "nnz": int(info.nnz), "columns": ncol, "views": nvsm,
                                             "weights": "fp16"},
                "roofline": {"bound": "hbm", "achieved": out_bytes / (t / 1e3) / 1e9, "peak": peak,
                             "unit": "GB/s", "frac": out_bytes / (t / 1e3) / 1e9 / peak,
                             "kernel": "ssm_cells_kernel (count + fill)", "algorithmic_bytes_per_launch": out_bytes,
                             "peak_source": peak_kind}}
    else:
        nvox = int(np.prod(rp.shape))
        vin = torch.rand(nvox, device="cuda", dtype=torch.float32)
        vout = torch.empty_like(vin)
        ta = np.ascontiguousarray(tables.tube_angles, np.float64)
        si = np.ascontiguousarray(tables.slice_indices, np.uint64)

        def one():
            C.check(C.lib().ctbb_gpu_rotate_device(ctx.handle, ctypes.byref(rp.geom), C.ptr(ta, ctypes.c_double),
                                                   C.ptr(si, ctypes.c_uint64), ctypes.c_void_p(vin.data_ptr()),
                                                   ctypes.c_void_p(vout.data_ptr()), C.ROTATE_ROTATING2FIXED))

        for _ in range(args.warmup):
            one()
        flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")  # larger than L2
        clocks.start()
        ms = []
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            one()
            b.record()
            b.synchronize()
            ms.append(a.elapsed_time(b))
        clocks.stop()
        t = float(np.median(ms))
        out_bytes = 8.0 * nvox
        line = {"metric": "voxels/s", "value": nvox / (t / 1e3), "unit": "voxels/s", "ms_per_step": t,
                "config": {"workload": args.workload, "stage": "rotate_slices_rotating2fixed",
                           "voxels": nvox, "l2": "256 MB buffer written between steps (L2 flushed)"},
                "roofline": {"bound": "hbm", "achieved": out_bytes / (t / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                             "frac": out_bytes / (t / 1e3) / 1e9 / peak, "kernel": "rotate_kernel",
                             "algorithmic_bytes_per_launch": out_bytes, "peak_source": peak_kind}}
    line.update({"n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
                 "dtype": line.get("dtype", "f32"), "data": "synthetic", "clocks": clocks.summary()})
    ctx.close()
    subprocess.run(["rm", "-rf", workdir])
    return line


def _stage_batch(args, C, ctx, torch, clocks):
    """--stage batch: the benchmark's config 4, 32 independent uneven scans
    (replicas.batch_specs: 128..512 squared, 8..64 rows, pitch 0.5..1.5, with
    or without the in-plane flying focal spot, 8..64 slices, random
    ellipsoids, quadratic penalty, FP32 weights), 20 iterations each, on one
    GPU through the batched persistent kernel (one launch per iteration for
    all scans of a batch, replayed from a CUDA graph). Scans are packed into
    batches that fit in device memory (a scan that does not fit starts the
    next batch). For each batch the first three iterations try the streamed
    kernel at 1 and 2 times the default concurrency and the shared-memory
    staged kernel, and the remaining 17 use the fastest.
    Metric: voxel updates of all scans over the device time of the ICD
    launches; the wall-clock rate including each scan's set-up (projector,
    matrix build, visiting order) is reported beside it."""
    from ctbb_icd_b200 import replicas as RP
    from ctbb_icd_b200 import workloads as W

    specs = RP.batch_specs(32, seed=0)
    order = sorted(range(len(specs)), key=lambda i: -RP.scan_cost(specs[i]))
    workdir = tempfile.mkdtemp(prefix="ctbb_batch_")
    n_iter = 20
    totals = {"updates": 0.0, "device_ms": 0.0, "entries": 0.0}
    batches = []
    t_wall = time.perf_counter()
    clocks.start()
    pending = list(order)
    while pending:
        scans = []
        while pending:
            # Leave room for the iteration's own buffers (graph, FP64
            # refresh of the largest scan) before packing another scan.
            if scans and torch.cuda.mem_get_info()[0] < 4 * 2 ** 30:
                break
            i = pending[0]
            sp = specs[i]
            d = os.path.join(workdir, sp["name"])
            os.makedirs(d, exist_ok=True)
            prm = dict(sp["prm"], sinogram_path=os.path.join(d, "raw.bin"), output_dir=d, output_file="o.img")
            open(prm["sinogram_path"], "wb").close()
            rp = C.configure_recon_params(W.write_prm(os.path.join(d, "s.prm"), prm))
            rc = ssm = None
            try:
                tables = C.slice_tables(rp)
                rc = C.Recon(rp, tables.slice_indices, ctx)
                ph = W.phantom_spec(dict(sp["phantom"], z_lo=min(prm["z_start"], prm["z_end"]),
                                         z_hi=max(prm["z_start"], prm["z_end"])))
                C.check(C.lib().ctbb_gpu_synth_raw(ctx.handle, ctypes.byref(rp.geom), ctypes.byref(ph),
                                                   ctypes.c_void_p(rc.raw_device_ptr())))
                ssm = C.Ssm.generate(rp, ctx, C.SSM_FP32)
                rc.set_volume(ssm, None)
            except C.CtbbError as e:
                for obj in (ssm, rc):
                    if obj is not None:
                        obj.free()
                if e.status != 7 or not scans:  # CTBB_ERR_OOM with scans pending: run them first
                    raise
                break
            scans.append((i, rp, rc, ssm))
            pending.pop(0)
        b = C.Batch([x[2] for x in scans], [x[3] for x in scans], ctx)
        n_vox = sum(int(np.prod(x[1].shape)) for x in scans)
        base = C.icd_opts(mode=C.ICD_GROUPED, weights=C.SSM_FP32)
        default_w = _batch_default_warps(ctx, [x[1] for x in scans])
        trials = []
        # (warps in flight, column stage): the streamed kernel at the default
        # and twice the default concurrency, the shared-memory staged kernel.
        for w, stage in ((default_w, 0), (max(4, 2 * default_w), 0), (4 * 148, 1)):
            st = b.iterate(1, C.icd_opts(mode=C.ICD_GROUPED, weights=C.SSM_FP32, warps_in_flight=w,
                                         stage_column=stage))
            trials.append((w, stage, st.device_ms, st.entries))
        best = min(trials, key=lambda t: t[2])
        st = b.iterate(n_iter - 3, C.icd_opts(mode=C.ICD_GROUPED, weights=C.SSM_FP32, warps_in_flight=best[0],
                                             stage_column=best[1]))
        dev_ms = sum(t[2] for t in trials) + st.device_ms
        totals["updates"] += n_vox * n_iter
        totals["device_ms"] += dev_ms
        totals["entries"] += sum(t[3] for t in trials) + st.entries
        costs = []
        for _, _, rc, ssm in scans:
            rc.refresh_residual(ssm)
            costs.append(rc.cost())
        batches.append({"scans": [specs[x[0]]["name"] for x in scans], "voxels": n_vox,
                        "warps_in_flight": best[0], "stage_column": best[1],
                        "trials_ms": [[t[0], t[1], round(t[2], 2)] for t in trials], "device_ms": round(dev_ms, 1),
                        "fp64_costs_after": costs})
        b.free()
        for _, _, rc, ssm in scans:
            rc.free()
            ssm.free()
        torch.cuda.synchronize()
    clocks.stop()
    wall = time.perf_counter() - t_wall
    subprocess.run(["rm", "-rf", workdir])
    value = totals["updates"] / (totals["device_ms"] / 1e3)
    return {"metric": "voxel-updates/s", "value": value, "unit": "voxel-updates/s",
            "ms_per_step": totals["device_ms"] / n_iter, "dtype": "f32",
            "config": {"workload": "32 uneven helical scans (config 4), 20 iterations each, quadratic penalty, "
                                   "FP32 weights, batched persistent kernel replayed from a CUDA graph",
                       "stage": "batch", "scans": len(specs), "batches": batches,
                       "voxel_updates": totals["updates"], "entries": totals["entries"],
                       "wall_s_including_setup": round(wall, 1),
                       "wall_rate_including_setup": totals["updates"] / wall}}


def _batch_default_warps(ctx, rps):
    """The batch kernel's default concurrency (icd_grouped.cu
    ctbb_gpu_batch_iterate): 0.4 x voxels / (3.2 x largest nx), within
    [4, 32 warps per SM]."""
    n = sum(float(np.prod(r.shape)) for r in rps)
    nx = max(int(r.geom.nx) for r in rps)
    return max(4, min(148 * 32, int(0.4 * n / (3.2 * nx))))


def _stage_cnn(args, C, ctx, torch, clocks):
    """--stage cnn: the warm-start network's tensor-core convolutions on a
    --cnn-shape volume (default 16 x 256 x 256): time per forward pass and
    per training step (forward, loss, backward, gradient accumulation), and
    the FLOP rate of the 32 -> 32 convolutions (2 x 27 x 32 x 32 FLOP per
    voxel each: 2 per residual block forward; forward, backward-data and
    weight gradient per block in a training step)."""
    import json as _json

    from ctbb_icd_b200 import learned as L

    shape = args.cnn_shape
    net = L.WarmStartNet(ctx, 4, seed=0)
    engine = C.CNN_ENGINE_TCGEN05 if args.cnn_engine == "tcgen05" else C.CNN_ENGINE_MMA_SYNC
    net.set_engine(engine)
    g = torch.Generator(device="cuda").manual_seed(0)
    x = (0.15 + 0.1 * torch.rand(*shape, device="cuda", generator=g)).contiguous()
    xc = (x + 0.002 * torch.randn(*shape, device="cuda", generator=g)).contiguous()
    nvox = x.numel()
    conv_flop = 2.0 * 27 * 32 * 32 * nvox

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(args.steps):
            fn()
        b.record()
        b.synchronize()
        return a.elapsed_time(b) / args.steps

    clocks.start()
    fwd_ms = timed(lambda: net.forward(x))
    train_ms = timed(lambda: net.accumulate_gradient(x, xc))
    clocks.stop()
    net.zero_gradient()
    net.free()
    fwd_tflops = 2 * 4 * conv_flop / (fwd_ms / 1e3) / 1e12
    peak = None
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            peak = _json.load(f).get("bf16_tflops")
    return {"metric": "network voxels/s", "value": nvox / (fwd_ms / 1e3), "unit": "voxels/s",
            "ms_per_step": fwd_ms, "dtype": "bf16 operands, fp32 accumulation",
            "config": {"workload": f"warm-start CNN forward, 4 residual blocks x 32 channels, volume {shape}",
                       "stage": "cnn", "engine": args.cnn_engine, "train_step_ms": train_ms,
                       "train_conv_tflops": 6 * 4 * conv_flop / (train_ms / 1e3) / 1e12},
            "roofline": {"bound": "tensor", "achieved": fwd_tflops, "peak": peak, "unit": "TFLOP/s",
                         "frac": fwd_tflops / peak if peak else None,
                         "kernel": "conv_mid_tc_kernel" if args.cnn_engine == "tcgen05" else "conv_mid_kernel",
                         "algorithmic_flops_per_pass": 2 * 4 * conv_flop,
                         "peak_source": "measured" if peak else None}}


def run_e2e(C, ctx, rp, tables, ssm, rc, opts, args, x_start):
    """The same metric through ctbb_gpu_icd (the icd_iteration drop-in) with
    pinned host buffers, over the same iteration range as the device-timed
    region: each call uploads the raw data and the iterate the timed region
    started from, creates the reconstruction state (FP64 A x refresh of the
    error sinogram included), runs `steps` iterations with the same settings
    and returns the image."""
    import torch

    raw = torch.empty(rp.raw_shape, dtype=torch.float32).pin_memory()
    C.check(C.lib().ctbb_gpu_recon_get_raw(rc.handle, C.ptr(raw.numpy(), ctypes.c_float)))
    x0 = torch.from_numpy(np.ascontiguousarray(x_start, np.float32)).pin_memory()
    vol = torch.empty_like(x0).pin_memory()
    g = C.GeomC.from_buffer_copy(rp.geom)
    g.num_iterations = args.steps
    si = np.ascontiguousarray(tables.slice_indices, np.uint64)
    st = C.IterStats()

    def one():
        vol.copy_(x0)
        C.check(C.lib().ctbb_gpu_icd(ctx.handle, ssm.handle, ctypes.byref(g), C.ptr(si, ctypes.c_uint64),
                                     C.ptr(raw.numpy(), ctypes.c_float), C.ptr(vol.numpy(), ctypes.c_float),
                                     ctypes.byref(opts), ctypes.byref(st)))

    one()  # warm-up
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        one()
    torch.cuda.synchronize()
    secs = time.perf_counter() - t0
    nvox = int(np.prod(rp.shape))
    # Kernel launches per call: residual refresh (forward projection, residual),
    # image conversion, entry count and visiting order (order keys, collision
    # split), then one ICD launch per iteration.
    launches_per = 6 + args.steps
    return {"value": nvox * args.steps * args.e2e_steps / secs, "seconds": secs,
            "updates": nvox * args.steps * args.e2e_steps,
            "h2d": int(raw.numel() * 4 + x0.numel() * 4), "d2h": int(vol.numel() * 4),
            "launches": launches_per * args.e2e_steps}


def read_traffic(kernel: str = "icd_grouped_kernel"):
    """DRAM bytes per launch of the ICD kernel from the committed ncu summary
    of that kernel on this workload."""
    p = os.path.join(ROOT, "profiles", f"{kernel.replace('_kernel', '')}_cfg2.md")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.strip().startswith("traffic_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


TTT_LADDER = (1000.0, 500.0, 200.0, 100.0, 50.0, 25.0, 10.0, 5.0, 2.0, 1.0, 0.5)


def time_to_tolerance_sample(ctx, tuned, seed=900, ref_iter=300, max_iter=80):
    """The second half of the benchmark metric on a bounded sample: wall time
    of plain grouped ICD and of the learned warm start to each RMSE tolerance
    (HU, inside the object support, interior slices) against a reference
    image, on a held-out scan of the network's training grid (cfg2's scanner,
    flying focal spot and penalty at 256 x 256 x 32, 1.17 mm voxels). The
    reference is the learned start followed by `ref_iter` iterations; both
    arms start from the zero image and run at most `max_iter` iterations with
    the main run's autotuned kernel settings. Reports each tolerance's times,
    the tightest tolerance both arms reach, and how far the reference itself
    still moved over its last ten iterations."""
    import ctbb_icd_b200 as C
    from ctbb_icd_b200 import learned as L

    t0 = time.time()
    net = L.WarmStartNet.load(ctx, L.WEIGHTS_PATH)
    scan = L.make_scan(ctx, L.TRAIN_WORKLOAD, seed, weights=C.SSM_FP16)
    opts = C.icd_opts(mode=C.ICD_GROUPED, weights=C.SSM_FP16, warps_per_voxel=tuned.warps_per_voxel,
                      warps_in_flight=tuned.warps_in_flight, entries_per_lane=tuned.entries_per_lane,
                      stage_column=tuned.stage_column, entry_pairs=tuned.entry_pairs)
    scan.rc.set_volume(scan.ssm, None)
    scan.rc.iterate(scan.ssm, net.n_early, net.early_opts(scan.rc, opts))
    scan.rc.warm_start(scan.ssm, net, scan.tables.tube_angles)
    done = 0
    while done < ref_iter - 10:
        n = min(50, ref_iter - 10 - done)
        scan.rc.iterate(scan.ssm, n, opts)
        scan.rc.refresh_residual(scan.ssm)
        done += n
    x_tail = scan.rc.volume()
    scan.rc.iterate(scan.ssm, 10, opts)
    scan.rc.refresh_residual(scan.ssm)
    x_ref = scan.rc.volume()
    motion = scan.error_hu(x_tail, x_ref)
    plain = L.time_to_tolerance(scan, x_ref, opts, tol_hu=min(TTT_LADDER), max_iter=max_iter, tols=TTT_LADDER)
    learned = L.time_to_tolerance(scan, x_ref, opts, tol_hu=min(TTT_LADDER), max_iter=max_iter, net=net,
                                  n_early=net.n_early, tols=TTT_LADDER)
    rows, tightest = [], None
    for tol in TTT_LADDER:
        a, b = plain["seconds_to"][str(tol)], learned["seconds_to"][str(tol)]
        rows.append([tol, None if a is None else round(a, 3), None if b is None else round(b, 3)])
        if a is not None and b is not None:
            tightest = (tol, a, b)
    scan.rc.free()
    scan.ssm.free()
    return {
        "workload": f"held-out seed {seed} of the warm-start training grid ({L.TRAIN_WORKLOAD}: "
                    "256x256x32 at 1.17 mm, cfg2 scanner, in-plane FFS, edge-preserving)",
        "reference": f"learned start + {ref_iter} iterations; moved {motion:.3f} HU RMSE over its last 10",
        "fields": ["hu", "plain_s", "learned_s"], "seconds_to_hu": rows,
        "tightest_both": None if tightest is None else
        {"hu": tightest[0], "plain_s": round(tightest[1], 3), "learned_s": round(tightest[2], 3),
         "learned_over_plain": round(tightest[2] / tightest[1], 3) if tightest[1] > 0 else None},
        "final_hu": {"plain": round(plain["trace"][-1][2], 3), "learned": round(learned["trace"][-1][2], 3),
                     "iterations": max_iter},
        "wall_s": round(time.time() - t0, 1),
    }


# --------------------------------------------------------------------------
# Reference arm / CPU baseline
# --------------------------------------------------------------------------
CPU_SAMPLE = dict(nx=64, nz=16, readings=3200)


def _sample_inrange_entries(g, slice_indices, colptr, idx):
    """In-range matrix entries per voxel of a sample (the icd_iteration.cpp:
    205-207 window test), from its matrix and slice table."""
    per_view = int(g.n_channels) * int(g.Nrows_projection)
    limit = int(g.Readings) * per_view
    half = int(g.num_views_for_system_matrix) // 2
    total = 0
    q = idx.astype(np.int64)
    for si in slice_indices:
        off = (int(si) - half) * per_view
        total += int(np.count_nonzero((q + off >= 0) & (q + off < limit)))
    return total / float(len(slice_indices) * (len(colptr) - 1))


def reference_sample(iterations, *, own_matrix, extra_builds=(), workdir=None):
    """Run the reference program (oracle/_ref, the CTBB_ICD sources built
    unmodified; icd_ref_cores = -O2 with OpenMP on every host processor) on a
    bounded sample of the benchmark workload: the same scanner, views per
    turn, flying focal spot, voxel size, slice thickness, phantom and
    penalty, on a 64 x 64 x 16 central sub-volume (3.75 cm FOV) over the 3200
    views around it. Geometry comes from the reference's own setup code and
    the raw frames from the oracle's CPU projector; no library of this
    package is loaded.

    own_matrix: the reference generates its matrix.bin itself (its
    generate_system_matrix_ffs time is reported); otherwise the oracle's
    builder writes it (byte-identical, tests/test_reference_run.py), which
    keeps the sample within seconds. extra_builds: other reference builds
    ("shipped" = -g with its hard-coded 11 threads, "O2" = -O2 with 11
    threads) timed for 2 iterations on the same matrix."""
    from ctbb_icd_b200 import workloads as W
    from oracle import reference_run as R

    if not R.available():
        return {"value": None, "unit": "voxel-updates/s", "cores": 0, "kind": "reference",
                "sample": "unavailable: the reference program is not built under oracle/_ref"}
    s = CPU_SAMPLE
    d = workdir or tempfile.mkdtemp(prefix="ctbb_ref_")
    w = W.workload(WORKLOAD)
    prm = R.central_subvolume(dict(w["prm"], num_iterations=iterations), s["nx"], s["nz"], s["readings"], d)
    prm_path = R.write_prm(os.path.join(d, "ref.prm"), prm)
    R.write_zero_raw(prm["sinogram_path"], prm["Readings"], prm["n_channels"], prm["Nrows"])
    fields, _, slices = R.setup_dump(prm_path)
    g = R.geometry(fields)
    ph = dict(w["phantom"], z_lo=min(prm["z_start"], prm["z_end"]), z_hi=max(prm["z_start"], prm["z_end"]))
    t0 = time.perf_counter()
    R.write_raw(prm["sinogram_path"], R.synth_raw(g, ph))
    synth_s = time.perf_counter() - t0
    matrix = os.path.join(d, "matrix.bin")
    if not own_matrix:
        R.write_matrix_bin(matrix, *R.oracle_matrix(g))
    ncpu = os.cpu_count() or 1
    rc, stamps = R.run("cores", prm_path, d)
    times = R.stage_times(stamps)
    if rc != 0 or len(times["iteration_s"]) < iterations:
        subprocess.run(["rm", "-rf", d])
        return {"value": None, "unit": "voxel-updates/s", "cores": ncpu, "kind": "reference",
                "sample": f"reference run failed (exit {rc}): " + " | ".join(l for _, l in stamps[-3:])}
    m = _read_colptr_idx(matrix, int(g.num_voxels_x * g.num_voxels_y))
    entries = _sample_inrange_entries(g, [sl[1] for sl in slices], *m)
    extra = {}
    for kind in extra_builds:
        p2 = R.write_prm(os.path.join(d, f"ref_{kind}.prm"), dict(prm, num_iterations=2, matrix_path=matrix,
                                                                   output_file=f"ref_{kind}.img"))
        rc2, st2 = R.run(kind, p2, d)
        extra[kind] = R.stage_times(st2)["iteration_s"] if rc2 == 0 else None
    subprocess.run(["rm", "-rf", d])
    nvox = s["nx"] * s["nx"] * s["nz"]
    per_iter = np.asarray(times["iteration_s"], np.float64)
    rate = nvox / float(np.median(per_iter))
    desc = (f"reference icd_iteration (CTBB_ICD sources built unmodified at -O2, OpenMP on all {ncpu} host "
            f"processors) on a {s['nx']}x{s['nx']}x{s['nz']} central sub-volume of the benchmark geometry "
            f"(3.75 cm FOV, {s['readings']} views, same scanner, voxel size, phantom and penalty; "
            f"{entries:.0f} in-range matrix entries per voxel vs {FULL_ENTRIES_PER_VOXEL:.0f} in the full "
            f"workload, rate not rescaled); median of {len(per_iter)} iterations {float(np.median(per_iter)):.3f} s")
    if times["ssm_s"] is not None:
        desc += f"; its own generate_system_matrix_ffs took {times['ssm_s']:.1f} s (single thread)"
    for kind, its in extra.items():
        label = {"shipped": "as shipped (-g, 11 threads)", "O2": "-O2 with its 11 threads"}.get(kind, kind)
        if its:
            desc += f"; {label}: {float(np.median(its)):.3f} s per iteration = {nvox / float(np.median(its)):.4g} vu/s"
    return {"value": rate, "unit": "voxel-updates/s", "cores": ncpu, "kind": "reference", "sample": desc,
            "seconds_per_iteration": per_iter.tolist(), "ssm_s": times["ssm_s"], "synth_s": synth_s,
            "entries_per_voxel_sample": entries, "extra_builds": extra}


# In-range matrix entries per voxel of the full benchmark workload (the
# 1.16e11 entries one iteration visits over 16,777,216 voxels, counted by the
# grouped kernel's entry counter on the GPU).
FULL_ENTRIES_PER_VOXEL = 116058564736 / 16777216


def _read_colptr_idx(path, ncol):
    buf = np.fromfile(path, np.uint8)
    colptr = np.zeros(ncol + 1, np.int64)
    parts = []
    pos = 0
    for c in range(ncol):
        n = int(buf[pos:pos + 8].view(np.uint64)[0])
        parts.append(buf[pos + 8:pos + 8 + 8 * n].view(np.int32)[0::2])
        pos += 8 + 8 * n
        colptr[c + 1] = colptr[c] + n
    return colptr, np.concatenate(parts) if parts else np.zeros(0, np.int32)


def cpu_sample(iterations=3):
    """CPU baseline for the benchmark line (rank 0, N = 1): the reference's
    ICD on the bounded sample, with the oracle-built matrix so the sample
    stays within tens of seconds."""
    return reference_sample(iterations, own_matrix=False)


def run_reference(args, rank, world):
    if rank != 0:
        return None
    r = reference_sample(args.warmup + args.steps, own_matrix=True, extra_builds=("shipped", "O2"))
    if not r.get("value"):
        return {"impl": "reference", "unavailable": r.get("sample", "reference run failed")}
    times = r["seconds_per_iteration"][-args.steps:]
    nvox = CPU_SAMPLE["nx"] ** 2 * CPU_SAMPLE["nz"]
    v = nvox * len(times) / float(np.sum(times))
    cb = dict(r, value=v)
    return {
        "impl": "reference", "metric": "voxel-updates/s", "value": v, "unit": "voxel-updates/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * float(np.mean(times)),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded phantom: water + 6 inserts + 40 ellipsoids, Poisson noise, oracle CPU projector)",
        "config": {"workload": WORKLOAD_TEXT, "sample": cb["sample"], "ssm_generation_s": r["ssm_s"],
                   "threads": r["cores"]},
        "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
        "e2e": {"value": v, "unit": "voxel-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--weights", choices=["fp16", "fp32"], default="fp16")
    ap.add_argument("--workload", default=WORKLOAD,
                    help="workload name from ctbb_icd_b200.workloads (the benchmark is cfg2)")
    ap.add_argument("--warps", type=int, default=0, help="warps in flight (0: auto)")
    ap.add_argument("--lattice", type=int, default=0)
    ap.add_argument("--wpv", type=int, default=1, help="warps per voxel update: 1, 4 or 8")
    ap.add_argument("--epl", type=int, default=0, help="entries per lane in flight: 8 or 16 (0: 8)")
    ap.add_argument("--no-autotune", dest="autotune", action="store_false",
                    help="skip the library's autotuner (warps per voxel, warps in flight, tile edge) and use "
                         "--wpv/--warps/--lattice as given")
    ap.add_argument("--no-e2e", dest="e2e", action="store_false")
    ap.add_argument("--e2e-steps", type=int, default=1, help="timed drop-in calls (each runs --steps iterations)")
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--no-ttt", dest="ttt", action="store_false",
                    help="skip the time-to-tolerance sample (plain vs learned warm start)")
    ap.add_argument("--no-clocks", dest="clocks", action="store_false", help="skip nvidia-smi clock sampling")
    ap.add_argument("--own-stream", action="store_true", help="run on the library's own stream")
    ap.add_argument("--stage", choices=["icd", "ssm", "rotate", "cnn", "batch"], default="icd",
                    help="icd (default): the grouped-ICD benchmark; ssm / rotate: time the matrix builder or the "
                         "slice rotation of the same workload on their own; cnn: the warm-start network; "
                         "batch: 32 uneven scans (config 4)")
    ap.add_argument("--cnn-shape", type=int, nargs=3, default=[16, 256, 256])
    ap.add_argument("--cnn-engine", choices=["tcgen05", "mma_sync"], default="mma_sync",
                    help="--stage cnn: tensor-core path of the 32 -> 32 convolutions")
    ap.add_argument("--entry-pairs", type=int, default=0, choices=[0, -1],
                    help="with --no-autotune: 0 reads FP16 matrices as entry pairs, -1 as single entries")
    ap.add_argument("--stack-align", type=int, default=0, choices=[0, 1],
                    help="with --no-autotune, 4 or 8 warps per voxel: start each sweep at its slice stack's "
                         "common data view")
    ap.add_argument("--l2-hints", type=int, default=0, choices=[0, 1],
                    help="with --no-autotune, 4 or 8 warps per voxel: matrix loads evict-first, e gathers "
                         "evict-last")
    ap.add_argument("--stage-column", type=int, default=-1,
                    help="with --no-autotune: 0 streams each column twice, 1/2 stage it in shared memory, "
                         "3 sweeps each slice stack in lockstep in one CTA, 4/5 bulk-copy each update's entry "
                         "pairs into one/two shared-memory stages, 6 the one-stage form with the next item claimed "
                         "ahead")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = None
    # The reference arm is rank 0's CPU work alone: no process group, and the
    # other ranks exit at once without touching a GPU.
    if world > 1 and args.impl != "reference":
        import datetime

        import torch
        import torch.distributed as tdist

        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        dist = tdist
    try:
        if args.impl == "reference":
            out = run_reference(args, rank, world)
        elif args.stage != "icd":
            out = run_stage(args) if rank == 0 else None
        else:
            out = run_ours(args, rank, world, dist)
        if rank == 0 and out is not None:
            print(json.dumps(out), flush=True)
    finally:
        if dist:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
